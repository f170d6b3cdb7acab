"""A caller of the reference's `ibp` package, written the way its own scripts call it
(`import ibp`; preprocess -> pinned clone -> get_compress_size -> compress_inplace ->
decompress_fetch onto 'cuda'; the round-trip pattern of the reference's tests/compress_test.py).
Run with the repository's dropin/ directory on PYTHONPATH, it exercises the engine through
exactly those calls.  Prints one "Match? <bool>" line per tensor."""
import ibp
import torch

torch.manual_seed(0)


def round_trip(original):
    mask, bitval = ibp.preprocess(original)
    packed = original.detach().clone().pin_memory()
    sizes = ibp.get_compress_size(packed, mask, bitval)
    torch.cuda.synchronize()
    raw = packed.numel() * packed.element_size()
    small = int(torch.sum(sizes))
    print(f"raw {raw} compressed {small} ({raw / small:.2f}x)")
    bitmask = ibp.compress_inplace(packed, mask, bitval)
    torch.cuda.synchronize()
    back = ibp.decompress_fetch(packed, mask, bitval, bitmask, torch.device("cuda"))
    print("Match?", torch.equal(original.to(torch.device("cuda")), back))


uniform32 = torch.rand([1200, 128], dtype=torch.float32).pin_memory()
round_trip(uniform32)
round_trip(uniform32.clone().pin_memory().view(dtype=torch.float64))
dense32 = torch.randint(2147483647, [100, 100], dtype=torch.int32).pin_memory()
round_trip(dense32)
round_trip(dense32.clone().pin_memory().view(dtype=torch.int64))
narrow32 = torch.randint(2147483647 // 100, [6, 100], dtype=torch.int32).pin_memory()
round_trip(narrow32)
round_trip(narrow32.clone().pin_memory().view(dtype=torch.int64))
