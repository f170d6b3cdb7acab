"""A caller of the reference's extension module, written the way its throughput scripts call
it (`import ibp_cuda as ibp`, every argument positional, a hand-made mask and bitval, the
average compressed length passed as a 0-d float tensor, an index array, impl None and 2; the
pattern of the reference's tests/decompression_thput.py).  Run with the repository's dropin/
directory on PYTHONPATH.  Prints one "Match? <bool>" line per case."""
import torch
import ibp_cuda as ibp

torch.manual_seed(1)
ROWS = 5000


def hand_mask(width, invariant_share):
    """A random mask over int32 columns with about `invariant_share` of the bits set."""
    bits = 32 * width
    mask = torch.zeros(width, dtype=torch.int32)
    for b in torch.randperm(bits)[: int(invariant_share * bits)].tolist():
        mask[b // 32] |= (1 << (b % 32)) if b % 32 != 31 else -(1 << 31)
    return mask


for width in (64, 256, 1024):
    for share in (0.25, 0.75, 0.97):
        mask = hand_mask(width, share)
        bitval = torch.randint(-(2 ** 31), 2 ** 31 - 1, (width,), dtype=torch.int32) & mask
        data = torch.randint(-(2 ** 31), 2 ** 31 - 1, (ROWS, width), dtype=torch.int32)
        data = (data & ~mask) | bitval  # every row fits the mask
        data[::97] = torch.randint(-(2 ** 31), 2 ** 31 - 1, data[::97].shape, dtype=torch.int32)
        m, bv = mask.to(torch.device("cuda")), bitval.to(torch.device("cuda"))
        packed = data.detach().clone().pin_memory()
        sizes = ibp.get_compress_size(packed, m, bv, None, None)
        torch.cuda.synchronize()
        avg_len = torch.sum(sizes) / (packed.numel() * packed.element_size()) * width
        bitmask = ibp.compress_inplace(packed, m, bv, None)
        torch.cuda.synchronize()
        index = torch.randint(0, ROWS, (3000,), device="cuda")
        for impl in (None, 2):
            out = ibp.decompress_fetch(packed, m, bv, bitmask, torch.device("cuda"), avg_len,
                                       index, None, None, impl, None)
            want = (data if impl is None else packed)[index.cpu()]
            print(f"width {width} share {share} impl {impl}:", end=" ")
            print("Match?", torch.equal(want, out.to(torch.device("cpu"))))
        whole = ibp.decompress_fetch(packed, m, bv, bitmask, torch.device("cuda"), avg_len, None,
                                     None, None, None, None)
        print(f"width {width} share {share} whole:", end=" ")
        print("Match?", torch.equal(data, whole.cpu()))
