"""Literal, slow emulation of the reference device code paths that define the
compressed layout -- used only to cross-check the CPU oracle's restatement.

Python integers stand in for the device registers; every shift follows PTX
semantics (shl/shr by >= the register width yield 0), which is what the
reference relies on when a mask word is 0 or all ones.

  compress_and_write      include/compress/ibp_compress_dev.cuh:7-97
  check_compress_size_*   include/misc/ibp_misc_dev.cuh:19-91
  decompress loop         include/decompress/ibp_decompress_dev.cuh:188-339
"""

M64 = (1 << 64) - 1


def _mask(w):
    return (1 << w) - 1


def shl(x, n, w):
    """PTX shl.b<w>: shift amounts >= w give 0."""
    return 0 if n >= w else (x << n) & _mask(w)


def shr(x, n, w):
    """PTX shr.u<w> (logical)."""
    return 0 if n >= w else (x & _mask(w)) >> n


def clz(x, w):
    x &= _mask(w)
    return w if x == 0 else w - x.bit_length()


def popc(x, w):
    return bin(x & _mask(w)).count("1")


def compressed_size(row, mask, bitval, w):
    """check_compress_size_warp: bytes of the compressed row, or the raw size."""
    v = len(row)
    wb = w // 8
    ctr = sum(popc(mask[j], w) for j in range(v) if (row[j] & mask[j]) == bitval[j])
    vec_bytes = v * wb
    meta = ((v + 7) // 8 + wb - 1) // wb * wb
    data = vec_bytes - ctr // 8
    data = (data + wb - 1) // wb * wb
    comp = meta + data
    return comp if comp < vec_bytes else vec_bytes


def compress_and_write(row, mask, bitval, w):
    """Word-by-word replay of the warp packer; returns the v output words."""
    v = len(row)
    wb = w // 8
    out = [0] * v
    bitmask_offset = ((v + 7) // 8 + wb - 1) // wb * wb  # bytes
    bitshift = 0
    for j in range(v):
        local_mask = mask[j] & _mask(w)
        val = row[j] & _mask(w)
        cur = w
        comp = (val & local_mask) == (bitval[j] & _mask(w))
        if comp:
            cur -= popc(local_mask, w)
        insert_size = w - popc(local_mask, w)
        compressed_val = 0
        if comp:
            num_bits = insert_size
            tis = clz(local_mask, w)
            num_inserted = 0
            while num_bits > 0:
                num_inserted += tis
                # (T)(((1ll << tis) - 1ll) << (W - num_inserted)), 64-bit signed ops
                part = (shl(1, tis, 64) - 1) & M64
                part = shl(part, w - num_inserted, 64)
                compressed_val |= val & part & _mask(w)
                num_bits -= tis
                local_mask = shl(local_mask, tis, w)
                shift = clz(~local_mask & _mask(w), w)
                local_mask = shl(local_mask, shift, w)
                val = shl(val, shift, w)
                tis = min(clz(local_mask, w), num_bits)
            out[j // w] |= 1 << (j % w)
        else:
            insert_size = w
            compressed_val = val
        fin = 0
        while insert_size > 0:
            elem = (bitmask_offset + bitshift // 8) // wb
            bit_offset = (bitmask_offset * 8 + bitshift) % w
            ib = min(insert_size, w - bit_offset)
            part = shl((shl(1, ib, 64) - 1) & M64, w - ib, 64)
            ins = (shl(compressed_val, fin, w) & part) >> bit_offset
            out[elem] |= ins & _mask(w)
            fin += ib
            insert_size -= ib
            bitshift += ib
        assert cur >= 0
    return out


def decompress_row(comp_row, mask, bitval, w):
    """Word-by-word replay of the decompress loop over the row's stream words."""
    v = len(comp_row)
    wb = w // 8
    mw = (((v + 7) // 8 + wb - 1) // wb * wb) // wb
    working = comp_row[mw:]
    out = [0] * v
    bitshift = 0
    for i in range(v):
        compressed = (comp_row[i // w] >> (i % w)) & 1
        num_bits = w
        if compressed:
            num_bits -= popc(mask[i], w)
        local_mask = mask[i] & _mask(w)
        if compressed:
            temp = bitval[i] & _mask(w)
            trs = min(num_bits, clz(local_mask, w))
        else:
            temp = 0
            trs = num_bits
        fin = 0
        while num_bits > 0:
            bit_offset = bitshift % w
            rb = min(trs, w - bit_offset)
            wd = working[bitshift // w] & _mask(w)
            part = shl((shl(1, rb, 64) - 1) & M64, w - rb, 64)
            term = (shl(wd, bit_offset, w) & part)
            term = shr(term, fin, 64)
            temp |= term & _mask(w)
            fin += rb
            num_bits -= rb
            bitshift += rb
            if compressed:
                local_mask = shl(local_mask, rb, w)
                shift = clz(~local_mask & _mask(w), w)
                local_mask = shl(local_mask, shift, w)
                fin += shift
                trs = min(clz(local_mask, w), num_bits)
            else:
                trs = num_bits
        out[i] = temp
    return out
