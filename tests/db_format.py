"""The on-disk k-mer database format restated in Python: a writer that lays
out the bytes from a sorted (key, count) list and a parser, independent of
the library's C writer and reader.  TEST INFRASTRUCTURE.

<path>.gkc_pre: "GKCP", u32 version 1, u32 k, lut_prefix_len l, suffix_bytes,
counter_bytes, min_count, max_count, u64 n, total; u64 lut[4^l + 1]; "GKCP".
<path>.gkc_suf: "GKCS", n x (low 2(k-l) key bits big-endian in
suffix_bytes, count little-endian in counter_bytes), "GKCS"."""
import struct

import numpy as np


def auto_lut(n, k):
    l = 1
    while l < 13 and (4 ** (l + 1)) * 8 <= n:
        l += 1
    return min(l, k - 1)


def key_ints(keys):
    """(n, kw) uint64 -> Python ints (low word first)."""
    keys = np.asarray(keys, np.uint64)
    if keys.ndim == 1:
        return [int(x) for x in keys]
    return [int(r[0]) | (int(r[1]) << 64 if keys.shape[1] > 1 else 0) for r in keys]


def layout(k, keys, counts, min_count, max_count, lut_len=0):
    """-> (pre bytes, suf bytes)."""
    ks = key_ints(keys)
    counts = [int(c) for c in counts]
    n = len(ks)
    l = lut_len if lut_len else auto_lut(n, k)
    shift = 2 * (k - l)
    sb = (shift + 7) // 8
    cmax = max(counts, default=0)
    cb = 1 if cmax < 256 else 2 if cmax < 65536 else 3 if cmax < (1 << 24) else 4
    prefixes = np.array([x >> shift for x in ks], np.uint64)
    lut = np.searchsorted(prefixes, np.arange(4 ** l + 1, dtype=np.uint64), side="left").astype(np.uint64)
    pre = b"GKCP" + struct.pack("<IIIIIIIQQ", 1, k, l, sb, cb, min_count, max_count, n, sum(counts)) \
        + lut.tobytes() + b"GKCP"
    mask = (1 << shift) - 1
    recs = b"".join((x & mask).to_bytes(sb, "big") + c.to_bytes(cb, "little") for x, c in zip(ks, counts))
    return pre, b"GKCS" + recs + b"GKCS"


def write(path, *args, **kw):
    pre, suf = layout(*args, **kw)
    with open(f"{path}.gkc_pre", "wb") as f:
        f.write(pre)
    with open(f"{path}.gkc_suf", "wb") as f:
        f.write(suf)


def parse(path):
    """-> (header dict, [(key, count)] in file order)."""
    pre = open(f"{path}.gkc_pre", "rb").read()
    suf = open(f"{path}.gkc_suf", "rb").read()
    assert pre[:4] == b"GKCP" and pre[-4:] == b"GKCP" and suf[:4] == b"GKCS" and suf[-4:] == b"GKCS"
    ver, k, l, sb, cb, mn, mx, n, total = struct.unpack_from("<IIIIIIIQQ", pre, 4)
    lut = np.frombuffer(pre, np.uint64, 4 ** l + 1, 4 + struct.calcsize("<IIIIIIIQQ"))
    shift = 2 * (k - l)
    out = []
    rec = sb + cb
    p = 0
    for i in range(n):
        while lut[p + 1] <= i:
            p += 1
        r = suf[4 + i * rec:4 + (i + 1) * rec]
        out.append(((p << shift) | int.from_bytes(r[:sb], "big"), int.from_bytes(r[sb:], "little")))
    return dict(version=ver, k=k, lut_prefix_len=l, suffix_bytes=sb, counter_bytes=cb, min_count=mn,
                max_count=mx, n_kmers=n, total_count=total), out
