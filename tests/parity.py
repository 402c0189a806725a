"""Canonical forms and digests used to compare partition and count outputs.

Partition parity is per bin, as a multiset of (length, packed bytes): order
within and across bins is free.  Count parity is per bin, as the sorted
(k-mer, count) array.
"""
import hashlib

import numpy as np


def partition_digest(multisets):
    h = hashlib.sha256()
    for b, items in enumerate(multisets):
        h.update(b"BIN" + int(b).to_bytes(4, "little") + len(items).to_bytes(8, "little"))
        for ln, data in items:
            h.update(int(ln).to_bytes(4, "little"))
            h.update(data)
    return h.hexdigest()


def counts_digest(bin_off, keys_lo, counts, keys_hi=None):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(bin_off, np.uint64).tobytes())
    h.update(np.ascontiguousarray(keys_lo, np.uint64).tobytes())
    if keys_hi is not None:
        h.update(np.ascontiguousarray(keys_hi, np.uint64).tobytes())
    h.update(np.ascontiguousarray(counts, np.uint32).tobytes())
    return h.hexdigest()


def bytes_digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def flatten_multisets(multisets):
    """(bin, len, byte_off, bytes) arrays in canonical (bin, len, bytes) order."""
    bins, lens, offs, data = [], [], [], []
    o = 0
    for b, items in enumerate(multisets):
        for ln, d in items:
            bins.append(b)
            lens.append(ln)
            offs.append(o)
            data.append(d)
            o += len(d)
    return (np.array(bins, np.uint32), np.array(lens, np.uint32), np.array(offs, np.uint64),
            np.frombuffer(b"".join(data), np.uint8).copy())
