"""Helpers for the GPU parity tests: run the library through the C ABI and
bring results back in the oracle's canonical forms."""
import numpy as np

import gkc_b200 as G
import oracle_ffi as F


def lib_partition(ctx, reads, offs, k, p, hpc, nbins):
    v = ctx.partition_host(reads, offs, G.params(k, p, nbins, hpc))
    bin_off, lens, boff, packed, mm = ctx.partition_copy_out(v)
    bins = np.repeat(np.arange(nbins, dtype=np.uint32), np.diff(bin_off).astype(np.int64))
    return F.Skms(bins, lens, boff, packed, minimizer=mm), v


def lib_counts(ctx, k, nbins, mode=G.MODE_BATCHED):
    v = ctx.count_device(G.params(k, 3 if k >= 3 else k, nbins), mode)
    bin_off, keys, counts = ctx.count_copy_out(v)
    res = dict(bin_off=bin_off, counts=counts, keys_lo=keys[:, 0].copy(),
               keys_hi=keys[:, 1].copy() if keys.shape[1] > 1 else None)
    return res, v


def assert_counts_equal(got, want):
    assert np.array_equal(got["bin_off"], want["bin_off"]), "bin offsets differ"
    assert np.array_equal(got["keys_lo"], want["keys_lo"]), "keys differ"
    if want.get("keys_hi") is not None:
        assert np.array_equal(got["keys_hi"], want["keys_hi"]), "high key words differ"
    assert np.array_equal(got["counts"], want["counts"]), "counts differ"
