"""The counting entry point that allocates nothing, checked against the one
that does.

Some callers cannot allocate device memory while they run: a program whose
own memory pool owns the GPU, a framework whose allocator holds all of HBM,
or a path where a cudaMalloc would stall the device or break a hard memory
cap.  They count a group of superkmers with
gkc_count_superkmers_device_noalloc, which takes its scratch memory from one
fixed array inside the library.  These tests call it through the C ABI on
device buffers and compare its sorted (k-mer, count) list with what
gkc_count_superkmers_host returns for the same superkmers, over two calls in a
row (the second call finds the first call's leftovers in the shared array).

This file is collected last so that a run stopping at its first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F

pytestmark = pytest.mark.gpu

GKC_OK, GKC_ERR_INVALID_ARG, GKC_ERR_CAPACITY = 0, 1, 6
MAX_SKM, MAX_KMERS = 1 << 17, 1 << 20


def superkmer_group(seed, n, k, lo, hi, pool=400):
    """n superkmers drawn with repeats from a pool of random ones (so that
    many k-mers occur more than once), plus a few poly-A ones; lengths in
    [lo, hi] with some shorter than k."""
    r = np.random.default_rng(seed)
    base_lens = r.integers(lo, hi + 1, pool).astype(np.uint32)
    base_lens[: pool // 20] = r.integers(1, k, pool // 20)  # no k-mer at all
    base = [r.integers(0, 256, int((ln + 3) // 4), dtype=np.uint8) for ln in base_lens]
    base[-1][:] = 0  # poly-A: one canonical k-mer many times
    pick = r.integers(0, pool, n)
    lens = base_lens[pick]
    packed = np.concatenate([base[i] for i in pick])
    return lens, packed


def n_kmers_of(lens, k):
    lens = lens.astype(np.int64)
    return int(np.maximum(lens - k + 1, 0).sum())


def count_with_alloc(ctx, k, lens, packed):
    nd = ctx.count_superkmers_host(k, lens, packed)
    bin_off = np.zeros(2, np.uint64)
    keys = np.zeros(max(nd, 1), np.uint64)
    counts = np.zeros(max(nd, 1), np.uint32)
    assert G.lib().gkc_count_copy_out(ctx.h, bin_off.ctypes.data,
                                      keys.ctypes.data, counts.ctypes.data) == GKC_OK
    return keys[:nd], counts[:nd]


def count_no_alloc(torch, k, lens, packed, capacity=None):
    """-> (status, keys, counts) from the no-allocation entry point."""
    d_lens = torch.from_numpy(lens.astype(np.uint32).view(np.int32)).cuda()
    d_packed = torch.from_numpy(packed.astype(np.uint8)).cuda()
    cap = n_kmers_of(lens, k) if capacity is None else capacity
    d_keys = torch.zeros(max(cap, 1), dtype=torch.int64, device="cuda")
    d_counts = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    nd = C.c_uint64(12345)
    st = G.lib().gkc_count_superkmers_device_noalloc(
        int(k), d_lens.data_ptr(), d_packed.data_ptr(), len(lens), cap, d_keys.data_ptr(),
        d_counts.data_ptr(), C.byref(nd), None)
    torch.cuda.synchronize()
    n = int(nd.value)
    keys = d_keys[:n].cpu().numpy().view(np.uint64)
    counts = d_counts[:n].cpu().numpy().view(np.uint32)
    return st, keys, counts


@pytest.fixture(scope="module")
def torch():
    import torch as T
    return T


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def test_two_calls_in_a_row_match_the_allocating_entry_point(torch, ctx):
    # a large group, then a smaller one with another k: the second call must
    # not see anything of the first in the shared scratch array
    for seed, n, k, lo, hi in [(11, 12000, 31, 20, 120), (12, 3000, 21, 10, 60)]:
        lens, packed = superkmer_group(seed, n, k, lo, hi)
        assert n_kmers_of(lens, k) <= MAX_KMERS
        want_keys, want_counts = count_with_alloc(ctx, k, lens, packed)
        st, keys, counts = count_no_alloc(torch, k, lens, packed)
        assert st == GKC_OK
        assert len(keys) == len(want_keys)
        assert np.array_equal(keys, want_keys)
        assert np.array_equal(counts, want_counts)
        assert int(counts.astype(np.int64).sum()) == n_kmers_of(lens, k)
        assert counts.max() > 1
        # and against the oracle's count of the same group
        boff = np.zeros(len(lens), np.uint64)
        boff[1:] = np.cumsum((lens.astype(np.uint64) + 3) // 4)[:-1]
        want = F.oracle_count_bins(F.Skms(np.zeros(len(lens), np.uint32), lens, boff, packed), k, 1)
        assert np.array_equal(keys, want["keys_lo"])
        assert np.array_equal(counts, want["counts"])


def test_a_call_allocates_no_device_memory(torch):
    k = 31
    lens, packed = superkmer_group(21, 4000, k, 20, 120)
    d_lens = torch.from_numpy(lens.astype(np.uint32).view(np.int32)).cuda()
    d_packed = torch.from_numpy(packed).cuda()
    cap = n_kmers_of(lens, k)
    d_keys = torch.zeros(cap, dtype=torch.int64, device="cuda")
    d_counts = torch.zeros(cap, dtype=torch.int32, device="cuda")
    nd = C.c_uint64(0)

    def call():
        return G.lib().gkc_count_superkmers_device_noalloc(
            k, d_lens.data_ptr(), d_packed.data_ptr(), len(lens), cap, d_keys.data_ptr(),
            d_counts.data_ptr(), C.byref(nd), None)

    assert call() == GKC_OK  # first call on the device: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call() == GKC_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_a_capturing_stream_is_refused(torch):
    k = 31
    lens, packed = superkmer_group(22, 100, k, 40, 60)
    d_lens = torch.from_numpy(lens.astype(np.uint32).view(np.int32)).cuda()
    d_packed = torch.from_numpy(packed).cuda()
    cap = n_kmers_of(lens, k)
    d_keys = torch.zeros(cap, dtype=torch.int64, device="cuda")
    d_counts = torch.zeros(cap, dtype=torch.int32, device="cuda")
    nd = C.c_uint64(0)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        st = G.lib().gkc_count_superkmers_device_noalloc(
            k, d_lens.data_ptr(), d_packed.data_ptr(), len(lens), cap, d_keys.data_ptr(),
            d_counts.data_ptr(), C.byref(nd), C.c_void_p(s.cuda_stream))
    assert st == GKC_ERR_INVALID_ARG
    del g


def test_group_at_the_kmer_limit(torch, ctx):
    k = 25
    r = np.random.default_rng(5)
    n = MAX_KMERS // 64  # superkmers of 64 k-mers: exactly the limit
    lens = np.full(n, 64 + k - 1, np.uint32)
    packed = r.integers(0, 256, n * int((64 + k - 1 + 3) // 4), dtype=np.uint8)
    packed[: 40 * 22] = 7  # a repeated stretch
    want_keys, want_counts = count_with_alloc(ctx, k, lens, packed)
    st, keys, counts = count_no_alloc(torch, k, lens, packed)
    assert st == GKC_OK
    assert np.array_equal(keys, want_keys)
    assert np.array_equal(counts, want_counts)


def test_sizes_beyond_the_limits_are_rejected(torch):
    k = 21
    # too many k-mers: 20000 superkmers of 80 k-mers each
    lens = np.full(20000, 80 + k - 1, np.uint32)
    packed = np.zeros(20000 * ((80 + k - 1 + 3) // 4), np.uint8)
    st, _, _ = count_no_alloc(torch, k, lens, packed)
    assert st == GKC_ERR_CAPACITY
    # too many superkmers (checked before any GPU work)
    lens = np.full(MAX_SKM + 1, 1, np.uint32)
    st, _, _ = count_no_alloc(torch, k, lens, np.zeros(MAX_SKM + 1, np.uint8))
    assert st == GKC_ERR_CAPACITY
    # output buffers smaller than the group's k-mers
    lens, packed = superkmer_group(3, 500, k, 30, 60)
    st, _, _ = count_no_alloc(torch, k, lens, packed, capacity=n_kmers_of(lens, k) - 1)
    assert st == GKC_ERR_CAPACITY
    # 128-bit keys are not supported here
    st, _, _ = count_no_alloc(torch, 33, lens, packed)
    assert st == GKC_ERR_INVALID_ARG
    # after the rejections the array still serves a normal call
    st, keys, counts = count_no_alloc(torch, k, lens, packed)
    assert st == GKC_OK and len(keys) > 0
