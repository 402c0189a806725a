"""The streaming host form (gkc_stream_submit / gkc_stream_wait): calls whose
upload, counting and download overlap give, call by call, the oracle's
per-bin sorted (k-mer, count) lists, with inputs of the same size (replays
of a captured pipeline with new reads) and of another size, reads cut from a
larger CSR, and the refusals: output room too small, pageable buffers."""
import ctypes as C

import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F
from gkc_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    return T


def pinned(torch, a):
    dt = {np.uint8: torch.uint8, np.uint64: torch.int64}[a.dtype.type]
    t = torch.empty(len(a), dtype=dt, pin_memory=True)
    t.numpy()[:] = a.view(t.numpy().dtype)
    return t


def outputs(torch, nbins, cap):
    return (torch.zeros(nbins + 1, dtype=torch.int64, pin_memory=True),
            torch.zeros(max(cap, 1), dtype=torch.int64, pin_memory=True),
            torch.zeros(max(cap, 1), dtype=torch.int32, pin_memory=True))


def expect(reads, offs, k, p, nbins):
    o = F.oracle_partition(reads, offs, k, p, 0, nbins)
    return F.oracle_count_bins(o, k, nbins)


def check(out, want, nd):
    bo, keys, counts = (t.numpy() for t in out)
    assert nd == len(want["keys_lo"])
    assert np.array_equal(bo.view(np.uint64), want["bin_off"])
    assert np.array_equal(keys[:nd].view(np.uint64), want["keys_lo"])
    assert np.array_equal(counts[:nd].view(np.uint32), want["counts"])


def test_overlapping_calls_match_the_oracle(torch):
    k, p, nb = 31, 11, 64
    batches = [synth.iid_reads(s, 700, 150, 0.002) for s in range(4)]  # same size, new reads
    batches.append(synth.iid_reads(9, 400, 150, 0.002))                 # another size
    batches.append(synth.iid_reads(10, 700, 150, 0.002))
    with G.Context(0) as ctx:
        prm = G.params(k, p, nb)
        ins = [(pinned(torch, r), pinned(torch, o)) for r, o in batches]
        cap = max(int(o[-1]) for _, o in batches)
        outs = [outputs(torch, nb, cap) for _ in batches]
        tickets = []
        for i, (r, o) in enumerate(ins):
            if i >= 2:  # at most two calls in flight
                nd, _ = ctx.stream_wait(tickets[i - 2])
                check(outs[i - 2], expect(*batches[i - 2], k, p, nb), nd)
            tickets.append(ctx.stream_submit(r, o, len(batches[i][1]) - 1, prm, *outs[i], cap))
        for i in (len(ins) - 2, len(ins) - 1):
            nd, nk = ctx.stream_wait(tickets[i])
            check(outs[i], expect(*batches[i], k, p, nb), nd)
            assert nk == int(np.maximum(np.diff(batches[i][1].astype(np.int64)) - k + 1, 0).sum())


def test_submitting_ahead_of_the_waits(torch):
    """Call i is submitted before call i - 2 is waited for (three host output
    sets), so uploads overlap downloads; every call still matches the oracle,
    and a fifth call without a wait is refused."""
    k, p, nb = 31, 11, 32
    batches = [synth.iid_reads(40 + s, 500 + 50 * s, 150, 0.002) for s in range(6)]
    with G.Context(0) as ctx:
        prm = G.params(k, p, nb)
        ins = [(pinned(torch, r), pinned(torch, o)) for r, o in batches]
        cap = max(int(o[-1]) for _, o in batches)
        outs = [outputs(torch, nb, cap) for _ in range(3)]
        tickets = []
        for i, (r, o) in enumerate(ins):
            tickets.append(ctx.stream_submit(r, o, len(batches[i][1]) - 1, prm, *outs[i % 3], cap))
            if i >= 2:
                nd, _ = ctx.stream_wait(tickets[i - 2])
                check(outs[(i - 2) % 3], expect(*batches[i - 2], k, p, nb), nd)
        # calls 4 and 5 still await their wait: two more are allowed, a third is not
        r, o = ins[0]
        fourth = outputs(torch, nb, cap)
        extra = [ctx.stream_submit(r, o, len(batches[0][1]) - 1, prm, *outs[0], cap),
                 ctx.stream_submit(r, o, len(batches[0][1]) - 1, prm, *fourth, cap)]
        with pytest.raises(G.GkcError):
            ctx.stream_submit(r, o, len(batches[0][1]) - 1, prm, *fourth, cap)
        for i in (4, 5):
            nd, _ = ctx.stream_wait(tickets[i])
            check(outs[i % 3], expect(*batches[i], k, p, nb), nd)
        for t, out in zip(extra, (outs[0], fourth)):
            nd, _ = ctx.stream_wait(t)
            check(out, expect(*batches[0], k, p, nb), nd)


def test_reads_cut_from_a_larger_csr(torch):
    k, p, nb = 25, 9, 16
    reads, offs = synth.iid_reads(21, 900, 120, 0.0)
    lo, hi = 300, 650  # reads [300, 650): offsets start at offs[300], not 0
    with G.Context(0) as ctx:
        r, o = pinned(torch, reads), pinned(torch, offs)
        cap = int(offs[hi] - offs[lo])
        out = outputs(torch, nb, cap)
        t = C.c_uint64()
        st = G.lib().gkc_stream_submit(ctx.h, C.byref(G.params(k, p, nb)), r.data_ptr(), o.data_ptr() + 8 * lo,
                                       hi - lo, out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), cap,
                                       C.byref(t))
        assert st == 0
        nd, _ = ctx.stream_wait(t.value)
        sub_offs = (offs[lo:hi + 1] - offs[lo]).astype(np.uint64)
        check(out, expect(reads[int(offs[lo]):int(offs[hi])], sub_offs, k, p, nb), nd)


def test_refusals(torch):
    k, p, nb = 31, 11, 8
    reads, offs = synth.iid_reads(31, 200, 150, 0.0)
    with G.Context(0) as ctx:
        prm = G.params(k, p, nb)
        r, o = pinned(torch, reads), pinned(torch, offs)
        small = outputs(torch, nb, 10)
        t = ctx.stream_submit(r, o, len(offs) - 1, prm, *small, 10)
        with pytest.raises(G.GkcError) as e:
            ctx.stream_wait(t)
        assert e.value.status == 6  # GKC_ERR_CAPACITY; the first 10 pairs are still copied
        # pageable output buffers are refused before any work
        pageable = np.zeros(nb + 1, np.uint64)
        out = outputs(torch, nb, 50000)
        tt = C.c_uint64()
        st = G.lib().gkc_stream_submit(ctx.h, C.byref(prm), r.data_ptr(), o.data_ptr(), len(offs) - 1,
                                       pageable.ctypes.data, out[1].data_ptr(), out[2].data_ptr(), 50000,
                                       C.byref(tt))
        assert st == 1
