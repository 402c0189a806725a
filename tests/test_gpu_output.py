"""Count output options (gkc_count_output): the per-bin frequency filter and
the merged global list, against the oracle's per-bin counts filtered and
merged in numpy."""
import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def reads_with_n(seed, n, lo, hi, n_rate):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(offs[-1]))].copy()
    b[r.random(len(b)) < n_rate] = ord("N")
    third = len(b) // 3
    # repeats (counts above 1), with N written as T in the copy: a k-mer that
    # holds an N counts as its N->T form, but its windows' minimizers differ,
    # so the two copies can land in different bins
    copy = b[:third].copy()
    copy[copy == ord("N")] = ord("T")
    b[third:2 * third] = copy
    return b, offs


def oracle_lists(reads, offs, k, p, nb):
    skm = F.oracle_partition(reads, offs, k, p, 0, nb)
    c = F.oracle_count_bins(skm, k, nb)
    keys = c["keys_lo"] if c["keys_hi"] is None else (c["keys_lo"].astype(object) |
                                                      (c["keys_hi"].astype(object) << 64))
    return c["bin_off"], keys, c["counts"]


def as_keys(keys2d):
    if keys2d.shape[1] == 1:
        return keys2d[:, 0]
    return keys2d[:, 0].astype(object) | (keys2d[:, 1].astype(object) << 64)


@pytest.mark.parametrize("k,p,nb", [(21, 7, 16), (41, 11, 8)])
def test_filter_and_merge_vs_oracle(ctx, k, p, nb):
    reads, offs = reads_with_n(7 + k, 3000, 60, 400, 0.02)
    ctx.pipeline_host(reads, offs, G.params(k, p, nb))
    bo, keys, counts = oracle_lists(reads, offs, k, p, nb)
    kw = 1 if k <= 32 else 2
    for lo, hi in [(1, 0xFFFFFFFF), (2, 0xFFFFFFFF), (1, 1), (3, 5)]:
        # per bin
        g_bo, g_keys, g_counts = ctx.count_output(lo, hi, False, kw, nb)
        keep = (counts >= lo) & (counts <= hi)
        want_bo = np.concatenate([[0], np.cumsum([keep[int(bo[b]):int(bo[b + 1])].sum() for b in range(nb)])])
        assert np.array_equal(g_bo, want_bo.astype(np.uint64))
        assert list(as_keys(g_keys)) == list(keys[keep])
        assert np.array_equal(g_counts, counts[keep])
        # merged: counts of a k-mer found in several bins added up, then filtered
        m_bo, m_keys, m_counts = ctx.count_output(lo, hi, True, kw)
        tot = {}
        for kk, cc in zip(keys, counts):
            tot[kk] = tot.get(kk, 0) + int(cc)
        mk = sorted(tot)
        mc = np.array([min(tot[x], 0xFFFFFFFF) for x in mk], np.uint64)
        sel = (mc >= lo) & (mc <= hi)
        assert list(as_keys(m_keys)) == [x for x, s in zip(mk, sel) if s]
        assert np.array_equal(m_counts.astype(np.uint64), mc[sel])
        assert m_bo[0] == 0 and m_bo[1] == len(m_counts)
    # some k-mer really is in two bins (reads hold N)
    assert len(tot) < len(keys)
