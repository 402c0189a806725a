"""The oracle (CPU restatement) against the reference's golden fixtures and,
where it was built here, against the reference compiled from its sources."""
import numpy as np
import pytest

import golden_cases as G
import oracle_ffi as F
import parity as P

FULL = sorted(G.index()["full"].keys())
DIGEST = sorted(G.index()["digest"].keys())


@pytest.mark.parametrize("name", FULL)
def test_oracle_matches_golden_full(name):
    meta, d = G.full_case(name)
    k, p, hpc, nb = meta["k"], meta["p"], meta["hpc"], meta["nbins"]
    skm = F.oracle_partition(d["reads"], d["offs"], k, p, hpc, nb)
    ms = skm.multisets(nb)
    assert ms == G.multisets_from_case(d, nb)
    assert P.partition_digest(ms) == meta["partition_sha256"]
    cnt = F.oracle_count_bins(skm, k, nb)
    assert np.array_equal(cnt["bin_off"], d["cnt_bin_off"])
    assert np.array_equal(cnt["keys_lo"], d["cnt_keys"])
    assert np.array_equal(cnt["counts"], d["cnt_counts"])
    # kmc_counting_GPU returns the number of distinct k-mers of its bin
    assert np.array_equal(np.diff(cnt["bin_off"]), d["cnt_returned"])


@pytest.mark.parametrize("name", DIGEST)
def test_oracle_matches_golden_digest(name):
    c = G.index()["digest"][name]
    reads, offs = G.digest_case_reads(c)
    assert P.bytes_digest(reads) == c["reads_sha256"]
    assert P.bytes_digest(offs) == c["offs_sha256"]
    skm = F.oracle_partition(reads, offs, c["k"], c["p"], c["hpc"], c["nbins"])
    ms = skm.multisets(c["nbins"])
    assert len(skm.bin) == c["n_skm"]
    assert P.partition_digest(ms) == c["partition_sha256"]
    cnt = F.oracle_count_bins(skm, c["k"], c["nbins"])
    assert int(cnt["counts"].astype(np.uint64).sum()) == c["n_kmers"]
    assert P.counts_digest(cnt["bin_off"], cnt["keys_lo"], cnt["counts"]) == c["counts_sha256"]


def _random_reads(seed, n, lo, hi, n_rate=0.01):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(b"ACGTacgtU", np.uint8)[r.integers(0, 9, int(offs[-1]))].copy()
    b[r.random(len(b)) < n_rate] = ord("N")
    return b, offs


@pytest.mark.skipif(not F.ref_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed,k,p,hpc,nb", [(1, 31, 11, 0, 256), (2, 21, 7, 1, 31),
                                              (3, 17, 9, 0, 5), (4, 27, 13, 1, 100),
                                              (5, 32, 16, 0, 64), (6, 12, 4, 0, 3)])
def test_oracle_matches_reference_random(seed, k, p, hpc, nb):
    reads, offs = _random_reads(seed, 150, k, 700)
    o = F.oracle_partition(reads, offs, k, p, hpc, nb)
    r = F.ref_partition(reads, offs, k, p, hpc, nb, batch_reads=37)
    assert o.multisets(nb) == r.multisets(nb)
    co = F.oracle_count_bins(o, k, nb)
    cr = F.ref_count_bins(r, k, nb)
    for key in ("bin_off", "keys_lo", "counts"):
        assert np.array_equal(co[key], cr[key])


def test_oracle_minimizer_clean_window_is_min_over_passing_pmers():
    """Without N the reference update rule reduces to the minimum over the
    window's passing forward / reverse-complement p-mers, else 4^p-1."""
    r = np.random.default_rng(9)
    k, p = 31, 11
    read = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, 400)].copy()
    mm = F.oracle_minimizers(read, k, p)
    code = {65: 0, 67: 1, 71: 2, 84: 3}
    c = np.array([code[x] for x in read])
    M = (1 << (2 * p)) - 1

    def passes(v):
        t = v >> (2 * (p - 3))
        return t not in (0, 4, 8)

    for s in range(len(read) - k + 1):
        best = M
        for j in range(s, s + k - p + 1):
            f = 0
            rc = 0
            for t in range(p):
                f = (f << 2) | int(c[j + t])
                rc = (rc << 2) | (3 - int(c[j + p - 1 - t]))
            if passes(f):
                best = min(best, f)
            if passes(rc):
                best = min(best, rc)
        assert mm[s] == best


def test_oracle_minimizer_position_definition():
    r = np.random.default_rng(10)
    k, p = 25, 15
    read = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, 300)].copy()
    mm, pos, st = F.oracle_minimizers(read, k, p, with_pos=True)
    for s in range(len(mm)):
        j = int(pos[s])
        assert j <= k - p
        seg = read[s + j:s + j + p].tobytes()
        comp = seg.translate(bytes.maketrans(b"ACGT", b"TGCA"))[::-1]
        enc = lambda x: int(x.translate(bytes.maketrans(b"ACGT", b"0123")), 4)
        assert (enc(seg) if st[s] == 0 else enc(comp)) == mm[s]


def test_oracle_hpc_runs():
    reads = np.frombuffer(b"AAACCGTTTTNNA" + b"G" + b"", np.uint8).copy()
    offs = np.array([0, 13, 14], np.uint64)
    out, ln, orig = F.oracle_hpc(reads, offs)
    assert list(ln) == [6, 1]
    assert out[:6].tobytes() == b"ACGTNA"
    assert list(orig[:6]) == [0, 3, 5, 6, 10, 12]


def test_oracle_short_reads_produce_nothing():
    reads = np.frombuffer(b"ACGTACGTAC" * 3, np.uint8).copy()
    offs = np.array([0, 5, 30], np.uint64)
    s = F.oracle_partition(reads, offs, 31, 11, 0, 16)
    assert len(s.bin) == 0


@pytest.mark.parametrize("filter_id", [1, 2, 3])
def test_oracle_filters_match_reference(filter_id):
    """Every FILTER_KERNEL variant of the reference, built from its sources,
    against the restatement with the same filter."""
    if not F.ref_available(filter_id):
        pytest.skip("reference tree absent: the per-filter builds were not made")
    reads, offs = _random_reads(40 + filter_id, 300, 31, 600)  # reads of at least k bases
    try:
        F.set_filter(filter_id)
        for k, p, hpc in [(31, 11, 0), (21, 9, 1)]:
            o = F.oracle_partition(reads, offs, k, p, hpc, 16)
            r = F.ref_partition(reads, offs, k, p, hpc, 16, batch_reads=41, filter_id=filter_id)
            assert o.multisets(16) == r.multisets(16)
            F.set_filter(0)
            assert o.multisets(16) != F.oracle_partition(reads, offs, k, p, hpc, 16).multisets(16)
            F.set_filter(filter_id)
    finally:
        F.set_filter(0)


@pytest.mark.skipif(not F.ref_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed,k,p,hpc,nb", [(50, 31, 11, 0, 256), (51, 21, 9, 1, 31), (52, 17, 7, 0, 5)])
def test_oracle_partition_sizes_match_reference(seed, k, p, hpc, nb):
    """Bases per bin as CalcSKMPartSize_instream adds them up, against the
    restatement's partition."""
    reads, offs = _random_reads(seed, 200, k, 700)
    want = F.ref_partition_sizes(reads, offs, k, p, hpc, nb, batch_reads=53)
    got = F.oracle_partition_sizes(F.oracle_partition(reads, offs, k, p, hpc, nb), nb)
    assert np.array_equal(got, want)


@pytest.mark.skipif(not F.ref_available(), reason="reference harness not built here")
def test_oracle_balance_report_matches_reference():
    """The avg / max / min / var / std / cv report of calVarStdev, as the text
    it logs, for size vectors below the reference's int-total limit."""
    r = np.random.default_rng(11)
    cases = [np.array([10, 20, 30, 45], np.uint64), np.full(64, 1000, np.uint64),
             np.array([7], np.uint64), r.integers(0, 100000, 256).astype(np.uint64),
             r.integers(1, 1 << 22, 500).astype(np.uint64)]
    for sizes in cases:
        assert int(sizes.sum()) < 2 ** 31
        assert F.balance_report(F.oracle_balance(sizes)) == F.ref_balance_report(sizes)


def test_oracle_partition_sizes_from_golden():
    """Per-bin bases of the fixtures' partitions equal the superkmer lengths
    each bin holds plus nothing else (the fixtures pin the partition)."""
    for name in FULL:
        meta, d = G.full_case(name)
        nb = meta["nbins"]
        skm = F.oracle_partition(d["reads"], d["offs"], meta["k"], meta["p"], meta["hpc"], nb)
        sizes = F.oracle_partition_sizes(skm, nb)
        want = np.zeros(nb, np.uint64)
        np.add.at(want, d["skm_bin"].astype(np.int64), d["skm_len"].astype(np.uint64))
        assert np.array_equal(sizes, want)


@pytest.mark.skipif(not F.ref_available(), reason="reference harness not built here")
def test_oracle_matches_reference_parameter_sweep():
    """Random (k, p, nbins, hpc, filter) combinations, each on its own random
    read set (reads of at least k bases, N and lower case included):
    partition multisets and per-bin counts equal the reference's."""
    r = np.random.default_rng(2024)
    try:
        for case in range(24):
            k = int(r.integers(5, 33))
            p = int(r.integers(3, min(16, k) + 1))
            nb = int(r.integers(1, 300))
            hpc = int(r.integers(0, 2))
            filt = int(r.integers(0, 4))
            if filt and not F.ref_available(filt):
                filt = 0
            reads, offs = _random_reads(1000 + case, 60, k, 400)
            F.set_filter(filt)
            o = F.oracle_partition(reads, offs, k, p, hpc, nb)
            ref = F.ref_partition(reads, offs, k, p, hpc, nb, batch_reads=17, filter_id=filt)
            assert o.multisets(nb) == ref.multisets(nb), (k, p, nb, hpc, filt)
            co, cr = F.oracle_count_bins(o, k, nb), F.ref_count_bins(ref, k, nb)
            for key in ("bin_off", "keys_lo", "counts"):
                assert np.array_equal(co[key], cr[key]), (k, p, nb, hpc, filt, key)
    finally:
        F.set_filter(0)
