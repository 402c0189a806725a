"""Parity of the CUDA path (through the C ABI) with the reference's golden
fixtures and with the oracle.  Partition: identical per-bin multisets of
(length, packed bytes).  Count: identical per-bin sorted (k-mer, count)."""
import numpy as np
import pytest

import gkc_b200 as G
import golden_cases as GC
import oracle_ffi as F
import parity as P
from gpu_helpers import assert_counts_equal, lib_counts, lib_partition

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(GC.index()["full"].keys()))
def test_golden_full(ctx, name):
    meta, d = GC.full_case(name)
    k, p, hpc, nb = meta["k"], meta["p"], meta["hpc"], meta["nbins"]
    skm, _ = lib_partition(ctx, d["reads"], d["offs"], k, p, hpc, nb)
    assert skm.multisets(nb) == GC.multisets_from_case(d, nb)
    got, _ = lib_counts(ctx, k, nb)
    want = dict(bin_off=d["cnt_bin_off"], keys_lo=d["cnt_keys"], counts=d["cnt_counts"])
    assert_counts_equal(got, want)


@pytest.mark.parametrize("name", sorted(GC.index()["digest"].keys()))
def test_golden_digest(ctx, name):
    c = GC.index()["digest"][name]
    reads, offs = GC.digest_case_reads(c)
    skm, v = lib_partition(ctx, reads, offs, c["k"], c["p"], c["hpc"], c["nbins"])
    assert v.n_superkmers == c["n_skm"]
    assert P.partition_digest(skm.multisets(c["nbins"])) == c["partition_sha256"]
    got, cv = lib_counts(ctx, c["k"], c["nbins"])
    assert cv.n_kmers == c["n_kmers"]
    assert P.counts_digest(got["bin_off"], got["keys_lo"], got["counts"]) == c["counts_sha256"]


def random_reads(seed, n, lo, hi, alphabet=b"ACGTacgtU", n_rate=0.01):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(alphabet, np.uint8)[r.integers(0, len(alphabet), int(offs[-1]))].copy()
    b[r.random(len(b)) < n_rate] = ord("N")
    return b, offs


CASES = [
    # seed, n, lo, hi, k, p, hpc, nbins
    (1, 400, 31, 900, 31, 11, 0, 256),
    (2, 300, 21, 700, 21, 7, 1, 31),
    (3, 200, 17, 5000, 17, 9, 0, 5),
    (4, 100, 40, 3000, 27, 13, 1, 100),
    (5, 300, 32, 400, 32, 16, 0, 64),
    (6, 500, 12, 100, 12, 4, 0, 3),
    (7, 200, 45, 500, 45, 15, 0, 128),    # 128-bit keys
    (8, 120, 63, 900, 63, 13, 0, 256),    # config-4 shape
    (9, 80, 64, 400, 64, 16, 1, 7),
]


@pytest.mark.parametrize("seed,n,lo,hi,k,p,hpc,nb", CASES)
def test_random_vs_oracle(ctx, seed, n, lo, hi, k, p, hpc, nb):
    reads, offs = random_reads(seed, n, lo, hi)
    o = F.oracle_partition(reads, offs, k, p, hpc, nb)
    skm, _ = lib_partition(ctx, reads, offs, k, p, hpc, nb)
    assert skm.multisets(nb) == o.multisets(nb)
    want = F.oracle_count_bins(o, k, nb)
    got, _ = lib_counts(ctx, k, nb)
    assert_counts_equal(got, want)


def test_short_and_empty_reads(ctx):
    reads = np.frombuffer(b"ACGTACGTAC" * 10, np.uint8).copy()
    offs = np.array([0, 0, 5, 5, 36, 37, 100], np.uint64)
    k, p, nb = 31, 11, 16
    o = F.oracle_partition(reads, offs, k, p, 0, nb)
    skm, _ = lib_partition(ctx, reads, offs, k, p, 0, nb)
    assert skm.multisets(nb) == o.multisets(nb)
    got, _ = lib_counts(ctx, k, nb)
    assert_counts_equal(got, F.oracle_count_bins(o, k, nb))


def test_empty_input(ctx):
    reads = np.zeros(0, np.uint8)
    offs = np.zeros(1, np.uint64)
    skm, v = lib_partition(ctx, reads, offs, 31, 11, 0, 8)
    assert v.n_superkmers == 0
    got, cv = lib_counts(ctx, 31, 8)
    assert cv.n_distinct == 0 and np.all(got["bin_off"] == 0)


def test_homopolymer_reads_oversize_bucket(ctx):
    """All-A reads: one superkmer per read, every k-mer equal -> one bucket far
    larger than shared memory (global MSD path, all-equal leaf)."""
    reads = np.frombuffer(b"A" * 20000 + b"C" * 3000 + b"A" * 9000, np.uint8).copy()
    offs = np.array([0, 20000, 23000, 32000], np.uint64)
    k, p, nb = 31, 11, 4
    o = F.oracle_partition(reads, offs, k, p, 0, nb)
    skm, _ = lib_partition(ctx, reads, offs, k, p, 0, nb)
    assert skm.multisets(nb) == o.multisets(nb)
    got, _ = lib_counts(ctx, k, nb)
    assert_counts_equal(got, F.oracle_count_bins(o, k, nb))


def test_low_complexity_oversize_mixed(ctx):
    """Mostly-A reads with sparse other bases: many distinct keys share long
    prefixes, so buckets overflow shared memory and split recursively."""
    r = np.random.default_rng(21)
    n, L = 60, 5000
    b = np.full(n * L, ord("A"), np.uint8)
    m = r.random(n * L) < 0.02
    b[m] = np.frombuffer(b"CGT", np.uint8)[r.integers(0, 3, int(m.sum()))]
    offs = np.arange(0, n * L + 1, L, dtype=np.uint64)
    k, p, nb = 31, 11, 2
    o = F.oracle_partition(b, offs, k, p, 0, nb)
    skm, _ = lib_partition(ctx, b, offs, k, p, 0, nb)
    assert skm.multisets(nb) == o.multisets(nb)
    got, _ = lib_counts(ctx, k, nb)
    assert_counts_equal(got, F.oracle_count_bins(o, k, nb))


def test_long_superkmer_beyond_tile_halo(ctx):
    """A superkmer spanning far more windows than one tile plus halo."""
    unit = b"A" * 9000
    rng = np.random.default_rng(3)
    tail = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 3000)].tobytes()
    reads = np.frombuffer(tail + unit + tail, np.uint8).copy()
    offs = np.array([0, len(reads)], np.uint64)
    k, p, nb = 25, 15, 64
    o = F.oracle_partition(reads, offs, k, p, 0, nb)
    skm, _ = lib_partition(ctx, reads, offs, k, p, 0, nb)
    assert skm.multisets(nb) == o.multisets(nb)


def test_pipeline_batched_matches_two_step(ctx):
    import torch
    reads, offs = random_reads(31, 3000, 150, 150, alphabet=b"ACGT", n_rate=0.001)
    k, p, nb = 31, 11, 256
    o = F.oracle_partition(reads, offs, k, p, 0, nb)
    want = F.oracle_count_bins(o, k, nb)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    for _ in range(3):  # first call captures the graph, later calls replay it
        pv, cv = ctx.pipeline_device(d_reads, len(reads), d_offs, len(offs) - 1, G.params(k, p, nb))
        bin_off, keys, counts = ctx.count_copy_out(cv)
        assert_counts_equal(dict(bin_off=bin_off, keys_lo=keys[:, 0], counts=counts), want)
    assert ctx.timings().graph_replayed == 1


def test_count_superkmers_host_one_bin(ctx):
    """kmc_counting_GPU drop-in: one bin's packed superkmers from the host."""
    meta, d = GC.full_case("iid_n")
    nb, k = meta["nbins"], meta["k"]
    for b in (0, 17, 255):
        sel = d["skm_bin"] == b
        lens = d["skm_len"][sel]
        chunks = [d["skm_bytes"][int(o):int(o) + (int(l) + 3) // 4] for o, l in zip(d["skm_off"][sel], lens)]
        packed = np.concatenate(chunks) if chunks else np.zeros(0, np.uint8)
        nd = ctx.count_superkmers_host(k, lens, packed)
        lo, hi = int(d["cnt_bin_off"][b]), int(d["cnt_bin_off"][b + 1])
        assert nd == hi - lo == int(d["cnt_returned"][b])
        _, keys, counts = ctx.count_copy_out(ctx.count_device(G.params(k, 3, 1)))
        assert np.array_equal(keys[:, 0], d["cnt_keys"][lo:hi])
        assert np.array_equal(counts, d["cnt_counts"][lo:hi])


@pytest.mark.parametrize("mode", [G.MODE_BATCHED, G.MODE_PLAIN])
def test_count_superkmers_host_fresh_context(mode):
    """A context that has never partitioned counts a superkmer group (with
    superkmers shorter than k among them) exactly as the oracle does."""
    r = np.random.default_rng(40 + mode)
    k, pool, n = 27, 300, 9000
    base_lens = r.integers(10, 110, pool).astype(np.uint32)
    base = [r.integers(0, 256, int((ln + 3) // 4), dtype=np.uint8) for ln in base_lens]
    pick = r.integers(0, pool, n)
    lens = base_lens[pick]
    packed = np.concatenate([base[i] for i in pick])
    boff = np.zeros(n, np.uint64)
    boff[1:] = np.cumsum((lens[:-1].astype(np.uint64) + 3) // 4)
    want = F.oracle_count_bins(F.Skms(np.zeros(n, np.uint32), lens, boff, packed), k, 1)
    with G.Context(0) as fresh:
        nd = fresh.count_superkmers_host(k, lens, packed, mode)
        assert nd == len(want["keys_lo"])
        _, keys, counts = fresh.count_copy_out(fresh.count_device(G.params(k, 3, 1), mode))
    assert np.array_equal(keys[:, 0], want["keys_lo"])
    assert np.array_equal(counts, want["counts"])


PLAIN_CASES = [
    (11, 300, 31, 900, 31, 11, 0, 256),
    (12, 200, 21, 700, 21, 7, 1, 31),
    (13, 100, 63, 600, 63, 13, 0, 64),
]


@pytest.mark.parametrize("seed,n,lo,hi,k,p,hpc,nb", PLAIN_CASES)
def test_plain_mode_vs_oracle(ctx, seed, n, lo, hi, k, p, hpc, nb):
    """The plain per-stage form (per-window minimizers, per-read superkmers,
    per-bin onesweep sort) gives the same partition and counts."""
    import torch
    reads, offs = random_reads(seed, n, lo, hi)
    o = F.oracle_partition(reads, offs, k, p, hpc, nb)
    want = F.oracle_count_bins(o, k, nb)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    pv, cv = ctx.pipeline_device(d_reads, len(reads), d_offs, len(offs) - 1, G.params(k, p, nb, hpc),
                                 mode=G.MODE_PLAIN)
    bo, lens, boff, packed, _ = ctx.partition_copy_out(pv)
    bins = np.repeat(np.arange(nb, dtype=np.uint32), np.diff(bo).astype(np.int64))
    assert F.Skms(bins, lens, boff, packed).multisets(nb) == o.multisets(nb)
    bin_off, keys, counts = ctx.count_copy_out(cv)
    got = dict(bin_off=bin_off, keys_lo=keys[:, 0].copy(), counts=counts,
               keys_hi=keys[:, 1].copy() if keys.shape[1] > 1 else None)
    assert_counts_equal(got, want)


def test_plain_count_after_fused_partition(ctx):
    meta, d = GC.full_case("mixed_defaults")
    k, p, hpc, nb = meta["k"], meta["p"], meta["hpc"], meta["nbins"]
    lib_partition(ctx, d["reads"], d["offs"], k, p, hpc, nb)
    got, _ = lib_counts(ctx, k, nb, mode=G.MODE_PLAIN)
    assert_counts_equal(got, dict(bin_off=d["cnt_bin_off"], keys_lo=d["cnt_keys"], counts=d["cnt_counts"]))


@pytest.mark.parametrize("seed,n,lo,hi,k,p,hpc,nb", [CASES[0], CASES[2], CASES[7]])
def test_sort_fallback_forced(ctx, seed, n, lo, hi, k, p, hpc, nb, monkeypatch):
    """With a probe limit of 0 every slice that has a collision falls back to
    the shared-memory / global-scratch sort (serialised through the scratch
    lock); results must not change."""
    monkeypatch.setenv("GKC_PROBE_LIMIT", "0")
    reads, offs = random_reads(seed, n, lo, hi)
    o = F.oracle_partition(reads, offs, k, p, hpc, nb)
    lib_partition(ctx, reads, offs, k, p, hpc, nb)
    got, _ = lib_counts(ctx, k, nb)
    assert_counts_equal(got, F.oracle_count_bins(o, k, nb))


@pytest.mark.parametrize("filter_id", [G.FILTER_ALL, G.FILTER_NEW, G.FILTER_SIGNATURE, G.FILTER_NEW2])
def test_minimizer_filters_vs_oracle(filter_id):
    """Each minimizer filter the reference can be built with (FILTER_KERNEL),
    chosen at run time: batched and plain partitions, counts and per-window
    minimizers against the oracle with the same filter."""
    import torch
    reads, offs = random_reads(60 + filter_id, 300, 40, 800)
    k, p, hpc, nb = 31, 11, 0, 64
    try:
        F.set_filter(filter_id)
        o = F.oracle_partition(reads, offs, k, p, hpc, nb)
        want = F.oracle_count_bins(o, k, nb)
        with G.Context(0) as c:
            c.set_filter(filter_id)
            skm, _ = lib_partition(c, reads, offs, k, p, hpc, nb)
            assert skm.multisets(nb) == o.multisets(nb)
            got, _ = lib_counts(c, k, nb)
            assert_counts_equal(got, want)
            d_reads = torch.from_numpy(reads).cuda()
            d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
            pv, cv = c.pipeline_device(d_reads, len(reads), d_offs, len(offs) - 1, G.params(k, p, nb, hpc),
                                       mode=G.MODE_PLAIN)
            bin_off, keys, counts = c.count_copy_out(cv)
            assert np.array_equal(keys[:, 0], want["keys_lo"]) and np.array_equal(counts, want["counts"])
            nbt = len(reads)
            d_mm = torch.zeros(nbt, dtype=torch.int32, device="cuda")
            c.minimizers_device(d_reads.data_ptr(), nbt, d_offs.data_ptr(), len(offs) - 1, G.params(k, p, 1),
                                d_mm.data_ptr(), None, None)
            mm = d_mm.cpu().numpy().view(np.uint32)
            for i in range(0, len(offs) - 1, 7):
                b, e = int(offs[i]), int(offs[i + 1])
                want_mm = F.oracle_minimizers(reads[b:e], k, p)
                assert np.array_equal(mm[b:b + len(want_mm)], want_mm)
    finally:
        F.set_filter(G.FILTER_NEW2)


@pytest.mark.parametrize("name", sorted(GC.index()["full"].keys()))
def test_partition_balance_golden(ctx, name):
    """Per-bin superkmer bases (CalcSKMPartSize_instream) and the calVarStdev
    summary of the context's partition: the bases against the fixture's
    superkmers, the summary against the oracle's, bit for bit."""
    meta, d = GC.full_case(name)
    k, p, hpc, nb = meta["k"], meta["p"], meta["hpc"], meta["nbins"]
    _, v = lib_partition(ctx, d["reads"], d["offs"], k, p, hpc, nb)
    sizes, st = ctx.partition_balance(v)
    want = np.zeros(nb, np.uint64)
    np.add.at(want, d["skm_bin"].astype(np.int64), d["skm_len"].astype(np.uint64))
    assert np.array_equal(sizes, want)
    assert st == F.oracle_balance(want)


@pytest.mark.parametrize("mode", [G.MODE_BATCHED, G.MODE_PLAIN])
def test_partition_balance_pipeline(ctx, mode):
    """After the whole pipeline in either mode, with HPC, the balance figures
    come from that run's partition."""
    import torch
    reads, offs = random_reads(70 + mode, 400, 30, 900)
    k, p, hpc, nb = 25, 9, 1, 37
    o = F.oracle_partition(reads, offs, k, p, hpc, nb)
    want = F.oracle_partition_sizes(o, nb)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    pv, _ = ctx.pipeline_device(d_reads, len(reads), d_offs, len(offs) - 1, G.params(k, p, nb, hpc), mode=mode)
    sizes, st = ctx.partition_balance(pv)
    assert np.array_equal(sizes, want)
    assert st == F.oracle_balance(want)


def test_random_parameter_sweep_vs_oracle(ctx):
    """Random (k, p, nbins, hpc, filter) combinations, k up to 64 and up to
    3000 bins (beyond the shared-memory bin placement): batched partition
    and counts, and plain-mode counts, against the oracle."""
    import torch
    r = np.random.default_rng(77)
    try:
        for case in range(16):
            k = int(r.integers(5, 65))
            p = int(r.integers(3, min(16, k) + 1))
            nb = int(r.choice([int(r.integers(1, 300)), int(r.integers(2049, 3001))]))
            hpc = int(r.integers(0, 2))
            filt = int(r.integers(0, 4))
            reads, offs = random_reads(500 + case, 150, k, 600)
            F.set_filter(filt)
            ctx.set_filter(filt)
            o = F.oracle_partition(reads, offs, k, p, hpc, nb)
            want = F.oracle_count_bins(o, k, nb)
            skm, _ = lib_partition(ctx, reads, offs, k, p, hpc, nb)
            assert skm.multisets(nb) == o.multisets(nb), (k, p, nb, hpc, filt)
            got, _ = lib_counts(ctx, k, nb)
            assert_counts_equal(got, want)
            d_reads = torch.from_numpy(reads).cuda()
            d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
            _, cv = ctx.pipeline_device(d_reads, len(reads), d_offs, len(offs) - 1, G.params(k, p, nb, hpc),
                                        mode=G.MODE_PLAIN)
            bin_off, keys, counts = ctx.count_copy_out(cv)
            got = dict(bin_off=bin_off, keys_lo=keys[:, 0].copy(), counts=counts,
                       keys_hi=keys[:, 1].copy() if keys.shape[1] > 1 else None)
            assert_counts_equal(got, want)
    finally:
        F.set_filter(0)
        ctx.set_filter(0)
