"""The serving loop: results are the same alone and in a concurrent mix,
admission respects the HBM budget, queued jobs can be cancelled, and the
per-job HBM estimate covers what a run allocates."""
import numpy as np
import pytest

import gkc_b200 as G
from gpu_helpers import assert_counts_equal

pytestmark = pytest.mark.gpu

GKC_ERR_BUDGET = 5


def iid_reads(seed, n, lo, hi):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(offs[-1]))].copy()
    b[r.random(len(b)) < 0.002] = ord("N")
    # repeat a stretch so that counts above 1 occur
    half = len(b) // 3
    b[half:2 * half] = b[:half]
    return b, offs


HOST_JOBS = [  # seed, n, lo, hi, k, p, nbins
    (1, 4000, 100, 300, 31, 11, 64),
    (2, 2500, 150, 150, 25, 11, 16),
    (3, 1500, 80, 2000, 45, 13, 32),
    (4, 6000, 150, 150, 21, 9, 256),
]
SYNTH_JOBS = [  # generator, seed, n_bases, k, p, hpc, nbins
    (G.GEN_GENOME_SHORT, 11, 3_000_000, 31, 11, False, 256),
    (G.GEN_GENOME_LONG, 12, 2_000_000, 25, 15, True, 64),
    (G.GEN_IID, 13, 1_000_000, 25, 11, False, 16),
]


def as_dict(res):
    bin_off, keys, counts = res
    return dict(bin_off=bin_off, keys_lo=keys[:, 0].copy(),
                keys_hi=keys[:, 1].copy() if keys.shape[1] > 1 else None, counts=counts)


def alone_host(ctx, seed, n, lo, hi, k, p, nb):
    reads, offs = iid_reads(seed, n, lo, hi)
    cv = ctx.pipeline_host(reads, offs, G.params(k, p, nb))
    return as_dict(ctx.count_copy_out(cv))


def run_all(srv):
    ids = []
    for seed, n, lo, hi, k, p, nb in HOST_JOBS:
        reads, offs = iid_reads(seed, n, lo, hi)
        ids.append(srv.submit(reads, offs, G.params(k, p, nb)))
    for gen, seed, nbases, k, p, hpc, nb in SYNTH_JOBS:
        ids.append(srv.submit_synth(G.params(k, p, nb, hpc), gen, seed, nbases))
    infos = [srv.wait(j) for j in ids]
    for i in infos:
        assert i.state == G.JOB_DONE, (i.state, i.status)
    res = [as_dict(srv.result(j)) for j in ids]
    for j in ids:
        srv.release(j)
    return infos, res


def test_results_same_alone_and_in_mix():
    # alone: host jobs through a plain context, every job through a one-slot server
    with G.Context(0) as ctx:
        want_host = [alone_host(ctx, *job) for job in HOST_JOBS]
    with G.Server(0, max_running=1) as one:
        infos1, alone = run_all(one)
    for a, w in zip(alone, want_host):
        assert_counts_equal(a, w)
    # one slot: jobs never overlap
    iv = sorted((i.start_s, i.end_s) for i in infos1)
    assert all(iv[t][1] <= iv[t + 1][0] + 1e-9 for t in range(len(iv) - 1))
    # the mix: four slots, all jobs submitted at once
    with G.Server(0, max_running=4) as four:
        infos4, mixed = run_all(four)
    for a, m in zip(alone, mixed):
        assert_counts_equal(m, a)
    iv = sorted((i.start_s, i.end_s) for i in infos4)
    overlaps = sum(1 for t in range(len(iv) - 1) if iv[t + 1][0] < iv[t][1])
    assert overlaps >= 1, "no two jobs ran at the same time"


def test_budget_admission_and_oversized_job():
    prm = G.params(31, 11, 64)
    reads, offs = iid_reads(21, 3000, 150, 150)
    est = G.job_hbm_estimate(prm, int(offs[-1]), len(offs) - 1)
    # room for one job at a time, however many slots are free
    with G.Server(0, hbm_budget=int(est * 1.6), max_running=4) as srv:
        ids = [srv.submit(reads, offs, prm) for _ in range(4)]
        big_r, big_o = iid_reads(22, 60000, 150, 150)
        assert G.job_hbm_estimate(prm, int(big_o[-1]), len(big_o) - 1) > est * 1.6
        big = srv.submit(big_r, big_o, prm)
        infos = [srv.wait(j) for j in ids]
        assert all(i.state == G.JOB_DONE for i in infos)
        iv = sorted((i.start_s, i.end_s) for i in infos)
        assert all(iv[t][1] <= iv[t + 1][0] + 1e-9 for t in range(len(iv) - 1))
        bi = srv.wait(big)
        assert bi.state == G.JOB_FAILED and bi.status == GKC_ERR_BUDGET
        first = srv.result(ids[0])
        for j in ids[1:]:
            r = srv.result(j)
            assert np.array_equal(r[1], first[1]) and np.array_equal(r[2], first[2])


def test_cancel_queued_job():
    prm = G.params(31, 11, 64)
    reads, offs = iid_reads(31, 20000, 150, 150)
    with G.Server(0, max_running=1) as srv:
        a = srv.submit(reads, offs, prm)
        b = srv.submit(reads, offs, prm)
        srv.cancel(b)
        assert srv.wait(b).state == G.JOB_CANCELLED
        assert srv.wait(a).state == G.JOB_DONE
        srv.release(b)
        with pytest.raises(G.GkcError):
            srv.poll(b)


@pytest.mark.parametrize("k,p,hpc", [(31, 11, False), (63, 13, False), (25, 15, True)])
def test_estimate_covers_a_run(k, p, hpc):
    reads, offs = iid_reads(41, 20000, 100, 400)
    prm = G.params(k, p, 256, hpc)
    with G.Context(0) as ctx:
        ctx.pipeline_host(reads, offs, prm)
        used = ctx.device_bytes()
    assert used <= G.job_hbm_estimate(prm, int(offs[-1]), len(offs) - 1)
