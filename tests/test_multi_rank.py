"""The multi-GPU host logic on CPU with gloo ranks: bench.py's per-rank read
ranges, slowest-rank time and whole-job rate, the reference arm on rank 0
only, and the bin-sharded exchange of gkc_b200.shard (every k-mer counted
once, by the owner of its bin)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import bench
    from gkc_b200 import synth
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wl = dict(bench.WORKLOADS["config2"], genome_len=200_000)
    first = bench.rank_first_read(wl, rank)
    g = synth.genome(2026, wl["genome_len"])
    reads, offs = synth.short_reads(2026, g, 50, wl["read_len"], wl["err"], first_read=first)
    local_ms = 100.0 + 50.0 * rank
    mx = bench.max_over_ranks(local_ms, dist, "cpu")
    rate = bench.whole_job_rate(1000, world, 2, mx)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), reads=reads, first=first, mx=mx, rate=rate)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    port = 29500 + (os.getpid() % 2000)
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0, r1 = (np.load(tmp_path / f"r{i}.npz") for i in range(2))
    assert int(r1["first"]) > int(r0["first"])  # disjoint read ranges
    assert not np.array_equal(r0["reads"], r1["reads"])
    assert float(r0["mx"]) == float(r1["mx"]) == 150.0  # the slowest rank
    assert float(r0["rate"]) == pytest.approx(1000 * 2 * 2 / 0.150)


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", LOCAL_RANK="1", RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config1",
                        "--steps", "1", "--warmup", "0", "--gpus", "2"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env.update(LOCAL_RANK="0", RANK="0")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config1",
                        "--steps", "1", "--warmup", "0", "--gpus", "2"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")


def _random_reads(seed, n, lo, hi):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(offs[-1]))].copy()
    b[r.random(len(b)) < 0.01] = ord("N")
    return b, offs


def _slice_reads(reads, offs, lo, hi):
    o = offs[lo:hi + 1]
    return reads[int(o[0]):int(o[-1])].copy(), (o - o[0]).astype(np.uint64)


SHARD_K, SHARD_P, SHARD_NB = 25, 9, 37


def _shard_rank_main(rank, world, port, out_dir):
    """One gloo rank of the bin-sharded count: its reads, the exchange of
    gkc_b200.shard over torch.distributed, the owned bins counted."""
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from shard_oracle_engine import OracleEngine
    import gkc_b200 as G
    from gkc_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    reads, offs = _random_reads(5, 240, 30, 400)
    n = len(offs) - 1
    # uneven shares: two ranks 1:4; three ranks with the middle one empty;
    # four ranks with every read on rank 2
    cuts = {2: [0, n // 5, n], 3: [0, n // 2, n // 2, n], 4: [0, 0, 0, n, n]}[world]
    r, o = _slice_reads(reads, offs, cuts[rank], cuts[rank + 1])
    nb = SHARD_NB if world < 4 else 4  # one bin per rank
    eng = OracleEngine(r, o, SHARD_K, SHARD_P, 0, nb)
    prm_local, bounds, _ = shard.exchange_dist(eng, G.params(SHARD_K, SHARD_P, nb))
    c = eng.count(prm_local.nbins)
    np.savez(os.path.join(out_dir, f"s{rank}.npz"), bounds=bounds, bin_off=c["bin_off"], keys=c["keys_lo"],
             counts=c["counts"], kmers=eng.local_kmers)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_bin_sharded_count_gloo(tmp_path, world):
    """Over gloo ranks, the owners' counts put together equal the counts of
    all reads on one rank: every k-mer counted once, by its bin's owner."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as F
    port = 31500 + (os.getpid() % 2000) + world
    mp.spawn(_shard_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    reads, offs = _random_reads(5, 240, 30, 400)
    nb = SHARD_NB if world < 4 else 4
    want = F.oracle_count_bins(F.oracle_partition(reads, offs, SHARD_K, SHARD_P, 0, nb), SHARD_K, nb)
    total_kmers = 0
    for rank in range(world):
        d = np.load(tmp_path / f"s{rank}.npz")
        lo, hi = int(d["bounds"][rank]), int(d["bounds"][rank + 1])
        for b in range(lo, hi):
            w0, w1 = int(want["bin_off"][b]), int(want["bin_off"][b + 1])
            g0, g1 = int(d["bin_off"][b - lo]), int(d["bin_off"][b - lo + 1])
            assert np.array_equal(d["keys"][g0:g1], want["keys_lo"][w0:w1])
            assert np.array_equal(d["counts"][g0:g1], want["counts"][w0:w1])
        total_kmers += int(d["kmers"].sum())
    assert total_kmers == int(want["counts"].astype(np.uint64).sum())


def test_owner_bounds():
    from gkc_b200 import shard
    assert list(shard.owner_bounds(256, 8)) == [0, 32, 64, 96, 128, 160, 192, 224, 256]
    assert list(shard.owner_bounds(37, 3)) == [0, 12, 24, 37]
    with pytest.raises(ValueError):
        shard.owner_bounds(3, 4)
