"""The multi-GPU host logic of bench.py (weak replicas, no data-path
collective) on CPU: two gloo ranks sample disjoint reads of one genome, the
job time is the slowest rank's, and the whole-job rate counts every rank's
units.  The reference arm runs on rank 0 only."""
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
