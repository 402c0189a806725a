"""Benchmark: canonical k-mers counted per second on one B200 (or N, weak).

Default workload: a 100 Mbp synthetic genome with 5%
of its length as 1-5 kbp segment copies (1% divergence), sampled as 150 bp
reads on both strands to 30x coverage (20 M reads, 3.0 G bases) with 0.5%
substitution errors; k=31, p=11, 256 bins.  Reads are generated on the device
from a seed.  One step = the batched, graph-captured pipeline
(partition -> expand -> sort -> count) over all reads, inputs resident in HBM.

With --gpus N > 1 (one process per GPU under torchrun) every rank generates
its own reads of the same genome (weak scaling); by default the bins are
sharded: each rank partitions its reads, the superkmers go to the owner of
their bin over NCCL (gkc_b200.shard), and each rank counts the bins it owns,
so every k-mer of the job is counted once.  --multi replicas runs N
independent single-GPU pipelines instead.

Printed: one JSON line (rank 0).  `--impl reference` times the reference's own
CPU implementation (oracle/_ref, compiled from the reference sources) on a
bounded sample of the same workload instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

WORKLOADS = {
    # name: generator, sizes, k, p, nbins
    "ns": dict(gen="genome", genome_len=100_000_000, coverage=30, read_len=150, err=0.005,
               k=31, p=11, nbins=256, hpc=0),
    "config2": dict(gen="genome", genome_len=10_000_000, coverage=30, read_len=150, err=0.005,
                    k=31, p=11, nbins=256, hpc=0),
    "config1": dict(gen="iid", n_reads=20000, read_len=150, n_rate=0.001, k=31, p=11, nbins=256,
                    hpc=0),
    "config4": dict(gen="genome", genome_len=100_000_000, coverage=30, read_len=250, err=0.005,
                    k=63, p=13, nbins=256, hpc=0),
    # a small case of the config-2 generator for profiler captures: 30x of a 3 Mbp genome (90 M bases,
    # 72 M k-mers), the same copies per k-mer as the 30x workloads
    "small": dict(gen="genome", genome_len=3_000_000, coverage=30, read_len=150, err=0.005,
                  k=31, p=11, nbins=256, hpc=0),
    # long reads: lognormal lengths (median 8 kbp, sigma 0.5, clipped to 1-50 kbp), 20x
    "config3": dict(gen="long", genome_len=100_000_000, coverage=20, median=8000.0, sigma=0.5,
                    min_len=1000, max_len=50000, k=25, p=15, nbins=256, hpc=1),
}
METRIC = "canonical k-mers counted/s"
SEED = 2026
_T0 = time.perf_counter()


def progress(what):
    """One line per bench leg on stderr (the JSON line stays alone on stdout)."""
    sys.stderr.write(f"[bench {time.perf_counter() - _T0:7.1f} s] {what}\n")
    sys.stderr.flush()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ns", choices=sorted(WORKLOADS))
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-reads", type=int, default=200_000)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--serve", action="store_true",
                    help="only the serving mix (config 5): 1000 jobs at 50/80/95%% load")
    ap.add_argument("--serve-jobs", type=int, default=None)
    ap.add_argument("--serve-loads", default="0.5,0.8,0.95",
                    help="loads of the serving mix, as fractions of the measured capacity")
    ap.add_argument("--serve-timeout", type=float, default=240.0,
                    help="seconds the default run gives its serving mix (a child process) before ending it")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default count-stage shapes instead of tuning them on a sample first")
    ap.add_argument("--multi", default=None, choices=["shard", "replicas"],
                    help="bins sharded by owner with a superkmer exchange (default when N > 1; "
                         "also runs with one rank when given), or independent replicas")
    return ap.parse_args()


# ----------------------------------------------------------------- helpers

def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(value, dist, device):
    """The largest value over all ranks (the job's time is its slowest rank)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_first_read(wl, rank):
    """Weak scaling: rank r samples reads [r * n, (r + 1) * n) of the same genome."""
    return rank * (wl["coverage"] * wl["genome_len"] // wl["read_len"])


def whole_job_rate(units_per_rank, world, steps, max_ms):
    """Units all ranks processed in the timed steps over the slowest rank's time."""
    return units_per_rank * world * steps / (max_ms / 1000.0)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(B, R, S, N, D, k):
    """Fixed byte model per stage (bytes that each stage must move at least
    once in the reference's dataflow): B bases, R reads, S superkmers,
    L superkmer bases, N k-mers, D distinct (k-mer, bin) pairs, w key bytes,
    P 8-bit LSD passes."""
    w = 8 if k <= 32 else 16
    P = math.ceil(2 * k / 8)
    L = N + S * (k - 1)
    part = B + 8 * (R + 1) + L / 4 + 8 * S
    expand = L / 4 + 8 * S + w * N
    sort = w * N + P * 2 * w * N
    count = w * N + (w + 4) * D
    return dict(partition=part, expand=expand, sort=sort, count=count,
                total=part + expand + sort + count, w=w, P=P, L=L)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------- workload (GPU)

def make_workload_device(wl, seed, rank, torch, G):
    """Reads (uint8) and offsets (int64 view of uint64) on the current device."""
    L = G.lib()
    dev = torch.cuda.current_device()
    if wl["gen"] == "iid":
        n = wl["n_reads"]
        reads = torch.empty(n * wl["read_len"] + 64, dtype=torch.uint8, device=dev)
        offs = torch.empty(n + 1, dtype=torch.int64, device=dev)
        st = L.gkc_synth_iid_reads(1, seed + rank, n, wl["read_len"], wl["n_rate"], reads.data_ptr(),
                                   offs.data_ptr())
        assert st == 0
        return reads, offs, n, n * wl["read_len"], None
    Gl = wl["genome_len"]
    genome = torch.empty(Gl, dtype=torch.uint8, device=dev)
    assert L.gkc_synth_genome(1, seed, Gl, 0.05, 0.01, genome.data_ptr()) == 0
    if wl["gen"] == "long":
        offs_h = long_read_offsets(wl, seed + rank, G)
        n = len(offs_h) - 1
        nb = int(offs_h[-1])
        reads = torch.empty(nb + 64, dtype=torch.uint8, device=dev)
        offs = torch.from_numpy(offs_h.view(np.int64)).to(dev)
        assert L.gkc_synth_long_reads(1, seed + rank, genome.data_ptr(), Gl, n, offs.data_ptr(),
                                      reads.data_ptr()) == 0
        return reads, offs, n, nb, genome
    n = wl["coverage"] * Gl // wl["read_len"]
    reads = torch.empty(n * wl["read_len"] + 64, dtype=torch.uint8, device=dev)
    offs = torch.empty(n + 1, dtype=torch.int64, device=dev)
    # each rank samples its own reads of the same genome (weak scaling)
    assert L.gkc_synth_short_reads(1, seed, genome.data_ptr(), Gl, rank_first_read(wl, rank), n, wl["read_len"],
                                   wl["err"], reads.data_ptr(), offs.data_ptr()) == 0
    return reads, offs, n, n * wl["read_len"], genome


def long_read_offsets(wl, seed, G, total=None):
    total = total or wl["genome_len"] * wl["coverage"]
    maxr = total // wl["min_len"] + 2
    offs = np.zeros(maxr + 1, np.uint64)
    n = G.lib().gkc_synth_long_read_offsets(seed, wl["median"], wl["sigma"], wl["min_len"], wl["max_len"],
                                            total, maxr, offs.ctypes.data)
    return offs[:n + 1].copy()


def host_sample(wl, seed, n_reads, genome_host=None):
    """The first n_reads reads of the workload, generated on the host."""
    from gkc_b200 import synth
    if wl["gen"] == "long":
        import gkc_b200 as G
        g = genome_host if genome_host is not None else synth.genome(seed, wl["genome_len"])
        g = np.ascontiguousarray(g, np.uint8)
        offs = long_read_offsets(wl, seed, G)[:n_reads + 1]
        out = np.zeros(int(offs[-1]) + 64, np.uint8)
        assert G.lib().gkc_synth_long_reads(0, seed, g.ctypes.data, len(g), len(offs) - 1,
                                            offs.ctypes.data, out.ctypes.data) == 0
        return out[:int(offs[-1])], offs
    if wl["gen"] == "iid":
        return synth.iid_reads(seed, min(n_reads, wl["n_reads"]), wl["read_len"], wl["n_rate"])
    g = genome_host if genome_host is not None else synth.genome(seed, wl["genome_len"])
    return synth.short_reads(seed, g, n_reads, wl["read_len"], wl["err"])


def cpu_reference_rate(reads, offs, wl, threads):
    """The reference's CPU path (partition kernels + SKMStore + Thrust-host
    counting, compiled from its sources) on a sample; returns k-mers/s."""
    import oracle_ffi as F
    t0 = time.perf_counter()
    distinct, kmers = F.ref_pipeline(reads, offs, wl["k"], wl["p"], wl["hpc"], wl["nbins"],
                                     batch_reads=2048, n_threads=threads)
    dt = time.perf_counter() - t0
    return kmers / dt, dt, kmers, distinct


def reference_parity(ctx, G, prm, reads, offs, wl, threads):
    """The CPU-baseline sample counted by the reference's own CPU path and by
    this library (through the host API), their per-bin sorted (k-mer, count)
    lists compared by digest (untimed)."""
    import oracle_ffi as F
    ref, _ = F.ref_pipeline_counts(reads, offs, wl["k"], wl["p"], wl["hpc"], wl["nbins"], batch_reads=2048,
                                   n_threads=threads)
    rd, _ = F.counts_digest64(ref["bin_off"], ref["keys_lo"], ref["counts"])
    cv = ctx.pipeline_host(reads, offs, prm, G.MODE_BATCHED)
    bo, keys, counts = ctx.count_copy_out(cv)
    gd, _ = F.counts_digest64(bo, keys[:, 0], counts)
    return {"reads": len(offs) - 1, "kmers": int(cv.n_kmers), "distinct": int(cv.n_distinct),
            "reference_distinct": int(len(ref["keys_lo"])), "digest": "%016x" % gd,
            "reference_digest": "%016x" % rd, "match": bool(gd == rd and np.array_equal(bo, ref["bin_off"])),
            "compared": "per-bin sorted (k-mer, count) lists of the CPU-baseline sample"}


def time_minimizer_emit(ctx, G, torch, stream, reads, offs, n_reads, n_bases, wl, reps=3):
    """HPC (gkc_hpc_device) then every window's minimizer, position and
    strand (gkc_minimizers_device) over the compressed reads; bytes moved at
    least: the reads and offsets in, the compressed reads, their offsets and
    original positions out and back in, 6 bytes per window out."""
    d_h = torch.empty(n_bases + 64, dtype=torch.uint8, device="cuda")
    d_ho = torch.empty(n_reads + 1, dtype=torch.int64, device="cuda")
    d_orig = torch.empty(n_bases + 16, dtype=torch.int32, device="cuda")
    d_mm = torch.empty(n_bases + 16, dtype=torch.int32, device="cuda")
    d_pos = torch.empty(n_bases + 16, dtype=torch.uint8, device="cuda")
    d_str = torch.empty(n_bases + 16, dtype=torch.int8, device="cuda")
    prm = G.params(wl["k"], wl["p"], wl["nbins"], False)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    t_hpc, t_mm = [], []
    for r in range(reps + 1):
        ev[0].record(stream)
        ctx.hpc_device(reads, n_bases, offs, n_reads, d_h, d_ho, d_orig)
        ev[1].record(stream)
        nb = int(d_ho[n_reads].item())
        ctx.minimizers_device(d_h, nb, d_ho, n_reads, prm, d_mm, d_pos, d_str)
        ev[2].record(stream)
        torch.cuda.synchronize()
        if r:
            t_hpc.append(ev[0].elapsed_time(ev[1]))
            t_mm.append(ev[1].elapsed_time(ev[2]))
    peak, kind = peaks()
    hpc_ms, mm_ms = float(np.median(t_hpc)), float(np.median(t_mm))
    b_hpc = n_bases + 8 * (n_reads + 1) + nb + 8 * (n_reads + 1) + 4 * nb
    b_mm = nb + 8 * (n_reads + 1) + 6 * nb
    return {"windows": nb, "hpc_ms": hpc_ms, "minimizer_ms": mm_ms,
            "windows_per_s": nb / ((hpc_ms + mm_ms) / 1000.0),
            "roofline": {"bound": "hbm", "kernel": "k_window_minimizers", "achieved": b_mm / (mm_ms / 1000.0) / 1e9,
                         "peak": peak, "peak_kind": kind, "unit": "GB/s",
                         "frac": b_mm / (mm_ms / 1000.0) / 1e9 / peak,
                         "model": "reads + offsets in, 4 + 1 + 1 bytes per window out"},
            "hpc_gbs": b_hpc / (hpc_ms / 1000.0) / 1e9}


def time_subsample(ctx, G, torch, stream, reads, offs, n_reads, n_bases, wl, reps=3, mod=4):
    """k-mers whose window minimizer % 4 == 0 with their position lists
    (gkc_subsample_positions_device)."""
    prm = G.params(wl["k"], wl["p"], wl["nbins"], False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts = []
    for r in range(reps + 1):
        e0.record(stream)
        v = ctx.subsample_positions_device(reads, n_bases, offs, n_reads, prm, mod)
        e1.record(stream)
        torch.cuda.synchronize()
        if r:
            ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    n_pos, nd = int(v.n_positions), int(v.n_distinct)
    w = 16
    P = math.ceil(2 * wl["k"] / 8)
    # model: reads in, selected (key, position) pairs sorted by LSD radix passes, keys + offsets + positions out
    model = n_bases + 8 * (n_reads + 1) + (w + 4) * n_pos * (1 + 2 * P) + w * nd + 8 * (nd + 1) + 4 * n_pos
    peak, kind = peaks()
    return {"positions": n_pos, "distinct": nd, "ms": ms, "positions_per_s": n_pos / (ms / 1000.0),
            "roofline": {"bound": "hbm", "achieved": model / (ms / 1000.0) / 1e9, "peak": peak, "peak_kind": kind,
                         "unit": "GB/s", "frac": model / (ms / 1000.0) / 1e9 / peak,
                         "model": "reads in; (key, position) pairs through 2k/8 LSD passes; lists out"}}


# ------------------------------------------------------------ reference arm

def run_reference(args, wl):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle_ffi as F
    if not F.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference tree absent at build time)"}))
        return
    threads = os.cpu_count() or 1
    # each step about min(10 s, 100 s / (steps + warm-up)) of CPU work, sized
    # from a calibration run on the first sample_reads(...) reads
    reads, offs = host_sample(wl, args.seed, sample_reads(args, wl))
    rate, _, kmers, _ = cpu_reference_rate(reads, offs, wl, threads)
    per_step = min(10.0, 100.0 / max(1, args.steps + args.warmup))
    n = scaled_sample(wl, len(offs) - 1, kmers, rate, per_step)
    if n > len(offs) - 1:
        reads, offs = host_sample(wl, args.seed, n)
    for _ in range(args.warmup):
        cpu_reference_rate(reads, offs, wl, threads)
    rates, secs, km = [], [], 0
    for _ in range(args.steps):
        r, dt, kmers, _ = cpu_reference_rate(reads, offs, wl, threads)
        rates.append(r)
        secs.append(dt)
        km = kmers
    value = float(np.median(rates))
    sample = f"first {len(offs) - 1} reads ({int(offs[-1])} bases, {km} k-mers) of workload {wl_name(args)}"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "kmers/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * float(np.median(secs)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": dict(config_dict(args, wl, len(offs) - 1, int(offs[-1])),
                       mode="the reference's CPU path: its partition kernels as host C++, SKMStore, "
                            "Thrust-host sort and run count", parallelism=f"{threads} host threads"),
        "cpu_baseline": {"value": value, "unit": "kmers/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "kmers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def host_read_pool(G, seed, n_bases):
    """Config-2 short reads (150 bp, 30x of a genome) made on the host, for
    the serving mix's host-read jobs: a job of b bases takes the first b // 150
    reads."""
    L = G.lib()
    n = n_bases // 150
    glen = max(n * 150 // 30, 1 << 16)
    genome = np.zeros(glen, np.uint8)
    assert L.gkc_synth_genome(0, seed, glen, 0.05, 0.01, genome.ctypes.data) == 0
    reads = np.zeros(n * 150 + 64, np.uint8)
    offs = np.zeros(n + 1, np.uint64)
    assert L.gkc_synth_short_reads(0, seed, genome.ctypes.data, glen, 0, n, 150, 0.005, reads.ctypes.data,
                                   offs.ctypes.data) == 0
    return reads, offs


def serve_mix(G, device, n_jobs, loads, seed, max_running=4, lo=1e5, hi=1e9, calib_jobs=40, host_frac=0.25,
              host_pool_bases=200_000_000, grace_s=30.0):
    """The serving mix: jobs of log-uniform size in [lo, hi] bases, each from
    the config-2 (short reads of a genome, 30x) or config-3 (long reads, 20x,
    HPC) generator at random, k in {25, 31}, Poisson arrivals at each load
    (a fraction of the capacity measured by a burst of calib_jobs jobs).
    Latency = job end - submission, on the server's clock.  A host_frac share
    of the config-2 jobs hands the server reads in host memory (taken from a
    pool made on the host, at most host_pool_bases bases), so their latency
    includes the upload; the others' reads are generated on the device when
    the job starts, inside its latency.  A job still unfinished grace_s
    seconds after the last submission is reported in "unfinished" (id, size,
    generator, k, state) instead of being waited for; out["stuck"] is then
    true and the server cannot be shut down cleanly (its worker still holds
    the job), so the caller ends the process."""
    import threading
    rng = np.random.default_rng(seed)
    pool_reads, pool_offs = host_read_pool(G, seed + 17, host_pool_bases)

    def draw(n):
        sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)
        gens = rng.choice([2, 3], n)
        gens = np.where((gens == 2) & (rng.random(n) < host_frac), 0, gens)  # 0: host reads (config-2 shape)
        return list(zip(sizes.tolist(), gens.tolist(), rng.choice([25, 31], n).tolist()))

    def submit(srv, sz, g, k, job_seed):
        if g == 0:
            nr = max(1, min(int(sz) // 150, len(pool_offs) - 1))
            return srv.submit(pool_reads[:int(pool_offs[nr])], pool_offs[:nr + 1], prm_for(2, k))
        return srv.submit_synth(prm_for(g, k), g, job_seed, sz)

    def prm_for(gen, k):
        return G.params(k, 15, 256, True) if gen == 3 else G.params(k, 11, 256)

    out = {"generators": "config-2 short reads 30x (p=11) / config-3 long reads 20x HPC (p=15)",
           "sizes_bases": [lo, hi], "k": [25, 31], "slots": max_running,
           "host_read_jobs": f"{host_frac:.0%} of the config-2 jobs, reads in host memory "
                             f"(at most {host_pool_bases:.0e} bases), upload inside the latency"}
    out["stuck"] = False
    srv = G.Server(device, max_running=max_running)
    try:
        def collect(ids, infos):
            for j in ids:
                infos.append(srv.wait(j))
                srv.release(j)

        cal = draw(calib_jobs)
        progress(f"serving: capacity from a burst of {calib_jobs} jobs")
        t0 = time.perf_counter()
        ids = [submit(srv, sz, g, k, seed * 7919 + i) for i, (sz, g, k) in enumerate(cal)]
        infos = []
        collect(ids, infos)
        wall = time.perf_counter() - t0
        cap = sum(int(i.n_bases) for i in infos) / wall
        out["capacity_bases_per_s"] = cap
        out["loads"] = {}
        for li, load in enumerate(loads):
            jobs = draw(n_jobs)
            progress(f"serving: {n_jobs} jobs at {load:.0%} load")
            mean_bases = float(np.mean([sz for sz, _, _ in jobs]))
            rate = load * cap / mean_bases
            gaps = rng.exponential(1.0 / rate, n_jobs)
            ids, infos, unfinished = [], [], []
            lock = threading.Lock()
            done = threading.Event()
            t_last = [None]  # host clock of the last submission

            def collector():
                k = 0
                while True:
                    with lock:
                        j = ids[k] if k < len(ids) else None
                    if j is None:
                        if done.is_set() and k >= len(ids):
                            return
                        time.sleep(0.001)
                        continue
                    while True:
                        info = srv.wait(j, 1.0)
                        if info.state in (2, 3, 4):  # done, failed, cancelled
                            infos.append(info)
                            srv.release(j)
                            break
                        if t_last[0] is not None and time.perf_counter() - t_last[0] > grace_s:
                            sz, g, kk = jobs[j - first_id]
                            unfinished.append({"job": j, "bases": int(sz), "generator": int(g), "k": int(kk),
                                               "state": "running" if info.state == 1 else "queued"})
                            break
                    k += 1

            th = threading.Thread(target=collector)
            first_id = None
            th.start()
            start, t = time.perf_counter(), 0.0
            for i, ((sz, g, k), gap) in enumerate(zip(jobs, gaps)):
                t += gap
                dt = start + t - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                jid = submit(srv, sz, g, k, seed * 100003 + li * 10007 + i)
                if first_id is None:
                    first_id = jid
                with lock:
                    ids.append(jid)
            t_last[0] = time.perf_counter()
            done.set()
            th.join()
            ok = [i for i in infos if i.state == 2]
            n_jobs_done = len(infos)
            lat = np.array([i.end_s - i.submit_s for i in ok])
            span = (max(i.end_s for i in ok) - min(i.submit_s for i in ok)) if ok else 0.0
            out["loads"][f"{load:.2f}"] = {
                "jobs": n_jobs, "failed": n_jobs_done - len(ok), "unfinished_count": len(unfinished),
                "failed_status": sorted({int(i.status) for i in infos if i.state != 2}),
                "p50_latency_s": float(np.percentile(lat, 50)) if ok else None,
                "p99_latency_s": float(np.percentile(lat, 99)) if ok else None,
                "mean_latency_s": float(lat.mean()) if ok else None,
                "kmers_per_s": sum(int(i.n_kmers) for i in ok) / span if span > 0 else None,
                "bases_per_s": sum(int(i.n_bases) for i in ok) / span if span > 0 else None,
                "offered_bases_per_s": load * cap, "span_s": span}
            if unfinished:
                out["loads"][f"{load:.2f}"]["unfinished"] = unfinished
                out["stuck"] = True
                break
    finally:
        if not out["stuck"]:
            srv.close()
    return out


def serve_child(args):
    """The default run's serving mix (200 jobs at 80% load) in a child
    process with a time limit, so that the throughput line is printed
    whatever the mix does; returns its "serving" object, or an error."""
    cmd = [sys.executable, os.path.abspath(__file__), "--serve", "--serve-jobs", str(args.serve_jobs or 200),
           "--serve-loads", "0.8", "--seed", str(args.seed)]
    try:
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                           timeout=args.serve_timeout, start_new_session=True)
    except subprocess.TimeoutExpired as e:
        tail = (e.stderr or "")[-400:] if isinstance(e.stderr, str) else ""
        return {"error": f"the serving mix did not finish within {args.serve_timeout:.0f} s", "stderr_tail": tail}
    line = next((ln for ln in reversed(r.stdout.splitlines()) if ln.startswith("{")), None)
    if line is None:
        return {"error": f"the serving mix exited {r.returncode} without a result", "stderr_tail": r.stderr[-400:]}
    res = json.loads(line).get("serving", {})
    if r.returncode != 0:
        res["exit_code"] = r.returncode
    return res


def run_serve(args):
    import torch
    import gkc_b200 as G
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    n = args.serve_jobs or 1000
    loads = tuple(float(x) for x in args.serve_loads.split(","))
    res = serve_mix(G, local, n, loads, args.seed)
    key = "0.80" if "0.80" in res["loads"] else sorted(res["loads"])[-1] if res["loads"] else None
    if key is None:
        print(json.dumps({"metric": "served canonical k-mers counted/s", "value": None, "serving": res}))
        sys.stdout.flush()
        os._exit(1)
    l80 = res["loads"][key]
    print(json.dumps({
        "metric": f"served canonical k-mers counted/s at {float(key):.0%} load (p50/p99 job latency in serving)",
        "value": l80["kmers_per_s"], "unit": "kmers/s", "n_gpus": 1, "steps": n, "warmup": 40,
        "ms_per_step": 1000 * l80["mean_latency_s"] if l80["mean_latency_s"] is not None else None,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"config5-serving-mix-{n}-jobs", "loads": list(loads)},
        "serving": res}))
    sys.stdout.flush()
    if res["stuck"]:
        # a worker still holds an unfinished job: the server cannot be joined
        sys.stderr.write("serving: unfinished jobs; ending the process without shutting the server down\n")
        os._exit(3)


def wl_name(args):
    return {"ns": "ns-100Mbp-30x-150bp-k31", "config2": "config2-10Mbp-30x-150bp-k31",
            "config1": "config1-iid-20000x150bp-k31", "config4": "config4-100Mbp-30x-250bp-k63",
            "config3": "config3-100Mbp-20x-long-hpc-k25", "small": "small-3Mbp-30x-150bp-k31"}[args.workload]


def scaled_sample(wl, n_cal, kmers_cal, rate, seconds):
    """Reads whose reference CPU run takes about `seconds`, from a
    calibration run of n_cal reads (kmers_cal k-mers at `rate` k-mers/s)."""
    per_read = max(kmers_cal / max(n_cal, 1), 1.0)
    n = int(seconds * rate / per_read)
    if wl["gen"] == "iid":
        return min(max(n, n_cal), wl["n_reads"])
    if wl["gen"] == "genome":
        return min(max(n, n_cal), wl["coverage"] * wl["genome_len"] // wl["read_len"])
    return max(n, n_cal)


def sample_reads(args, wl):
    """Reads in the bounded CPU-baseline sample (about 30 M bases of long reads)."""
    if wl["gen"] == "iid":
        return wl["n_reads"]
    if wl["gen"] == "long":
        return max(100, int(30e6 // wl["median"]))
    return args.cpu_sample_reads


def config_dict(args, wl, n_reads, n_bases):
    d = {"workload": wl_name(args), "reads": n_reads, "bases": n_bases, "k": wl["k"], "p": wl["p"],
         "nbins": wl["nbins"], "hpc": bool(wl["hpc"]), "seed": args.seed,
         "l2": "inputs larger than L2 (reads + superkmers + keys >> 126 MB)",
         "mode": "batched, graph-captured", "parallelism": f"weak-replicas{args.gpus}"}
    if args.multi == "shard" or (args.gpus > 1 and args.multi is None):
        d.update(mode="partition; superkmer all-to-all to bin owners (NCCL); owned bins counted",
                 parallelism=f"weak-bin-shard{args.gpus}")
    if wl["gen"] == "genome":
        d.update(genome_bp=wl["genome_len"], coverage=wl["coverage"], read_len=wl["read_len"],
                 error_rate=wl["err"])
    if wl["gen"] == "long":
        d.update(genome_bp=wl["genome_len"], coverage=wl["coverage"],
                 read_len=f"lognormal median {wl['median']:.0f} sigma {wl['sigma']} clipped {wl['min_len']}-{wl['max_len']}",
                 errors="5%: 40% substitution, 30% insertion, 30% deletion (indels likelier in homopolymers)")
    return d


# ------------------------------------------------------------------ our arm

def run_ours(args, wl):
    import torch
    import gkc_b200 as G

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    progress("workload")
    reads, offs, n_reads, n_bases, genome = make_workload_device(wl, args.seed, rank, torch, G)
    torch.cuda.synchronize()
    prm = G.params(wl["k"], wl["p"], wl["nbins"], wl["hpc"])
    ctx = G.Context(local)
    stream = torch.cuda.Stream()  # graphs cannot be captured on the legacy default stream
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    # launch shapes of the count stage, chosen by timing candidates on a
    # sample of the reads (outside the timed region)
    tune = None
    if not args.no_tune:
        progress("tuning the count stage on a sample")
        rep = ctx.autotune_device(reads, n_bases, offs, n_reads, prm, force=True)
        tune = {"chosen": rep.chosen.as_dict(), "defaults": rep.defaults.as_dict(),
                "sample_bases": int(rep.sample_bases), "candidates": int(rep.candidates),
                "count_ms_sample_default": float(rep.default_ms), "count_ms_sample_tuned": float(rep.tuned_ms),
                "tuned_over_default": float(rep.default_ms / rep.tuned_ms) if rep.tuned_ms > 0 else None}

    def step():
        return ctx.pipeline_device(reads, n_bases, offs, n_reads, prm, G.MODE_BATCHED)

    progress("warm-up")
    for _ in range(max(args.warmup, 3)):
        pv, cv = step()
    torch.cuda.synchronize()
    progress("timed steps")

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    stage_acc = {}
    launches = 0
    barrier()
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            pv, cv = step()
            t = ctx.timings()
            launches += int(t.launches)
            for name, ms in t.stages().items():
                stage_acc.setdefault(name, []).append(ms)
        e1.record(stream)
        barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    clocks = clk.summary()

    N, D, S = int(cv.n_kmers), int(cv.n_distinct), int(pv.n_superkmers)
    B, R = int(pv.n_bases), int(pv.n_reads)
    ms_step = ms_total / args.steps
    value = whole_job_rate(N, world, args.steps, ms_total)
    stages = {k: float(np.mean(v)) for k, v in stage_acc.items()}
    model = algorithmic_bytes(B, R, S, N, D, wl["k"])
    peak, peak_kind = peaks()

    # dominant stage and its model bytes per launch: the partition kernel; the
    # expansion (the histogram kernel walks the superkmers and writes every
    # canonical key); sort + count (the bucket scatter, the count kernel and
    # the compaction of its runs)
    stages["sort_count"] = stages.get("coarse_scatter", 0.0) + stages.get("coarse_count", 0.0) + \
        stages.get("finish", 0.0)
    kernel_bytes = {"partition": model["partition"], "coarse_hist": model["expand"],
                    "sort_count": model["sort"] + model["count"]}
    dom = max(kernel_bytes, key=lambda s: stages.get(s, 0.0))
    dom_ms = stages[dom]
    achieved = kernel_bytes[dom] / (dom_ms / 1000.0) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as f:
                td = json.load(f)
            per_unit = td.get(wl_name(args), {}).get(dom)
            if per_unit is not None:
                traffic = per_unit["dram_bytes_per_kmer"] * N
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "model": "fixed algorithmic-bytes model: partition B+8(R+1)+L/4+8S, expand L/4+8S+wN, sort wN+2PwN, count wN+(w+4)D",
                "model_bytes_per_launch": kernel_bytes[dom], "ms_per_launch": dom_ms}
    if traffic:
        roofline["frac_dram_traffic"] = traffic / (dom_ms / 1000.0) / 1e9 / peak
    roofline["stages"] = {n: {"model_bytes": b, "ms": stages.get(n, 0.0),
                              "frac": (b / (stages[n] / 1000.0) / 1e9 / peak) if stages.get(n) else None}
                          for n, b in kernel_bytes.items()}
    pipeline = {"model_bytes": model["total"], "ms": ms_step,
                "achieved_gbs": model["total"] / (ms_step / 1000.0) / 1e9,
                "frac_of_hbm_roofline": model["total"] / (ms_step / 1000.0) / 1e9 / peak,
                "bases_per_s": B * world / (ms_step / 1000.0), "superkmers": S, "kmers": N,
                "distinct": D}

    result = {
        "metric": METRIC, "value": value, "unit": "kmers/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64" if wl["k"] <= 32 else "u128", "data": "synthetic",
        "config": config_dict(args, wl, n_reads, n_bases), "roofline": roofline,
        "pipeline": pipeline, "stages_ms": stages, "gpu_launches": launches, "clocks": clocks,
    }
    if tune is not None:
        result["tune"] = tune

    # plain per-stage form on the same input, its whole output compared with
    # the batched one on the device (bin offsets, every key and count)
    if not args.no_plain and rank == 0:
        progress("plain per-stage form")
        kw = 1 if wl["k"] <= 32 else 2
        nd_b = int(cv.n_distinct)
        # the plain form allocates its own buffers: with 16-byte keys the
        # batched ones are given back first (both key sets do not fit), and
        # the two outputs are compared in host memory
        wide = wl["k"] > 32
        where = "cpu" if wide else "cuda"
        batched_out = (torch.empty(wl["nbins"] + 1, dtype=torch.int64, device=where),
                       torch.empty(max(nd_b * kw, 1), dtype=torch.int64, device=where),
                       torch.empty(max(nd_b, 1), dtype=torch.int32, device=where))
        assert G.lib().gkc_count_copy_out(ctx.h, *(t.data_ptr() for t in batched_out)) == 0
        torch.cuda.synchronize()
        if wide:
            assert G.lib().gkc_ctx_release_workspace(ctx.h) == 0
        pe0 = torch.cuda.Event(enable_timing=True)
        pe1 = torch.cuda.Event(enable_timing=True)
        ctx.pipeline_device(reads, n_bases, offs, n_reads, prm, G.MODE_PLAIN)  # warm-up
        torch.cuda.synchronize()
        pe0.record(stream)
        for _ in range(args.plain_steps):
            ppv, pcv = ctx.pipeline_device(reads, n_bases, offs, n_reads, prm, G.MODE_PLAIN)
        pe1.record(stream)
        torch.cuda.synchronize()
        p_ms = pe0.elapsed_time(pe1) / args.plain_steps
        same = int(pcv.n_distinct) == nd_b
        if same:
            plain_out = tuple(torch.empty_like(t) for t in batched_out)
            assert G.lib().gkc_count_copy_out(ctx.h, *(t.data_ptr() for t in plain_out)) == 0
            torch.cuda.synchronize()
            same = all(torch.equal(a, b) for a, b in zip(batched_out, plain_out))
            del plain_out
        del batched_out
        torch.cuda.empty_cache()
        result["plain"] = {"value": N / (p_ms / 1000.0), "unit": "kmers/s", "ms_per_step": p_ms,
                           "steps": args.plain_steps, "batched_over_plain": p_ms / ms_step,
                           "same_output_as_batched": bool(same),
                           "compared": "bin offsets, every key and every count, " +
                                       ("in host memory" if wide else "on the device"),
                           "launches_per_step": int(ctx.timings().launches)}
        # restore the batched result in the context
        if wide:
            assert G.lib().gkc_ctx_release_workspace(ctx.h) == 0
        step()

    # the workload's application outputs, each timed on its own: config 3's
    # per-window (minimizer, position, strand) emit after HPC, config 4's
    # sub-sampled k-mers with position lists (minimizer % 4 == 0)
    if rank == 0 and wl["gen"] == "long":
        result["minimizer_emit"] = time_minimizer_emit(ctx, G, torch, stream, reads, offs, n_reads, n_bases, wl)
    if rank == 0 and wl["k"] > 32:
        # its own workspaces: the count pipeline's 16-byte key arrays are given back first
        assert G.lib().gkc_ctx_release_workspace(ctx.h) == 0
        result["subsample_positions"] = time_subsample(ctx, G, torch, stream, reads, offs, n_reads, n_bases, wl)
        assert G.lib().gkc_ctx_release_workspace(ctx.h) == 0

    # the CPU baseline's reads: the workload's first reads, copied from the
    # device (at most 10 M reads, enough for about 10 s of reference CPU work)
    cpu_sample = None
    if not args.no_cpu and rank == 0 and world == 1:
        n_max = min(n_reads, 10_000_000)
        so = offs[:n_max + 1].cpu().numpy().view(np.uint64).copy()
        cpu_sample = (reads[:int(so[-1])].cpu().numpy(), so)

    # end to end through the host API: pinned host reads in, the full sorted
    # list out, every step.  Headline: the streaming form (gkc_stream_submit /
    # gkc_stream_wait), where one step's upload, the previous step's counting
    # and the one before's download overlap; beside it the one-call form
    # (gkc_pipeline_host + gkc_count_copy_out), each step in turn.
    if not args.no_e2e:
        progress("end to end from host memory")
        h_reads = torch.empty(n_bases, dtype=torch.uint8, pin_memory=True)
        h_offs = torch.empty(n_reads + 1, dtype=torch.int64, pin_memory=True)
        h_reads.copy_(reads[:n_bases])
        h_offs.copy_(offs)
        kw = 1 if wl["k"] <= 32 else 2
        cap = D + D // 64 + 1024
        # the streaming form holds two calls' device buffers: with 16-byte keys
        # at this size they do not fit, and the one-call form is the e2e figure
        streaming = wl["k"] <= 32
        # three host output sets: call i is submitted before call i - 2 is
        # waited for, so its upload overlaps call i - 2's download
        outs = [(torch.empty(wl["nbins"] + 1, dtype=torch.int64, pin_memory=True),
                 torch.empty(cap * kw, dtype=torch.int64, pin_memory=True),
                 torch.empty(cap, dtype=torch.int32, pin_memory=True)) for _ in range(3 if streaming else 1)]
        nr = h_reads.numpy()
        no = h_offs.numpy().view(np.uint64)
        del reads  # the host path uploads its own copy
        torch.cuda.empty_cache()
        # the plain form's buffers are not needed again; the streaming form
        # holds two calls' inputs and outputs
        assert G.lib().gkc_ctx_release_workspace(ctx.h) == 0

        if streaming:
            def submit(i):
                o = outs[i % 3]
                return ctx.stream_submit(h_reads, h_offs, n_reads, prm, o[0], o[1], o[2], cap)

            for t in (submit(0), submit(1)):  # the first call of each slot captures its graph
                ctx.stream_wait(t)
            barrier()
            e_steps = max(args.e2e_steps, 4)
            t0 = time.perf_counter()
            tickets = []
            for i in range(e_steps):
                tickets.append(submit(i))
                if i >= 2:
                    ctx.stream_wait(tickets[i - 2])
            for t in tickets[-2:]:
                nd, nk = ctx.stream_wait(t)
            torch.cuda.synchronize()
            e_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0, dist, "cuda")
            assert nd == D and nk == N, (nd, D, nk, N)
            result["e2e"] = {"value": whole_job_rate(N, world, e_steps, e_ms), "unit": "kmers/s",
                             "h2d_bytes_per_step": n_bases + (n_reads + 1) * 8,
                             "d2h_bytes_per_step": (wl["nbins"] + 1) * 8 + nd * 8 * kw + nd * 4,
                             "ms_per_step": e_ms / e_steps, "steps": e_steps,
                             "api": "gkc_stream_submit + gkc_stream_wait (pinned host buffers; calls overlap)",
                             "clock": "host clock between device synchronisations"}
        # the one-call form, each step in turn
        progress("end to end, one call at a time")
        h_binoff, h_keys, h_counts = outs[0]

        def e2e_step():
            c = ctx.pipeline_host(nr, no, prm, G.MODE_BATCHED)
            st = G.lib().gkc_count_copy_out(ctx.h, h_binoff.data_ptr(), h_keys.data_ptr(), h_counts.data_ptr())
            assert st == 0
            return c

        e2e_step()
        barrier()
        ee0 = torch.cuda.Event(enable_timing=True)
        ee1 = torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        for _ in range(args.e2e_steps):
            c = e2e_step()
        ee1.record(stream)
        barrier()
        s_ms = max_over_ranks(ee0.elapsed_time(ee1), dist, "cuda")
        one_call = {"value": whole_job_rate(N, world, args.e2e_steps, s_ms),
                    "ms_per_step": s_ms / args.e2e_steps, "steps": args.e2e_steps,
                    "api": "gkc_pipeline_host + gkc_count_copy_out"}
        if streaming:
            result["e2e"]["one_call_form"] = one_call
        else:
            result["e2e"] = dict(one_call, unit="kmers/s", h2d_bytes_per_step=n_bases + (n_reads + 1) * 8,
                                 d2h_bytes_per_step=(wl["nbins"] + 1) * 8 + D * 8 * kw + D * 4,
                                 clock="CUDA events on the pipeline's stream",
                                 note="16-byte keys: two calls' buffers do not fit the device at this size, "
                                      "so the streaming form is not run")

    # CPU baseline: the reference's own CPU path on a bounded sample (rank 0, N=1)
    if not args.no_cpu and rank == 0 and world == 1:
        import oracle_ffi as F
        if F.ref_available():
            progress("reference CPU path on a sample")
            threads = os.cpu_count() or 1
            n_cal = min(sample_reads(args, wl), cpu_sample[1].size - 1)
            cal_o = cpu_sample[1][:n_cal + 1]
            rate, _, kmers, _ = cpu_reference_rate(cpu_sample[0][:int(cal_o[-1])], cal_o, wl, threads)
            n = min(scaled_sample(wl, n_cal, kmers, rate, 10.0), cpu_sample[1].size - 1)
            so = cpu_sample[1][:n + 1]
            sr = cpu_sample[0][:int(so[-1])]
            rate, dt, km, _ = cpu_reference_rate(sr, so, wl, threads)
            result["cpu_baseline"] = {
                "value": rate, "unit": "kmers/s", "cores": threads, "kind": "reference",
                "sample": f"first {len(so) - 1} reads ({int(so[-1])} bases, {km} k-mers) of the workload, {dt:.2f} s"}
            if wl["k"] > 32:
                result["cpu_baseline"]["note"] = ("the reference keeps k-mers in 64-bit words (k <= 32): "
                                                  "at this k its CPU path is a timing figure only")
                result["parity"] = {"reads": len(so) - 1, "match": None,
                                    "note": "the reference's keys are 64-bit: no comparison at k > 32"}
            else:
                progress("parity against the reference on that sample")
                result["parity"] = reference_parity(ctx, G, prm, sr, so, wl, threads)
        else:
            result["cpu_baseline"] = {"value": None, "unit": "kmers/s", "cores": 0, "kind": "reference",
                                      "sample": "oracle/_ref not built"}
    ctx.close()
    # served latency: a shorter serving mix at 80% load (full mix: --serve)
    if not args.no_serve and rank == 0 and world == 1:
        del ctx
        torch.cuda.empty_cache()
        progress("serving mix")
        result["serving"] = serve_child(args)
    if rank == 0:
        print(json.dumps(result))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------- our arm, bins sharded

def run_shard(args, wl):
    """N > 1: every rank partitions its own reads, the superkmers go to the
    owners of their bins (three NCCL all-to-alls), every rank counts the bins
    it owns.  One step = partition + exchange + count; the whole-job rate
    counts the k-mers all ranks counted over the slowest rank's time."""
    import datetime
    import torch
    import torch.distributed as dist
    import gkc_b200 as G
    from gkc_b200 import shard

    for key, val in (("MASTER_ADDR", "127.0.0.1"), ("MASTER_PORT", "29511"), ("RANK", "0"), ("WORLD_SIZE", "1")):
        os.environ.setdefault(key, val)  # one rank without a launcher
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    reads, offs, n_reads, n_bases, genome = make_workload_device(wl, args.seed, rank, torch, G)
    torch.cuda.synchronize()
    prm = G.params(wl["k"], wl["p"], wl["nbins"], wl["hpc"])
    ctx = G.Context(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    stage_acc = {"partition": [], "exchange": [], "count": []}
    state = {"launches": 0}

    def step(record=False, host=None):
        ev[0].record(stream)
        if host is None:
            pv = ctx.partition_device(reads, n_bases, offs, n_reads, prm)
        else:
            pv = ctx.partition_host(host[0], host[1], prm)
        state["launches"] += int(ctx.timings().launches)
        own = dict(kmers=int(pv.n_kmers), skm=int(pv.n_superkmers), bases=int(pv.n_bases),
                   reads=int(pv.n_reads), bytes=int(pv.n_packed_bytes))
        ev[1].record(stream)
        eng = shard.DeviceEngine(ctx, pv, dev)
        prm_local, bounds, _ = shard.exchange_dist(eng, prm)
        state["launches"] += eng.launches
        ev[2].record(stream)
        cv = ctx.count_device(prm_local, G.MODE_BATCHED)
        state["launches"] += int(ctx.timings().launches)
        ev[3].record(stream)
        if record:
            ev[3].synchronize()
            for name, a, b in (("partition", 0, 1), ("exchange", 1, 2), ("count", 2, 3)):
                stage_acc[name].append(ev[a].elapsed_time(ev[b]))
        return own, cv, prm_local, bounds

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    state["launches"] = 0
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            own, cv, prm_local, bounds = step(record=True)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    clocks = clk.summary()
    launches = state["launches"]

    counted = torch.tensor([int(cv.n_kmers), own["kmers"], int(cv.n_distinct)], dtype=torch.int64, device=dev)
    dist.all_reduce(counted)
    total_kmers, own_total, distinct_total = (int(x) for x in counted.tolist())
    ms_step = ms_total / args.steps
    value = total_kmers * args.steps / (ms_total / 1000.0)
    stages = {k: float(np.mean(v)) for k, v in stage_acc.items()}
    # HBM roofline of the count stage (the owned bins) and the partition stage
    N, D, S = int(cv.n_kmers), int(cv.n_distinct), own["skm"]
    model_own = algorithmic_bytes(own["bases"], own["reads"], S, own["kmers"], D, wl["k"])
    model_cnt = algorithmic_bytes(0, 0, 0, N, D, wl["k"])
    kernel_bytes = {"partition": model_own["partition"],
                    "count": model_cnt["expand"] + model_cnt["sort"] + model_cnt["count"]}
    dom = max(kernel_bytes, key=lambda s: stages[s])
    peak, peak_kind = peaks()
    achieved = kernel_bytes[dom] / (stages[dom] / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                "model": "fixed algorithmic-bytes model: partition B+8(R+1)+L/4+8S, expand L/4+8S+wN, sort wN+2PwN, count wN+(w+4)D",
                "model_bytes_per_launch": kernel_bytes[dom], "ms_per_launch": stages[dom]}
    sent = 8 * S + own["bytes"]  # descriptors + packed bytes, all destinations
    leaves = sent * (world - 1) / world
    exchange = {"bytes_sent_per_rank": sent, "bytes_leaving_rank_est": leaves, "ms": stages["exchange"],
                "gbs_leaving": leaves / (stages["exchange"] / 1000.0) / 1e9,
                "peer_copy_gbs_measured": 770.0,
                "frac_of_peer_copy": leaves / (stages["exchange"] / 1000.0) / 1e9 / 770.0}
    result = {
        "metric": METRIC, "value": value, "unit": "kmers/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64" if wl["k"] <= 32 else "u128", "data": "synthetic",
        "config": config_dict(args, wl, n_reads, n_bases), "roofline": roofline, "exchange": exchange,
        "stages_ms": stages, "gpu_launches": launches, "clocks": clocks,
        "check": {"kmers_counted": total_kmers, "kmers_partitioned": own_total,
                  "distinct_over_owners": distinct_total, "owned_bins_rank0": [int(bounds[0]), int(bounds[1])]},
    }

    if not args.no_e2e:
        h_reads = torch.empty(n_bases, dtype=torch.uint8, pin_memory=True)
        h_offs = torch.empty(n_reads + 1, dtype=torch.int64, pin_memory=True)
        h_reads.copy_(reads[:n_bases])
        h_offs.copy_(offs)
        host = (h_reads.numpy(), h_offs.numpy().view(np.uint64))
        kw = 1 if wl["k"] <= 32 else 2
        cap = 2 * int(cv.n_distinct) + 1024
        h_binoff = torch.empty(wl["nbins"] + 1, dtype=torch.int64, pin_memory=True)
        h_keys = torch.empty(cap * kw, dtype=torch.int64, pin_memory=True)
        h_counts = torch.empty(cap, dtype=torch.int32, pin_memory=True)
        del reads
        torch.cuda.empty_cache()
        L = G.lib()

        def e2e_step():
            o, c, pl, _ = step(host=host)
            assert int(c.n_distinct) <= cap
            assert L.gkc_count_copy_out(ctx.h, h_binoff.data_ptr(), h_keys.data_ptr(), h_counts.data_ptr()) == 0
            return c

        e2e_step()
        torch.cuda.synchronize()
        dist.barrier()
        ee0 = torch.cuda.Event(enable_timing=True)
        ee1 = torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        for _ in range(args.e2e_steps):
            c = e2e_step()
        ee1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        e_ms = max_over_ranks(ee0.elapsed_time(ee1), dist, "cuda")
        nd = int(c.n_distinct)
        result["e2e"] = {"value": total_kmers * args.e2e_steps / (e_ms / 1000.0), "unit": "kmers/s",
                         "h2d_bytes_per_step": n_bases + (n_reads + 1) * 8,
                         "d2h_bytes_per_step": (int(prm_local.nbins) + 1) * 8 + nd * 8 * kw + nd * 4,
                         "ms_per_step": e_ms / args.e2e_steps, "steps": args.e2e_steps,
                         "api": "gkc_partition_host + exchange + gkc_count_device + gkc_count_copy_out"}
    ctx.close()
    if rank == 0:
        print(json.dumps(result))
    dist.barrier()
    dist.destroy_process_group()


def main():
    args = parse()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
    elif args.serve:
        run_serve(args)
    elif args.multi == "shard" or (dist_env()[1] > 1 and args.multi is None):
        run_shard(args, wl)
    else:
        run_ours(args, wl)


if __name__ == "__main__":
    main()
