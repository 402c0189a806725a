"""Bin sharding on the GPU: the pack and import kernels (gkc_exchange_pack,
gkc_partition_import) with the exchange of gkc_b200.shard.  Several ranks
are contexts on one device exchanging through exchange_local (no kernel
waits on another); one NCCL rank runs exchange_dist.  The owners' counts put
together must equal the oracle's counts of all reads."""
import os

import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F
from gkc_b200 import shard

pytestmark = pytest.mark.gpu


def _reads(seed, n, lo, hi):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    b = np.frombuffer(b"ACGTacgtU", np.uint8)[r.integers(0, 9, int(offs[-1]))].copy()
    b[r.random(len(b)) < 0.01] = ord("N")
    return b, offs


def _to_dev(torch, reads, offs, lo, hi):
    o = offs[lo:hi + 1]
    r = reads[int(o[0]):int(o[-1])].copy()
    o = (o - o[0]).astype(np.uint64)
    return torch.from_numpy(r).cuda(), torch.from_numpy(o.view(np.int64)).cuda(), len(r), len(o) - 1


def _check_owner(ctx, cv, bounds, rank, want, kw):
    bin_off, keys, counts = ctx.count_copy_out(cv)
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    for b in range(lo, hi):
        w0, w1 = int(want["bin_off"][b]), int(want["bin_off"][b + 1])
        g0, g1 = int(bin_off[b - lo]), int(bin_off[b - lo + 1])
        assert np.array_equal(keys[g0:g1, 0], want["keys_lo"][w0:w1]), b
        if kw > 1:
            assert np.array_equal(keys[g0:g1, 1], want["keys_hi"][w0:w1]), b
        assert np.array_equal(counts[g0:g1], want["counts"][w0:w1]), b


CASES = [
    # world, mode, k, p, hpc, nbins
    (1, G.MODE_BATCHED, 31, 11, 0, 64),
    (2, G.MODE_BATCHED, 31, 11, 0, 256),
    (3, G.MODE_PLAIN, 21, 9, 1, 37),
    (4, G.MODE_BATCHED, 45, 15, 0, 64),   # 128-bit keys
]


@pytest.mark.parametrize("world,mode,k,p,hpc,nb", CASES)
def test_virtual_ranks_on_one_device(world, mode, k, p, hpc, nb):
    import torch
    reads, offs = _reads(80 + world, 600, 50, 700)
    want = F.oracle_count_bins(F.oracle_partition(reads, offs, k, p, hpc, nb), k, nb)
    prm = G.params(k, p, nb, hpc)
    n = len(offs) - 1
    cuts = [n * r // world for r in range(world + 1)]
    if world > 1:
        cuts[1] = max(1, n // (3 * world))  # uneven shares
    ctxs = [G.Context(0) for _ in range(world)]
    try:
        engines, keep = [], []
        for r in range(world):
            d_reads, d_offs, nbytes, nreads = _to_dev(torch, reads, offs, cuts[r], cuts[r + 1])
            keep.append((d_reads, d_offs))
            v = ctxs[r].partition_device(d_reads, nbytes, d_offs, nreads, prm)
            engines.append(shard.DeviceEngine(ctxs[r], v))
        bounds, prms = shard.exchange_local(engines, prm)
        kmers = 0
        for r in range(world):
            assert engines[r].view.nbins == prms[r].nbins
            kmers += engines[r].view.n_kmers
            cv = ctxs[r].count_device(prms[r], mode)
            _check_owner(ctxs[r], cv, bounds, r, want, 2 if k > 32 else 1)
        assert kmers == int(want["counts"].astype(np.uint64).sum())
    finally:
        for c in ctxs:
            c.close()


def test_imported_partition_matches_oracle_bins():
    """The imported partition of each owner holds exactly the superkmers of
    its bins (as multisets of length and packed bytes)."""
    import torch
    reads, offs = _reads(90, 300, 40, 600)
    k, p, nb, world = 27, 11, 48, 3
    o = F.oracle_partition(reads, offs, k, p, 0, nb)
    want = o.multisets(nb)
    n = len(offs) - 1
    cuts = [n * r // world for r in range(world + 1)]
    ctxs = [G.Context(0) for _ in range(world)]
    try:
        engines, keep = [], []
        for r in range(world):
            d_reads, d_offs, nbytes, nreads = _to_dev(torch, reads, offs, cuts[r], cuts[r + 1])
            keep.append((d_reads, d_offs))
            engines.append(shard.DeviceEngine(ctxs[r], ctxs[r].partition_device(d_reads, nbytes, d_offs, nreads,
                                                                                G.params(k, p, nb))))
        bounds, _ = shard.exchange_local(engines, G.params(k, p, nb))
        for r in range(world):
            bo, lens, boff, packed, mm = ctxs[r].partition_copy_out(engines[r].view)
            nbl = int(bounds[r + 1] - bounds[r])
            bins = np.repeat(np.arange(nbl, dtype=np.uint32), np.diff(bo).astype(np.int64))
            got = F.Skms(bins, lens, boff, packed).multisets(nbl)
            assert got == want[int(bounds[r]):int(bounds[r + 1])]
            assert np.all(mm == 0xFFFFFFFF)
            sizes, _ = ctxs[r].partition_balance(engines[r].view)
            assert np.array_equal(sizes, F.oracle_partition_sizes(o, nb)[int(bounds[r]):int(bounds[r + 1])])
    finally:
        for c in ctxs:
            c.close()


def test_nccl_single_rank_exchange():
    """exchange_dist over a one-rank NCCL group: the real collective path."""
    import torch
    import torch.distributed as dist
    reads, offs = _reads(91, 400, 60, 500)
    k, p, nb = 31, 11, 32
    want = F.oracle_count_bins(F.oracle_partition(reads, offs, k, p, 0, nb), k, nb)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(29000 + os.getpid() % 2000)
    import datetime
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        with G.Context(0) as c:
            d_reads, d_offs, nbytes, nreads = _to_dev(torch, reads, offs, 0, len(offs) - 1)
            cv, bounds = shard.sharded_count_device(c, d_reads, nbytes, d_offs, nreads, G.params(k, p, nb))
            _check_owner(c, cv, bounds, 0, want, 1)
    finally:
        dist.destroy_process_group()
