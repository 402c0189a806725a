"""Bin sharding over several GPUs, one process per GPU.

Every rank partitions its own reads.  Owner r of G holds the contiguous bins
[r*nbins//G, (r+1)*nbins//G) and counts them after one exchange of packed
superkmers, so every k-mer of the job is counted once, by the owner of its
bin.  The exchange is three all-to-alls: a small one of run sizes and per-bin
counts, then the superkmer descriptors, then their packed bytes.

The steps are kept apart so that one piece of logic serves every transport:
  pack (SendPlan)   what one rank sends, built on its device
  exchange_dist     the transfer between processes (torch.distributed:
                    NCCL between GPUs, gloo on CPU)
  exchange_local    the transfer between engines of one process (several
                    contexts sharing one device)
  receive           the received runs imported as the rank's partition
An engine does pack and receive; DeviceEngine is the CUDA one, through the C
ABI (gkc_exchange_pack / gkc_partition_import).
"""
from dataclasses import dataclass

import numpy as np

import gkc_b200 as G


def owner_bounds(nbins, world):
    """bin_lo[r] .. bin_lo[r+1]: the bins rank r owns (world + 1 entries)."""
    if nbins < world:
        raise ValueError(f"{nbins} bins cannot be shared by {world} ranks")
    return np.array([r * nbins // world for r in range(world + 1)], np.uint32)


@dataclass
class SendPlan:
    desc: object          # int64 tensor: descriptors, destination after destination
    data: object          # uint8 tensor: packed bytes, destination after destination
    skm_split: np.ndarray  # superkmers per destination
    byte_split: np.ndarray  # bytes per destination
    meta: object          # int64 tensor: per destination [skm, bytes, bin_skm..., bin_kmers...]
    meta_split: list


def make_plan(torch, device, bounds, desc, data, skm_split, byte_split, bin_skm, bin_kmers):
    """Adds the metadata runs: destination d gets its run sizes and, for each
    of its bins, this rank's superkmers and k-mers there."""
    parts, split = [], []
    for d in range(len(bounds) - 1):
        lo, hi = int(bounds[d]), int(bounds[d + 1])
        run = np.concatenate([[skm_split[d], byte_split[d]], bin_skm[lo:hi], bin_kmers[lo:hi]]).astype(np.int64)
        parts.append(run)
        split.append(len(run))
    meta = torch.from_numpy(np.concatenate(parts)).to(device)
    return SendPlan(desc, data, np.asarray(skm_split, np.uint64), np.asarray(byte_split, np.uint64), meta, split)


def parse_meta(recv_meta, n_src, nbl):
    """Received metadata (one run of 2 + 2*nbl words per sender) ->
    (skm per sender, bytes per sender, sender x bin superkmers, sender x bin k-mers)."""
    m = np.asarray(recv_meta, np.int64).reshape(n_src, 2 + 2 * nbl).astype(np.uint64)
    return m[:, 0].copy(), m[:, 1].copy(), m[:, 2:2 + nbl].copy(), m[:, 2 + nbl:].copy()


def local_params(prm, bounds, rank):
    return G.params(prm.k, prm.p, int(bounds[rank + 1] - bounds[rank]), prm.hpc)


class DeviceEngine:
    """The CUDA engine: a context holding this rank's partition."""

    def __init__(self, ctx, view, device="cuda"):
        import torch
        self.torch, self.ctx, self.view, self.device = torch, ctx, view, device
        self.launches = 0  # kernels the pack and the import launched

    def _settle(self):
        # torch's stream and the library's are different: buffers pass
        # between them only when the producing stream is done
        self.torch.cuda.current_stream(self.device).synchronize()

    def pack(self, bounds):
        t = self.torch
        desc = t.empty(int(self.view.n_superkmers), dtype=t.int64, device=self.device)
        data = t.empty(int(self.view.n_packed_bytes), dtype=t.uint8, device=self.device)
        self._settle()  # memory torch hands out may still be read by its stream
        skm_split, byte_split, bin_skm, bin_kmers = self.ctx.exchange_pack(self.view, bounds, desc, data)
        self.launches += int(self.ctx.timings().launches)
        data = data[:int(byte_split.sum())]
        return make_plan(t, self.device, bounds, desc, data, skm_split, byte_split, bin_skm, bin_kmers)

    def receive(self, prm_local, seg_bin_skm, seg_bin_kmers, seg_bytes, recv_desc, recv_bytes):
        self._settle()  # the received runs were written on torch's side
        self.view = self.ctx.partition_import(prm_local, seg_bin_skm, seg_bin_kmers, seg_bytes, recv_desc,
                                              recv_bytes)
        self.launches += int(self.ctx.timings().launches)
        return self.view


def exchange_dist(engine, prm, group=None):
    """The exchange between the ranks of a process group; every rank calls it
    with the same prm.  -> (local params, owner bounds, received view)."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    bounds = owner_bounds(prm.nbins, world)
    plan = engine.pack(bounds)
    nbl = int(bounds[rank + 1] - bounds[rank])
    recv_meta = torch.empty(world * (2 + 2 * nbl), dtype=torch.int64, device=engine.device)
    dist.all_to_all_single(recv_meta, plan.meta, [2 + 2 * nbl] * world, plan.meta_split, group=group)
    seg_skm, seg_bytes, seg_bin_skm, seg_bin_kmers = parse_meta(recv_meta.cpu().numpy(), world, nbl)
    recv_desc = torch.empty(int(seg_skm.sum()), dtype=torch.int64, device=engine.device)
    dist.all_to_all_single(recv_desc, plan.desc, [int(x) for x in seg_skm], [int(x) for x in plan.skm_split],
                           group=group)
    recv_bytes = torch.empty(int(seg_bytes.sum()), dtype=torch.uint8, device=engine.device)
    dist.all_to_all_single(recv_bytes, plan.data, [int(x) for x in seg_bytes], [int(x) for x in plan.byte_split],
                           group=group)
    prm_local = local_params(prm, bounds, rank)
    view = engine.receive(prm_local, seg_bin_skm, seg_bin_kmers, seg_bytes, recv_desc, recv_bytes)
    return prm_local, bounds, view


def exchange_local(engines, prm):
    """The same exchange among engines of one process (rank = list index).
    -> (owner bounds, [local params per rank])."""
    import torch
    world = len(engines)
    bounds = owner_bounds(prm.nbins, world)
    plans = [e.pack(bounds) for e in engines]
    # run starts inside every sender's buffers
    moff = [np.concatenate([[0], np.cumsum(p.meta_split)]) for p in plans]
    soff = [np.concatenate([[0], np.cumsum(p.skm_split.astype(np.int64))]) for p in plans]
    boff = [np.concatenate([[0], np.cumsum(p.byte_split.astype(np.int64))]) for p in plans]
    out = []
    for r, e in enumerate(engines):
        nbl = int(bounds[r + 1] - bounds[r])
        meta = torch.cat([p.meta[int(moff[s][r]):int(moff[s][r + 1])].cpu() for s, p in enumerate(plans)])
        seg_skm, seg_bytes, seg_bin_skm, seg_bin_kmers = parse_meta(meta.numpy(), world, nbl)
        recv_desc = torch.cat([p.desc[int(soff[s][r]):int(soff[s][r + 1])] for s, p in enumerate(plans)])
        recv_bytes = torch.cat([p.data[int(boff[s][r]):int(boff[s][r + 1])] for s, p in enumerate(plans)])
        prm_local = local_params(prm, bounds, r)
        e.receive(prm_local, seg_bin_skm, seg_bin_kmers, seg_bytes, recv_desc, recv_bytes)
        out.append(prm_local)
    return bounds, out


def sharded_count_device(ctx, d_reads, n_bytes, d_offs, n_reads, prm, group=None, mode=G.MODE_BATCHED,
                         device="cuda"):
    """This rank's reads partitioned, superkmers exchanged by bin owner, the
    owned bins counted.  -> (count view of the owned bins, owner bounds):
    local bin b is global bin bounds[rank] + b."""
    view = ctx.partition_device(d_reads, n_bytes, d_offs, n_reads, prm)
    prm_local, bounds, _ = exchange_dist(DeviceEngine(ctx, view, device), prm, group)
    return ctx.count_device(prm_local, mode), bounds
