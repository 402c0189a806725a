"""An exchange engine built on the oracle, for the multi-rank host-logic
tests on CPU (gloo): the same SendPlan / receive contract as the CUDA engine
(gkc_b200.shard.DeviceEngine), restated with numpy over the oracle's
partition.  TEST INFRASTRUCTURE."""
import numpy as np
import torch

import oracle_ffi as F
from gkc_b200 import shard


class OracleEngine:
    device = "cpu"

    def __init__(self, reads, offs, k, p, hpc, nbins):
        self.k, self.nbins = k, nbins
        s = F.oracle_partition(reads, offs, k, p, hpc, nbins)
        order = np.argsort(s.bin, kind="stable")  # bin order
        self.bin = s.bin[order].astype(np.int64)
        self.len = s.len[order].astype(np.uint64)
        self.chunks = [s.bytes[int(o):int(o) + (int(n) + 3) // 4] for o, n in zip(s.byte_off[order], s.len[order])]
        self.local = None

    def pack(self, bounds):
        nb = (self.len + 3) // 4
        dest = np.searchsorted(bounds, self.bin, side="right") - 1
        world = len(bounds) - 1
        skm_split = np.bincount(dest, minlength=world).astype(np.uint64)
        byte_split = np.bincount(dest, weights=nb, minlength=world).astype(np.uint64)
        off = np.concatenate([[0], np.cumsum(nb)]).astype(np.uint64)[:-1]
        run_start = np.concatenate([[0], np.cumsum(byte_split)]).astype(np.uint64)[dest]
        desc = (((off - run_start) << np.uint64(24)) | self.len).view(np.int64)
        data = np.concatenate(self.chunks) if self.chunks else np.zeros(0, np.uint8)
        bin_skm = np.bincount(self.bin, minlength=self.nbins).astype(np.uint64)
        km = np.where(self.len >= self.k, self.len - np.uint64(self.k - 1), 0)
        bin_kmers = np.bincount(self.bin, weights=km, minlength=self.nbins).astype(np.uint64)
        return shard.make_plan(torch, "cpu", bounds, torch.from_numpy(desc.copy()), torch.from_numpy(data.copy()),
                               skm_split, byte_split, bin_skm, bin_kmers)

    def receive(self, prm_local, seg_bin_skm, seg_bin_kmers, seg_bytes, recv_desc, recv_bytes):
        """Local partition in bin order, senders in order inside a bin."""
        d = recv_desc.numpy().view(np.uint64)
        data = recv_bytes.numpy()
        nbl = prm_local.nbins
        starts = np.concatenate([[0], np.cumsum(seg_bin_skm.sum(axis=1))]).astype(np.int64)
        bstarts = np.concatenate([[0], np.cumsum(seg_bytes)]).astype(np.uint64)
        bins, lens, offs, src = [], [], [], []
        for s in range(len(seg_bytes)):
            run = d[starts[s]:starts[s + 1]]
            bins.append(np.repeat(np.arange(nbl), seg_bin_skm[s].astype(np.int64)))
            lens.append(run & np.uint64(0xFFFFFF))
            offs.append((run >> np.uint64(24)) + bstarts[s])
            src.append(np.full(len(run), s))
        bins, lens, offs, src = (np.concatenate(x) if x else np.zeros(0, np.int64) for x in (bins, lens, offs, src))
        order = np.lexsort((src, bins))  # bin-major, then sender; stable inside a run
        self.local = F.Skms(bins[order].astype(np.uint32), lens[order].astype(np.uint32),
                            offs[order].astype(np.uint64), data)
        self.local_kmers = seg_bin_kmers.sum(axis=0)
        return self.local

    def count(self, nbl):
        return F.oracle_count_bins(self.local, self.k, nbl)
