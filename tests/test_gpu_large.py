"""Parity at the stated size of config 2 (10 Mbp genome, 30x of 150 bp reads:
2 M reads, 300 M bases, 240 M k-mers, 43.6 M distinct): the library's
partition and per-bin counts against 64-bit digests of the reference's own
output on the same reads (tests/golden/make_golden.py, "large" cases), for
the batched pipeline over several graph replays and for the plain per-stage
form.  The reads are generated on the device and checked byte for byte
against the host generator's digest first."""
import hashlib

import numpy as np
import pytest

import gkc_b200 as G
import golden_cases as GC
import oracle_ffi as F

pytestmark = pytest.mark.gpu


def _case():
    return GC.index()["large"]["config2"]


@pytest.fixture(scope="module")
def device_reads():
    import torch
    c = _case()
    L = G.lib()
    g = torch.empty(c["genome_len"], dtype=torch.uint8, device="cuda")
    assert L.gkc_synth_genome(1, c["seed"], c["genome_len"], 0.05, 0.01, g.data_ptr()) == 0
    n = c["coverage"] * c["genome_len"] // c["read_len"]
    reads = torch.empty(n * c["read_len"] + 64, dtype=torch.uint8, device="cuda")
    offs = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    assert L.gkc_synth_short_reads(1, c["seed"], g.data_ptr(), c["genome_len"], 0, n, c["read_len"], c["err"],
                                   reads.data_ptr(), offs.data_ptr()) == 0
    torch.cuda.synchronize()
    nb = n * c["read_len"]
    assert hashlib.sha256(reads[:nb].cpu().numpy().tobytes()).hexdigest() == c["reads_sha256"]
    return reads, offs, n, nb


def _digests(ctx, pv, cv, nbins):
    bin_off, lens, boff, packed, _ = ctx.partition_copy_out(pv)
    bins = np.repeat(np.arange(nbins, dtype=np.uint32), np.diff(bin_off).astype(np.int64))
    sd, _, _ = F.skm_digest64(bins, lens, boff, packed, nbins)
    bo, keys, counts = ctx.count_copy_out(cv)
    cd, _ = F.counts_digest64(bo, keys[:, 0], counts)
    return "%016x" % sd, "%016x" % cd


@pytest.mark.parametrize("mode", [G.MODE_BATCHED, G.MODE_PLAIN])
def test_config2_full_size(device_reads, mode):
    import torch
    c = _case()
    reads, offs, n, nb = device_reads
    prm = G.params(c["k"], c["p"], c["nbins"], c["hpc"])
    with G.Context(0) as ctx:
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        replays = 3 if mode == G.MODE_BATCHED else 1
        for r in range(replays):
            pv, cv = ctx.pipeline_device(reads, nb, offs, n, prm, mode)
            assert int(pv.n_superkmers) == c["n_skm"]
            assert int(cv.n_kmers) == c["n_kmers"]
            assert int(cv.n_distinct) == c["n_distinct"], f"replay {r}"
            sd, cd = _digests(ctx, pv, cv, c["nbins"])
            assert sd == c["skm_digest64"], f"partition differs (replay {r})"
            assert cd == c["counts_digest64"], f"counts differ (replay {r})"
