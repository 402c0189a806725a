"""Generates the golden fixtures in this directory from the REFERENCE itself:
its kernels, superkmer store and counting step compiled from its sources
(oracle/Makefile -> oracle/_ref/libgkcref.so).  Run in a tree where that
library was built:  python tests/golden/make_golden.py

Small cases store inputs and full outputs (case_<name>.npz); larger cases
store the generator parameters plus SHA-256 digests (golden.json), their
reads being regenerated by gkc_b200.synth.  The "large" cases (config 2 at its
stated size: 2 M reads, 240 M k-mers) store 64-bit digests instead
(oracle_ffi.counts_digest64 / skm_digest64), which the GPU tests recompute
on the library's output; `--large` regenerates only those.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle_ffi as F  # noqa: E402
import parity as P  # noqa: E402
from gkc_b200 import synth  # noqa: E402


def mixed_reads(seed, n, lo, hi):
    """Reads of lengths in [lo, hi] with N, lowercase and U mixed in."""
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    tot = int(offs[-1])
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, tot)].copy()
    b[r.random(tot) < 0.01] = ord("N")
    b[r.random(tot) < 0.003] = ord("U")
    lc = r.random(tot) < 0.02
    b[lc] |= 0x20
    return b, offs


def homopolymer_reads(seed, n, lo, hi):
    """Reads built from runs of 1-6 equal bases (for HPC)."""
    r = np.random.default_rng(seed)
    out, offs = [], [0]
    for _ in range(n):
        L = int(r.integers(lo, hi + 1))
        s = []
        while len(s) < L:
            s.extend([b"ACGTN"[int(r.integers(0, 4 if r.random() > 0.01 else 5))]] * int(r.integers(1, 7)))
        out.append(bytes(s[:L]))
        offs.append(offs[-1] + L)
    return np.frombuffer(b"".join(out), np.uint8).copy(), np.array(offs, np.uint64)


FULL_CASES = {
    # name: (reads generator, k, p, hpc, nbins)
    "iid_n": (lambda: synth.iid_reads(7, 300, 150, 0.01), 31, 11, 0, 256),
    "mixed_defaults": (lambda: mixed_reads(11, 200, 21, 600), 21, 7, 0, 31),
    "hpc": (lambda: homopolymer_reads(13, 60, 40, 2000), 25, 15, 1, 64),
    "k32": (lambda: mixed_reads(17, 150, 32, 400), 32, 16, 0, 17),
    "exact_k": (lambda: mixed_reads(19, 100, 31, 33), 31, 11, 0, 256),
}

DIGEST_CASES = {
    # config 1 at its stated size
    "config1": dict(gen="iid", seed=1, n_reads=20000, read_len=150, n_rate=0.001, k=31, p=11,
                    hpc=0, nbins=256),
    # genome-derived short reads (config-2 generator at 200 kbp)
    "genome200k": dict(gen="genome", seed=2, genome_len=200000, coverage=30, read_len=150,
                       err=0.005, k=31, p=11, hpc=0, nbins=256),
}


def gen_digest_case(c):
    if c["gen"] == "iid":
        return synth.iid_reads(c["seed"], c["n_reads"], c["read_len"], c["n_rate"])
    g = synth.genome(c["seed"], c["genome_len"])
    n = c["coverage"] * c["genome_len"] // c["read_len"]
    return synth.short_reads(c["seed"], g, n, c["read_len"], c["err"])


LARGE_CASES = {
    # config 2 at its stated size: 10 Mbp genome, 30x of 150 bp reads (2 M reads)
    "config2": dict(gen="genome", seed=2026, genome_len=10_000_000, coverage=30, read_len=150,
                    err=0.005, k=31, p=11, hpc=0, nbins=256),
}


def make_large(index):
    index.setdefault("large", {})
    for name, c in LARGE_CASES.items():
        reads, offs = gen_digest_case(c)
        skm = F.ref_partition(reads, offs, c["k"], c["p"], c["hpc"], c["nbins"], n_threads=os.cpu_count())
        sd, _, _ = F.skm_digest64(skm.bin, skm.len, skm.byte_off, skm.bytes, c["nbins"])
        cnt = F.ref_count_bins(skm, c["k"], c["nbins"], n_threads=os.cpu_count())
        cd, _ = F.counts_digest64(cnt["bin_off"], cnt["keys_lo"], cnt["counts"])
        d = dict(c)
        d.update(reads_sha256=P.bytes_digest(reads), n_reads=len(offs) - 1, n_skm=int(len(skm.bin)),
                 skm_bases=int(skm.len.astype(np.uint64).sum()), n_distinct=int(len(cnt["keys_lo"])),
                 n_kmers=int(cnt["counts"].astype(np.uint64).sum()),
                 skm_digest64="%016x" % sd, counts_digest64="%016x" % cd)
        index["large"][name] = d
        print(name, d["n_skm"], d["n_distinct"], d["n_kmers"], d["skm_digest64"], d["counts_digest64"])


def run_ref(reads, offs, k, p, hpc, nbins):
    skm = F.ref_partition(reads, offs, k, p, hpc, nbins)
    ms = skm.multisets(nbins)
    cnt = F.ref_count_bins(skm, k, nbins)
    return ms, cnt


def main():
    assert F.ref_available(), "build oracle/_ref first (make -C oracle)"
    if "--large" in sys.argv:
        with open(os.path.join(HERE, "golden.json")) as f:
            index = json.load(f)
        make_large(index)
        with open(os.path.join(HERE, "golden.json"), "w") as f:
            json.dump(index, f, indent=1, sort_keys=True)
        return
    index = {"full": {}, "digest": {}}
    for name, (gen, k, p, hpc, nbins) in FULL_CASES.items():
        reads, offs = gen()
        ms, cnt = run_ref(reads, offs, k, p, hpc, nbins)
        fb, fl, fo, fd = P.flatten_multisets(ms)
        np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), reads=reads, offs=offs,
                            skm_bin=fb, skm_len=fl, skm_off=fo, skm_bytes=fd,
                            cnt_bin_off=cnt["bin_off"], cnt_keys=cnt["keys_lo"],
                            cnt_counts=cnt["counts"], cnt_returned=cnt["returned"])
        index["full"][name] = dict(k=k, p=p, hpc=hpc, nbins=nbins, n_reads=len(offs) - 1,
                                   n_skm=len(fb), n_distinct=int(len(cnt["keys_lo"])),
                                   partition_sha256=P.partition_digest(ms),
                                   counts_sha256=P.counts_digest(cnt["bin_off"], cnt["keys_lo"],
                                                                 cnt["counts"]))
        print(name, index["full"][name]["n_skm"], index["full"][name]["n_distinct"])
    for name, c in DIGEST_CASES.items():
        reads, offs = gen_digest_case(c)
        ms, cnt = run_ref(reads, offs, c["k"], c["p"], c["hpc"], c["nbins"])
        n_skm = sum(len(b) for b in ms)
        d = dict(c)
        d.update(reads_sha256=P.bytes_digest(reads), offs_sha256=P.bytes_digest(offs),
                 n_skm=n_skm, skm_bases=int(sum(l for b in ms for l, _ in b)),
                 n_distinct=int(len(cnt["keys_lo"])),
                 n_kmers=int(cnt["counts"].astype(np.uint64).sum()),
                 partition_sha256=P.partition_digest(ms),
                 counts_sha256=P.counts_digest(cnt["bin_off"], cnt["keys_lo"], cnt["counts"]))
        index["digest"][name] = d
        print(name, n_skm, d["n_distinct"], d["n_kmers"])
    make_large(index)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
