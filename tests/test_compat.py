"""The drop-in for GKC's two GPU entry points (gkc_b200/compat/gkc_compat.cpp):
it compiles as C++14 against GKC's own headers and defines the functions
they declare (CPU test, where the GKC tree exists), and a driver written the
way GKC's own driver calls GenSuperkmerGPU (with SKMStore::add_skms as the
callback) and kmc_counting_GPU (from a pool of threads) gets the oracle's
per-bin superkmer multisets and sorted (k-mer, count) lists (GPU test)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_ffi as F
from gkc_b200 import build as B
from gkc_b200 import synth

GKC_SRC = os.environ.get("GKC_REFERENCE_DIR", "/root/reference")


@pytest.mark.skipif(not os.path.isfile(os.path.join(GKC_SRC, "gkc_cuda.hpp")),
                    reason="GKC source tree not present (the drop-in is compiled against its headers)")
def test_compiles_against_gkc_headers_as_cpp14():
    lib = B.build_compat(GKC_SRC)
    names = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True).stdout
    for sym in ("GenSuperkmerGPU(PinnedCSR&, int, int, bool, CUDAParams, CountTask, int, std::function<void (T_h_data)>)",
                "kmc_counting_GPU(unsigned char, SKMStore&, int, unsigned short, unsigned short, "
                "std::vector<T_kmc, std::allocator<T_kmc> >&)",
                "PinnedCSR::PinnedCSR(std::vector<ReadPtr, std::allocator<ReadPtr> >&, bool)",
                "PinnedCSR::~PinnedCSR()", "GPUReset(int)", "CalcSKMPartSize_instream("):
        assert sym in names, sym
    assert os.access(B.COMPAT_DRIVER, os.X_OK)


def run_driver(reads, offs, k, p, hpc, nbins, threads=4):
    with tempfile.TemporaryDirectory() as d:
        src, out = os.path.join(d, "reads.bin"), os.path.join(d, "out.bin")
        with open(src, "wb") as f:
            f.write(np.uint64(len(offs) - 1).tobytes())
            f.write(np.ascontiguousarray(offs, np.uint64).tobytes())
            f.write(np.ascontiguousarray(reads, np.uint8).tobytes())
        r = subprocess.run([B.COMPAT_DRIVER, src, str(k), str(p), str(hpc), str(nbins), str(threads), out],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        data = open(out, "rb").read()
    pos = 0

    def take(fmt, n=1):
        nonlocal pos
        a = np.frombuffer(data, fmt, n, pos)
        pos += a.nbytes
        return a

    ms = []
    for _ in range(nbins):
        items = []
        for _ in range(int(take(np.uint64)[0])):
            ln = int(take(np.uint32)[0])
            items.append((ln, bytes(take(np.uint8, (ln + 3) // 4))))
        ms.append(sorted(items))
    ret, keys, counts, bin_off = [], [], [], [0]
    for _ in range(nbins):
        ret.append(int(take(np.uint64)[0]))
        m = int(take(np.uint64)[0])
        for _ in range(m):
            keys.append(int(take(np.uint64)[0]))
            counts.append(int(take(np.uint32)[0]))
        bin_off.append(len(keys))
    return ms, ret, np.array(bin_off, np.uint64), np.array(keys, np.uint64), np.array(counts, np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["config1", "hpc"])
def test_driver_matches_oracle(case):
    if not os.access(B.COMPAT_DRIVER, os.X_OK):
        pytest.fail("the drop-in's test driver was not built (gkc_b200.build.build_compat)")
    if case == "config1":
        reads, offs = synth.iid_reads(3, 6000, 150, 0.001)  # three batches of 2048 reads
        k, p, hpc, nbins = 31, 11, 0, 64
    else:
        r = np.random.default_rng(4)
        parts, offs = [], [0]
        for _ in range(300):
            L = int(r.integers(60, 400))
            s = np.repeat(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, L)], r.integers(1, 4, L))[:L]
            parts.append(s)
            offs.append(offs[-1] + len(s))
        reads, offs = np.concatenate(parts), np.array(offs, np.uint64)
        k, p, hpc, nbins = 25, 15, 1, 32
    ms, ret, bin_off, keys, counts = run_driver(reads, offs, k, p, hpc, nbins)
    o = F.oracle_partition(reads, offs, k, p, hpc, nbins)
    assert ms == [sorted(b) for b in o.multisets(nbins)]
    want = F.oracle_count_bins(o, k, nbins)
    assert np.array_equal(bin_off, want["bin_off"])
    assert np.array_equal(keys, want["keys_lo"])
    assert np.array_equal(counts, want["counts"])
    assert ret == [int(x) for x in np.diff(want["bin_off"])]
