"""CPU-side checks of the shipped library: it loads, exports every symbol the
public header declares, rejects use without a device, and its host-side
generators produce the same bytes as the numpy mirror."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import gkc_b200 as G
from gkc_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "gkc", "gkc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gkc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    L = G.lib()
    missing = [s for s in header_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert L.gkc_abi_version() == 1


def test_binding_covers_header():
    bound = {n for n, _, _ in G.SIGNATURES}
    assert set(header_symbols()) <= bound


def test_status_strings():
    L = G.lib()
    assert L.gkc_status_string(0) == b"ok"
    assert L.gkc_status_string(5) == b"HBM budget exceeded"


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and False, reason="")
def test_ctx_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    st = G.lib().gkc_ctx_create(0, 0, C.byref(h))
    assert st == 3  # GKC_ERR_NO_DEVICE


def test_host_iid_generator_matches_numpy():
    n, L = 50, 150
    out = np.zeros(n * L, np.uint8)
    offs = np.zeros(n + 1, np.uint64)
    assert G.lib().gkc_synth_iid_reads(0, 5, n, L, 0.01, out.ctypes.data, offs.ctypes.data) == 0
    r2, o2 = synth.iid_reads(5, n, L, 0.01)
    assert np.array_equal(out, r2) and np.array_equal(offs, o2)


def test_host_genome_and_short_reads_match_numpy():
    Gl = 60000
    g = np.zeros(Gl, np.uint8)
    assert G.lib().gkc_synth_genome(0, 3, Gl, 0.05, 0.01, g.ctypes.data) == 0
    g2 = synth.genome(3, Gl)
    assert np.array_equal(g, g2)
    n, L = 300, 150
    out = np.zeros(n * L, np.uint8)
    offs = np.zeros(n + 1, np.uint64)
    assert G.lib().gkc_synth_short_reads(0, 3, g.ctypes.data, Gl, 7, n, L, 0.005, out.ctypes.data,
                                         offs.ctypes.data) == 0
    r2, o2 = synth.short_reads(3, g2, n, L, 0.005, first_read=7)
    assert np.array_equal(out, r2)


def test_host_long_reads_are_deterministic():
    Gl = 100000
    g = np.zeros(Gl, np.uint8)
    G.lib().gkc_synth_genome(0, 4, Gl, 0.05, 0.01, g.ctypes.data)
    offs = np.zeros(1001, np.uint64)
    n = G.lib().gkc_synth_long_read_offsets(4, 8000.0, 0.6, 1000, 50000, 200000, 1000, offs.ctypes.data)
    assert 5 < n < 200 and offs[n] >= 200000
    lens = np.diff(offs[:n + 1])
    assert lens.min() >= 1000 and lens.max() <= 50000
    a = np.zeros(int(offs[n]), np.uint8)
    b = np.zeros(int(offs[n]), np.uint8)
    for buf in (a, b):
        assert G.lib().gkc_synth_long_reads(0, 4, g.ctypes.data, Gl, n, offs.ctypes.data, buf.ctypes.data) == 0
    assert np.array_equal(a, b)
    assert set(np.unique(a).tolist()) <= set(b"ACGT")


def test_c_consumer_of_the_header(tmp_path):
    """The header compiles as C11 with warnings as errors, and a C program
    linked against the library calls its host-side entry points."""
    import shutil
    import subprocess
    import db_format as D
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "consumer"
    libdir = os.path.join(ROOT, "gkc_b200")
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_consumer", "consumer.c"), "-o", str(exe), "-L", libdir,
                    "-lgkc_b200", f"-Wl,-rpath,{libdir}"], check=True)
    fa = tmp_path / "r.fa"
    fa.write_text(">a\nACGTACGT\n>b two lines\nGGGGCCCC\nAAAA\n")
    D.write(str(tmp_path / "db"), 31, np.array([[5], [77], [1 << 40]], np.uint64),
            np.array([2, 9, 300], np.uint32), 1, 1000)
    r = subprocess.run([str(exe), str(fa), str(tmp_path / "db")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok ") == 12


def test_cpp_nccl_sharding_example_compiles(tmp_path):
    """The C++ driver of the bin-sharded count over NCCL
    (tests/c_consumer/shard_nccl.cpp) compiles against the header."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    cuda_inc = "/usr/local/cuda/include"
    nccl_dirs = [d for d in ("/usr/include",) if os.path.exists(os.path.join(d, "nccl.h"))]
    if cxx is None or not nccl_dirs or not os.path.exists(os.path.join(cuda_inc, "cuda_runtime.h")):
        pytest.skip("no C++ compiler, CUDA headers or NCCL header")
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-c", "-I", os.path.join(ROOT, "include"),
                    "-I", cuda_inc, "-I", nccl_dirs[0],
                    os.path.join(ROOT, "tests", "c_consumer", "shard_nccl.cpp"), "-o", str(tmp_path / "s.o")],
                   check=True)
