"""Builds the in-tree shared library gkc_b200/libgkc_b200.so for sm_100a.

Each .cu under csrc/ is compiled with nvcc (in parallel) into _build/ and
linked into one shared library.  Usage: python -m gkc_b200.build [--force]
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgkc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "--extended-lambda", "-I" + os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _deps_mtime():
    return max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)) if os.listdir(CSRC) else 0


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime():
        return obj
    cmd = [NVCC] + ARCH + FLAGS + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + cmd[1:]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


COMPAT_SRC = os.path.join(HERE, "compat", "gkc_compat.cpp")
COMPAT_DIR = os.path.join(BUILD, "compat")
COMPAT_LIB = os.path.join(COMPAT_DIR, "libgkc_compat.so")
COMPAT_DRIVER = os.path.join(COMPAT_DIR, "compat_driver")


def build_compat(gkc_src_dir):
    """Compiles the drop-in for GKC's GPU entry points (compat/gkc_compat.cpp)
    as C++14 against the GKC source tree's own headers (gkc_cuda.hpp,
    kmer_counting.hpp, superkmers.hpp), as a GKC build would, into
    _build/compat/libgkc_compat.so, plus the test driver that uses it the way
    GKC's driver does.  Returns the library path."""
    os.makedirs(COMPAT_DIR, exist_ok=True)
    lib = build()
    cuda = os.path.dirname(os.path.dirname(NVCC))
    inc = ["-I" + gkc_src_dir, "-I" + os.path.join(HERE, "..", "include"), "-I" + os.path.join(cuda, "include")]
    link = ["-L" + HERE, "-lgkc_b200", "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-lpthread",
            "-Wl,-rpath," + HERE + ":" + COMPAT_DIR + ":" + os.path.join(cuda, "lib64")]
    cmds = [["g++", "-std=c++14", "-O2", "-fPIC", "-shared", "-w"] + inc + [COMPAT_SRC, "-o", COMPAT_LIB] + link,
            ["g++", "-std=c++14", "-O2", "-w"] + inc +
            [os.path.join(HERE, "..", "tests", "c_consumer", "compat_driver.cpp"), "-o", COMPAT_DRIVER,
             "-L" + COMPAT_DIR, "-lgkc_compat"] + link]
    for cmd in cmds:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compat build failed:\n" + " ".join(cmd) + "\n" + r.stderr)
    return COMPAT_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
