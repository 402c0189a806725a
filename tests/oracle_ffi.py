"""ctypes bindings to the oracle libraries under oracle/ (test infrastructure only).

liboracle.so is the plain-C restatement; oracle/_ref/libgkcref.so is the
reference's own code compiled from its sources (present only where it was
built).  Results are returned as numpy arrays.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgkcref.so")

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)


class OrcSkms(C.Structure):
    _fields_ = [("n_skm", C.c_uint64), ("n_bytes", C.c_uint64), ("bin", u32p), ("len", u32p),
                ("byte_off", u64p), ("read_id", u64p), ("start", u32p), ("minimizer", u32p),
                ("bytes", u8p)]


class OrcCounts(C.Structure):
    _fields_ = [("nbins", C.c_uint32), ("n_distinct", C.c_uint64), ("bin_off", u64p),
                ("keys_lo", u64p), ("keys_hi", u64p), ("counts", u32p)]


class OrcPos(C.Structure):
    _fields_ = [("n_distinct", C.c_uint64), ("n_pos", C.c_uint64), ("keys_lo", u64p),
                ("keys_hi", u64p), ("pos_off", u64p), ("pos", u32p)]


class RefSkms(C.Structure):
    _fields_ = [("n_skm", C.c_uint64), ("n_bytes", C.c_uint64), ("bin", u32p), ("len", u32p),
                ("byte_off", u64p), ("bytes", u8p)]


class RefCounts(C.Structure):
    _fields_ = [("nbins", C.c_uint32), ("n_distinct", C.c_uint64), ("bin_off", u64p),
                ("keys", u64p), ("counts", u32p), ("returned", u64p)]


def _arr(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(int(n),)).astype(dtype, copy=True)


def _ptr(a, t):
    return a.ctypes.data_as(t)


_orc = None
_ref = None


def oracle():
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE_SO)
        lib.orc_partition.argtypes = [u8p, u64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(OrcSkms)]
        lib.orc_count_bins.argtypes = [C.POINTER(OrcSkms), C.c_int, C.c_int, C.POINTER(OrcCounts)]
        lib.orc_count_packed.argtypes = [u32p, u64p, u8p, C.c_uint64, C.c_int, C.POINTER(OrcCounts)]
        lib.orc_window_minimizers.argtypes = [u8p, C.c_int32, C.c_int, C.c_int, u32p]
        lib.orc_window_minimizer_pos.argtypes = [u8p, C.c_int32, C.c_int, C.c_int, u32p, u8p,
                                                 C.POINTER(C.c_int8)]
        lib.orc_hpc.argtypes = [u8p, u64p, C.c_int64, u8p, C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32)]
        lib.orc_subsample_positions.argtypes = [u8p, u64p, C.c_int64, C.c_int, C.c_int, C.c_uint32,
                                                C.POINTER(OrcPos)]
        lib.orc_skms_free.argtypes = [C.POINTER(OrcSkms)]
        lib.orc_counts_free.argtypes = [C.POINTER(OrcCounts)]
        lib.orc_poslists_free.argtypes = [C.POINTER(OrcPos)]
        _orc = lib
    return _orc


# the reference built as shipped (new_filter2) and with its other FILTER_KERNEL variants
REF_FILTER_SO = {0: REF_SO, 1: REF_SO.replace("libgkcref", "libgkcref_mm_filter"),
                 2: REF_SO.replace("libgkcref", "libgkcref_new_filter"),
                 3: REF_SO.replace("libgkcref", "libgkcref_sign_filter")}
_refs = {}


def ref_available(filter_id=0):
    return os.path.exists(REF_FILTER_SO[filter_id])


def set_filter(filter_id):
    """Minimizer filter of the C restatement for later calls (0 = new_filter2)."""
    lib = oracle()
    lib.orc_set_filter.argtypes = [C.c_int]
    lib.orc_set_filter(int(filter_id))


def reference(filter_id=0):
    global _ref
    if filter_id in _refs:
        return _refs[filter_id]
    if filter_id != 0 or _ref is None:
        lib = C.CDLL(REF_FILTER_SO[filter_id])
        lib.ref_partition.argtypes = [C.c_char_p, u64p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.POINTER(RefSkms)]
        lib.ref_count_bins.argtypes = [C.POINTER(RefSkms), C.c_int, C.c_int, C.c_int,
                                       C.POINTER(RefCounts)]
        lib.ref_pipeline.argtypes = [C.c_char_p, u64p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_int, u64p, u64p]
        lib.ref_pipeline_counts.argtypes = [C.c_char_p, u64p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_int, C.c_int, u64p, C.POINTER(RefCounts)]
        lib.ref_skms_free.argtypes = [C.POINTER(RefSkms)]
        lib.ref_counts_free.argtypes = [C.POINTER(RefCounts)]
        lib.ref_partition_sizes.argtypes = [C.c_char_p, u64p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_int, C.c_int, u64p]
        lib.ref_cal_var_stdev.argtypes = [u64p, C.c_int, C.c_char_p, C.c_int]
        _refs[filter_id] = lib
        if filter_id == 0:
            _ref = lib
    return _refs.get(filter_id, _ref)


class Skms:
    """Superkmers as flat arrays: bin, len, byte_off into `bytes`."""

    def __init__(self, bin, length, byte_off, data, minimizer=None, read_id=None, start=None):
        self.bin = bin
        self.len = length
        self.byte_off = byte_off
        self.bytes = data
        self.minimizer = minimizer
        self.read_id = read_id
        self.start = start

    def multisets(self, nbins):
        """Per bin: sorted list of (len, packed bytes) -- the partition parity form."""
        out = [[] for _ in range(nbins)]
        for i in range(len(self.bin)):
            nb = (int(self.len[i]) + 3) // 4
            o = int(self.byte_off[i])
            out[int(self.bin[i])].append((int(self.len[i]), self.bytes[o:o + nb].tobytes()))
        for b in out:
            b.sort()
        return out


def oracle_partition(reads, offs, k, p, hpc, nbins):
    lib = oracle()
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    s = OrcSkms()
    rc = lib.orc_partition(_ptr(reads, u8p), _ptr(offs, u64p), len(offs) - 1, k, p, int(hpc), nbins,
                           C.byref(s))
    assert rc == 0, rc
    out = Skms(_arr(s.bin, s.n_skm, np.uint32), _arr(s.len, s.n_skm, np.uint32),
               _arr(s.byte_off, s.n_skm, np.uint64), _arr(s.bytes, s.n_bytes, np.uint8),
               _arr(s.minimizer, s.n_skm, np.uint32), _arr(s.read_id, s.n_skm, np.uint64),
               _arr(s.start, s.n_skm, np.uint32))
    lib.orc_skms_free(C.byref(s))
    return out


def _counts_from(c, wide):
    nb = c.nbins
    res = dict(bin_off=_arr(c.bin_off, nb + 1, np.uint64),
               keys_lo=_arr(c.keys_lo, c.n_distinct, np.uint64),
               counts=_arr(c.counts, c.n_distinct, np.uint32))
    res["keys_hi"] = _arr(c.keys_hi, c.n_distinct, np.uint64) if wide else None
    return res


def oracle_count_bins(skms, k, nbins):
    lib = oracle()
    s = OrcSkms()
    s.n_skm = len(skms.bin)
    s.n_bytes = len(skms.bytes)
    keep = [np.ascontiguousarray(skms.bin, np.uint32), np.ascontiguousarray(skms.len, np.uint32),
            np.ascontiguousarray(skms.byte_off, np.uint64),
            np.ascontiguousarray(skms.bytes if len(skms.bytes) else np.zeros(1, np.uint8), np.uint8)]
    s.bin = _ptr(keep[0], u32p)
    s.len = _ptr(keep[1], u32p)
    s.byte_off = _ptr(keep[2], u64p)
    s.bytes = _ptr(keep[3], u8p)
    c = OrcCounts()
    rc = lib.orc_count_bins(C.byref(s), k, nbins, C.byref(c))
    assert rc == 0, rc
    res = _counts_from(c, k > 32)
    lib.orc_counts_free(C.byref(c))
    return res


def oracle_minimizers(read, k, p, with_pos=False):
    lib = oracle()
    read = np.ascontiguousarray(read, dtype=np.uint8)
    W = max(0, len(read) - k + 1)
    mm = np.zeros(max(W, 1), np.uint32)
    if not with_pos:
        lib.orc_window_minimizers(_ptr(read, u8p), len(read), k, p, _ptr(mm, u32p))
        return mm[:W]
    pos = np.zeros(max(W, 1), np.uint8)
    st = np.zeros(max(W, 1), np.int8)
    lib.orc_window_minimizer_pos(_ptr(read, u8p), len(read), k, p, _ptr(mm, u32p), _ptr(pos, u8p),
                                 st.ctypes.data_as(C.POINTER(C.c_int8)))
    return mm[:W], pos[:W], st[:W]


def oracle_hpc(reads, offs):
    lib = oracle()
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    n = len(offs) - 1
    out = np.zeros(max(len(reads), 1), np.uint8)
    ln = np.zeros(max(n, 1), np.int32)
    orig = np.zeros(max(len(reads), 1), np.int32)
    lib.orc_hpc(_ptr(reads, u8p), _ptr(offs, u64p), n, _ptr(out, u8p),
                ln.ctypes.data_as(C.POINTER(C.c_int32)), orig.ctypes.data_as(C.POINTER(C.c_int32)))
    return out[:len(reads)], ln[:n], orig[:len(reads)]


def oracle_subsample(reads, offs, k, p, mod):
    lib = oracle()
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    r = OrcPos()
    rc = lib.orc_subsample_positions(_ptr(reads, u8p), _ptr(offs, u64p), len(offs) - 1, k, p, mod,
                                     C.byref(r))
    assert rc == 0
    res = dict(keys_lo=_arr(r.keys_lo, r.n_distinct, np.uint64),
               keys_hi=_arr(r.keys_hi, r.n_distinct, np.uint64),
               pos_off=_arr(r.pos_off, r.n_distinct + 1, np.uint64),
               pos=_arr(r.pos, r.n_pos, np.uint32))
    lib.orc_poslists_free(C.byref(r))
    return res


def ref_partition(reads, offs, k, p, hpc, nbins, batch_reads=2048, n_threads=4, filter_id=0):
    lib = reference(filter_id)
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    s = RefSkms()
    rc = lib.ref_partition(reads.ctypes.data_as(C.c_char_p), _ptr(offs, u64p), len(offs) - 1, k, p,
                           int(hpc), nbins, batch_reads, n_threads, C.byref(s))
    assert rc == 0
    out = Skms(_arr(s.bin, s.n_skm, np.uint32), _arr(s.len, s.n_skm, np.uint32),
               _arr(s.byte_off, s.n_skm, np.uint64), _arr(s.bytes, s.n_bytes, np.uint8))
    lib.ref_skms_free(C.byref(s))
    return out


def ref_count_bins(skms, k, nbins, n_threads=4):
    lib = reference()
    s = RefSkms()
    keep = [np.ascontiguousarray(skms.bin, np.uint32), np.ascontiguousarray(skms.len, np.uint32),
            np.ascontiguousarray(skms.byte_off, np.uint64),
            np.ascontiguousarray(skms.bytes if len(skms.bytes) else np.zeros(1, np.uint8), np.uint8)]
    s.n_skm = len(skms.bin)
    s.n_bytes = len(skms.bytes)
    s.bin = _ptr(keep[0], u32p)
    s.len = _ptr(keep[1], u32p)
    s.byte_off = _ptr(keep[2], u64p)
    s.bytes = _ptr(keep[3], u8p)
    c = RefCounts()
    rc = lib.ref_count_bins(C.byref(s), k, nbins, n_threads, C.byref(c))
    assert rc == 0
    res = dict(bin_off=_arr(c.bin_off, nbins + 1, np.uint64),
               keys_lo=_arr(c.keys, c.n_distinct, np.uint64),
               counts=_arr(c.counts, c.n_distinct, np.uint32),
               returned=_arr(c.returned, nbins, np.uint64), keys_hi=None)
    lib.ref_counts_free(C.byref(c))
    return res


def ref_pipeline(reads, offs, k, p, hpc, nbins, batch_reads=2048, n_threads=1):
    lib = reference()
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    d = np.zeros(1, np.uint64)
    km = np.zeros(1, np.uint64)
    rc = lib.ref_pipeline(reads.ctypes.data_as(C.c_char_p), _ptr(offs, u64p), len(offs) - 1, k, p,
                          int(hpc), nbins, batch_reads, n_threads, _ptr(d, u64p), _ptr(km, u64p))
    assert rc == 0
    return int(d[0]), int(km[0])


def ref_pipeline_counts(reads, offs, k, p, hpc, nbins, batch_reads=2048, n_threads=1):
    """The reference's CPU path with its per-bin sorted (k-mer, count) lists
    kept (k <= 32); returns (counts dict as ref_count_bins, k-mers)."""
    lib = reference()
    reads = np.ascontiguousarray(reads, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    km = np.zeros(1, np.uint64)
    c = RefCounts()
    rc = lib.ref_pipeline_counts(reads.ctypes.data_as(C.c_char_p), _ptr(offs, u64p), len(offs) - 1, k, p,
                                 int(hpc), nbins, batch_reads, n_threads, _ptr(km, u64p), C.byref(c))
    assert rc == 0
    res = dict(bin_off=_arr(c.bin_off, nbins + 1, np.uint64),
               keys_lo=_arr(c.keys, c.n_distinct, np.uint64),
               counts=_arr(c.counts, c.n_distinct, np.uint32), keys_hi=None)
    lib.ref_counts_free(C.byref(c))
    return res, int(km[0])


def counts_digest64(bin_off, keys_lo, counts, keys_hi=None):
    """(digest over all bins, per-bin digests) of per-bin sorted (k-mer,
    count) lists; the same function digests the GPU's and the reference's."""
    lib = oracle()
    lib.orc_counts_digest.restype = C.c_uint64
    lib.orc_counts_digest.argtypes = [u64p, C.c_uint32, u64p, u64p, u32p, u64p]
    bo = np.ascontiguousarray(bin_off, np.uint64)
    kl = np.ascontiguousarray(keys_lo, np.uint64)
    kh = None if keys_hi is None else np.ascontiguousarray(keys_hi, np.uint64)
    cn = np.ascontiguousarray(counts, np.uint32)
    nb = len(bo) - 1
    per = np.zeros(max(nb, 1), np.uint64)
    if len(kl) == 0:
        kl = np.zeros(1, np.uint64)
        cn = np.zeros(1, np.uint32)
    tot = lib.orc_counts_digest(_ptr(bo, u64p), nb, _ptr(kl, u64p), None if kh is None else _ptr(kh, u64p),
                                _ptr(cn, u32p), _ptr(per, u64p))
    return int(tot), per[:nb]


def skm_digest64(bins, lens, byte_off, data, nbins):
    """(digest, per-bin digests, per-bin counts) of a partition as per-bin
    multisets of (length, packed bytes)."""
    lib = oracle()
    lib.orc_skm_multiset_digest.restype = C.c_uint64
    lib.orc_skm_multiset_digest.argtypes = [u32p, u32p, u64p, u8p, C.c_uint64, C.c_uint32, u64p, u64p]
    b = np.ascontiguousarray(bins, np.uint32)
    ln = np.ascontiguousarray(lens, np.uint32)
    bo = np.ascontiguousarray(byte_off, np.uint64)
    d = np.ascontiguousarray(data if len(data) else np.zeros(1, np.uint8), np.uint8)
    per = np.zeros(nbins, np.uint64)
    cnt = np.zeros(nbins, np.uint64)
    tot = lib.orc_skm_multiset_digest(_ptr(b, u32p), _ptr(ln, u32p), _ptr(bo, u64p), _ptr(d, u8p), len(b),
                                      nbins, _ptr(per, u64p), _ptr(cnt, u64p))
    return int(tot), per, cnt


class OrcBalance(C.Structure):
    _fields_ = [("total", C.c_uint64), ("mean", C.c_uint64), ("max", C.c_uint64), ("min", C.c_uint64),
                ("variance", C.c_double), ("stdev", C.c_double), ("cv", C.c_double)]


def oracle_partition_sizes(skms, nbins):
    """Bases per bin of an oracle (or any) partition: the sum of its superkmer lengths."""
    sizes = np.zeros(nbins, np.uint64)
    np.add.at(sizes, np.asarray(skms.bin, np.int64), np.asarray(skms.len, np.uint64))
    return sizes


def oracle_balance(sizes):
    lib = oracle()
    lib.orc_balance_stats.argtypes = [u64p, C.c_int, C.POINTER(OrcBalance)]
    sizes = np.ascontiguousarray(sizes, np.uint64)
    st = OrcBalance()
    lib.orc_balance_stats(_ptr(sizes, u64p), len(sizes), C.byref(st))
    return {f: getattr(st, f) for f, _ in OrcBalance._fields_}


def balance_report(st):
    """The text calVarStdev logs (experiment.cpp:30-35) for a summary:
    integers as they are, doubles as an ostream prints them by default
    (six significant digits, printf %g)."""
    return ("SKM TOT_LEN=%d\n" % st["total"] +
            "AVG=%d\tMAX=%d\tmin=%d\tvar=%g\tSTD=%g\tCV=%g\n\n"
            % (st["mean"], st["max"], st["min"], st["variance"], st["stdev"], st["cv"]))


def ref_partition_sizes(reads, offs, k, p, hpc, nbins, batch_reads=2048, n_threads=4, filter_id=0):
    lib = reference(filter_id)
    reads = np.ascontiguousarray(reads, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    sizes = np.zeros(nbins, np.uint64)
    rc = lib.ref_partition_sizes(reads.tobytes(), _ptr(offs, u64p), len(offs) - 1, k, p, int(hpc),
                                 nbins, batch_reads, n_threads, _ptr(sizes, u64p))
    assert rc == 0, rc
    return sizes


def ref_balance_report(sizes):
    lib = reference()
    sizes = np.ascontiguousarray(sizes, np.uint64)
    buf = C.create_string_buffer(1024)
    n = lib.ref_cal_var_stdev(_ptr(sizes, u64p), len(sizes), buf, len(buf))
    assert n < len(buf)
    return buf.value.decode()


REF_LOADER_SO = os.path.join(ROOT, "oracle", "_ref", "libgkcref_loader.so")


def ref_loader_available():
    return os.path.exists(REF_LOADER_SO)


def ref_load_reads(path, n_threads=1, buffer_size=0):
    """The reads the reference's ReadLoader (read_loader.hpp) delivers for a
    file, in order: (reads uint8, offs uint64)."""
    lib = C.CDLL(REF_LOADER_SO)
    lib.ref_load_reads.argtypes = [C.c_char_p, C.c_int, C.c_uint64, u64p, C.POINTER(C.c_void_p),
                                   C.POINTER(C.c_void_p)]
    lib.ref_free_reads.argtypes = [C.c_void_p, C.c_void_p]
    n = np.zeros(1, np.uint64)
    r, o = C.c_void_p(), C.c_void_p()
    assert lib.ref_load_reads(os.fsencode(path), n_threads, buffer_size, _ptr(n, u64p), C.byref(r), C.byref(o)) == 0
    nr = int(n[0])
    offs = np.ctypeslib.as_array(C.cast(o, u64p), shape=(nr + 1,)).copy()
    reads = (np.ctypeslib.as_array(C.cast(r, u8p), shape=(int(offs[-1]),)).copy() if offs[-1]
             else np.zeros(0, np.uint8))
    lib.ref_free_reads(r, o)
    return reads, offs
