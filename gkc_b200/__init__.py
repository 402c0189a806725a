"""gkc_b200: B200-native k-mer partitioning and counting.

Thin ctypes binding over the C ABI in include/gkc/gkc.h (libgkc_b200.so,
built in-tree by gkc_b200.build).  There is no fallback: if the shared
library is missing, loading fails with an error.

Host-level calls take numpy arrays; device-level calls take torch CUDA
tensors (torch is used only to hold device memory).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgkc_b200.so")

MODE_BATCHED = 0
MODE_PLAIN = 1

FILTER_NEW2, FILTER_ALL, FILTER_NEW, FILTER_SIGNATURE = 0, 1, 2, 3

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "no CUDA device",
          4: "out of device memory", 5: "HBM budget exceeded", 6: "capacity exceeded",
          7: "device-side wait timed out", 8: "not ready", 9: "cancelled", 10: "not found",
          11: "internal error"}


class GkcError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"gkc status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("k", C.c_int), ("p", C.c_int), ("hpc", C.c_int), ("nbins", C.c_int)]


class PartitionView(C.Structure):
    _fields_ = [("n_reads", C.c_uint64), ("n_bases", C.c_uint64), ("n_superkmers", C.c_uint64),
                ("n_packed_bytes", C.c_uint64), ("n_kmers", C.c_uint64), ("nbins", C.c_uint32),
                ("bin_skm_off", C.c_void_p), ("bin_kmer_off", C.c_void_p), ("skm_desc", C.c_void_p),
                ("skm_minimizer", C.c_void_p), ("packed", C.c_void_p), ("hpc_reads", C.c_void_p),
                ("hpc_offs", C.c_void_p), ("hpc_orig_pos", C.c_void_p)]


class BalanceStats(C.Structure):
    _fields_ = [("total", C.c_uint64), ("mean", C.c_uint64), ("max", C.c_uint64), ("min", C.c_uint64),
                ("variance", C.c_double), ("stdev", C.c_double), ("cv", C.c_double)]


class DbInfo(C.Structure):
    _fields_ = [("k", C.c_uint32), ("lut_prefix_len", C.c_uint32), ("suffix_bytes", C.c_uint32),
                ("counter_bytes", C.c_uint32), ("min_count", C.c_uint32), ("max_count", C.c_uint32),
                ("n_kmers", C.c_uint64), ("total_count", C.c_uint64)]


class CountView(C.Structure):
    _fields_ = [("n_distinct", C.c_uint64), ("n_kmers", C.c_uint64), ("nbins", C.c_uint32),
                ("key_words", C.c_int), ("bin_off", C.c_void_p), ("keys", C.c_void_p),
                ("counts", C.c_void_p)]


class PoslistView(C.Structure):
    _fields_ = [("n_distinct", C.c_uint64), ("n_positions", C.c_uint64), ("key_words", C.c_int),
                ("keys", C.c_void_p), ("pos_off", C.c_void_p), ("positions", C.c_void_p)]


MAX_STAGES = 8


class Timings(C.Structure):
    _fields_ = [("partition_ms", C.c_float), ("count_ms", C.c_float), ("total_ms", C.c_float),
                ("h2d_ms", C.c_float), ("d2h_ms", C.c_float), ("launches", C.c_uint32),
                ("graph_replayed", C.c_uint32), ("n_stages", C.c_uint32),
                ("stage_ms", C.c_float * MAX_STAGES)]

    def stages(self):
        L = lib()
        return {L.gkc_stage_name(i).decode(): float(self.stage_ms[i]) for i in range(self.n_stages)}


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("n_bases", C.c_uint64),
                ("n_kmers", C.c_uint64), ("n_distinct", C.c_uint64), ("nbins", C.c_uint32),
                ("key_words", C.c_int), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("end_s", C.c_double), ("hbm_bytes", C.c_uint64)]


class TuneParams(C.Structure):
    _fields_ = [("coarse_target", C.c_uint32), ("chunk_kmers", C.c_uint32),
                ("count_ctas_per_sm", C.c_uint32), ("reserved", C.c_uint32)]

    def as_dict(self):
        return {"coarse_target": int(self.coarse_target), "chunk_kmers": int(self.chunk_kmers),
                "count_ctas_per_sm": int(self.count_ctas_per_sm)}


class TuneReport(C.Structure):
    _fields_ = [("chosen", TuneParams), ("defaults", TuneParams), ("default_ms", C.c_float),
                ("tuned_ms", C.c_float), ("candidates", C.c_uint32), ("from_cache", C.c_int),
                ("sample_bases", C.c_uint64)]


# (name, restype, argtypes) for every exported symbol of include/gkc/gkc.h
vp, u64, u32, i32, dbl = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_double
P = C.POINTER
SIGNATURES = [
    ("gkc_abi_version", C.c_int, []),
    ("gkc_stage_name", C.c_char_p, [C.c_int]),
    ("gkc_status_string", C.c_char_p, [C.c_int]),
    ("gkc_ctx_create", C.c_int, [C.c_int, u64, P(vp)]),
    ("gkc_ctx_destroy", None, [vp]),
    ("gkc_ctx_last_error", C.c_char_p, [vp]),
    ("gkc_ctx_set_stream", C.c_int, [vp, vp]),
    ("gkc_ctx_set_filter", C.c_int, [vp, C.c_int]),
    ("gkc_ctx_synchronize", C.c_int, [vp]),
    ("gkc_ctx_device_bytes", u64, [vp]),
    ("gkc_ctx_release_workspace", C.c_int, [vp]),
    ("gkc_last_timings", C.c_int, [vp, P(Timings)]),
    ("gkc_partition_device", C.c_int, [vp, P(Params), vp, u64, vp, u64, P(PartitionView)]),
    ("gkc_partition_host", C.c_int, [vp, P(Params), vp, vp, u64, P(PartitionView)]),
    ("gkc_partition_copy_out", C.c_int, [vp, vp, vp, vp, vp, vp]),
    ("gkc_partition_balance", C.c_int, [vp, vp, u32, P(BalanceStats)]),
    ("gkc_exchange_pack", C.c_int, [vp, u32, vp, vp, u64, vp, u64, vp, vp, vp, vp]),
    ("gkc_partition_import", C.c_int, [vp, P(Params), u32, vp, vp, vp, vp, vp, P(PartitionView)]),
    ("gkc_count_device", C.c_int, [vp, P(Params), C.c_int, P(CountView)]),
    ("gkc_count_superkmers_host", C.c_int, [vp, C.c_int, vp, vp, u64, C.c_int, P(u64)]),
    ("gkc_count_copy_out", C.c_int, [vp, vp, vp, vp]),
    ("gkc_count_output", C.c_int, [vp, u32, u32, C.c_int, P(u64), vp, vp, vp]),
    ("gkc_count_superkmers_device_noalloc", C.c_int, [C.c_int, vp, vp, u64, u64, vp, vp, P(u64), vp]),
    ("gkc_tune_get", C.c_int, [vp, P(TuneParams)]),
    ("gkc_tune_set", C.c_int, [vp, P(TuneParams)]),
    ("gkc_autotune_device", C.c_int, [vp, P(Params), vp, u64, vp, u64, C.c_int, P(TuneReport)]),
    ("gkc_tune_cache_lookup", C.c_int, [C.c_int, P(Params), u64, u64, P(TuneParams)]),
    ("gkc_tune_cache_store", C.c_int, [C.c_int, P(Params), u64, u64, P(TuneParams)]),
    ("gkc_tune_cache_clear", None, []),
    ("gkc_tune_cache_save", C.c_int, [C.c_char_p]),
    ("gkc_tune_cache_load", C.c_int, [C.c_char_p]),
    ("gkc_pipeline_device", C.c_int, [vp, P(Params), C.c_int, vp, u64, vp, u64, P(PartitionView),
                                      P(CountView)]),
    ("gkc_pipeline_host", C.c_int, [vp, P(Params), C.c_int, vp, vp, u64, P(CountView)]),
    ("gkc_stream_submit", C.c_int, [vp, P(Params), vp, vp, u64, vp, vp, vp, u64, P(u64)]),
    ("gkc_stream_wait", C.c_int, [vp, u64, P(u64), P(u64)]),
    ("gkc_minimizers_device", C.c_int, [vp, P(Params), vp, u64, vp, u64, vp, vp, vp]),
    ("gkc_subsample_positions_device", C.c_int, [vp, P(Params), u32, vp, u64, vp, u64,
                                                 P(PoslistView)]),
    ("gkc_hpc_device", C.c_int, [vp, vp, u64, vp, u64, vp, vp, vp]),
    ("gkc_fastx_load", C.c_int, [C.c_char_p, C.c_int, C.c_int, P(vp), P(vp), P(u64)]),
    ("gkc_fastx_load_ex", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, P(vp), P(vp), P(u64)]),
    ("gkc_fastx_free", None, [vp, vp, C.c_int]),
    ("gkc_db_write", C.c_int, [vp, C.c_char_p, u32, u32, C.c_int]),
    ("gkc_db_open", C.c_int, [C.c_char_p, P(vp)]),
    ("gkc_db_close", None, [vp]),
    ("gkc_db_get_info", C.c_int, [vp, P(DbInfo)]),
    ("gkc_db_lookup", C.c_int, [vp, vp, u64, vp]),
    ("gkc_db_read", C.c_int, [vp, u64, u64, vp, vp]),
    ("gkc_server_create", C.c_int, [C.c_int, u64, C.c_int, P(vp)]),
    ("gkc_server_destroy", None, [vp]),
    ("gkc_server_submit", C.c_int, [vp, P(Params), vp, vp, u64, P(u64)]),
    ("gkc_server_submit_device_synth", C.c_int, [vp, P(Params), C.c_int, u64, u64, P(u64)]),
    ("gkc_server_poll", C.c_int, [vp, u64, P(JobInfo)]),
    ("gkc_server_wait", C.c_int, [vp, u64, dbl, P(JobInfo)]),
    ("gkc_server_cancel", C.c_int, [vp, u64]),
    ("gkc_server_copy_result", C.c_int, [vp, u64, vp, vp, vp]),
    ("gkc_server_release", C.c_int, [vp, u64]),
    ("gkc_job_hbm_estimate", u64, [P(Params), u64, u64]),
    ("gkc_synth_iid_reads", C.c_int, [C.c_int, u64, u64, u32, dbl, vp, vp]),
    ("gkc_synth_genome", C.c_int, [C.c_int, u64, u64, dbl, dbl, vp]),
    ("gkc_synth_short_reads", C.c_int, [C.c_int, u64, vp, u64, u64, u64, u32, dbl, vp, vp]),
    ("gkc_synth_long_read_offsets", u64, [u64, dbl, dbl, u32, u32, u64, u64, vp]),
    ("gkc_synth_long_reads", C.c_int, [C.c_int, u64, vp, u64, u64, vp, vp]),
]

_lib = None


def lib():
    """Loads libgkc_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m gkc_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    """Address of a numpy array or a torch tensor."""
    if a is None:
        return None
    if isinstance(a, int):  # a raw device address
        return a or None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def params(k, p, nbins, hpc=False):
    return Params(int(k), int(p), int(bool(hpc)), int(nbins))


class Context:
    """One device context (reference: GPUReset + the per-call CUDA state of
    GenSuperkmerGPU / kmc_counting_GPU)."""

    def __init__(self, device=0, hbm_budget=0):
        self._L = lib()
        h = C.c_void_p()
        st = self._L.gkc_ctx_create(int(device), int(hbm_budget), C.byref(h))
        if st != 0:
            raise GkcError(st, "gkc_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            self._L.gkc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st != 0:
            msg = self._L.gkc_ctx_last_error(self.h)
            raise GkcError(st, f"{what}: {msg.decode() if msg else ''}")

    def timings(self):
        t = Timings()
        self._check(self._L.gkc_last_timings(self.h, C.byref(t)), "timings")
        return t

    def device_bytes(self):
        return int(self._L.gkc_ctx_device_bytes(self.h))

    def set_filter(self, filter_id):
        """Minimizer filter for later calls (FILTER_*)."""
        self._check(self._L.gkc_ctx_set_filter(self.h, int(filter_id)), "set_filter")

    def set_stream(self, stream_ptr):
        self._check(self._L.gkc_ctx_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    # ---- partition ----
    def partition_host(self, reads, offs, prm):
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        v = PartitionView()
        self._check(self._L.gkc_partition_host(self.h, C.byref(prm), _ptr(reads), _ptr(offs),
                                               len(offs) - 1, C.byref(v)), "partition_host")
        return v

    def partition_device(self, d_reads, n_bytes, d_offs, n_reads, prm):
        v = PartitionView()
        self._check(self._L.gkc_partition_device(self.h, C.byref(prm), _ptr(d_reads), int(n_bytes),
                                                 _ptr(d_offs), int(n_reads), C.byref(v)),
                    "partition_device")
        return v

    def partition_copy_out(self, view):
        """-> (bin_off, lens, byte_off, packed, minimizer) numpy arrays."""
        n, nb = int(view.n_superkmers), int(view.nbins)
        bin_off = np.zeros(nb + 1, np.uint64)
        lens = np.zeros(max(n, 1), np.uint32)
        boff = np.zeros(max(n, 1), np.uint64)
        packed = np.zeros(max(int(view.n_packed_bytes), 1), np.uint8)
        mm = np.zeros(max(n, 1), np.uint32)
        self._check(self._L.gkc_partition_copy_out(self.h, _ptr(bin_off), _ptr(lens), _ptr(boff),
                                                   _ptr(packed), _ptr(mm)), "partition_copy_out")
        return bin_off, lens[:n], boff[:n], packed[:int(view.n_packed_bytes)], mm[:n]

    def partition_balance(self, view):
        """-> (bases per bin, summary dict) of the context's partition (the
        view its partition call returned): the per-bin superkmer bases and the
        avg / max / min / var / std / cv summary of the reference's
        partition-size report."""
        nbins = int(view.nbins)
        sizes = np.zeros(max(nbins, 1), np.uint64)
        st = BalanceStats()
        self._check(self._L.gkc_partition_balance(self.h, _ptr(sizes), len(sizes), C.byref(st)), "partition_balance")
        return sizes[:nbins], {f: getattr(st, f) for f, _ in BalanceStats._fields_}

    def db_write(self, path, min_count=1, max_count=0xFFFFFFFF, lut_prefix_len=0):
        """The merged count list (within [min_count, max_count]) as an on-disk
        database <path>.gkc_pre / <path>.gkc_suf; read it with Database."""
        self._check(self._L.gkc_db_write(self.h, os.fsencode(path), int(min_count), int(max_count),
                                         int(lut_prefix_len)), "db_write")

    # ---- superkmer exchange (bin sharding over several GPUs) ----
    def exchange_pack(self, view, bin_lo, d_send_desc, d_send_bytes):
        """Runs of the context's partition per destination (owner r holds bins
        [bin_lo[r], bin_lo[r+1])) written to the two device tensors;
        -> (skm_split, byte_split, bin_skm, bin_kmers) numpy arrays."""
        bin_lo = np.ascontiguousarray(bin_lo, np.uint32)
        nd, nb = len(bin_lo) - 1, int(view.nbins)
        skm_split, byte_split = np.zeros(nd, np.uint64), np.zeros(nd, np.uint64)
        bin_skm, bin_kmers = np.zeros(max(nb, 1), np.uint64), np.zeros(max(nb, 1), np.uint64)
        self._check(self._L.gkc_exchange_pack(self.h, nd, _ptr(bin_lo), _ptr(d_send_desc), d_send_desc.numel(),
                                              _ptr(d_send_bytes), d_send_bytes.numel(), _ptr(skm_split),
                                              _ptr(byte_split), _ptr(bin_skm), _ptr(bin_kmers)), "exchange_pack")
        return skm_split, byte_split, bin_skm[:nb], bin_kmers[:nb]

    def partition_import(self, prm, seg_bin_skm, seg_bin_kmers, seg_bytes, d_desc, d_bytes):
        """The senders' runs (concatenated in sender order in the two device
        tensors) as this context's partition of prm.nbins local bins."""
        seg_bin_skm = np.ascontiguousarray(seg_bin_skm, np.uint64)
        seg_bin_kmers = np.ascontiguousarray(seg_bin_kmers, np.uint64)
        seg_bytes = np.ascontiguousarray(seg_bytes, np.uint64)
        v = PartitionView()
        self._check(self._L.gkc_partition_import(self.h, C.byref(prm), len(seg_bytes), _ptr(seg_bin_skm),
                                                 _ptr(seg_bin_kmers), _ptr(seg_bytes), _ptr(d_desc),
                                                 _ptr(d_bytes), C.byref(v)), "partition_import")
        return v

    # ---- count ----
    def count_device(self, prm, mode=MODE_BATCHED):
        v = CountView()
        self._check(self._L.gkc_count_device(self.h, C.byref(prm), int(mode), C.byref(v)),
                    "count_device")
        return v

    def count_superkmers_host(self, k, lens, packed, mode=MODE_BATCHED):
        lens = np.ascontiguousarray(lens, np.uint32)
        packed = np.ascontiguousarray(packed, np.uint8)
        nd = C.c_uint64()
        self._check(self._L.gkc_count_superkmers_host(self.h, int(k), _ptr(lens), _ptr(packed),
                                                      len(lens), int(mode), C.byref(nd)),
                    "count_superkmers_host")
        return int(nd.value)

    def count_copy_out(self, view):
        """-> (bin_off, keys (n, key_words) uint64, counts)."""
        nd, nb, kw = int(view.n_distinct), int(view.nbins), int(view.key_words)
        bin_off = np.zeros(nb + 1, np.uint64)
        keys = np.zeros(max(nd * kw, 1), np.uint64)
        counts = np.zeros(max(nd, 1), np.uint32)
        self._check(self._L.gkc_count_copy_out(self.h, _ptr(bin_off), _ptr(keys), _ptr(counts)),
                    "count_copy_out")
        return bin_off, keys[:nd * kw].reshape(nd, kw), counts[:nd]

    def count_output(self, min_count=1, max_count=0xFFFFFFFF, merged=False, key_words=1, nbins=None):
        """-> (bin_off, keys (n, key_words), counts): the last count result
        filtered to min_count <= count <= max_count, per bin or merged."""
        n = C.c_uint64()
        self._check(self._L.gkc_count_output(self.h, int(min_count), int(max_count), int(bool(merged)),
                                             C.byref(n), None, None, None), "count_output")
        nn = int(n.value)
        nb = 1 if merged else int(nbins)
        bin_off = np.zeros(nb + 1, np.uint64)
        keys = np.zeros(max(nn * key_words, 1), np.uint64)
        counts = np.zeros(max(nn, 1), np.uint32)
        self._check(self._L.gkc_count_output(self.h, int(min_count), int(max_count), int(bool(merged)),
                                             C.byref(n), _ptr(bin_off), _ptr(keys), _ptr(counts)),
                    "count_output")
        return bin_off, keys[:nn * key_words].reshape(nn, key_words), counts[:nn]

    # ---- launch-shape tuning ----
    def tune_get(self):
        t = TuneParams()
        self._check(self._L.gkc_tune_get(self.h, C.byref(t)), "tune_get")
        return t

    def tune_set(self, tp=None):
        self._check(self._L.gkc_tune_set(self.h, C.byref(tp) if tp is not None else None), "tune_set")

    def autotune_device(self, d_reads, n_bytes, d_offs, n_reads, prm, force=False):
        """Times candidate count-stage shapes on a sample of the reads and
        keeps the fastest on this context; -> TuneReport."""
        r = TuneReport()
        self._check(self._L.gkc_autotune_device(self.h, C.byref(prm), _ptr(d_reads), int(n_bytes),
                                                _ptr(d_offs), int(n_reads), int(bool(force)), C.byref(r)),
                    "autotune_device")
        return r

    # ---- pipeline ----
    def pipeline_device(self, d_reads, n_bytes, d_offs, n_reads, prm, mode=MODE_BATCHED):
        pv, cv = PartitionView(), CountView()
        self._check(self._L.gkc_pipeline_device(self.h, C.byref(prm), int(mode), _ptr(d_reads),
                                                int(n_bytes), _ptr(d_offs), int(n_reads),
                                                C.byref(pv), C.byref(cv)), "pipeline_device")
        return pv, cv

    def pipeline_host(self, reads, offs, prm, mode=MODE_BATCHED):
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        cv = CountView()
        self._check(self._L.gkc_pipeline_host(self.h, C.byref(prm), int(mode), _ptr(reads),
                                              _ptr(offs), len(offs) - 1, C.byref(cv)),
                    "pipeline_host")
        return cv

    def stream_submit(self, reads, offs, n_reads, prm, bin_off, keys, counts, capacity):
        """Streaming host form: page-locked tensors in and out; -> ticket."""
        t = C.c_uint64()
        self._check(self._L.gkc_stream_submit(self.h, C.byref(prm), _ptr(reads), _ptr(offs), int(n_reads),
                                              _ptr(bin_off), _ptr(keys), _ptr(counts), int(capacity),
                                              C.byref(t)), "stream_submit")
        return int(t.value)

    def stream_wait(self, ticket):
        """-> (n_distinct, n_kmers) once the call's results are in host memory."""
        nd, nk = C.c_uint64(), C.c_uint64()
        self._check(self._L.gkc_stream_wait(self.h, int(ticket), C.byref(nd), C.byref(nk)), "stream_wait")
        return int(nd.value), int(nk.value)

    def minimizers_device(self, d_reads, n_bytes, d_offs, n_reads, prm, d_mm, d_pos, d_strand):
        self._check(self._L.gkc_minimizers_device(self.h, C.byref(prm), _ptr(d_reads), int(n_bytes),
                                                  _ptr(d_offs), int(n_reads), _ptr(d_mm),
                                                  _ptr(d_pos), _ptr(d_strand)), "minimizers")

    def subsample_positions_device(self, d_reads, n_bytes, d_offs, n_reads, prm, mod):
        v = PoslistView()
        self._check(self._L.gkc_subsample_positions_device(self.h, C.byref(prm), int(mod),
                                                           _ptr(d_reads), int(n_bytes), _ptr(d_offs),
                                                           int(n_reads), C.byref(v)), "subsample")
        return v

    def hpc_device(self, d_reads, n_bytes, d_offs, n_reads, d_out, d_out_offs, d_orig):
        self._check(self._L.gkc_hpc_device(self.h, _ptr(d_reads), int(n_bytes), _ptr(d_offs),
                                           int(n_reads), _ptr(d_out), _ptr(d_out_offs),
                                           _ptr(d_orig)), "hpc")


def skms_from_copy(bin_off, lens, boff, packed):
    """Per-superkmer bin ids from the bin offsets (for parity checks)."""
    nb = len(bin_off) - 1
    bins = np.repeat(np.arange(nb, dtype=np.uint32), np.diff(bin_off).astype(np.int64))
    return bins, lens, boff, packed


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = range(5)
GEN_IID, GEN_GENOME_SHORT, GEN_GENOME_LONG = 1, 2, 3


class Server:
    """Continuous-batching counting server on one device (gkc_server_*)."""

    def __init__(self, device=0, hbm_budget=0, max_running=4):
        self._L = lib()
        h = C.c_void_p()
        st = self._L.gkc_server_create(int(device), int(hbm_budget), int(max_running), C.byref(h))
        if st != 0:
            raise GkcError(st, "gkc_server_create")
        self.h = h

    def close(self):
        if self.h:
            self._L.gkc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st != 0:
            raise GkcError(st, what)

    def submit(self, reads, offs, prm):
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        jid = C.c_uint64()
        self._check(self._L.gkc_server_submit(self.h, C.byref(prm), _ptr(reads), _ptr(offs),
                                              len(offs) - 1, C.byref(jid)), "submit")
        return int(jid.value)

    def submit_synth(self, prm, generator, seed, n_bases):
        jid = C.c_uint64()
        self._check(self._L.gkc_server_submit_device_synth(self.h, C.byref(prm), int(generator),
                                                           int(seed), int(n_bases), C.byref(jid)),
                    "submit_device_synth")
        return int(jid.value)

    def poll(self, jid):
        info = JobInfo()
        self._check(self._L.gkc_server_poll(self.h, int(jid), C.byref(info)), "poll")
        return info

    def wait(self, jid, timeout=-1.0):
        info = JobInfo()
        st = self._L.gkc_server_wait(self.h, int(jid), float(timeout), C.byref(info))
        if st not in (0, 8):
            raise GkcError(st, "wait")
        return info

    def cancel(self, jid):
        self._check(self._L.gkc_server_cancel(self.h, int(jid)), "cancel")

    def result(self, jid):
        """-> (bin_off, keys (n, key_words), counts) of a finished job."""
        info = self.poll(jid)
        nd, nb, kw = int(info.n_distinct), int(info.nbins), int(info.key_words)
        bin_off = np.zeros(nb + 1, np.uint64)
        keys = np.zeros(max(nd * kw, 1), np.uint64)
        counts = np.zeros(max(nd, 1), np.uint32)
        self._check(self._L.gkc_server_copy_result(self.h, int(jid), _ptr(bin_off), _ptr(keys),
                                                   _ptr(counts)), "copy_result")
        return bin_off, keys[:nd * kw].reshape(nd, kw), counts[:nd]

    def release(self, jid):
        self._check(self._L.gkc_server_release(self.h, int(jid)), "release")


def job_hbm_estimate(prm, n_bases, n_reads):
    return int(lib().gkc_job_hbm_estimate(C.byref(prm), int(n_bases), int(n_reads)))


class Database:
    """Reader of an on-disk k-mer database (gkc_db_open; no GPU needed)."""

    def __init__(self, path):
        self._L = lib()
        self.h = C.c_void_p()
        st = self._L.gkc_db_open(os.fsencode(path), C.byref(self.h))
        if st != 0:
            raise GkcError(st, f"gkc_db_open {path}")
        i = DbInfo()
        self._L.gkc_db_get_info(self.h, C.byref(i))
        self.info = {f: int(getattr(i, f)) for f, _ in DbInfo._fields_}
        self.key_words = 1 if self.info["k"] <= 32 else 2

    def close(self):
        if self.h:
            self._L.gkc_db_close(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def lookup(self, keys):
        """Counts of keys (n x key_words uint64, or n uint64 for k <= 32); 0 if absent."""
        keys = np.ascontiguousarray(keys, np.uint64)
        n = keys.shape[0]
        out = np.zeros(max(n, 1), np.uint32)
        st = self._L.gkc_db_lookup(self.h, _ptr(keys), n, _ptr(out))
        if st != 0:
            raise GkcError(st, "gkc_db_lookup")
        return out[:n]

    def read(self, first=0, n=None):
        """(keys n x key_words, counts) of records first .. first+n-1."""
        if n is None:
            n = self.info["n_kmers"] - first
        keys = np.zeros((max(n, 1), self.key_words), np.uint64)
        counts = np.zeros(max(n, 1), np.uint32)
        st = self._L.gkc_db_read(self.h, int(first), int(n), _ptr(keys), _ptr(counts))
        if st != 0:
            raise GkcError(st, "gkc_db_read")
        return keys[:n], counts[:n]


FASTX_JOIN_LINES, FASTX_FORMAT_FROM_CONTENT = 1, 2


def load_fastx(path, threads=0, flags=0):
    """(reads uint8, offs uint64) of a FASTA / FASTQ file (gkc_fastx_load_ex):
    by default the reference's record rules (format from the file name, one
    sequence line per FASTA record); flags FASTX_JOIN_LINES,
    FASTX_FORMAT_FROM_CONTENT."""
    L = lib()
    r, o, n = C.c_void_p(), C.c_void_p(), C.c_uint64()
    st = L.gkc_fastx_load_ex(os.fsencode(path), int(threads), 0, int(flags), C.byref(r), C.byref(o), C.byref(n))
    if st != 0:
        raise GkcError(st, f"gkc_fastx_load {path}")
    try:
        nr = int(n.value)
        offs = np.ctypeslib.as_array(C.cast(o, C.POINTER(C.c_uint64)), shape=(nr + 1,)).copy()
        nb = int(offs[-1])
        reads = (np.ctypeslib.as_array(C.cast(r, C.POINTER(C.c_uint8)), shape=(nb,)).copy()
                 if nb else np.zeros(0, np.uint8))
    finally:
        L.gkc_fastx_free(r, o, 0)
    return reads, offs
