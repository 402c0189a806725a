/* gkc-b200: B200-native k-mer partitioning and counting (C ABI).
 *
 * Drop-in boundary for GKC's partition-and-count path.  Every entry point
 * names the reference interface it replaces (paths relative to the GKC
 * project root).  All entry points return a gkc_status; none exits the
 * process (the reference's CUDA_CHECK calls exit(1), gkc_cuda.hpp:4-9).
 * Plain pointers and sizes only: no C++ or framework types cross this ABI.
 *
 * Data conventions
 *   reads    concatenated read bytes (ASCII; A/C/G/T/U in either case are
 *            bases, anything else behaves like N)
 *   offs     n_reads + 1 uint64 offsets into reads; read r is
 *            reads[offs[r], offs[r+1]).  Device entry points require
 *            offs[0] == 0; host entry points rebase.
 *   superkmer descriptor (uint64): (packed byte offset << 24) | length in bases
 *   packed   2 bits per base (A0 C1 G2 T3, N as T), first base in the top
 *            bits of the first byte, each superkmer starting on a byte
 *            boundary, last byte zero padded (superkmers.hpp:63-71)
 *   k-mer    2k-bit canonical key min(x, revcomp(x)); k <= 32 keys are
 *            uint64, k <= 64 keys are 16 bytes (low word first)
 */
#ifndef GKC_GKC_H
#define GKC_GKC_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GKC_ABI_VERSION 1

typedef enum gkc_status {
  GKC_OK = 0,
  GKC_ERR_INVALID_ARG = 1,
  GKC_ERR_CUDA = 2,
  GKC_ERR_NO_DEVICE = 3,
  GKC_ERR_OUT_OF_MEMORY = 4,
  GKC_ERR_BUDGET = 5,          /* request exceeds the context's HBM budget */
  GKC_ERR_CAPACITY = 6,        /* internal buffer too small even after retry */
  GKC_ERR_DEVICE_TIMEOUT = 7,  /* a bounded device-side wait expired */
  GKC_ERR_NOT_READY = 8,
  GKC_ERR_CANCELLED = 9,
  GKC_ERR_NOT_FOUND = 10,
  GKC_ERR_INTERNAL = 11
} gkc_status;

typedef struct gkc_ctx gkc_ctx;

/* Parameters of one partition / count run.  Reference: K_kmer, P_minimizer,
 * HPC and SKM_partitions of GenSuperkmerGPU (gkc_cuda.hpp:58-61). */
typedef struct gkc_params {
  int k;      /* 1..64 (reference: k <= 32) */
  int p;      /* 3..16, p <= k */
  int hpc;    /* collapse homopolymer runs before partitioning */
  int nbins;  /* superkmer partitions: bin = minimizer % nbins */
} gkc_params;

typedef enum gkc_mode {
  GKC_MODE_BATCHED = 0, /* persistent kernels, whole pipeline in one CUDA graph */
  GKC_MODE_PLAIN = 1    /* per-stage, per-batch / per-bin launches */
} gkc_mode;

/* Device-resident partition (valid until the next call on the context). */
typedef struct gkc_partition_view {
  uint64_t n_reads, n_bases;      /* after HPC when enabled */
  uint64_t n_superkmers, n_packed_bytes, n_kmers;
  uint32_t nbins;
  const uint64_t *bin_skm_off;    /* nbins+1: superkmers of bin b are [off[b], off[b+1]) */
  const uint64_t *bin_kmer_off;   /* nbins+1: k-mer prefix per bin */
  const uint64_t *skm_desc;       /* bin-ordered descriptors */
  const uint32_t *skm_minimizer;  /* bin-ordered minimizer values */
  const uint8_t *packed;
  const char *hpc_reads;          /* HPC only: compacted reads, offsets, */
  const uint64_t *hpc_offs;       /*   and in-read original position of  */
  const int32_t *hpc_orig_pos;    /*   every kept base; else NULL        */
} gkc_partition_view;

/* Device-resident counts: per bin, ascending canonical keys with counts. */
typedef struct gkc_count_view {
  uint64_t n_distinct, n_kmers;
  uint32_t nbins;
  int key_words;             /* 1 (k <= 32) or 2 (k <= 64) uint64 per key */
  const uint64_t *bin_off;   /* nbins+1 */
  const uint64_t *keys;      /* n_distinct * key_words */
  const uint32_t *counts;    /* n_distinct, clamped to 2^32-1 */
} gkc_count_view;

#define GKC_MAX_STAGES 8
typedef struct gkc_timings {
  float partition_ms, count_ms, total_ms, h2d_ms, d2h_ms;
  uint32_t launches;        /* kernels launched by the last pipeline call */
  uint32_t graph_replayed;  /* 1 if the batched pipeline ran from a cached graph */
  uint32_t n_stages;        /* batched pipeline: device time of each stage */
  float stage_ms[GKC_MAX_STAGES];
} gkc_timings;
/* Name of stage i of the batched pipeline ("partition", "sort_count", ...). */
const char *gkc_stage_name(int i);

/* ---- context (reference: GPUReset gkc_cuda.cu:367-373; CUDAParams.device_id) ---- */
gkc_status gkc_ctx_create(int device_id, uint64_t hbm_budget_bytes, gkc_ctx **out);
void gkc_ctx_destroy(gkc_ctx *ctx);
const char *gkc_ctx_last_error(const gkc_ctx *ctx);
const char *gkc_status_string(gkc_status s);
gkc_status gkc_ctx_set_stream(gkc_ctx *ctx, void *cuda_stream);
/* Which p-mers may be minimizers (the reference chooses one at compile time,
 * FILTER_KERNEL at gkc_cuda.cu:6, among the variants at :196-227).  The
 * setting applies to every later call on the context. */
typedef enum gkc_filter {
  GKC_FILTER_NEW2 = 0,      /* new_filter2, the reference's choice (default):
                               the top three bases are not AAA, ACA or AGA */
  GKC_FILTER_ALL = 1,       /* mm_filter: every p-mer */
  GKC_FILTER_NEW = 2,       /* new_filter: 2nd and 3rd bases not both A */
  GKC_FILTER_SIGNATURE = 3  /* sign_filter: KMC2 signatures */
} gkc_filter;
gkc_status gkc_ctx_set_filter(gkc_ctx *ctx, int filter);
gkc_status gkc_ctx_synchronize(gkc_ctx *ctx);
uint64_t gkc_ctx_device_bytes(const gkc_ctx *ctx);
gkc_status gkc_ctx_release_workspace(gkc_ctx *ctx);
gkc_status gkc_last_timings(const gkc_ctx *ctx, gkc_timings *out);
int gkc_abi_version(void);

/* ---- partition (reference: GenSuperkmerGPU gkc_cuda.cu:376-541 with the
 *      process_func SKMStore::add_skms, superkmers.hpp:167-186) ---- */
gkc_status gkc_partition_device(gkc_ctx *ctx, const gkc_params *prm, const char *d_reads,
                                uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                gkc_partition_view *out);
gkc_status gkc_partition_host(gkc_ctx *ctx, const gkc_params *prm, const char *reads,
                              const uint64_t *offs, uint64_t n_reads, gkc_partition_view *out);
/* Copies the context's partition to host arrays sized from the view:
 * bin_skm_off[nbins+1], skm_len[n_superkmers], skm_byte_off[n_superkmers]
 * (into `packed`), packed[n_packed_bytes], minimizer[n_superkmers] (may be NULL;
 * all 0xFFFFFFFF for an imported partition, which carries none). */
gkc_status gkc_partition_copy_out(gkc_ctx *ctx, uint64_t *bin_skm_off, uint32_t *skm_len,
                                  uint64_t *skm_byte_off, uint8_t *packed, uint32_t *minimizer);

/* Balance of the context's partition.  bin_bases[b] (room for `capacity`
 * entries, at least nbins, or NULL) = the bases of the superkmers of bin b,
 * each superkmer counted with its k-1 overlap (reference: the part_sizes
 * that CalcSKMPartSize_instream, gkc_cuda.cu:350-365, adds up over all
 * batches).  The summary is the one
 * calVarStdev (experiment.cpp:18-37) logs: mean is the integer quotient,
 * variance the mean of (size - mean)^2 with each square taken in 64-bit
 * unsigned arithmetic and summed in double, in bin order.  `total` is the
 * exact 64-bit sum; the reference accumulates it in an int, so its figures
 * agree only while the total is below 2^31. */
typedef struct gkc_balance_stats {
  uint64_t total, mean, max, min;
  double variance, stdev, cv; /* cv = stdev / mean */
} gkc_balance_stats;
gkc_status gkc_partition_balance(gkc_ctx *ctx, uint64_t *bin_bases, uint32_t capacity,
                                 gkc_balance_stats *stats);

/* ---- superkmer exchange for bin sharding over several GPUs (no reference
 *      counterpart: the reference runs on one GPU).  Every GPU partitions
 *      its own reads; owner r of n_dest holds bins [bin_lo[r], bin_lo[r+1])
 *      and counts them after the exchange.  The transfer itself (an
 *      all-to-all of descriptors and one of bytes, split as returned) is the
 *      caller's. ---- */
/* Sender side, on the context's partition: for each destination in turn,
 * its superkmers' descriptors (bin order; byte offsets relative to that
 * destination's run of bytes) go to d_send_desc and their packed bytes to
 * d_send_bytes; skm_split and byte_split (n_dest entries each) receive the
 * run sizes, bin_skm and bin_kmers (nbins entries each, may be NULL) the
 * superkmers and k-mers of every bin.  Capacities equal to the view's
 * n_superkmers and n_packed_bytes always suffice. */
gkc_status gkc_exchange_pack(gkc_ctx *ctx, uint32_t n_dest, const uint32_t *bin_lo,
                             uint64_t *d_send_desc, uint64_t desc_capacity, uint8_t *d_send_bytes,
                             uint64_t bytes_capacity, uint64_t *skm_split, uint64_t *byte_split,
                             uint64_t *bin_skm, uint64_t *bin_kmers);
/* Receiver side: the runs of n_src senders, concatenated in sender order in
 * d_desc and d_bytes, become the context's partition with prm->nbins local
 * bins, ordered by bin and, inside a bin, by sender.  seg_bin_skm and
 * seg_bin_kmers hold n_src rows of nbins counts (the sender's bin_skm /
 * bin_kmers for this owner's bins), seg_bytes the n_src byte-run sizes.  The
 * inputs are copied before the call returns.  The resulting view has no
 * minimizers (skm_minimizer is NULL); gkc_count_device counts it. */
gkc_status gkc_partition_import(gkc_ctx *ctx, const gkc_params *prm, uint32_t n_src,
                                const uint64_t *seg_bin_skm, const uint64_t *seg_bin_kmers,
                                const uint64_t *seg_bytes, const uint64_t *d_desc,
                                const uint8_t *d_bytes, gkc_partition_view *out);

/* ---- counting (reference: kmc_counting_GPU kmer_counting.cu:59-199, per bin) ---- */
/* Counts the context's current partition, all bins. */
gkc_status gkc_count_device(gkc_ctx *ctx, const gkc_params *prm, gkc_mode mode,
                            gkc_count_view *out);
/* One group of packed superkmers in host memory (one bin), as
 * kmc_counting_GPU takes one SKMStore: lengths and each superkmer's bytes
 * back to back.  The distinct count is returned in *n_distinct; the sorted
 * list can then be fetched with gkc_count_copy_out. */
gkc_status gkc_count_superkmers_host(gkc_ctx *ctx, int k, const uint32_t *skm_len,
                                     const uint8_t *packed, uint64_t n_skm, gkc_mode mode,
                                     uint64_t *n_distinct);
/* Copies the last count result: bin_off[nbins+1], keys[n_distinct*key_words],
 * counts[n_distinct]; any pointer may be NULL, and each may point to host or
 * to device memory. */
gkc_status gkc_count_copy_out(gkc_ctx *ctx, uint64_t *bin_off, uint64_t *keys, uint32_t *counts);
/* Counts one group of packed superkmers already in device memory without
 * allocating anything.  No counterpart in the reference: it exists for callers
 * that cannot allocate device memory while they run (a program that owns the
 * whole GPU through its own memory pool, a framework whose allocator holds all
 * of HBM, or a path where a cudaMalloc would stall the device or break a hard
 * memory cap).  It needs no context; it runs on the calling thread's current
 * device and on `cuda_stream` (NULL: the default stream), and returns after
 * the stream has finished its work.
 *   Input: skm_len[n_skm] and the packed bytes back to back, as for
 *   gkc_count_superkmers_host (k <= 32).  Output: the distinct canonical
 *   k-mers in ascending order in d_keys_out and their counts in d_counts_out;
 *   both must hold out_capacity >= the group's k-mer count entries (the key
 *   buffer is also the sort's second buffer).  *n_distinct receives the count.
 * Scratch memory is one fixed array of about 23 MB of device memory inside
 * the library, held by every GPU that loads it until the process exits.  It
 * bounds a call to 131,072 superkmers and 1,048,576 k-mers: larger groups are
 * rejected with GKC_ERR_CAPACITY (GKC_ERR_INVALID_ARG for k > 32).  The first
 * call on a device looks up the array's device address, and with CUDA's lazy
 * module loading (the default) that lookup is what loads the library's
 * kernels and the array onto the device: make the first call at start-up,
 * before a memory pool claims the rest of HBM and before any stream capture.
 * The address is kept for the process's life, so the entry point must not be
 * used after cudaDeviceReset.  Every call waits on its stream (to read the
 * group's size, then the result); on a stream that is capturing it returns
 * GKC_ERR_INVALID_ARG without queuing work.  All calls share the one array
 * and each leaves its contents behind (the next call clears what must start
 * at zero), so calls that overlap on the GPU, from different streams or
 * threads, race and must not be made. */
gkc_status gkc_count_superkmers_device_noalloc(int k, const uint32_t *d_skm_len,
                                               const uint8_t *d_packed, uint64_t n_skm,
                                               uint64_t out_capacity, uint64_t *d_keys_out,
                                               uint32_t *d_counts_out, uint64_t *n_distinct,
                                               void *cuda_stream);

/* Output options over the last count result (reference: the min/max
 * frequency filter of kmc_counting_GPU, kmer_counting.cu:188-190, defaults
 * utilities.hpp:109, commented out there; the merged global list,
 * README.md:17,31-33).  merged = 0: per bin, the (k-mer, count) pairs with
 * min_count <= count <= max_count; merged = 1: one sorted list over all bins,
 * the counts of a k-mer found in several bins added up (clamped to
 * UINT32_MAX), then the same filter.  *n_out receives the number of pairs;
 * when bin_off (nbins+1 entries, or 2 when merged), keys (n_out * key_words)
 * and counts (n_out) are not NULL they receive the list.  Calling first with
 * NULL arrays to size them and again to copy computes the list once. */
gkc_status gkc_count_output(gkc_ctx *ctx, uint32_t min_count, uint32_t max_count, int merged,
                            uint64_t *n_out, uint64_t *bin_off, uint64_t *keys, uint32_t *counts);

/* ---- on-disk k-mer database, KMC-style: a prefix lookup table and
 *      fixed-width (suffix, counter) records in key order (no reference
 *      code; README.md:17 names KMC3's counting as the use case).  Files
 *      <path>.gkc_pre and <path>.gkc_suf:
 *        gkc_pre  "GKCP", u32 version 1, u32 k, lut_prefix_len l, suffix_bytes,
 *                 counter_bytes, min_count, max_count, u64 n_kmers,
 *                 total_count, u64 lut[4^l + 1] (first record of each
 *                 prefix = key >> 2(k-l)), "GKCP"
 *        gkc_suf  "GKCS", n_kmers x (the key's low 2(k-l) bits big-endian in
 *                 suffix_bytes, count little-endian in counter_bytes), "GKCS"
 *      Integers little-endian.  counter_bytes is the fewest (1..4) that hold
 *      the largest count. ---- */
typedef struct gkc_db gkc_db;
typedef struct gkc_db_info {
  uint32_t k, lut_prefix_len, suffix_bytes, counter_bytes, min_count, max_count;
  uint64_t n_kmers, total_count;
} gkc_db_info;
/* Writes the merged list of the last count result (gkc_count_output with
 * merged = 1 and the given bounds).  lut_prefix_len 0 picks about eight
 * records per table entry; otherwise 1..13 and below k. */
gkc_status gkc_db_write(gkc_ctx *ctx, const char *path, uint32_t min_count, uint32_t max_count,
                        int lut_prefix_len);
/* Host reader (maps the records; needs no GPU). */
gkc_status gkc_db_open(const char *path, gkc_db **out);
void gkc_db_close(gkc_db *db);
gkc_status gkc_db_get_info(const gkc_db *db, gkc_db_info *out);
/* counts[i] = count of keys[i] (key_words per key as in the count view), 0 if absent. */
gkc_status gkc_db_lookup(const gkc_db *db, const uint64_t *keys, uint64_t n, uint32_t *counts);
/* Records first .. first+n-1 as keys and counts (either may be NULL). */
gkc_status gkc_db_read(const gkc_db *db, uint64_t first, uint64_t n, uint64_t *keys, uint32_t *counts);

/* ---- launch-shape tuning (the reference fixes its launch shape by hand:
 *      NUM_BLOCKS_PER_GRID, NUM_THREADS_PER_BLOCK and the stream count,
 *      experiment.cpp:234-238).  Shapes of the batched count stage that need
 *      no rebuild: the largest mean keys per count bucket (the coarse digit
 *      width of each bin follows from it), the k-mers per histogram chunk
 *      (a power of two) and the count kernel's CTAs per SM.  Zero fields
 *      mean the default. ---- */
typedef struct gkc_tune_params {
  uint32_t coarse_target;      /* 256 .. 65536; default 8192 */
  uint32_t chunk_kmers;        /* 4096 .. 2^22, a power of two; default 65536 */
  uint32_t count_ctas_per_sm;  /* 1 .. 4; default 2 */
  uint32_t reserved;
} gkc_tune_params;
typedef struct gkc_tune_report {
  gkc_tune_params chosen, defaults;
  float default_ms, tuned_ms;  /* count stages on the sample, median of 3 replays */
  uint32_t candidates;         /* shapes timed */
  int from_cache;              /* 1: taken from the cache, nothing timed */
  uint64_t sample_bases;
} gkc_tune_report;
gkc_status gkc_tune_get(const gkc_ctx *ctx, gkc_tune_params *out);
/* NULL restores the defaults.  Applies to the context's later calls. */
gkc_status gkc_tune_set(gkc_ctx *ctx, const gkc_tune_params *p);
/* Chooses the shapes for this input's class by timing candidates on a sample
 * of the reads (the first ones, about 2^30 bases; run with the bin count
 * scaled down so its bins hold as many bases as the full input's), one
 * dimension at a time from the defaults, and sets them on the context.  The
 * choice is cached per (SM count, key width, read-length class: mean above
 * 1 kbp or not, bin count, bases per bin in factors of 4); a cached choice is
 * used without timing unless force != 0.  The context's partition and count
 * results are replaced by the sample's. */
gkc_status gkc_autotune_device(gkc_ctx *ctx, const gkc_params *prm, const char *d_reads, uint64_t n_bytes,
                               const uint64_t *d_offs, uint64_t n_reads, int force, gkc_tune_report *out);
/* The process-wide cache (host only, needs no GPU). */
gkc_status gkc_tune_cache_lookup(int sm_count, const gkc_params *prm, uint64_t n_bases, uint64_t n_reads,
                                 gkc_tune_params *out);
gkc_status gkc_tune_cache_store(int sm_count, const gkc_params *prm, uint64_t n_bases, uint64_t n_reads,
                                const gkc_tune_params *p);
void gkc_tune_cache_clear(void);
/* Text file, one entry per line; load merges into the cache. */
gkc_status gkc_tune_cache_save(const char *path);
gkc_status gkc_tune_cache_load(const char *path);

/* ---- whole pipeline: reads -> superkmer partitions -> sorted (k-mer, count)
 *      (reference: process_reads_count + gen_skm_and_count_with_TP,
 *      experiment.cpp:76-89,156-219) ---- */
gkc_status gkc_pipeline_device(gkc_ctx *ctx, const gkc_params *prm, gkc_mode mode,
                               const char *d_reads, uint64_t n_bytes, const uint64_t *d_offs,
                               uint64_t n_reads, gkc_partition_view *part, gkc_count_view *cnt);
gkc_status gkc_pipeline_host(gkc_ctx *ctx, const gkc_params *prm, gkc_mode mode,
                             const char *reads, const uint64_t *offs, uint64_t n_reads,
                             gkc_count_view *cnt);

/* ---- streaming host form: consecutive calls overlap.  Each submitted call
 *      is copied in, counted and its result copied out into the caller's
 *      buffers on separate streams, so that one call's upload, the previous
 *      call's counting and the one before's download run at the same time
 *      (two calls' inputs and outputs are held on the device).  All buffers
 *      must be page-locked host memory (cudaHostAlloc or cudaHostRegister),
 *      read or written by the device until gkc_stream_wait returns for the
 *      call; a call's results go to bin_off[nbins+1], keys and counts (room
 *      for `capacity` pairs).  The reads of a call may be cut from a larger
 *      CSR (offs[0] need not be 0).  A call whose reads have the size of the
 *      call two before (the same buffer slot) replays that call's captured
 *      pipeline; another size captures anew, which waits for the device.
 *      gkc_stream_wait blocks until the call's results are in host memory
 *      and returns its status; at most two calls may be in flight, and the
 *      context's device views do not describe them.  (No reference
 *      counterpart: the reference uploads, computes and downloads each batch
 *      in turn, gkc_cuda.cu:414-498.) ---- */
/* The download of call t is three DMA copies, enqueued once its pipeline is
 * done: by gkc_stream_wait(t), or by the next gkc_stream_submit when call t
 * has finished by then.  Up to four calls may await their wait (a fifth
 * submit returns GKC_ERR_INVALID_ARG before doing anything); call t
 * reuses call t-2's device buffers, so submitting t before waiting for t-2
 * (with a third set of host outputs) lets t's upload run during t-2's
 * download. */
gkc_status gkc_stream_submit(gkc_ctx *ctx, const gkc_params *prm, const char *reads, const uint64_t *offs,
                             uint64_t n_reads, uint64_t *bin_off, uint64_t *keys, uint32_t *counts,
                             uint64_t capacity, uint64_t *ticket);
gkc_status gkc_stream_wait(gkc_ctx *ctx, uint64_t ticket, uint64_t *n_distinct, uint64_t *n_kmers);

/* ---- per-window minimizers with position and strand (reference declares
 *      d_mm_pos / d_mm_strand, gkc_cuda.cu:159-160, but never fills them).
 *      Arrays have n_bytes entries indexed by window start in the CSR;
 *      windows that do not fit in their read hold minimizer 0xFFFFFFFF. ---- */
gkc_status gkc_minimizers_device(gkc_ctx *ctx, const gkc_params *prm, const char *d_reads,
                                 uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                 uint32_t *d_minimizer, uint8_t *d_pos, int8_t *d_strand);

/* ---- sub-sampled counting with position lists: k-mers whose window
 *      minimizer % mod == 0, each with the ascending list of its window start
 *      offsets in the CSR (README.md:16 use case; no reference code). ---- */
typedef struct gkc_poslist_view {
  uint64_t n_distinct, n_positions;
  int key_words;
  const uint64_t *keys;      /* ascending */
  const uint64_t *pos_off;   /* n_distinct + 1 */
  const uint32_t *positions;
} gkc_poslist_view;
gkc_status gkc_subsample_positions_device(gkc_ctx *ctx, const gkc_params *prm, uint32_t mod,
                                          const char *d_reads, uint64_t n_bytes,
                                          const uint64_t *d_offs, uint64_t n_reads,
                                          gkc_poslist_view *out);

/* ---- homopolymer compression alone (reference: GPU_HPCEncoding
 *      gkc_cuda.cu:164-192, with the per-read start index) ---- */
gkc_status gkc_hpc_device(gkc_ctx *ctx, const char *d_reads, uint64_t n_bytes,
                          const uint64_t *d_offs, uint64_t n_reads, char *d_out_reads,
                          uint64_t *d_out_offs, int32_t *d_orig_pos);

/* ---- FASTA / FASTQ ingest (reference: ReadLoader, read_loader.hpp:44-196,
 *      :276-321, :470-520).  Reads the file on n_threads threads (0: all
 *      cores) into one read CSR, in file order: *reads holds the sequences
 *      back to back, *offs their n_reads+1 offsets.  By default the
 *      reference's rules: FASTQ when the file name ends in 'q', else FASTA
 *      (:285); FASTQ: the second line of each 4-line record; FASTA: the line
 *      after each header (the reference reads two-line records).  Flags:
 *      GKC_FASTX_JOIN_LINES joins all lines of a FASTA record up to the next
 *      header; GKC_FASTX_FORMAT_FROM_CONTENT takes the format from the first
 *      byte ('>' or '@') instead of the name.  A '\r' before a line end is
 *      dropped.  A file that does not start as its format does is refused
 *      (GKC_ERR_INVALID_ARG).  With pinned != 0 the arrays are page-locked
 *      (fast host-to-device copies).  Free them with gkc_fastx_free and the
 *      same `pinned`.  No GPU is needed unless pinned != 0. ---- */
#define GKC_FASTX_JOIN_LINES 1
#define GKC_FASTX_FORMAT_FROM_CONTENT 2
gkc_status gkc_fastx_load(const char *path, int n_threads, int pinned, char **reads, uint64_t **offs,
                          uint64_t *n_reads);
gkc_status gkc_fastx_load_ex(const char *path, int n_threads, int pinned, int flags, char **reads,
                             uint64_t **offs, uint64_t *n_reads);
void gkc_fastx_free(char *reads, uint64_t *offs, int pinned);

/* ---- serving: continuous batching of counting jobs against an HBM budget ---- */
typedef struct gkc_server gkc_server;
typedef enum gkc_job_state {
  GKC_JOB_QUEUED = 0,
  GKC_JOB_RUNNING = 1,
  GKC_JOB_DONE = 2,
  GKC_JOB_FAILED = 3,
  GKC_JOB_CANCELLED = 4
} gkc_job_state;
typedef struct gkc_job_info {
  gkc_job_state state;
  gkc_status status;
  uint64_t n_bases, n_kmers, n_distinct;
  uint32_t nbins;
  int key_words;
  double submit_s, start_s, end_s;   /* seconds since server start */
  uint64_t hbm_bytes;                /* admitted budget */
} gkc_job_info;
gkc_status gkc_server_create(int device_id, uint64_t hbm_budget_bytes, int max_running,
                             gkc_server **out);
void gkc_server_destroy(gkc_server *srv);
/* The server copies the reads; the caller may free them after return. */
gkc_status gkc_server_submit(gkc_server *srv, const gkc_params *prm, const char *reads,
                             const uint64_t *offs, uint64_t n_reads, uint64_t *job_id);
gkc_status gkc_server_submit_device_synth(gkc_server *srv, const gkc_params *prm, int generator,
                                          uint64_t seed, uint64_t n_bases, uint64_t *job_id);
gkc_status gkc_server_poll(gkc_server *srv, uint64_t job_id, gkc_job_info *info);
gkc_status gkc_server_wait(gkc_server *srv, uint64_t job_id, double timeout_s, gkc_job_info *info);
gkc_status gkc_server_cancel(gkc_server *srv, uint64_t job_id);
gkc_status gkc_server_copy_result(gkc_server *srv, uint64_t job_id, uint64_t *bin_off,
                                  uint64_t *keys, uint32_t *counts);
gkc_status gkc_server_release(gkc_server *srv, uint64_t job_id);
uint64_t gkc_job_hbm_estimate(const gkc_params *prm, uint64_t n_bases, uint64_t n_reads);

/* ---- synthetic workloads (seeded; same bytes on host and device) ---- */
gkc_status gkc_synth_iid_reads(int on_device, uint64_t seed, uint64_t n_reads, uint32_t read_len,
                               double n_rate, char *out, uint64_t *offs);
gkc_status gkc_synth_genome(int on_device, uint64_t seed, uint64_t genome_len,
                            double seg_fraction, double divergence, uint8_t *genome_codes);
gkc_status gkc_synth_short_reads(int on_device, uint64_t seed, const uint8_t *genome_codes,
                                 uint64_t genome_len, uint64_t first_read, uint64_t n_reads,
                                 uint32_t read_len, double err_rate, char *out, uint64_t *offs);
/* Long-read lengths (host only): lognormal(median, sigma) clipped to
 * [min_len, max_len], until the sum reaches total_bases; returns the count. */
uint64_t gkc_synth_long_read_offsets(uint64_t seed, double median, double sigma, uint32_t min_len,
                                     uint32_t max_len, uint64_t total_bases, uint64_t max_reads,
                                     uint64_t *offs);
gkc_status gkc_synth_long_reads(int on_device, uint64_t seed, const uint8_t *genome_codes,
                                uint64_t genome_len, uint64_t n_reads, const uint64_t *offs,
                                char *out);

#ifdef __cplusplus
}
#endif
#endif
