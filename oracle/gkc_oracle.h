/* Oracle for the GKC partition-and-count path: a plain-C CPU restatement.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library calls, links or
 * loads this code; only the tests, the smoke check and the benchmark's CPU
 * baseline leg use it, and only to check results.
 *
 * Parity of the k <= 32 partition and count semantics (including the
 * N-smear of the minimizer kernel and the run-collapse of HPC) is pinned
 * against the reference's own implementation compiled from its sources
 * (oracle/Makefile -> oracle/_ref) and the golden fixtures under
 * tests/golden/.  The k > 32 (128-bit) keys, the per-window
 * (minimizer, position, strand) emission and the sub-sampled position lists
 * have no counterpart in the reference; for those this restatement IS the
 * definition ("parity unpinned").
 */
#ifndef GKC_ORACLE_H
#define GKC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Superkmers in read order (reads in CSR order, superkmers left to right). */
typedef struct {
  uint64_t n_skm;
  uint64_t n_bytes;
  uint32_t *bin;      /* minimizer % nbins of the superkmer's first window */
  uint32_t *len;      /* bases */
  uint64_t *byte_off; /* offset of the packed bytes in `bytes` */
  uint64_t *read_id;  /* read the superkmer came from */
  uint32_t *start;    /* first window (= first base) inside the (HPC) read */
  uint32_t *minimizer;
  uint8_t *bytes;     /* 2 bits per base, MSB first, each superkmer byte-aligned */
} orc_skms;

/* Per-bin sorted (k-mer, count) lists. keys_hi is NULL for k <= 32. */
typedef struct {
  uint32_t nbins;
  uint64_t n_distinct;
  uint64_t *bin_off; /* nbins + 1 */
  uint64_t *keys_lo;
  uint64_t *keys_hi;
  uint32_t *counts;
} orc_counts;

/* Sub-sampled k-mers with position lists (CSR). */
typedef struct {
  uint64_t n_distinct;
  uint64_t n_pos;
  uint64_t *keys_lo;
  uint64_t *keys_hi;
  uint64_t *pos_off; /* n_distinct + 1 */
  uint32_t *pos;     /* global base offsets in the read CSR */
} orc_poslists;

int orc_version(void);
/* Minimizer filter for later calls: 0 new_filter2 (default), 1 every p-mer,
 * 2 new_filter, 3 sign_filter (the reference's FILTER_KERNEL variants). */
void orc_set_filter(int filter);

/* Run-collapse of each read (HPC).  out_reads uses the input CSR layout;
 * out_len[r] = number of runs; orig_pos[offs[r] + j] = in-read index of the
 * first base of run j. */
void orc_hpc(const uint8_t *reads, const uint64_t *offs, int64_t n_reads,
             uint8_t *out_reads, int32_t *out_len, int32_t *orig_pos);

/* Canonical minimizer of every k-window of one read, reference semantics
 * (including non-ACGTU bytes).  mm has len-k+1 entries. */
void orc_window_minimizers(const uint8_t *read, int32_t len, int k, int p, uint32_t *mm);

/* Minimizer position inside each window (0..k-p) and strand (0 forward,
 * 1 reverse complement, -1 palindromic p-mer; 255/0 when no p-mer passes). */
void orc_window_minimizer_pos(const uint8_t *read, int32_t len, int k, int p,
                              uint32_t *mm, uint8_t *pos, int8_t *strand);

/* Superkmer partition of all reads. Returns 0 on success. */
int orc_partition(const uint8_t *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                  int hpc, int nbins, orc_skms *out);
void orc_skms_free(orc_skms *s);

/* Count canonical k-mers of the superkmers, per bin (k <= 64). */
int orc_count_bins(const orc_skms *s, int k, int nbins, orc_counts *out);
void orc_counts_free(orc_counts *c);

/* Count from raw packed superkmer arrays (one group = one bin). */
int orc_count_packed(const uint32_t *len, const uint64_t *byte_off, const uint8_t *bytes,
                     uint64_t n_skm, int k, orc_counts *out);

/* k-mers whose window minimizer % mod == 0, with the sorted list of their
 * window start offsets (global, in the read CSR). HPC off. */
int orc_subsample_positions(const uint8_t *reads, const uint64_t *offs, int64_t n_reads,
                            int k, int p, uint32_t mod, orc_poslists *out);
void orc_poslists_free(orc_poslists *p);

/* Partition balance.  sizes[b] = bases of the superkmers of bin b, each
 * superkmer with its k-1 overlap (the part_sizes of CalcSKMPartSize_instream,
 * gkc_cuda.cu:350-365); the summary calVarStdev logs (experiment.cpp:18-37)
 * with the total kept in 64 bits. */
typedef struct {
  uint64_t total, mean, max, min;
  double variance, stdev, cv;
} orc_balance;
void orc_partition_sizes(const orc_skms *s, int nbins, uint64_t *sizes);
void orc_balance_stats(const uint64_t *sizes, int n, orc_balance *out);

void orc_free(void *p);

/* Digests of large outputs (test infrastructure): per bin, a sum of mixed
 * words over the bin's sorted (key, count) list, the index in the bin
 * included; and a multiset digest of a partition's (length, packed bytes)
 * per bin.  Each returns the digest over all bins; the per-bin arrays may be
 * NULL.  keys_hi is NULL for 64-bit keys. */
uint64_t orc_counts_digest(const uint64_t *bin_off, uint32_t nbins, const uint64_t *keys_lo,
                           const uint64_t *keys_hi, const uint32_t *counts, uint64_t *bin_digest);
uint64_t orc_skm_multiset_digest(const uint32_t *bin, const uint32_t *len, const uint64_t *byte_off,
                                 const uint8_t *bytes, uint64_t n_skm, uint32_t nbins,
                                 uint64_t *bin_digest, uint64_t *bin_count);

#ifdef __cplusplus
}
#endif
#endif
