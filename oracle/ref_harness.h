// C entry points of the reference harness (oracle/_ref/libgkcref.so).
// TEST INFRASTRUCTURE: the reference's own kernels (gkc_cuda.cu), superkmer
// store (superkmers.hpp) and counting step (kmer_counting.cu, Thrust host
// backend), compiled from the reference sources and driven the way
// GenSuperkmerGPU (gkc_cuda.cu:376-541) and gen_skm_and_count_with_TP
// (experiment.cpp:156-219) drive them.
#pragma once
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint64_t n_skm;
  uint64_t n_bytes;
  uint32_t *bin;
  uint32_t *len;
  uint64_t *byte_off;
  uint8_t *bytes;
} ref_skms;

typedef struct {
  uint32_t nbins;
  uint64_t n_distinct;
  uint64_t *bin_off;   // nbins + 1
  uint64_t *keys;
  uint32_t *counts;
  uint64_t *returned;  // per bin: kmc_counting_GPU's return value
} ref_counts;

// Partition: batches of batch_reads reads (the reference uses
// NUM_BLOCKS_PER_GRID * NUM_THREADS_PER_BLOCK = 2048), n_threads batches in
// flight, superkmers dumped from the per-bin SKMStore queues.
int ref_partition(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                  int hpc, int nbins, int batch_reads, int n_threads, ref_skms *out);
void ref_skms_free(ref_skms *s);

// Bases of the superkmers of each bin as CalcSKMPartSize_instream
// (gkc_cuda.cu:350-365) adds them up over the batches; nbins <= 512.
int ref_partition_sizes(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                        int hpc, int nbins, int batch_reads, int n_threads, uint64_t *sizes);

// The report calVarStdev (experiment.cpp:18-37) logs for the sizes, as text
// (its two log lines); returns the text length.
int ref_cal_var_stdev(const uint64_t *sizes, int n, char *buf, int cap);

// Per-bin counting through kmc_counting_GPU; the sorted keys and run lengths
// it computes (and discards) are captured.  k <= 32.
int ref_count_bins(const ref_skms *s, int k, int nbins, int n_threads, ref_counts *out);
void ref_counts_free(ref_counts *c);

// Whole reference CPU path (partition + per-bin count in a thread pool);
// returns the summed distinct count (experiment.cpp:203-211) and k-mers.
int ref_pipeline(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int hpc,
                 int nbins, int batch_reads, int n_threads, uint64_t *distinct_out,
                 uint64_t *kmers_out);

// The same with the per-bin sorted (k-mer, count) lists returned (k <= 32).
int ref_pipeline_counts(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                        int hpc, int nbins, int batch_reads, int n_threads, uint64_t *kmers_out,
                        ref_counts *out);

#ifdef __cplusplus
}
#endif
