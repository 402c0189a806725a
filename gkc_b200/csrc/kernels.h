// Kernel argument blocks and launch helpers shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace gkc {

struct PartArgs {
  int filter;            // minimizer filter (FILTER_*)
  const uint8_t *reads;  // concatenated read bytes (CSR), offsets rebased to 0
  uint64_t nbytes;       // byte count (an upper bound when nbytes_dev is set)
  const uint64_t *nbytes_dev;  // optional: device-side byte count
  int aligned16;         // reads is 16-byte aligned
  const uint32_t *rs_bits;  // read-start bitmap, bit nbytes set
  uint64_t rs_words;
  int k, p, nbins, nbins_smem;
  uint64_t *skm_desc;    // (packed byte offset << 24) | length in bases
  uint32_t *skm_mm;      // minimizer of the superkmer
  uint64_t *skm_gpos;    // optional: global position of its first base
  uint8_t *packed;       // 2-bit packed superkmer bases
  unsigned long long *cursors;  // [0] superkmers, [1] packed bytes (16-byte rounded per tile)
  uint64_t cap_skm, cap_bytes;
  unsigned long long *bin_nskm, *bin_nkmers;
  uint32_t *err;
};

constexpr int kPartThreads = 512;
constexpr int kPartTile = 4096;
size_t partition_smem_bytes(int nbins_smem);
__global__ void k_partition(PartArgs a);
constexpr int kBinChunk = 8192;          // superkmers per placement chunk
constexpr int kBinRound = 2048;          // superkmers grouped by bin at a time
constexpr int kBinPlaceThreads = 512;
size_t bin_place_smem_bytes(uint32_t nbins);
constexpr int kBinPlaceMaxBins = 2048;   // larger bin counts use k_bin_scatter
__global__ void k_bin_count(const unsigned long long *n_skm_ptr, const uint32_t *mm, uint32_t nbins,
                            uint64_t nch_cap, unsigned long long *mat, const uint32_t *err);
__global__ void k_bin_place(const unsigned long long *n_skm_ptr, const uint64_t *desc, const uint32_t *mm,
                            uint32_t nbins, uint64_t nch_cap, const uint64_t *off, uint64_t *out_desc,
                            uint32_t *out_mm, const uint32_t *err);
__global__ void k_read_start_bits(const uint64_t *offs, uint64_t n_reads, uint32_t *bits);
__global__ void k_bin_scatter(const unsigned long long *n_skm_ptr, const uint64_t *desc,
                              const uint32_t *mm, uint32_t nbins, const uint64_t *bin_start,
                              unsigned long long *bin_fill, uint64_t *out_desc, uint32_t *out_mm,
                              const uint64_t *gpos, uint64_t *out_gpos, const uint32_t *err);
__global__ void k_bin_prefix(const unsigned long long *bin_nskm,
                             const unsigned long long *bin_nkmers, uint32_t nbins,
                             uint64_t *bin_start, uint64_t *bin_kstart);

// ---- counting ----
struct CountPlan {
  // inputs
  uint32_t nbins;
  const uint64_t *bin_start;   // superkmers per bin (exclusive prefix, nbins+1)
  const uint64_t *bin_kstart;  // k-mers per bin (exclusive prefix, nbins+1)
  uint32_t coarse_target;      // desired largest mean keys per coarse bucket
  uint32_t max_bits;           // coarse bucket bits cap (<= kCoarseMaxBits)
  uint64_t chunk_kmers;        // k-mers per expansion chunk
  int k;
  const uint32_t *err;         // nothing is planned after an upstream overflow
  // outputs
  uint32_t *bin_bits;          // coarse bucket bits per bin
  uint64_t *bucket_base;       // first coarse bucket of each bin (nbins+1)
  uint64_t *chunk_base;        // first chunk of each bin (nbins+1)
  uint64_t *hist_base;         // first (digit, chunk) entry of each bin (nbins+1)
};
__global__ void k_count_plan(CountPlan pl);

struct ExpandArgs {
  const uint64_t *desc;        // bin-ordered superkmer descriptors
  const uint64_t *koff;        // k-mer offset of each bin-ordered superkmer (n + 1)
  const uint8_t *packed;
  uint32_t nbins;
  const uint64_t *bin_start;
  const uint64_t *bin_kstart;
  const uint64_t *chunk_base;
  const uint64_t *hist_base;
  const uint64_t *bucket_base;
  const uint32_t *bin_bits;
  uint64_t chunk_kmers;
  int k;
  uint64_t *chunk_s0;          // first superkmer of each chunk
  uint32_t *hist;              // (bin, chunk, digit) counts, then write offsets in the bin
  void *keys;                  // scatter output (uint64 or u128)
  void *flat;                  // the keys in k-mer order (written by the histogram, read by the scatter)
  uint64_t keys_cap;          // of keys and flat
  uint32_t *big_list;          // buckets of at least big_min keys (listed by the scan, counted first)
  unsigned long long *big_count;  // zeroed
  uint64_t big_min;
  uint32_t *err;
};
__global__ void k_chunk_first(ExpandArgs a);
template <typename K> __global__ void k_bucket_hist(ExpandArgs a);
__global__ void k_bucket_scan(ExpandArgs a, uint64_t *bucket_start, uint64_t *bucket_size, uint32_t *bucket_bin);
template <typename K> __global__ void k_bucket_scatter(ExpandArgs a);
constexpr int kBucketScanThreads = 1024;
constexpr int kBucketHistThreads = 256;
constexpr int kBucketScatterThreads = 1024;
template <typename K> size_t bucket_scatter_smem_bytes();
__global__ void k_skm_nk(const uint64_t *desc, const unsigned long long *n_skm_dev, int k,
                         unsigned long long *nk);

struct SortCountArgs {
  uint32_t nbins;
  int k;
  const uint64_t *bucket_base;    // buckets per bin (prefix, nbins + 1)
  const uint32_t *bin_bits;
  const uint64_t *bucket_start;   // first key of each bucket
  const uint64_t *bucket_size;
  const uint32_t *bucket_bin;     // bin of each bucket
  const void *keys;               // bucketed keys
  void *scratch;                  // oversized buckets, placed by sub-bucket at their own key range
  uint32_t *slice_starts;         // per CTA: sub-bucket starts of its current large bucket (4097 each)
  void *stage_keys;               // runs of bucket g at [bucket_start[g], + its distinct count)
  uint32_t *stage_counts;
  uint64_t stage_cap;
  unsigned long long *bucket_d;   // distinct keys of each bucket
  unsigned long long *ticket;     // zeroed
  const uint32_t *big_list;       // buckets of at least big_min keys, taken before the others
  const unsigned long long *big_count;
  unsigned long long *big_ticket;  // zeroed
  uint64_t big_min;
  uint32_t *err;
};
template <typename K> __global__ void k_bucket_count(SortCountArgs a);
template <typename K> size_t bucket_count_smem_bytes();
template <typename K> uint64_t bucket_count_cap();  // keys of the largest bucket counted in shared memory
template <typename K>
__global__ void k_compact_runs(const K *stage_keys, const uint32_t *stage_counts, const uint64_t *bucket_start,
                               const unsigned long long *bucket_d, const uint64_t *bucket_out,
                               const uint64_t *bucket_base, uint32_t nbins, K *out_keys, uint32_t *out_counts,
                               uint64_t *bin_out, const uint32_t *err);
constexpr int kBucketCountThreads = 512;
constexpr uint32_t kCoarseTarget = 8192;
constexpr uint32_t kCoarseMaxBits = 12;
constexpr uint64_t kChunkKmers = 65536;

// device-wide exclusive scan of uint64 counters (n <= 2^31)
void scan_u64(const unsigned long long *in, uint64_t *out, uint64_t n, uint64_t *block_tmp,
              cudaStream_t st);
size_t scan_u64_tmp_words(uint64_t n);
// the same over a device-side length min(*n_dev, n_cap); out[n] = total
void scan_u64_dev(const unsigned long long *in, uint64_t *out, uint64_t n_cap, const uint64_t *n_dev,
                  uint64_t *block_tmp, cudaStream_t st);

}  // namespace gkc

namespace gkc {
__global__ void k_hpc_count(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            unsigned long long *run_len);
__global__ void k_hpc_write(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            const uint64_t *hpc_offs, uint8_t *out, int32_t *orig_pos);
// Run-length pass over sorted keys (distinct keys + first indices).
uint64_t rle_block_count(uint64_t n);
template <typename K>
void rle_runs(const K *sorted, uint64_t n, unsigned long long *blk, uint64_t *blk_off, uint64_t *tmp,
              const unsigned long long *cursor, K *out_keys, uint64_t *starts, cudaStream_t st);

}  // namespace gkc
