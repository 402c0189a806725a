// Kernel argument blocks and launch helpers shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace gkc {

struct PartArgs {
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
  uint32_t target_bucket;      // desired mean keys per bucket
  uint32_t max_bits;           // bucket bits cap (<= 12)
  uint32_t chunk_skm;          // superkmers per expansion chunk
  int k;
  const uint32_t *err;         // nothing is planned after an upstream overflow
  // outputs
  uint32_t *bin_bits;          // bucket bits per bin
  uint64_t *bucket_base;       // first bucket of each bin (nbins+1)
  uint64_t *chunk_base;        // first chunk of each bin (nbins+1)
};
__global__ void k_count_plan(CountPlan pl);

struct ExpandArgs {
  const uint64_t *desc;        // bin-ordered superkmer descriptors
  const uint8_t *packed;
  uint32_t nbins;
  const uint64_t *bin_start;
  const uint64_t *chunk_base;
  const uint32_t *bin_bits;
  const uint64_t *bucket_base;
  uint32_t chunk_skm;
  int k;
  unsigned long long *bucket_count;   // histogram pass output
  unsigned long long *bucket_cursor;  // scatter pass: running fill
  void *keys;                         // scatter pass output (uint64 or u128)
  uint64_t keys_cap;
  uint32_t *err;
};
template <typename K> __global__ void k_bucket_hist(ExpandArgs a);
template <typename K> __global__ void k_bucket_scatter(ExpandArgs a);

struct SortCountArgs {
  const uint64_t *bucket_start;   // n_buckets + 1 (device exclusive prefix of bucket sizes)
  const uint64_t *n_buckets_dev;  // device-side bucket count (bucket_base[nbins])
  const uint64_t *bucket_base;    // per bin
  const uint32_t *bin_bits;
  uint32_t nbins;
  int k;
  void *keys;                     // bucketed keys (sorted output may alias it)
  void *out_keys;
  uint32_t *out_counts;
  uint64_t *bucket_out;           // exclusive output offset per bucket (n_buckets + 1)
  unsigned long long *status;     // look-back words, zeroed
  unsigned long long *ticket;     // zeroed
  void *scratch;                  // 2 * scratch_keys keys for oversized buckets
  uint64_t scratch_keys;
  uint32_t *scratch_cnt;          // 16 * 4096 counters
  uint32_t *err;
  unsigned long long *prof;       // optional cycle counters (GKC_PROFILE_SORT), else null
};
template <typename K> __global__ void k_sort_count(SortCountArgs a);
template <typename K> size_t sort_count_smem_bytes();
template <typename K> int sort_count_cap();
constexpr int kSortThreads = 512;

__global__ void k_bin_out_offsets(const uint64_t *bucket_out, const uint64_t *bucket_base,
                                  uint32_t nbins, uint64_t *bin_out);

// device-wide exclusive scan of uint64 counters (n <= 2^31)
void scan_u64(const unsigned long long *in, uint64_t *out, uint64_t n, uint64_t *block_tmp,
              cudaStream_t st);
size_t scan_u64_tmp_words(uint64_t n);

}  // namespace gkc

namespace gkc {
__global__ void k_hpc_count(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            unsigned long long *run_len);
__global__ void k_hpc_write(const uint8_t *reads, const uint64_t *offs, uint64_t n_reads,
                            const uint64_t *hpc_offs, uint8_t *out, int32_t *orig_pos);
}  // namespace gkc
