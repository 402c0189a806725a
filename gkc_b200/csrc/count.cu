// Canonical k-mer counting from bin-grouped superkmers (batched path).
//
// Semantics follow kmc_counting_GPU (kmer_counting.cu:95-191): every k-mer of
// every superkmer of a bin, canonicalised as min(x, revcomp(x)), sorted
// ascending, run-length counted (count clamped to 2^32-1), per bin.
//
// Device layout:
//   1. k_bucket_hist   - expands each bin's superkmers (rolling forward and
//                        reverse-complement keys) and histograms the top
//                        `bin_bits[b]` bits of the canonical key per bin;
//   2. scan            - bucket sizes -> bucket offsets;
//   3. k_bucket_scatter- re-expands and writes every key into its (bin,
//                        prefix) bucket, runs staged through shared memory;
//   4. k_sort_count    - persistent: one bucket per CTA iteration, taken in
//                        key order; the bucket is sorted in shared memory
//                        (one MSD counting pass on the next digit, leaves by
//                        insertion sort, large leaves by a bitonic network),
//                        run-length counted, and written at its output offset
//                        found by a decoupled look-back over the buckets
//                        before it.  Buckets larger than shared memory are
//                        split by MSD passes through global scratch.
#include "common.cuh"
#include "kernels.h"

namespace gkc {

// ------------------------------------------------------------------ planning

__global__ void k_count_plan(CountPlan pl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool dead = (*pl.err & (ERR_CAPACITY | ERR_BAD_READ)) != 0;
  uint64_t bb = 0, cb = 0;
  for (uint32_t b = 0; b < pl.nbins; b++) {
    uint64_t nk = dead ? 0 : pl.bin_kstart[b + 1] - pl.bin_kstart[b];
    uint64_t ns = dead ? 0 : pl.bin_start[b + 1] - pl.bin_start[b];
    uint32_t bits = 0;
    while (bits < pl.max_bits && (int)bits < 2 * pl.k && (nk >> bits) > pl.target_bucket) bits++;
    pl.bin_bits[b] = bits;
    pl.bucket_base[b] = bb;
    bb += 1ull << bits;
    pl.chunk_base[b] = cb;
    cb += (ns + pl.chunk_skm - 1) / pl.chunk_skm;
  }
  pl.bucket_base[pl.nbins] = bb;
  pl.chunk_base[pl.nbins] = cb;
}

// ----------------------------------------------------------------- expansion

// Calls f(canonical key) for every k-mer of one packed superkmer.  The
// forward key rolls in from the right; the reverse complement rolls in from
// the top, so min(x, rc) is the reference's canonicalkmer (kmer_counting.cu:33-44).
template <typename K, typename F>
GKC_DEV void expand_skm(const uint8_t *packed, uint64_t desc, int k, F &&f) {
  const uint64_t off = desc >> 24;
  const uint32_t len = (uint32_t)(desc & 0xFFFFFFu);
  if (len < (uint32_t)k) return;
  const K mask = kmer_mask<K>(k);
  const int top = 2 * k - 2;
  K x = 0, r = 0;
  const uint8_t *src = packed + off;
  uint32_t byte = 0;
  for (uint32_t i = 0; i < len; i++) {
    if ((i & 3u) == 0) byte = __ldg(src + (i >> 2));
    uint32_t c = (byte >> (6 - 2 * (i & 3u))) & 3u;
    x = ((x << 2) | (K)c) & mask;
    r = (r >> 2) | ((K)(3u - c) << top);
    if (i + 1 >= (uint32_t)k) f(x < r ? x : r);
  }
}

// bin owning chunk c: the b with chunk_base[b] <= c < chunk_base[b+1]
GKC_DEV uint32_t chunk_bin(const uint64_t *chunk_base, uint32_t nbins, uint64_t c) {
  uint32_t lo = 0, hi = nbins - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (chunk_base[mid] <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

constexpr int EX_NT = 256;

template <typename K>
__global__ void __launch_bounds__(EX_NT) k_bucket_hist(ExpandArgs a) {
  extern __shared__ uint32_t hist[];  // 1 << max bits
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = chunk_bin(a.chunk_base, a.nbins, c);
    const uint32_t nbits = a.bin_bits[b], nd = 1u << nbits;
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT) hist[d] = 0;
    __syncthreads();
    const uint64_t s0 = a.bin_start[b] + (c - a.chunk_base[b]) * a.chunk_skm;
    const uint64_t s1 = min(s0 + a.chunk_skm, a.bin_start[b + 1]);
    for (uint64_t i = s0 + threadIdx.x; i < s1; i += EX_NT) {
      expand_skm<K>(a.packed, a.desc[i], a.k, [&](K key) {
        atomicAdd(&hist[key_digit<K>(key, key_bits, 0, (int)nbits)], 1u);
      });
    }
    __syncthreads();
    const uint64_t bb = a.bucket_base[b];
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT)
      if (hist[d]) atomicAdd(&a.bucket_count[bb + d], (unsigned long long)hist[d]);
    __syncthreads();
  }
}

template <typename K>
__global__ void __launch_bounds__(EX_NT) k_bucket_scatter(ExpandArgs a) {
  extern __shared__ unsigned long long sh_base[];      // 1 << max bits
  uint32_t *hist = reinterpret_cast<uint32_t *>(sh_base + 4096);
  K *keys = reinterpret_cast<K *>(a.keys);
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = chunk_bin(a.chunk_base, a.nbins, c);
    const uint32_t nbits = a.bin_bits[b], nd = 1u << nbits;
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT) hist[d] = 0;
    __syncthreads();
    const uint64_t s0 = a.bin_start[b] + (c - a.chunk_base[b]) * a.chunk_skm;
    const uint64_t s1 = min(s0 + a.chunk_skm, a.bin_start[b + 1]);
    for (uint64_t i = s0 + threadIdx.x; i < s1; i += EX_NT) {
      expand_skm<K>(a.packed, a.desc[i], a.k, [&](K key) {
        atomicAdd(&hist[key_digit<K>(key, key_bits, 0, (int)nbits)], 1u);
      });
    }
    __syncthreads();
    const uint64_t bb = a.bucket_base[b];
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT) {
      uint32_t h = hist[d];
      sh_base[d] = h ? atomicAdd(&a.bucket_cursor[bb + d], (unsigned long long)h) : 0ull;
      hist[d] = 0;
    }
    __syncthreads();
    for (uint64_t i = s0 + threadIdx.x; i < s1; i += EX_NT) {
      expand_skm<K>(a.packed, a.desc[i], a.k, [&](K key) {
        uint32_t d = key_digit<K>(key, key_bits, 0, (int)nbits);
        uint64_t slot = sh_base[d] + atomicAdd(&hist[d], 1u);
        if (slot < a.keys_cap) keys[slot] = key;
        else atomicOr(a.err, ERR_CAPACITY);
      });
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- look-back

constexpr unsigned long long LB_AGG = 1ull << 62, LB_PRE = 2ull << 62;
constexpr unsigned long long LB_VAL = (1ull << 62) - 1;

GKC_DEV void st_release(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
GKC_DEV unsigned long long ld_acquire(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
GKC_DEV uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Sum of the outputs of buckets [0, i) (waits, bounded, for predecessors).
GKC_DEV uint64_t lookback_prefix(unsigned long long *status, uint64_t i, uint32_t *err) {
  uint64_t excl = 0;
  if (i == 0) return 0;
  uint64_t j = i - 1;
  uint64_t t0 = globaltimer_ns();
  uint32_t it = 0;
  while (true) {
    unsigned long long v = ld_acquire(status + j);
    unsigned long long flag = v & ~LB_VAL;
    if (flag == 0) {
      if (++it > (1u << 24) || globaltimer_ns() - t0 > 8000000000ull) {
        atomicOr(err, ERR_SPIN_TIMEOUT);
        return excl;
      }
      nanosleep_backoff(it);
      continue;
    }
    excl += v & LB_VAL;
    if (flag == LB_PRE || j == 0) return excl;
    j--;
  }
}

// -------------------------------------------------------- shared-memory sort

constexpr int SC_NT = kSortThreads;
constexpr int SC_DMAX = 12;           // bits per MSD counting pass
constexpr int SC_SMAX = 32;           // leaves up to this size: insertion sort
constexpr int SC_BIGMAX = 256;        // larger leaves recorded per pass

template <typename K> struct SortCap;
template <> struct SortCap<uint64_t> { static constexpr int value = 5632; };
template <> struct SortCap<u128> { static constexpr int value = 2816; };

template <typename K>
struct SortSmem {
  K A[SortCap<K>::value];
  K B[SortCap<K>::value];
  uint32_t cnt[1 << SC_DMAX];
  uint32_t tmp[64];
  uint32_t big_s[SC_BIGMAX], big_m[SC_BIGMAX];
  uint32_t n_big;
  uint32_t D;
  uint64_t bucket, excl, n, start;
  // oversized-bucket frames
  struct Frame {
    uint64_t off, len;
    int skip, src, split, d;
    uint32_t cursor;
  } fr[24];
  int depth;
  int act;              // action decided by thread 0 for the oversize walk
  uint64_t c_off, c_len;
  int c_skip, c_src;
  uint64_t out;
};

template <typename K> int sort_count_cap() { return SortCap<K>::value; }
template <typename K> size_t sort_count_smem_bytes() { return sizeof(SortSmem<K>); }
template int sort_count_cap<uint64_t>();
template int sort_count_cap<u128>();
template size_t sort_count_smem_bytes<uint64_t>();
template size_t sort_count_smem_bytes<u128>();

GKC_DEV int ceil_log2_u32(uint32_t n) { return n <= 1 ? 0 : 32 - __clz(n - 1); }

// Exclusive scan of cnt[0, nd) in place; returns the total.
GKC_DEV uint32_t scan_counters(uint32_t *cnt, uint32_t nd, uint32_t *tmp) {
  const uint32_t per = (nd + SC_NT - 1) / SC_NT;
  const uint32_t c0 = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t j = c0; j < c0 + per && j < nd; j++) s += cnt[j];
  uint32_t total;
  uint32_t run = block_exclusive_scan<SC_NT>(s, tmp, &total);
  for (uint32_t j = c0; j < c0 + per && j < nd; j++) {
    uint32_t v = cnt[j];
    cnt[j] = run;
    run += v;
  }
  __syncthreads();
  return total;
}

// In-place ascending sort of A[0, m) with a comparator network in which every
// comparator puts the smaller key at the lower index, so indices >= m can be
// treated as +infinity (the "flip" form of bitonic sort).
template <typename K>
GKC_DEV void bitonic_sort(K *A, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = threadIdx.x; i < P / 2; i += SC_NT) {
      uint32_t blk = i / half, off = i % half;
      uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m) {
        K x = A[lo], y = A[hi];
        if (y < x) { A[lo] = y; A[hi] = x; }
      }
    }
    __syncthreads();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < P / 2; i += SC_NT) {
        uint32_t blk = i / stride, off = i % stride;
        uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m) {
          K x = A[lo], y = A[hi];
          if (y < x) { A[lo] = y; A[hi] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// Sorts S.A[0, n) ascending; keys agree on their top `skip` bits.
template <typename K>
GKC_DEV void smem_sort(SortSmem<K> &S, uint32_t n, int key_bits, int skip) {
  const int R = key_bits - skip;
  if (n <= 1 || R <= 0) return;
  const int d = max(1, min(min(SC_DMAX, R), ceil_log2_u32(n)));
  const uint32_t nd = 1u << d;
  for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) S.cnt[j] = 0;
  if (threadIdx.x == 0) S.n_big = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT)
    atomicAdd(&S.cnt[key_digit<K>(S.A[i], key_bits, skip, d)], 1u);
  __syncthreads();
  scan_counters(S.cnt, nd, S.tmp);
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT) {
    K x = S.A[i];
    uint32_t pos = atomicAdd(&S.cnt[key_digit<K>(x, key_bits, skip, d)], 1u);
    S.B[pos] = x;
  }
  __syncthreads();
  // cnt[j] is now the end of leaf j
  for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) {
    uint32_t s = j ? S.cnt[j - 1] : 0u, e = S.cnt[j], m = e - s;
    if (m <= (uint32_t)SC_SMAX) {
      for (uint32_t t = 0; t < m; t++) {
        K x = S.B[s + t];
        uint32_t q = t;
        while (q > 0 && x < S.A[s + q - 1]) {
          S.A[s + q] = S.A[s + q - 1];
          q--;
        }
        S.A[s + q] = x;
      }
    } else {
      uint32_t slot = atomicAdd(&S.n_big, 1u);
      if (slot < (uint32_t)SC_BIGMAX) {
        S.big_s[slot] = s;
        S.big_m[slot] = m;
      }
    }
  }
  __syncthreads();
  const uint32_t nbig = min(S.n_big, (uint32_t)SC_BIGMAX);
  for (uint32_t t = 0; t < nbig; t++) {
    const uint32_t s = S.big_s[t], m = S.big_m[t];
    for (uint32_t i = threadIdx.x; i < m; i += SC_NT) S.A[s + i] = S.B[s + i];
    __syncthreads();
    bitonic_sort<K>(S.A + s, m);
  }
  // big leaves beyond the list (at most n / SC_SMAX exist, so only when
  // n > SC_BIGMAX * SC_SMAX) are sorted by one more bitonic pass overall.
  if (S.n_big > (uint32_t)SC_BIGMAX) {
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) {
      uint32_t s = j ? S.cnt[j - 1] : 0u, e = S.cnt[j];
      if (e - s > (uint32_t)SC_SMAX)
        for (uint32_t i = s; i < e; i++) S.A[i] = S.B[i];
    }
    __syncthreads();
    bitonic_sort<K>(S.A, n);
  }
  __syncthreads();
}

// Run-length pass over sorted S.A[0, n): run starts go to S.B viewed as
// uint32 (run j spans [rs[j], rs[j+1])).  Returns the number of runs.
template <typename K>
GKC_DEV uint32_t smem_runs(SortSmem<K> &S, uint32_t n) {
  uint32_t *rs = reinterpret_cast<uint32_t *>(S.B);
  const uint32_t per = (n + SC_NT - 1) / SC_NT;
  const uint32_t c0 = threadIdx.x * per;
  uint32_t cntr = 0;
  for (uint32_t i = c0; i < c0 + per && i < n; i++) cntr += (i == 0 || S.A[i] != S.A[i - 1]);
  uint32_t total;
  uint32_t idx = block_exclusive_scan<SC_NT>(cntr, S.tmp, &total);
  for (uint32_t i = c0; i < c0 + per && i < n; i++)
    if (i == 0 || S.A[i] != S.A[i - 1]) rs[idx++] = i;
  if (threadIdx.x == 0) rs[total] = n;
  __syncthreads();
  return total;
}

template <typename K>
GKC_DEV void write_runs(SortSmem<K> &S, uint32_t D, K *out_keys, uint32_t *out_counts,
                        uint64_t out) {
  const uint32_t *rs = reinterpret_cast<const uint32_t *>(S.B);
  for (uint32_t j = threadIdx.x; j < D; j += SC_NT) {
    out_keys[out + j] = S.A[rs[j]];
    out_counts[out + j] = rs[j + 1] - rs[j];
  }
}

template <typename K>
GKC_DEV void load_keys(K *dst, const K *src, uint32_t n) {
  for (uint32_t i = threadIdx.x; i < n; i += SC_NT) dst[i] = src[i];
}

// Oversized bucket: MSD passes through global scratch, depth first in key
// order; sub-buckets that fit are finished in shared memory.
template <typename K>
GKC_DEV void oversize_bucket(SortSmem<K> &S, const SortCountArgs &a, K *keys, K *out_keys,
                             uint64_t start, uint64_t n, int skip0, uint64_t excl) {
  const int key_bits = 2 * a.k;
  const int CAP = SortCap<K>::value;
  K *half[2] = {reinterpret_cast<K *>(a.scratch), reinterpret_cast<K *>(a.scratch) + a.scratch_keys};
  if (n > a.scratch_keys) {
    if (threadIdx.x == 0) {
      atomicOr(a.err, ERR_OVERSIZE_SCRATCH);
      S.out = excl;
    }
    __syncthreads();
    return;
  }
  for (uint64_t i = threadIdx.x; i < n; i += SC_NT) half[0][i] = keys[start + i];
  if (threadIdx.x == 0) {
    S.depth = 0;
    S.fr[0] = {0, n, skip0, 0, 0, 0, 0};
    S.out = excl;
  }
  __threadfence_block();
  __syncthreads();
  while (S.depth >= 0) {
    const int dep = S.depth;
    uint32_t *gc = a.scratch_cnt + (size_t)dep * 4096;
    if (!S.fr[dep].split) {
      const uint64_t off = S.fr[dep].off, len = S.fr[dep].len;
      const int skip = S.fr[dep].skip, src = S.fr[dep].src;
      const int d = min(SC_DMAX, key_bits - skip);
      const uint32_t nd = 1u << d;
      for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) S.cnt[j] = 0;
      __syncthreads();
      for (uint64_t i = threadIdx.x; i < len; i += SC_NT)
        atomicAdd(&S.cnt[key_digit<K>(half[src][off + i], key_bits, skip, d)], 1u);
      __syncthreads();
      scan_counters(S.cnt, nd, S.tmp);
      for (uint64_t i = threadIdx.x; i < len; i += SC_NT) {
        K x = half[src][off + i];
        uint32_t pos = atomicAdd(&S.cnt[key_digit<K>(x, key_bits, skip, d)], 1u);
        half[1 - src][off + pos] = x;
      }
      __syncthreads();
      for (uint32_t j = threadIdx.x; j < nd; j += SC_NT) gc[j] = S.cnt[j];  // leaf ends
      __threadfence_block();
      __syncthreads();
      if (threadIdx.x == 0) {
        S.fr[dep].split = 1;
        S.fr[dep].d = d;
        S.fr[dep].cursor = 0;
      }
      __syncthreads();
    }
    // thread 0 walks to the next non-empty child and decides what to do
    if (threadIdx.x == 0) {
      S.act = 0;  // 0: frame done
      auto &F = S.fr[dep];
      const uint32_t nd = 1u << F.d;
      while (F.cursor < nd) {
        uint32_t j = F.cursor++;
        uint64_t s = j ? gc[j - 1] : 0, e = gc[j];
        if (e == s) continue;
        S.c_off = F.off + s;
        S.c_len = e - s;
        S.c_skip = F.skip + F.d;
        S.c_src = 1 - F.src;
        if (S.c_len <= (uint64_t)CAP) S.act = 1;            // finish in shared memory
        else if (S.c_skip >= key_bits) S.act = 2;           // all keys equal
        else S.act = 3;                                     // split further
        break;
      }
      if (S.act == 3) {
        S.depth = dep + 1;
        S.fr[dep + 1] = {S.c_off, S.c_len, S.c_skip, S.c_src, 0, 0, 0};
      } else if (S.act == 0) {
        S.depth = dep - 1;
      }
    }
    __syncthreads();
    const int act = S.act;
    if (act == 1) {
      const uint32_t m = (uint32_t)S.c_len;
      load_keys<K>(S.A, half[S.c_src] + S.c_off, m);
      __syncthreads();
      smem_sort<K>(S, m, key_bits, S.c_skip);
      uint32_t D = smem_runs<K>(S, m);
      write_runs<K>(S, D, out_keys, a.out_counts, S.out);
      __syncthreads();
      if (threadIdx.x == 0) S.out += D;
    } else if (act == 2) {
      if (threadIdx.x == 0) {
        out_keys[S.out] = half[S.c_src][S.c_off];
        a.out_counts[S.out] = S.c_len > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)S.c_len;
        S.out += 1;
      }
    }
    __syncthreads();
  }
}

template <typename K>
__global__ void __launch_bounds__(SC_NT, 2) k_sort_count(SortCountArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  SortSmem<K> &S = *reinterpret_cast<SortSmem<K> *>(smem_raw);
  K *keys = reinterpret_cast<K *>(a.keys);
  K *out_keys = reinterpret_cast<K *>(a.out_keys);
  const int key_bits = 2 * a.k;
  const int CAP = SortCap<K>::value;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ)) return;  // keys incomplete: the host re-runs
  const uint64_t n_buckets = *a.n_buckets_dev;
  while (true) {
    if (threadIdx.x == 0) S.bucket = atomicAdd(a.ticket, 1ull);
    __syncthreads();
    const uint64_t i = S.bucket;
    if (i >= n_buckets) break;
    const uint64_t start = a.bucket_start[i], n = a.bucket_start[i + 1] - start;
    // bucket -> bin -> prefix bits shared by the bucket's keys
    uint32_t lo = 0, hi = a.nbins - 1;
    while (lo < hi) {
      uint32_t mid = (lo + hi + 1) >> 1;
      if (a.bucket_base[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const int skip = (int)a.bin_bits[lo];
    long long t0 = clock64();
    if (n <= (uint64_t)CAP) {
      load_keys<K>(S.A, keys + start, (uint32_t)n);
      __syncthreads();
      long long t1 = clock64();
      smem_sort<K>(S, (uint32_t)n, key_bits, skip);
      long long t2 = clock64();
      const uint32_t D = smem_runs<K>(S, (uint32_t)n);
      long long t3 = clock64();
      if (threadIdx.x == 0 && a.prof) {
        atomicAdd(a.prof + 0, (unsigned long long)(t1 - t0));
        atomicAdd(a.prof + 1, (unsigned long long)(t2 - t1));
        atomicAdd(a.prof + 2, (unsigned long long)(t3 - t2));
        atomicAdd(a.prof + 6, 1ull);
        atomicAdd(a.prof + 7, (unsigned long long)S.n_big);
        atomicAdd(a.prof + 8, (unsigned long long)n);
      }
      if (threadIdx.x == 0) {
        if (i == 0) {
          S.excl = 0;
          st_release(a.status, LB_PRE | D);
        } else {
          st_release(a.status + i, LB_AGG | D);
          S.excl = lookback_prefix(a.status, i, a.err);
          st_release(a.status + i, LB_PRE | (S.excl + D));
        }
        a.bucket_out[i] = S.excl;
        if (i + 1 == n_buckets) a.bucket_out[i + 1] = S.excl + D;
      }
      __syncthreads();
      long long t4 = clock64();
      write_runs<K>(S, D, out_keys, a.out_counts, S.excl);
      __syncthreads();
      if (threadIdx.x == 0 && a.prof) {
        atomicAdd(a.prof + 3, (unsigned long long)(t4 - t3));
        atomicAdd(a.prof + 4, (unsigned long long)(clock64() - t4));
      }
    } else {
      if (threadIdx.x == 0 && a.prof) atomicAdd(a.prof + 5, 1ull);
      if (threadIdx.x == 0) S.excl = lookback_prefix(a.status, i, a.err);
      __syncthreads();
      const uint64_t excl = S.excl;
      oversize_bucket<K>(S, a, keys, out_keys, start, n, skip, excl);
      if (threadIdx.x == 0) {
        st_release(a.status + i, LB_PRE | S.out);
        a.bucket_out[i] = excl;
        if (i + 1 == n_buckets) a.bucket_out[i + 1] = S.out;
      }
      __syncthreads();
    }
  }
}

__global__ void k_bin_out_offsets(const uint64_t *bucket_out, const uint64_t *bucket_base,
                                  uint32_t nbins, uint64_t *bin_out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins; b += gridDim.x * blockDim.x)
    bin_out[b] = bucket_out[bucket_base[b]];
}

template __global__ void k_bucket_hist<uint64_t>(ExpandArgs);
template __global__ void k_bucket_hist<u128>(ExpandArgs);
template __global__ void k_bucket_scatter<uint64_t>(ExpandArgs);
template __global__ void k_bucket_scatter<u128>(ExpandArgs);
template __global__ void k_sort_count<uint64_t>(SortCountArgs);
template __global__ void k_sort_count<u128>(SortCountArgs);

}  // namespace gkc
