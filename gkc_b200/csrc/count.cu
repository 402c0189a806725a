// Canonical k-mer counting from bin-grouped superkmers (batched path).
//
// Semantics follow kmc_counting_GPU (kmer_counting.cu:95-191): every k-mer of
// every superkmer of a bin, canonicalised as min(x, revcomp(x)), sorted
// ascending, run-length counted (count clamped to 2^32-1), per bin.
//
// The keys of a bin are split into 2^cb coarse buckets by the top bits of an
// order-preserving map of the key (eq_map), so a bin's sorted list is the
// concatenation of its buckets' sorted lists.  Device stages:
//   1. k_bucket_hist    - per chunk of a bin's k-mers, a histogram of coarse
//                         digits.  A canonical key's digit depends only on its
//                         top 32 bits, which are min(top of x, top of
//                         revcomp x): the first 16 bases and the reverse
//                         complement of the last 16, two 32-bit rolling
//                         windows (no 64-bit expansion);
//   2. k_bucket_scan    - one CTA per bin turns the (chunk, digit) counts
//                         into each chunk's write offset per digit and each
//                         bucket's start and size;
//   3. k_bucket_scatter - expands every k-mer once and writes it at its
//                         chunk's offset for its digit plus its rank there
//                         (a shared-memory atomic);
//   4. k_bucket_count   - persistent, one bucket per ticket: counting sort by
//                         sub-bucket in shared memory, each thread sorting and
//                         run-length encoding a few sub-buckets, a block scan,
//                         the runs staged at the bucket's own key range and
//                         its distinct count recorded (buckets are counted
//                         independently of one another); k_compact_runs then
//                         moves them to the scan of the counts.  A bucket
//                         larger than shared memory is placed by sub-bucket in
//                         a scratch area and counted in slices; a single
//                         sub-bucket too large for a slice is aggregated in a
//                         shared-memory hash table over key ranges that are
//                         halved until a range's distinct keys fit.
#include "common.cuh"
#include "kernels.h"

namespace gkc {

// ------------------------------------------------------------ key digits

// Top 32 bits of a 2k-bit key, left-aligned when the key is shorter.
template <typename K>
GKC_DEV uint32_t key_top32(K x, int key_bits) {
  return key_bits >= 32 ? (uint32_t)(x >> (key_bits - 32)) : (uint32_t)((uint64_t)x << (32 - key_bits));
}

// Order-preserving map of a canonical key's top 32 bits t that spreads
// canonical keys evenly: the canonical key of a uniform k-mer is the smaller
// of two near-independent uniform values, whose distribution function is
// 1 - (1 - u)^2; v = 2^32 (1 - (1 - t / 2^32)^2), non-decreasing in t.
GKC_DEV uint32_t eq_map(uint32_t t) {
  if (t == 0) return 0;
  const uint64_t s = (1ull << 32) - t;  // 1 .. 2^32 - 1
  return (uint32_t)((0ull - s * s) >> 32);
}

GKC_DEV uint32_t coarse_of(uint32_t v, int cb) { return cb ? v >> (32 - cb) : 0u; }

template <typename K>
GKC_DEV uint32_t coarse_digit(K x, int key_bits, int cb) {
  return coarse_of(eq_map(key_top32<K>(x, key_bits)), cb);
}

// The sb bits of the key's map below its cb coarse bits (cb + sb <= 32).
template <typename K>
GKC_DEV uint32_t sub_digit(K x, int key_bits, int cb, int sb) {
  if (sb == 0) return 0u;
  const uint32_t v = eq_map(key_top32<K>(x, key_bits));
  return (v >> (32 - cb - sb)) & ((1u << sb) - 1u);
}

// ------------------------------------------------------------------ planning

__global__ void k_count_plan(CountPlan pl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool dead = (*pl.err & (ERR_CAPACITY | ERR_BAD_READ)) != 0;
  uint64_t bb = 0, cb = 0, hb = 0;
  for (uint32_t b = 0; b < pl.nbins; b++) {
    const uint64_t nk = dead ? 0 : pl.bin_kstart[b + 1] - pl.bin_kstart[b];
    uint32_t bits = 0;
    while (bits < pl.max_bits && (int)bits < 2 * pl.k && (nk >> bits) > pl.coarse_target) bits++;
    const uint64_t nch = (nk + pl.chunk_kmers - 1) / pl.chunk_kmers;
    pl.bin_bits[b] = bits;
    pl.bucket_base[b] = bb;
    pl.chunk_base[b] = cb;
    pl.hist_base[b] = hb;
    bb += 1ull << bits;
    cb += nch;
    hb += nch << bits;
  }
  pl.bucket_base[pl.nbins] = bb;
  pl.chunk_base[pl.nbins] = cb;
  pl.hist_base[pl.nbins] = hb;
}

GKC_DEV uint32_t find_bin(const uint64_t *base, uint32_t nbins, uint64_t c) {
  uint32_t lo = 0, hi = nbins - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (base[mid] <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Number of k-mers of each bin-ordered superkmer (for the k-mer prefix).
__global__ void k_skm_nk(const uint64_t *desc, const unsigned long long *n_skm_dev, int k,
                         unsigned long long *nk) {
  const uint64_t n = *n_skm_dev;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t len = (uint32_t)(desc[i] & 0xFFFFFFu);
    nk[i] = len >= (uint32_t)k ? len - k + 1 : 0;
  }
}

// First superkmer of every chunk: the last superkmer of the bin whose k-mer
// prefix is at most the chunk's first k-mer.
__global__ void k_chunk_first(ExpandArgs a) {
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n_chunks;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t q0 = a.bin_kstart[b] + (c - a.chunk_base[b]) * a.chunk_kmers;
    uint64_t lo = a.bin_start[b], hi = a.bin_start[b + 1] - 1;
    while (lo < hi) {
      const uint64_t mid = (lo + hi + 1) >> 1;
      if (a.koff[mid] <= q0) lo = mid; else hi = mid - 1;
    }
    a.chunk_s0[c] = lo;
  }
}

// ------------------------------------------------------- k-mer runs

// The superkmer of the bin holding k-mer q: the last one in [lo, hi] whose
// k-mer prefix is at most q.
GKC_DEV uint64_t skm_of_kmer(const uint64_t *koff, uint64_t lo, uint64_t hi, uint64_t q) {
  while (lo < hi) {
    const uint64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(koff + mid) <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Thread tid's k-mers of chunk c: a contiguous run [*q, *qe) of about
// chunk_kmers / nt k-mers, and the superkmer holding its first k-mer
// (searched between the chunk's first superkmer and the next chunk's).
GKC_DEV uint64_t thread_run(const ExpandArgs &a, uint64_t c, uint32_t b, uint64_t j, int nt, uint64_t *q,
                            uint64_t *qe) {
  const uint64_t q0 = a.bin_kstart[b] + j * a.chunk_kmers;
  const uint64_t q1 = min(q0 + a.chunk_kmers, a.bin_kstart[b + 1]);
  const uint64_t per = (q1 - q0 + nt - 1) / nt;
  *q = min(q0 + per * threadIdx.x, q1);
  *qe = min(*q + per, q1);
  const uint64_t lo = a.chunk_s0[c];
  const uint64_t hi = (c + 1 < a.chunk_base[b + 1]) ? a.chunk_s0[c + 1] : a.bin_start[b + 1] - 1;
  return skm_of_kmer(a.koff, lo, hi, *q);
}

// 16 bases of a packed superkmer from base index pos, first base in the top
// bits (2 bits per base, MSB first; bytes past the end read as padding).
GKC_DEV uint32_t bases16(const uint8_t *packed, uint64_t off, uint32_t pos) {
  const uint8_t *p = packed + off + (pos >> 2);
  const uint32_t sh = 2 * (pos & 3u);
  uint32_t v = ((uint32_t)__ldg(p) << 24) | ((uint32_t)__ldg(p + 1) << 16) | ((uint32_t)__ldg(p + 2) << 8) |
               (uint32_t)__ldg(p + 3);
  if (sh) v = (v << sh) | ((uint32_t)__ldg(p + 4) >> (8 - sh));
  return v;
}

// Reverse complement of the 16 bases of w.
GKC_DEV uint32_t revcomp16(uint32_t w) {
  const uint32_t y = __brev(~w);
  return ((y >> 1) & 0x55555555u) | ((y & 0x55555555u) << 1);
}

// The 2k bits of bases [o, o+k) of a packed superkmer at byte `off`.
template <typename K>
GKC_DEV K extract_kmer(const uint8_t *packed, uint64_t off, uint32_t o, int k);

template <>
GKC_DEV uint64_t extract_kmer<uint64_t>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  const uint8_t *p = packed + off + (o >> 2);
  const int sh = 2 * (o & 3);
  uint64_t hi = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) hi = (hi << 8) | __ldg(p + i);
  const uint64_t v = sh ? ((hi << sh) | (uint64_t)(__ldg(p + 8) >> (8 - sh))) : hi;
  return v >> (64 - 2 * k);
}

template <>
GKC_DEV u128 extract_kmer<u128>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  const uint8_t *p = packed + off + (o >> 2);
  const int sh = 2 * (o & 3);
  u128 hi = 0;
#pragma unroll
  for (int i = 0; i < 16; i++) hi = (hi << 8) | (u128)__ldg(p + i);
  const u128 v = sh ? ((hi << sh) | (u128)(__ldg(p + 16) >> (8 - sh))) : hi;
  return v >> (128 - 2 * k);
}

// Bases of a packed superkmer from index j on, each byte read once.
struct BaseStream {
  const uint8_t *p;
  uint32_t j, byte;
  GKC_DEV void init(const uint8_t *src, uint32_t j0) {
    p = src;
    j = j0;
    byte = __ldg(p + (j >> 2));
  }
  GKC_DEV uint32_t next() {
    if ((j & 3u) == 0) byte = __ldg(p + (j >> 2));
    const uint32_t c = (byte >> (6 - 2 * (j & 3u))) & 3u;
    j++;
    return c;
  }
};

// ----------------------------------------------------------- 1. histogram

constexpr int HS_NT = 256;

// Per chunk of a bin's k-mers, the histogram of coarse digits.  Each thread
// walks a contiguous run of about chunk_kmers / 256 k-mers through its
// superkmers; the digit needs only the top 32 bits of the canonical key,
// min(first 16 bases, reverse complement of the last 16), from two 32-bit
// rolling windows (h = min(k, 16) bases each).
__global__ void __launch_bounds__(HS_NT) k_bucket_hist(ExpandArgs a) {
  __shared__ uint32_t hist[1 << kCoarseMaxBits];
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int k = a.k;
  const int h = k < 16 ? k : 16;
  const uint32_t hmask = h == 16 ? 0xFFFFFFFFu : ((1u << (2 * h)) - 1u);
  const int hsh = 32 - 2 * h;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t j = c - a.chunk_base[b];
    const int cb = (int)a.bin_bits[b];
    const uint32_t nd = 1u << cb;
    for (uint32_t d = threadIdx.x; d < nd; d += HS_NT) hist[d] = 0;
    __syncthreads();
    uint64_t q, qe;
    uint64_t s = thread_run(a, c, b, j, HS_NT, &q, &qe);
    while (q < qe) {
      const uint64_t ks = __ldg(a.koff + s), ke = __ldg(a.koff + s + 1);
      if (ke <= q) {  // a superkmer without k-mers, or one already passed
        s++;
        continue;
      }
      const uint64_t off = __ldg(a.desc + s) >> 24;
      const uint32_t o = (uint32_t)(q - ks);
      uint32_t cnt = (uint32_t)(min(qe, ke) - q);
      uint32_t fw = bases16(a.packed, off, o) >> hsh;
      uint32_t rc = revcomp16(bases16(a.packed, off, o + k - h)) & hmask;
      BaseStream sf, sr;
      sf.init(a.packed + off, o + h);
      sr.init(a.packed + off, o + k);
      q += cnt;
      s++;
      while (true) {
        atomicAdd(&hist[coarse_of(eq_map(min(fw, rc) << hsh), cb)], 1u);
        if (--cnt == 0) break;
        fw = ((fw << 2) | sf.next()) & hmask;
        rc = (rc >> 2) | ((3u - sr.next()) << (2 * h - 2));
      }
    }
    __syncthreads();
    uint32_t *row = a.hist + a.hist_base[b] + j * nd;  // the chunk's row, digits contiguous
    for (uint32_t d = threadIdx.x; d < nd; d += HS_NT) row[d] = hist[d];
    __syncthreads();
  }
}

// ----------------------------------------------------------------- 2. scan

// One CTA per bin: column sums of the bin's (chunk, digit) counts, an
// exclusive scan over digits (the bucket starts), then every chunk's write
// offset per digit, written over its count; offsets are relative to the
// bin's first key.
constexpr int BS_NT = 1024;
__global__ void __launch_bounds__(BS_NT) k_bucket_scan(ExpandArgs a, uint64_t *bucket_start,
                                                       uint64_t *bucket_size) {
  __shared__ uint32_t tmp[64];
  constexpr int DPT = (1 << kCoarseMaxBits) / BS_NT;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  for (uint32_t b = blockIdx.x; b < a.nbins; b += gridDim.x) {
    const uint32_t nd = 1u << a.bin_bits[b];
    const uint64_t nch = a.chunk_base[b + 1] - a.chunk_base[b];
    if (a.bin_kstart[b + 1] - a.bin_kstart[b] >= (1ull << 32)) {  // offsets in a bin are 32-bit
      if (threadIdx.x == 0) atomicOr(a.err, ERR_BIN_TOO_LARGE);
      continue;
    }
    uint32_t *M = a.hist + a.hist_base[b];
    // thread t holds the contiguous digits [t * DPT, t * DPT + DPT)
    uint32_t col[DPT];
#pragma unroll
    for (int u = 0; u < DPT; u++) col[u] = 0;
    for (uint64_t jj = 0; jj < nch; jj++) {
#pragma unroll
      for (int u = 0; u < DPT; u++) {
        const uint32_t d = threadIdx.x * DPT + u;
        if (d < nd) col[u] += M[jj * nd + d];
      }
    }
    uint32_t s = 0;
#pragma unroll
    for (int u = 0; u < DPT; u++) s += col[u];
    uint32_t tot;
    uint32_t run = block_exclusive_scan<BS_NT>(s, tmp, &tot);
    const uint64_t g0 = a.bucket_base[b];
    uint32_t start[DPT];
#pragma unroll
    for (int u = 0; u < DPT; u++) {
      const uint32_t d = threadIdx.x * DPT + u;
      start[u] = run;
      if (d < nd) {
        bucket_start[g0 + d] = a.bin_kstart[b] + run;
        bucket_size[g0 + d] = col[u];
      }
      run += col[u];
    }
    for (uint64_t jj = 0; jj < nch; jj++) {
#pragma unroll
      for (int u = 0; u < DPT; u++) {
        const uint32_t d = threadIdx.x * DPT + u;
        if (d < nd) {
          const uint32_t v = M[jj * nd + d];
          M[jj * nd + d] = start[u];
          start[u] += v;
        }
      }
    }
    __syncthreads();
  }
}

// -------------------------------------------------------------- 3. scatter

constexpr int SC_THREADS = 256;

// Expands every k-mer once and writes it to its bucket: the chunk's write
// offset per digit (from the scan) plus the key's rank among the chunk's keys
// of that digit, taken with a shared-memory atomic.  Threads walk contiguous
// runs as in the histogram; the first k-mer of each superkmer segment is
// extracted whole, the rest rolled in (kmer_counting.cu:99-112, canonical
// form :33-44).
template <typename K>
__global__ void __launch_bounds__(SC_THREADS) k_bucket_scatter(ExpandArgs a) {
  __shared__ uint32_t cnt[1 << kCoarseMaxBits];
  __shared__ uint32_t gbase[1 << kCoarseMaxBits];
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  K *keys = reinterpret_cast<K *>(a.keys);
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int k = a.k, key_bits = 2 * k, top = 2 * k - 2;
  const K mask = kmer_mask<K>(k);
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t j = c - a.chunk_base[b];
    const int cb = (int)a.bin_bits[b];
    const uint32_t nd = 1u << cb;
    const uint64_t kbase = a.bin_kstart[b];
    const uint32_t *row = a.hist + a.hist_base[b] + j * nd;
    for (uint32_t d = threadIdx.x; d < nd; d += SC_THREADS) {
      gbase[d] = row[d];
      cnt[d] = 0;
    }
    __syncthreads();
    uint64_t q, qe;
    uint64_t s = thread_run(a, c, b, j, SC_THREADS, &q, &qe);
    while (q < qe) {
      const uint64_t ks = __ldg(a.koff + s), ke = __ldg(a.koff + s + 1);
      if (ke <= q) {
        s++;
        continue;
      }
      const uint64_t off = __ldg(a.desc + s) >> 24;
      const uint32_t o = (uint32_t)(q - ks);
      uint32_t n = (uint32_t)(min(qe, ke) - q);
      K x = extract_kmer<K>(a.packed, off, o, k);
      K r = revcomp_k<K>(x, k);
      BaseStream bs;
      bs.init(a.packed + off, o + k);
      q += n;
      s++;
      while (true) {
        const K key = x < r ? x : r;
        const uint32_t d = coarse_digit<K>(key, key_bits, cb);
        const uint64_t slot = kbase + gbase[d] + atomicAdd(&cnt[d], 1u);
        if (slot < a.keys_cap) keys[slot] = key;
        else atomicOr(a.err, ERR_CAPACITY);
        if (--n == 0) break;
        const uint32_t cc = bs.next();
        x = ((x << 2) | (K)cc) & mask;
        r = (r >> 2) | ((K)(3u - cc) << top);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- 4. count

template <typename K> struct CountShape;
template <> struct CountShape<uint64_t> { static constexpr int NT = 512, CAP = 8192; };
template <> struct CountShape<u128> { static constexpr int NT = 512, CAP = 4096; };
constexpr int CC_SB_MAX = 12;        // sub-bucket bits
constexpr int CC_NSUB_MAX = 1 << CC_SB_MAX;
constexpr uint32_t CC_SEG_MAX = 64;  // longer per-thread segments are sorted by warps
constexpr int CC_BIG_LIST = 128;
constexpr int CC_STACK = 2 * 129 + 2;  // key-range halving: at most 128 levels, two entries each

// Heavy-slice hash table: keys, counts and a slot state (0 free, 1 being
// written, 2 holds a key), inside the key area of the shared memory.
template <typename K> struct HeavyTab {
  static constexpr int SLOTS = (CountShape<K>::CAP * sizeof(K)) / (sizeof(K) + 8);
  static constexpr int N = SLOTS >= 4096 ? 4096 : (SLOTS >= 2048 ? 2048 : 1024);
  K key[N];
  uint32_t cnt[N];
  uint32_t state[N];
};

template <typename K>
struct CountSmem {
  static constexpr int CAP = CountShape<K>::CAP, NT = CountShape<K>::NT;
  union {
    K A[CAP];  // keys of a bucket or a slice
    HeavyTab<K> h;
  } u;
  // run counts; cursors of the oversized path (as 32-bit words)
  uint16_t C[CAP > 2 * CC_NSUB_MAX ? CAP : 2 * CC_NSUB_MAX];
  uint32_t cnt[CC_NSUB_MAX + 1];  // sub-bucket counts, then starts
  uint32_t seg_pos[NT];           // output position of each thread's runs (exclusive scan)
  uint32_t seg_src[NT];           // first run of each thread's segment in A
  uint32_t big[CC_BIG_LIST];      // threads whose segments are sorted by warps
  uint32_t tmp[64];
  uint32_t nbig, hfill, nsub;
  int flag, sp;
  uint64_t g, start, n, out_base, run, tbase;
  uint32_t b;
  K stk_lo[CC_STACK], stk_hi[CC_STACK];
};

template <typename K> size_t bucket_count_smem_bytes() { return sizeof(CountSmem<K>); }
template size_t bucket_count_smem_bytes<uint64_t>();
template size_t bucket_count_smem_bytes<u128>();

// In-place ascending sort of A[0, m) by one warp (bitonic network whose
// comparators put the smaller key first, so indices >= m act as +infinity).
template <typename K>
GKC_DEV void warp_sort(K *A, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = lane; i < P / 2; i += 32) {
      const uint32_t blk = i / half, off = i % half;
      const uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m) {
        const K x = A[lo], y = A[hi];
        if (y < x) {
          A[lo] = y;
          A[hi] = x;
        }
      }
    }
    __syncwarp();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = lane; i < P / 2; i += 32) {
        const uint32_t blk = i / stride, off = i % stride;
        const uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m) {
          const K x = A[lo], y = A[hi];
          if (y < x) {
            A[lo] = y;
            A[hi] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// The same network over (key, count) pairs, by the whole block.
template <typename K, int NT>
GKC_DEV void block_sort_pairs(K *A, uint32_t *cv, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = threadIdx.x; i < P / 2; i += NT) {
      const uint32_t blk = i / half, off = i % half;
      const uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m && A[hi] < A[lo]) {
        const K x = A[lo];
        A[lo] = A[hi];
        A[hi] = x;
        const uint32_t c = cv[lo];
        cv[lo] = cv[hi];
        cv[hi] = c;
      }
    }
    __syncthreads();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < P / 2; i += NT) {
        const uint32_t blk = i / stride, off = i % stride;
        const uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m && A[hi] < A[lo]) {
          const K x = A[lo];
          A[lo] = A[hi];
          A[hi] = x;
          const uint32_t c = cv[lo];
          cv[lo] = cv[hi];
          cv[hi] = c;
        }
      }
      __syncthreads();
    }
  }
}

// Exclusive scan of S.cnt[0, nsub) in place (thread-contiguous groups).
template <typename K, int NT>
GKC_DEV void scan_sub(CountSmem<K> &S, uint32_t nsub) {
  const uint32_t per = (nsub + NT - 1) / NT, c0 = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t jj = c0; jj < c0 + per && jj < nsub; jj++) s += S.cnt[jj];
  uint32_t tot;
  uint32_t run = block_exclusive_scan<NT>(s, S.tmp, &tot);
  for (uint32_t jj = c0; jj < c0 + per && jj < nsub; jj++) {
    const uint32_t v = S.cnt[jj];
    S.cnt[jj] = run;
    run += v;
  }
  __syncthreads();
}

// The m keys in S.u.A are grouped by sub-bucket: sub-bucket jb + jj starts at
// S.cnt[jb + jj] - s0 for jj in [0, nsl) (the last one ends at m).  Each
// thread sorts the sub-buckets it owns and run-length encodes them in place
// (keys in A, counts in C); longer segments are sorted by warps first.  Sets
// S.seg_src / S.seg_pos (exclusive scan of the run counts) and returns the
// slice's distinct keys.
template <typename K, int NT>
GKC_DEV uint32_t slice_runs(CountSmem<K> &S, uint32_t m, uint32_t jb, uint32_t nsl, uint32_t s0) {
  const int tid = threadIdx.x;
  K *A = S.u.A;
  auto start_of = [&](uint32_t jj) -> uint32_t { return jj < nsl ? S.cnt[jb + jj] - s0 : m; };
  const uint32_t j0 = (uint32_t)(((uint64_t)tid * nsl) / NT), j1 = (uint32_t)(((uint64_t)(tid + 1) * nsl) / NT);
  const uint32_t s = start_of(j0), e = start_of(j1);
  if (tid == 0) S.nbig = 0;
  __syncthreads();
  bool big = e - s > CC_SEG_MAX;
  if (big) {
    const uint32_t t = atomicAdd(&S.nbig, 1u);
    if (t < (uint32_t)CC_BIG_LIST) S.big[t] = (uint32_t)tid;
    else big = false;  // list full: sorted by its own thread
  }
  if (!big) {
    for (uint32_t jj = j0; jj < j1; jj++) {
      const uint32_t b0 = start_of(jj), b1 = start_of(jj + 1);
      for (uint32_t p = b0 + 1; p < b1; p++) {
        const K x = A[p];
        uint32_t q = p;
        while (q > b0 && x < A[q - 1]) {
          A[q] = A[q - 1];
          q--;
        }
        A[q] = x;
      }
    }
  }
  __syncthreads();
  const uint32_t nbig = min(S.nbig, (uint32_t)CC_BIG_LIST);
  for (uint32_t t = threadIdx.x >> 5; t < nbig; t += NT / 32) {
    const uint32_t ow = S.big[t];
    const uint32_t oj0 = (uint32_t)(((uint64_t)ow * nsl) / NT), oj1 = (uint32_t)(((uint64_t)(ow + 1) * nsl) / NT);
    const uint32_t os = start_of(oj0);
    warp_sort<K>(A + os, start_of(oj1) - os);
  }
  __syncthreads();
  uint32_t u = 0;
  for (uint32_t i = s; i < e;) {
    const K x = A[i];
    uint32_t c = 1;
    i++;
    while (i < e && A[i] == x) {
      c++;
      i++;
    }
    A[s + u] = x;
    S.C[s + u] = (uint16_t)c;  // c <= m <= CAP < 2^16
    u++;
  }
  uint32_t D;
  const uint32_t pos = block_exclusive_scan<NT>(u, S.tmp, &D);
  S.seg_pos[tid] = pos;
  S.seg_src[tid] = s;
  __syncthreads();
  return D;
}

// Writes the D runs of the slice (S.seg_* from slice_runs) to the staging
// arrays at [ob, ob+D), coalesced: output i comes from the thread whose runs
// cover it.
template <typename K, int NT>
GKC_DEV void write_runs(CountSmem<K> &S, const SortCountArgs &a, uint32_t D, uint64_t ob) {
  K *out_keys = reinterpret_cast<K *>(a.stage_keys);
  for (uint32_t i = threadIdx.x; i < D; i += NT) {
    uint32_t lo = 0, hi = NT - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (S.seg_pos[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const uint32_t src = S.seg_src[lo] + (i - S.seg_pos[lo]);
    if (ob + i < a.stage_cap) {
      out_keys[ob + i] = S.u.A[src];
      a.stage_counts[ob + i] = S.C[src];
    } else {
      atomicOr(a.err, ERR_CAPACITY);
    }
  }
}

// One sub-bucket of n keys at tmp[0, n), too many for shared memory: key
// ranges are aggregated in the hash table; a range whose distinct keys fill
// more than 3/4 of it is halved and both halves retried (lower first).  Runs
// are appended to the staging arrays at S.out_base + S.run.
template <typename K, int NT>
GKC_DEV void heavy_slice(CountSmem<K> &S, const SortCountArgs &a, const K *src, uint64_t n) {
  constexpr int HN = HeavyTab<K>::N;
  HeavyTab<K> &T = S.u.h;
  K *out_keys = reinterpret_cast<K *>(a.stage_keys);
  const int tid = threadIdx.x;
  if (tid == 0) {
    S.sp = 1;
    S.stk_lo[0] = (K)0;
    S.stk_hi[0] = ~(K)0;
  }
  __syncthreads();
  while (true) {
    if (S.sp == 0) break;
    const K lo = S.stk_lo[S.sp - 1], hi = S.stk_hi[S.sp - 1];
    for (int s = tid; s < HN; s += NT) {
      T.cnt[s] = 0;
      T.state[s] = 0;
    }
    __syncthreads();
    if (tid == 0) {
      S.sp--;
      S.flag = 0;
      S.hfill = 0;
    }
    __syncthreads();
    for (uint64_t i = tid; i < n; i += NT) {
      const K x = src[i];
      if (x < lo || x > hi) continue;
      uint64_t hh = (uint64_t)x ^ (uint64_t)(x >> (4 * sizeof(K))) ^ (uint64_t)(x >> (8 * sizeof(K) - 8));
      hh = (hh ^ (hh >> 29)) * 0xBF58476D1CE4E5B9ull;
      uint32_t slot = (uint32_t)(hh >> 40) & (HN - 1);
      for (uint32_t probes = 0;; probes++) {
        if (probes >= (uint32_t)HN || *(volatile int *)&S.flag) {
          S.flag = 1;
          break;
        }
        uint32_t st = *(volatile uint32_t *)&T.state[slot];
        if (st == 0) {
          if (atomicCAS(&T.state[slot], 0u, 1u) == 0u) {
            T.key[slot] = x;
            __threadfence_block();
            atomicExch(&T.state[slot], 2u);
            atomicAdd(&T.cnt[slot], 1u);
            if (atomicAdd(&S.hfill, 1u) + 1 > (uint32_t)(HN * 3 / 4)) S.flag = 1;
            break;
          }
          st = 1;
        }
        if (st == 1) {  // another thread is writing this slot's key
          uint32_t w = 0;
          while ((st = *(volatile uint32_t *)&T.state[slot]) != 2u && ++w < (1u << 22)) {
          }
          if (st != 2u) {
            atomicOr(a.err, ERR_SPIN_TIMEOUT);
            S.flag = 1;
            break;
          }
        }
        if (*(volatile K *)&T.key[slot] == x) {
          atomicAdd(&T.cnt[slot], 1u);
          break;
        }
        slot = (slot + 1) & (HN - 1);
      }
    }
    __syncthreads();
    if (S.flag && lo < hi) {
      if (tid == 0) {
        const K mid = lo + ((hi - lo) >> 1);
        if (S.sp + 2 <= CC_STACK) {
          S.stk_lo[S.sp] = mid + 1;  // upper half below the lower half
          S.stk_hi[S.sp] = hi;
          S.stk_lo[S.sp + 1] = lo;
          S.stk_hi[S.sp + 1] = mid;
          S.sp += 2;
        } else {
          atomicOr(a.err, ERR_BOUNDS);
        }
      }
      __syncthreads();
      continue;
    }
    // the occupied slots to the front (through registers), sorted, written
    constexpr int PT = HN / NT;
    K mk[PT];
    uint32_t mc[PT], mine = 0;
#pragma unroll
    for (int u = 0; u < PT; u++) {
      const int s = u * NT + tid;
      if (T.state[s] == 2u) {
        mk[mine] = T.key[s];
        mc[mine] = T.cnt[s];
        mine++;
      }
    }
    __syncthreads();
    if (tid == 0) S.hfill = 0;
    __syncthreads();
    const uint32_t first = atomicAdd(&S.hfill, mine);
#pragma unroll
    for (int u = 0; u < PT; u++)
      if ((uint32_t)u < mine) {
        T.key[first + u] = mk[u];
        T.cnt[first + u] = mc[u];
      }
    __syncthreads();
    const uint32_t nd = S.hfill;
    block_sort_pairs<K, NT>(T.key, T.cnt, nd);
    const uint64_t ob = S.out_base + S.run;
    for (uint32_t i = tid; i < nd; i += NT) {
      if (ob + i < a.stage_cap) {
        out_keys[ob + i] = T.key[i];
        a.stage_counts[ob + i] = T.cnt[i];
      } else {
        atomicOr(a.err, ERR_CAPACITY);
      }
    }
    __syncthreads();
    if (tid == 0) S.run += nd;
    __syncthreads();
  }
}

template <typename K>
__global__ void __launch_bounds__(CountShape<K>::NT, 2) k_bucket_count(SortCountArgs a) {
  constexpr int NT = CountShape<K>::NT, CAP = CountShape<K>::CAP, KPT = CAP / NT;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  CountSmem<K> &S = *reinterpret_cast<CountSmem<K> *>(smem_raw);
  const K *keys = reinterpret_cast<const K *>(a.keys);
  K *tmp = reinterpret_cast<K *>(a.scratch);
  const int key_bits = 2 * a.k;
  const int room = key_bits < 32 ? key_bits : 32;  // bits of the map
  const int tid = threadIdx.x;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  const uint64_t n_buckets = a.bucket_base[a.nbins];
  while (true) {
    if (tid == 0) {
      S.g = atomicAdd(a.ticket, 1ull);
      if (S.g < n_buckets) {
        S.b = find_bin(a.bucket_base, a.nbins, S.g);
        S.start = a.bucket_start[S.g];
        S.n = a.bucket_size[S.g];
      }
    }
    __syncthreads();
    const uint64_t g = S.g;
    if (g >= n_buckets) break;
    const uint64_t start = S.start, n = S.n;
    const uint32_t b = S.b;
    const int cb = (int)a.bin_bits[b];
    if (n <= (uint64_t)CAP) {
      // ---- the whole bucket in shared memory
      const uint32_t m = (uint32_t)n;
      int sb = 0;
      while (sb < CC_SB_MAX && (2u << sb) <= m) sb++;
      sb = min(sb, room - cb);
      const uint32_t nsub = 1u << sb;
      for (uint32_t jj = tid; jj < nsub; jj += NT) S.cnt[jj] = 0;
      __syncthreads();
      K xs[KPT];
      uint32_t rk[(KPT + 1) / 2];
#pragma unroll
      for (int u = 0; u < (KPT + 1) / 2; u++) rk[u] = 0;
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t i = u * NT + tid;
        if (i < m) {
          xs[u] = keys[start + i];
          const uint32_t r = atomicAdd(&S.cnt[sub_digit<K>(xs[u], key_bits, cb, sb)], 1u);
          rk[u / 2] |= r << (16 * (u & 1));
        }
      }
      __syncthreads();
      scan_sub<K, NT>(S, nsub);
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t i = u * NT + tid;
        if (i < m)
          S.u.A[S.cnt[sub_digit<K>(xs[u], key_bits, cb, sb)] + ((rk[u / 2] >> (16 * (u & 1))) & 0xFFFFu)] = xs[u];
      }
      __syncthreads();
      const uint32_t D = slice_runs<K, NT>(S, m, 0, nsub, 0);
      // the runs go to the staging arrays at the bucket's own key range
      // (its keys are all in registers or shared memory by now); a later
      // pass moves them to their final place
      if (tid == 0) a.bucket_d[g] = D;
      write_runs<K, NT>(S, a, D, start);
      __syncthreads();
      continue;
    }

    // ---- oversized bucket: placed by sub-bucket in the scratch area, then
    // counted in slices of at most CAP keys in key order
    const int sb = max(0, min(CC_SB_MAX, room - cb));
    const uint32_t nsub = 1u << sb;
    if (tid == 0) {
      S.flag = 0;
      const unsigned long long at = atomicAdd(a.scratch_cursor, (unsigned long long)n);
      if (at + n > a.scratch_keys) {
        atomicOr(a.err, ERR_OVERSIZE_SCRATCH);
        S.flag = 1;
      }
      S.tbase = at;
    }
    for (uint32_t jj = tid; jj < nsub; jj += NT) S.cnt[jj] = 0;
    __syncthreads();
    if (S.flag) {  // no room: an empty result (the host re-runs with a larger area)
      if (tid == 0) a.bucket_d[g] = 0;
      __syncthreads();
      continue;
    }
    K *place = tmp + S.tbase;
    for (uint64_t i = tid; i < n; i += NT) atomicAdd(&S.cnt[sub_digit<K>(keys[start + i], key_bits, cb, sb)], 1u);
    __syncthreads();
    scan_sub<K, NT>(S, nsub);
    static_assert(sizeof(S.C) / 4 >= CC_NSUB_MAX, "cursors fit in C");
    uint32_t *cur = reinterpret_cast<uint32_t *>(S.C);
    for (uint32_t jj = tid; jj < nsub; jj += NT) cur[jj] = S.cnt[jj];
    __syncthreads();
    for (uint64_t i = tid; i < n; i += NT) {
      const K x = keys[start + i];
      place[atomicAdd(&cur[sub_digit<K>(x, key_bits, cb, sb)], 1u)] = x;
    }
    __threadfence_block();
    __syncthreads();
    if (tid == 0) {
      S.out_base = start;  // staged at the bucket's own key range (all its keys are in the scratch area)
      S.run = 0;
    }
    __syncthreads();
    uint32_t jlo = 0;
    while (jlo < nsub) {
      // next slice: sub-buckets [jlo, jhi), at most CAP keys, or one heavy sub-bucket
      const uint32_t s0 = S.cnt[jlo];
      uint32_t lo = jlo + 1, hi = nsub;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        const uint64_t e = mid < nsub ? S.cnt[mid] : n;
        if (e - s0 <= (uint64_t)CAP) lo = mid; else hi = mid - 1;
      }
      const uint32_t jhi = lo;
      const uint64_t se = jhi < nsub ? S.cnt[jhi] : n;
      const uint64_t ns = se - s0;
      if (ns <= (uint64_t)CAP) {
        const uint32_t m = (uint32_t)ns;
        for (uint32_t i = tid; i < m; i += NT) S.u.A[i] = place[s0 + i];
        __syncthreads();
        const uint32_t D = slice_runs<K, NT>(S, m, jlo, jhi - jlo, s0);
        write_runs<K, NT>(S, a, D, S.out_base + S.run);
        __syncthreads();
        if (tid == 0) S.run += D;
        __syncthreads();
      } else {
        heavy_slice<K, NT>(S, a, place + s0, ns);
      }
      jlo = jhi;
    }
    if (tid == 0) a.bucket_d[g] = S.run;
    __syncthreads();
  }
}

// Moves each bucket's staged runs to its final offset (the exclusive scan of
// the buckets' distinct counts), one warp per bucket; bin_out[b] is the
// offset of the bin's first bucket.
template <typename K>
__global__ void k_compact_runs(const K *stage_keys, const uint32_t *stage_counts, const uint64_t *bucket_start,
                               const unsigned long long *bucket_d, const uint64_t *bucket_out,
                               const uint64_t *bucket_base, uint32_t nbins, K *out_keys, uint32_t *out_counts,
                               uint64_t *bin_out, const uint32_t *err) {
  if (*err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  const uint64_t nb = bucket_base[nbins];
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = t; b <= nbins; b += nt) bin_out[b] = bucket_out[bucket_base[b]];
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t g = t >> 5; g < nb; g += nt >> 5) {
    const uint64_t s = bucket_start[g], d = bucket_d[g], o = bucket_out[g];
    for (uint64_t i = lane; i < d; i += 32) {
      out_keys[o + i] = stage_keys[s + i];
      out_counts[o + i] = stage_counts[s + i];
    }
  }
}

template __global__ void k_compact_runs<uint64_t>(const uint64_t *, const uint32_t *, const uint64_t *,
                                                  const unsigned long long *, const uint64_t *, const uint64_t *,
                                                  uint32_t, uint64_t *, uint32_t *, uint64_t *, const uint32_t *);
template __global__ void k_compact_runs<u128>(const u128 *, const uint32_t *, const uint64_t *,
                                              const unsigned long long *, const uint64_t *, const uint64_t *,
                                              uint32_t, u128 *, uint32_t *, uint64_t *, const uint32_t *);
template __global__ void k_bucket_scatter<uint64_t>(ExpandArgs);
template __global__ void k_bucket_scatter<u128>(ExpandArgs);
template __global__ void k_bucket_count<uint64_t>(SortCountArgs);
template __global__ void k_bucket_count<u128>(SortCountArgs);

}  // namespace gkc
