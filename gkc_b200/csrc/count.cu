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
//                         digits.  Warps take 32 consecutive k-mers at a time,
//                         one per lane: each lane finds its superkmer by a
//                         search over the next 32 superkmers' k-mer ends and
//                         extracts its k-mer from aligned 8-byte words;
//   2. k_bucket_scan    - one CTA per bin turns the (chunk, digit) counts
//                         into each chunk's write offset per digit and each
//                         bucket's start, size and bin;
//   3. k_bucket_scatter - expands every k-mer once the same way and writes
//                         it at its chunk's offset for its digit plus its
//                         rank there (a shared-memory atomic);
//   4. k_bucket_count   - persistent, buckets taken by ticket, each counted
//                         on its own: its keys aggregated in a shared-memory
//                         hash table and the distinct (key, count) pairs
//                         sorted by a bitonic network; a bucket with too many
//                         distinct keys is counting-sorted by sub-bucket
//                         instead (the digit that follows the common prefix
//                         of its smallest and largest key), each sub-bucket
//                         reduced by its thread or a warp.  The runs are staged at the bucket's own key
//                         range and its distinct count recorded;
//                         k_compact_runs then moves them to the scan of the
//                         counts.  A bucket larger than shared memory is
//                         placed by sub-bucket in a scratch area and counted
//                         in slices; a single sub-bucket too large for a slice
//                         is aggregated in a shared-memory hash table over key
//                         ranges that are halved until a range's distinct keys
//                         fit.
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

// Bits of a key type, its leading zeros, and the sb bits that follow the
// first cp bits (keys of one bucket share their first cp bits, the common
// prefix of the bucket's smallest and largest key, so these digits order the
// bucket's keys by their first differing bits whatever the distribution).
template <typename K> constexpr int key_type_bits() { return 8 * (int)sizeof(K); }
GKC_DEV int key_clz(uint64_t x) { return __clzll((long long)x); }
GKC_DEV int key_clz(u128 x) {
  const uint64_t hi = (uint64_t)(x >> 64);
  return hi ? __clzll((long long)hi) : 64 + __clzll((long long)(uint64_t)x);
}
template <typename K>
GKC_DEV uint32_t prefix_digit(K x, int cp, int sb) {
  if (sb == 0) return 0u;  // sb <= key bits - cp, so cp < key bits here
  return (uint32_t)((K)(x << cp) >> (key_type_bits<K>() - sb));
}
// The sub-bucket bits of a bucket of m keys whose smallest and largest keys
// are lo and hi: about two sub-buckets per key, at most CC_SB_MAX bits, and
// no more than the bits below the common prefix.
template <typename K>
GKC_DEV void prefix_split(K lo, K hi, uint64_t m, int sb_max, int *cp, int *sb) {
  *cp = lo == hi ? key_type_bits<K>() : key_clz((K)(lo ^ hi));
  int b = 0;
  while (b < sb_max && ((uint64_t)1 << b) < 2 * m) b++;
  *sb = min(b, key_type_bits<K>() - *cp);
}

// Pulls the 128-byte line holding p into L2 (no register waits for it).
GKC_DEV void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

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

// Packed bases are read as aligned 8-byte words, byte-swapped so that the
// stream's first base is in the top bits (2 bits per base, MSB first within
// a byte).  A word is loaded only when it holds a wanted base, so reads end
// within 7 bytes past the last superkmer.
GKC_DEV uint64_t be_word(const uint8_t *packed, uint64_t w) {
  const uint64_t x = __ldg(reinterpret_cast<const unsigned long long *>(packed) + w);
  return ((uint64_t)__byte_perm((uint32_t)x, 0, 0x0123) << 32) | __byte_perm((uint32_t)(x >> 32), 0, 0x0123);
}

// nb <= 64 bits of the stream from bit position pos, left-aligned.
GKC_DEV uint64_t stream_bits(const uint8_t *packed, uint64_t pos, int nb) {
  const uint64_t w = pos >> 6;
  const int r = (int)(pos & 63);
  uint64_t v = be_word(packed, w) << r;
  if (r + nb > 64) v |= be_word(packed, w + 1) >> (64 - r);
  return v;
}

// The 2k bits of bases [o, o+k) of a packed superkmer at byte `off`.
template <typename K>
GKC_DEV K extract_kmer(const uint8_t *packed, uint64_t off, uint32_t o, int k);

template <>
GKC_DEV uint64_t extract_kmer<uint64_t>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  return stream_bits(packed, 8 * off + 2 * (uint64_t)o, 2 * k) >> (64 - 2 * k);
}

template <>
GKC_DEV u128 extract_kmer<u128>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  const uint64_t pos = 8 * off + 2 * (uint64_t)o;
  const int nb = 2 * k;  // 66 .. 128
  const uint64_t hi = stream_bits(packed, pos, 64);
  const uint64_t lo = stream_bits(packed, pos + 64, nb - 64);
  const u128 v = ((u128)hi << 64) | lo;
  return v >> (128 - nb);
}

// The k-mers [qa, qb) of one bin, taken by the calling warp 32 at a time,
// lane i the i-th of each group: each lane finds its superkmer among the 32
// from the group's first one (a search over their k-mer ends relative to the
// group's first k-mer, held one per lane), extracts its k-mer and passes the
// canonical key to emit(key, valid) (called by every lane; valid is false
// past qb).  s0 is the superkmer holding k-mer qa, s_end the bin's end
// (k-mer offsets up to koff[s_end] are read).  The next group's offsets are
// loaded before this group's k-mers are extracted.
template <typename K, typename Emit>
GKC_DEV void warp_kmers(const ExpandArgs &a, uint64_t qa, uint64_t qb, uint64_t s0, uint64_t s_end, Emit &&emit) {
  const uint32_t lane = threadIdx.x & 31u;
  const int k = a.k;
  uint64_t base = s0;
  uint64_t e = base + 1 + lane <= s_end ? __ldg(a.koff + base + 1 + lane) : ~0ull;  // end of superkmer base + lane
  uint64_t kb = __ldg(a.koff + base);                                                // start of superkmer base
  for (uint64_t q0 = qa; q0 < qb; q0 += 32) {
    // superkmer `base` holds q0 or ends at it, so e >= q0
    const uint32_t rel = (uint32_t)min(e - q0, (uint64_t)64);
    uint32_t cnt = 0;  // superkmers from `base` on that end at or before q0 + lane
#pragma unroll
    for (uint32_t st = 16; st > 0; st >>= 1)
      if (__shfl_sync(0xffffffffu, rel, cnt + st - 1) <= lane) cnt += st;
    const uint32_t prev = __shfl_sync(0xffffffffu, rel, cnt ? cnt - 1 : 0);
    const uint32_t r31 = __shfl_sync(0xffffffffu, rel, 31);
    const bool valid = q0 + lane < qb;
    uint64_t s = base + cnt;
    uint64_t o = cnt ? (uint64_t)(lane - prev) : q0 - kb + lane;  // the k-mer's index in its superkmer
    if (valid && lane >= r31) {  // 32 superkmers (some without k-mers) end before this k-mer
      const uint64_t q = q0 + lane;
      s = skm_of_kmer(a.koff, base + 32, s_end - 1, q);
      o = q - __ldg(a.koff + s);
    }
    const uint64_t nbase = __shfl_sync(0xffffffffu, s, 31);  // holds the next group's first k-mer or precedes it
    uint64_t ne = e, nkb = kb;
    if (q0 + 32 < qb) {
      ne = nbase + 1 + lane <= s_end ? __ldg(a.koff + nbase + 1 + lane) : ~0ull;
      nkb = __ldg(a.koff + nbase);
    }
    K key = 0;
    if (valid) {
      const uint64_t off = __ldg(a.desc + s) >> 24;
      const K x = extract_kmer<K>(a.packed, off, (uint32_t)o, k);
      const K r = revcomp_k<K>(x, k);
      key = x < r ? x : r;
    }
    emit(key, valid);
    base = nbase;
    e = ne;
    kb = nkb;
  }
}

// The k-mers of chunk c (bin b, j-th chunk of the bin) taken by warp w of W:
// [*qa, *qb) and the superkmer holding *qa.
GKC_DEV uint64_t warp_run(const ExpandArgs &a, uint64_t c, uint32_t b, uint64_t j, int w, int W, uint64_t *qa,
                          uint64_t *qb) {
  const uint64_t q0 = a.bin_kstart[b] + j * a.chunk_kmers;
  const uint64_t q1 = min(q0 + a.chunk_kmers, a.bin_kstart[b + 1]);
  const uint64_t per = ((q1 - q0 + W - 1) / W + 31) & ~31ull;
  *qa = min(q0 + per * w, q1);
  *qb = min(*qa + per, q1);
  const uint64_t lo = a.chunk_s0[c];
  const uint64_t hi = (c + 1 < a.chunk_base[b + 1]) ? a.chunk_s0[c + 1] : a.bin_start[b + 1] - 1;
  return skm_of_kmer(a.koff, lo, hi, *qa);
}

// ----------------------------------------------------------- 1. histogram

constexpr int HS_NT = 256;

// Expands every k-mer once (k-mer extraction and canonical form:
// kmer_counting.cu:99-112, 33-44) into `flat`, in k-mer order, and counts
// the coarse digits of each chunk of a bin's k-mers; each warp takes a
// contiguous share of the chunk, 32 consecutive k-mers at a time, so the
// writes are coalesced.
template <typename K>
__global__ void __launch_bounds__(HS_NT) k_bucket_hist(ExpandArgs a) {
  __shared__ uint32_t hist[1 << kCoarseMaxBits];
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  K *flat = reinterpret_cast<K *>(a.flat);
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  const int w = threadIdx.x >> 5;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t j = c - a.chunk_base[b];
    const int cb = (int)a.bin_bits[b];
    const uint32_t nd = 1u << cb;
    for (uint32_t d = threadIdx.x; d < nd; d += HS_NT) hist[d] = 0;
    __syncthreads();
    uint64_t qa, qb;
    const uint64_t s0 = warp_run(a, c, b, j, w, HS_NT / 32, &qa, &qb);
    if (qa < qb && qb <= a.keys_cap) {
      uint64_t q = qa + (threadIdx.x & 31u);
      warp_kmers<K>(a, qa, qb, s0, a.bin_start[b + 1], [&](K key, bool valid) {
        if (valid) {
          flat[q] = key;
          atomicAdd(&hist[coarse_digit<K>(key, key_bits, cb)], 1u);
        }
        q += 32;
      });
    } else if (qa < qb && (threadIdx.x & 31u) == 0) {
      atomicOr(a.err, ERR_CAPACITY);
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
                                                       uint64_t *bucket_size, uint32_t *bucket_bin) {
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
        bucket_bin[g0 + d] = b;
        if (col[u] >= a.big_min) a.big_list[atomicAdd(a.big_count, 1ull)] = (uint32_t)(g0 + d);
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

constexpr int SC_THREADS = 1024;
// keys per scatter tile: the tile, its digits and three digit tables fill
// most of the shared memory of one CTA per SM
template <typename K> constexpr int sc_tile() { return sizeof(K) == 8 ? 16384 : 8192; }

// Moves every key of `flat` to its bucket.  Each CTA takes whole chunks, a
// tile of SC_TILE keys at a time: the tile is counting-sorted by digit in
// shared memory (a key's rank within its digit from a shared-memory atomic),
// then written out in that order, so the keys of one digit leave as a
// contiguous run at the chunk's write offset for the digit (from the scan)
// plus the digit's keys of the chunk's earlier tiles.
template <typename K>
__global__ void __launch_bounds__(SC_THREADS, 1) k_bucket_scatter(ExpandArgs a) {
  constexpr int SC_TILE = sc_tile<K>(), KPT = SC_TILE / SC_THREADS;
  constexpr int ND = 1 << kCoarseMaxBits;
  extern __shared__ __align__(16) uint8_t sc_smem[];
  K *S = reinterpret_cast<K *>(sc_smem);                      // the tile, by digit
  uint16_t *Sd = reinterpret_cast<uint16_t *>(S + SC_TILE);   // digits of S
  uint32_t *gbase = reinterpret_cast<uint32_t *>(Sd + SC_TILE);  // chunk's write offsets
  uint32_t *done = gbase + ND;                                // digit's keys of the chunk's earlier tiles
  uint32_t *toff = done + ND;                                 // tile counts, then tile offsets (ND + 1)
  uint32_t *tmp = toff + ND + 1;                              // block scan
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  K *keys = reinterpret_cast<K *>(a.keys);
  const K *flat = reinterpret_cast<const K *>(a.flat);
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  const int tid = threadIdx.x;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t j = c - a.chunk_base[b];
    const int cb = (int)a.bin_bits[b];
    const uint32_t nd = 1u << cb;
    const uint64_t kbase = a.bin_kstart[b];
    const uint64_t q0 = kbase + j * a.chunk_kmers;
    const uint64_t q1 = min(q0 + a.chunk_kmers, a.bin_kstart[b + 1]);
    const uint32_t *row = a.hist + a.hist_base[b] + j * nd;
    for (uint32_t d = tid; d < nd; d += SC_THREADS) {
      gbase[d] = row[d];
      done[d] = 0;
    }
    for (uint64_t t0 = q0; t0 < q1; t0 += SC_TILE) {
      const uint32_t tn = (uint32_t)min((uint64_t)SC_TILE, q1 - t0);
      // the chunk's next tile into L2 while this one is sorted and written
      constexpr int KPL = 128 / (int)sizeof(K);  // keys per line
      for (uint64_t i = t0 + SC_TILE + (uint64_t)tid * KPL; i < q1 && i < t0 + 2 * (uint64_t)SC_TILE;
           i += (uint64_t)SC_THREADS * KPL)
        prefetch_l2(flat + i);
      for (uint32_t d = tid; d < nd; d += SC_THREADS) toff[d] = 0;
      __syncthreads();
      K xs[KPT];
      uint32_t rk[KPT / 2];  // ranks within the digit, two 16-bit halves (< SC_TILE)
#pragma unroll
      for (int u = 0; u < KPT / 2; u++) rk[u] = 0;
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t i = u * SC_THREADS + tid;
        if (i < tn) {
          xs[u] = flat[t0 + i];
          rk[u / 2] |= atomicAdd(&toff[coarse_digit<K>(xs[u], key_bits, cb)], 1u) << (16 * (u & 1));
        }
      }
      __syncthreads();
      // exclusive scan of the tile counts, thread-contiguous digits
      const uint32_t per = (nd + SC_THREADS - 1) / SC_THREADS, d0 = tid * per;
      uint32_t sum = 0;
      for (uint32_t d = d0; d < d0 + per && d < nd; d++) sum += toff[d];
      uint32_t total;
      uint32_t run = block_exclusive_scan<SC_THREADS>(sum, tmp, &total);
      for (uint32_t d = d0; d < d0 + per && d < nd; d++) {
        const uint32_t v = toff[d];
        toff[d] = run;
        run += v;
      }
      if (tid == 0) toff[nd] = total;
      __syncthreads();
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t i = u * SC_THREADS + tid;
        if (i < tn) {
          const uint32_t d = coarse_digit<K>(xs[u], key_bits, cb);
          const uint32_t at = toff[d] + ((rk[u / 2] >> (16 * (u & 1))) & 0xFFFFu);
          S[at] = xs[u];
          Sd[at] = (uint16_t)d;
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < tn; i += SC_THREADS) {
        const uint32_t d = Sd[i];
        const uint64_t slot = kbase + gbase[d] + done[d] + (i - toff[d]);
        if (slot < a.keys_cap) keys[slot] = S[i];
        else atomicOr(a.err, ERR_CAPACITY);
      }
      __syncthreads();
      for (uint32_t d = tid; d < nd; d += SC_THREADS) done[d] += toff[d + 1] - toff[d];
      __syncthreads();  // before the next tile clears toff
    }
  }
}

template <typename K> size_t bucket_scatter_smem_bytes() {
  constexpr int ND = 1 << kCoarseMaxBits;
  static_assert(sc_tile<K>() <= 65536 && sc_tile<K>() % SC_THREADS == 0, "16-bit ranks, whole rounds");
  return (size_t)sc_tile<K>() * (sizeof(K) + 2) + 4 * (3 * ND + 1 + 64);
}
template size_t bucket_scatter_smem_bytes<uint64_t>();
template size_t bucket_scatter_smem_bytes<u128>();

// ---------------------------------------------------------------- 4. count

template <typename K> struct CountShape;
template <> struct CountShape<uint64_t> { static constexpr int NT = 512, CAP = 8192; };
template <> struct CountShape<u128> { static constexpr int NT = 512, CAP = 4096; };
constexpr int CC_SB_MAX = 12;        // sub-bucket bits
constexpr int CC_NSUB_MAX = 1 << CC_SB_MAX;
constexpr uint32_t CC_THREAD_MAX = 8;  // larger sub-buckets are reduced by warps
constexpr int CC_BIG_LIST = 1024;      // > CAP / (CC_THREAD_MAX + 1): every larger sub-bucket fits
constexpr uint32_t CC_TICKETS = 4;     // buckets taken per ticket
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
  uint16_t big[CC_BIG_LIST];      // sub-buckets reduced by warps
  uint32_t tmp[64];
  uint32_t nbig, hfill, nsub;
  int flag, sp;
  uint64_t g, start, n, out_base, run, tbase;
  uint64_t pf_start, pf_n;        // the next bucket's keys, prefetched into L2
  K red[64];                      // block min / max
  uint32_t b;
  union {
    struct {
      K lo[CC_STACK], hi[CC_STACK];
    } stk;                       // key-range stack of the heavy path
    uint16_t dc[CC_NSUB_MAX];    // distinct keys of each sub-bucket of a slice
  } w;
};

static_assert(CountShape<uint64_t>::CAP / (CC_THREAD_MAX + 1) < CC_BIG_LIST, "big list holds every large sub-bucket");
static_assert(CountShape<u128>::CAP / (CC_THREAD_MAX + 1) < CC_BIG_LIST, "big list holds every large sub-bucket");

template <typename K> size_t bucket_count_smem_bytes() { return sizeof(CountSmem<K>); }
template <typename K> uint64_t bucket_count_cap() { return CountShape<K>::CAP; }
template uint64_t bucket_count_cap<uint64_t>();
template uint64_t bucket_count_cap<u128>();
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

template <typename K>
GKC_DEV void insertion_sort(K *A, uint32_t b0, uint32_t b1) {
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

// Run-length encodes the sorted A[b0, b1) in place (keys in A, counts in C
// from b0); returns the number of runs.
template <typename K>
GKC_DEV uint32_t rle_in_place(K *A, uint16_t *C, uint32_t b0, uint32_t b1) {
  uint32_t u = 0;
  for (uint32_t i = b0; i < b1;) {
    const K x = A[i];
    uint32_t c = 1;
    i++;
    while (i < b1 && A[i] == x) {
      c++;
      i++;
    }
    A[b0 + u] = x;
    C[b0 + u] = (uint16_t)c;  // c <= m <= CAP < 2^16
    u++;
  }
  return u;
}

template <typename K> GKC_DEV K shfl_xor_k(K v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
template <> GKC_DEV u128 shfl_xor_k<u128>(u128 v, int m) {
  const uint64_t lo = __shfl_xor_sync(0xffffffffu, (uint64_t)v, m);
  const uint64_t hi = __shfl_xor_sync(0xffffffffu, (uint64_t)(v >> 64), m);
  return ((u128)hi << 64) | lo;
}
template <typename K> GKC_DEV K shfl_up_k(K v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <> GKC_DEV u128 shfl_up_k<u128>(u128 v, int d) {
  const uint64_t lo = __shfl_up_sync(0xffffffffu, (uint64_t)v, d);
  const uint64_t hi = __shfl_up_sync(0xffffffffu, (uint64_t)(v >> 64), d);
  return ((u128)hi << 64) | lo;
}

// Smallest and largest of the block's (lo, hi) pairs, in every thread.
template <typename K, int NT>
GKC_DEV void block_minmax(CountSmem<K> &S, K &lo, K &hi) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    const K a = shfl_xor_k<K>(lo, m), b = shfl_xor_k<K>(hi, m);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if (lane == 0) {
    S.red[w] = lo;
    S.red[32 + w] = hi;
  }
  __syncthreads();
  lo = S.red[0];
  hi = S.red[32];
  for (int i = 1; i < NT / 32; i++) {
    lo = S.red[i] < lo ? S.red[i] : lo;
    hi = S.red[32 + i] > hi ? S.red[32 + i] : hi;
  }
  __syncthreads();
}

GKC_DEV uint32_t warp_exclusive_scan(uint32_t c, uint32_t *total) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t inc = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= (uint32_t)d) inc += t;
  }
  *total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - c;
}

// Sorts A[b0, b0 + n), n <= 32 R, with the calling warp: lane l holds
// positions l R .. l R + R - 1 in registers (positions past n hold the
// largest key, so the first n sorted positions are A's keys), a bitonic
// network over 32 R positions; then run-length encodes the sorted keys in
// place (keys in A, counts in C from b0).  Returns the number of runs.
template <typename K, int R>
GKC_DEV uint32_t warp_sort_rle(K *A, uint16_t *C, uint32_t b0, uint32_t n) {
  constexpr uint32_t N = 32 * R;
  const uint32_t lane = threadIdx.x & 31u;
  K v[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const uint32_t e = lane * R + r;
    v[r] = e < n ? A[b0 + e] : ~(K)0;
  }
#pragma unroll
  for (uint32_t size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride < (uint32_t)R) {
#pragma unroll
        for (int r = 0; r < R; r++)
          if ((r & stride) == 0) {
            const bool asc = ((lane * R + r) & size) == 0;
            const K x = v[r], y = v[r + stride];
            const bool sw = asc ? (y < x) : (x < y);
            v[r] = sw ? y : x;
            v[r + stride] = sw ? x : y;
          }
      } else {
        const int lm = (int)(stride / R);
#pragma unroll
        for (int r = 0; r < R; r++) {
          const K y = shfl_xor_k<K>(v[r], lm);
          const bool asc = ((lane * R + r) & size) == 0;
          const bool low = (lane & (uint32_t)lm) == 0;  // the lower position of the pair
          const bool keep_min = low == asc;
          v[r] = keep_min ? (y < v[r] ? y : v[r]) : (v[r] < y ? y : v[r]);
        }
      }
    }
  }
  // run heads among the first n positions
  const K before = shfl_up_k<K>(v[R - 1], 1);
  uint32_t hb = 0;
#pragma unroll
  for (int r = 0; r < R; r++) {
    const uint32_t e = lane * R + r;
    const K p = r == 0 ? before : v[r > 0 ? r - 1 : 0];
    if (e < n && (e == 0 || p != v[r])) hb |= 1u << r;
  }
  uint32_t D;
  const uint32_t rank0 = warp_exclusive_scan(__popc(hb), &D);
  __syncwarp();
  uint32_t rank = rank0;
#pragma unroll
  for (int r = 0; r < R; r++)
    if ((hb >> r) & 1u) {
      A[b0 + rank] = v[r];
      C[b0 + rank] = (uint16_t)(lane * R + r);  // the run's first position, < 32 R
      rank++;
    }
  __syncwarp();
  uint32_t nxt[R];
  rank = rank0;
#pragma unroll
  for (int r = 0; r < R; r++)
    if ((hb >> r) & 1u) {
      nxt[r] = rank + 1 < D ? C[b0 + rank + 1] : n;
      rank++;
    }
  __syncwarp();
  rank = rank0;
#pragma unroll
  for (int r = 0; r < R; r++)
    if ((hb >> r) & 1u) {
      C[b0 + rank] = (uint16_t)(nxt[r] - (lane * R + r));
      rank++;
    }
  __syncwarp();
  return D;
}

template <typename K> GKC_DEV K warp_min_k(K v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    const K y = shfl_xor_k<K>(v, m);
    v = y < v ? y : v;
  }
  return v;
}

// Run-length encodes A[b0, b0 + n) with the calling warp when it holds at
// most 32 distinct keys: each round takes the smallest key above the last
// one and counts its copies.  Returns the number of runs, or 0 (A untouched)
// when there are more.
template <typename K>
GKC_DEV uint32_t warp_select_rle(K *A, uint16_t *C, uint32_t b0, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u;
  K mine = 0;
  uint32_t mine_c = 0, d = 0, seen = 0;
  K last = 0;
  while (seen < n) {
    if (d == 32) return 0;
    K lo = ~(K)0;
    bool any = false;
    for (uint32_t i = lane; i < n; i += 32) {
      const K x = A[b0 + i];
      if ((d == 0 || last < x) && (!any || x < lo)) {
        lo = x;
        any = true;
      }
    }
    // lanes with nothing above `last` offer the largest key, which is only
    // taken when no lane has a smaller one; the copies counted below decide
    const K key = warp_min_k<K>(lo);
    uint32_t c = 0;
    for (uint32_t i = lane; i < n; i += 32) c += A[b0 + i] == key ? 1u : 0u;
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) c += __shfl_xor_sync(0xffffffffu, c, m);
    if (lane == d) {
      mine = key;
      mine_c = c;
    }
    last = key;
    seen += c;
    d++;
  }
  __syncwarp();
  if (lane < d) {
    A[b0 + lane] = mine;
    C[b0 + lane] = (uint16_t)mine_c;
  }
  __syncwarp();
  return d;
}

// The m keys in S.u.A are grouped by sub-bucket: sub-bucket jb + jj starts at
// S.cnt[jb + jj] - s0 for jj in [0, nsl) (the last one ends at m).  Each
// sub-bucket is reduced to its runs in place: by the thread that owns it
// (insertion sort) when it holds at most CC_THREAD_MAX keys, else by a warp
// (a register bitonic sort up to 128 keys; above that, rounds that take the
// next smallest key while there are at most 32 distinct ones; else a bitonic
// sort in shared memory).  A k-mer seen many times fills a sub-bucket with
// copies of itself and of its sequencing-error variants, which share its
// leading bases.  Each thread then packs the runs of the sub-buckets it owns
// together from their first key on (keys in A, counts in C).  Sets
// S.seg_src / S.seg_pos (exclusive scan of the run counts) and returns the
// slice's distinct keys.
template <typename K, int NT>
GKC_DEV uint32_t slice_runs(CountSmem<K> &S, uint32_t m, uint32_t jb, uint32_t nsl, uint32_t s0) {
  const int tid = threadIdx.x;
  K *A = S.u.A;
  uint16_t *dc = S.w.dc;
  auto start_of = [&](uint32_t jj) -> uint32_t { return jj < nsl ? S.cnt[jb + jj] - s0 : m; };
  const uint32_t j0 = (uint32_t)(((uint64_t)tid * nsl) / NT), j1 = (uint32_t)(((uint64_t)(tid + 1) * nsl) / NT);
  if (tid == 0) S.nbig = 0;
  __syncthreads();
  for (uint32_t jj = j0; jj < j1; jj++) {
    const uint32_t b0 = start_of(jj), b1 = start_of(jj + 1);
    if (b1 - b0 <= CC_THREAD_MAX) {
      insertion_sort<K>(A, b0, b1);
      dc[jj] = (uint16_t)rle_in_place<K>(A, S.C, b0, b1);
    } else {
      S.big[atomicAdd(&S.nbig, 1u)] = (uint16_t)jj;  // fewer than CC_BIG_LIST (static_assert)
    }
  }
  __syncthreads();
  const uint32_t nbig = S.nbig, lane = threadIdx.x & 31u;
  for (uint32_t t = threadIdx.x >> 5; t < nbig; t += NT / 32) {
    const uint32_t jj = S.big[t];
    const uint32_t b0 = start_of(jj), n = start_of(jj + 1) - b0;
    uint32_t d;
    if (n <= 32) {
      d = warp_sort_rle<K, 1>(A, S.C, b0, n);
    } else if (n <= 64) {
      d = warp_sort_rle<K, 2>(A, S.C, b0, n);
    } else if (n <= 128) {
      d = warp_sort_rle<K, 4>(A, S.C, b0, n);
    } else {
      d = warp_select_rle<K>(A, S.C, b0, n);
      if (d == 0) {
        warp_sort<K>(A + b0, n);
        if (lane == 0) d = rle_in_place<K>(A, S.C, b0, b0 + n);
        d = __shfl_sync(0xffffffffu, d, 0);
      }
    }
    if (lane == 0) dc[jj] = (uint16_t)d;
    __syncwarp();
  }
  __syncthreads();
  const uint32_t s = start_of(j0);
  uint32_t u = 0;
  for (uint32_t jj = j0; jj < j1; jj++) {
    const uint32_t b0 = start_of(jj), d = dc[jj];
    if (b0 != s + u)
      for (uint32_t i = 0; i < d; i++) {
        A[s + u + i] = A[b0 + i];
        S.C[s + u + i] = S.C[b0 + i];
      }
    u += d;
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
    S.w.stk.lo[0] = (K)0;
    S.w.stk.hi[0] = ~(K)0;
  }
  __syncthreads();
  while (true) {
    if (S.sp == 0) break;
    const K lo = S.w.stk.lo[S.sp - 1], hi = S.w.stk.hi[S.sp - 1];
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
          S.w.stk.lo[S.sp] = mid + 1;  // upper half below the lower half
          S.w.stk.hi[S.sp] = hi;
          S.w.stk.lo[S.sp + 1] = lo;
          S.w.stk.hi[S.sp + 1] = mid;
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

// Sorts the 32 R keys (with counts) at Kb / Cb by the calling warp in
// registers: lane l holds positions r 32 + l, a bitonic network (strides
// below 32 across lanes by shuffles, larger ones across a lane's registers).
template <int R, typename CT>
GKC_DEV void warp_sort_run(uint64_t *Kb, CT *Cb) {
  const uint32_t lane = threadIdx.x & 31u;
  uint64_t v[R];
  uint32_t c[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    v[r] = Kb[r * 32 + lane];
    c[r] = Cb[r * 32 + lane];
  }
#pragma unroll
  for (uint32_t size = 2; size <= 32u * R; size <<= 1) {
#pragma unroll
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int rs = (int)(stride / 32);
#pragma unroll
        for (int r = 0; r < R; r++)
          if ((r & rs) == 0) {
            const bool asc = ((r * 32 + lane) & size) == 0;
            const uint64_t x = v[r], y = v[r + rs];
            if (asc ? (y < x) : (x < y)) {
              v[r] = y;
              v[r + rs] = x;
              const uint32_t t = c[r];
              c[r] = c[r + rs];
              c[r + rs] = t;
            }
          }
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) {
          const bool asc = ((r * 32 + lane) & size) == 0;
          const uint64_t y = __shfl_xor_sync(0xffffffffu, v[r], stride);
          const uint32_t cy = __shfl_xor_sync(0xffffffffu, c[r], stride);
          const bool keep_min = ((lane & stride) == 0) == asc;
          if (keep_min ? (y < v[r]) : (v[r] < y)) {
            v[r] = y;
            c[r] = cy;
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    Kb[r * 32 + lane] = v[r];
    Cb[r * 32 + lane] = (CT)c[r];
  }
}

// Merges the sorted runs of length L of (sk, sc) pairwise into (dk, dc): each
// thread writes P / NT consecutive outputs (at least one), starting from a
// merge-path search of its first one.
template <int NT, typename CT>
GKC_DEV void merge_round(const uint64_t *sk, const CT *sc, uint64_t *dk, CT *dc, uint32_t P, uint32_t L) {
  const uint32_t per = P >= (uint32_t)NT ? P / NT : 1u;
  const uint32_t o0 = threadIdx.x * per;
  if (o0 < P) {
    const uint32_t a0 = o0 & ~(2 * L - 1);
    const uint64_t *A = sk + a0, *Bk = sk + a0 + L;
    const uint32_t o = o0 - a0;
    uint32_t lo = o > L ? o - L : 0u, hi = o < L ? o : L;
    while (lo < hi) {  // i = outputs before o taken from A (ties from A first)
      const uint32_t mid = (lo + hi) >> 1;
      if (A[mid] <= Bk[o - mid - 1]) lo = mid + 1; else hi = mid;
    }
    uint32_t i = lo, j = o - lo;
    for (uint32_t t = 0; t < per; t++) {
      if (j >= L || (i < L && A[i] <= Bk[j])) {
        dk[o0 + t] = A[i];
        dc[o0 + t] = sc[a0 + i];
        i++;
      } else {
        dk[o0 + t] = Bk[j];
        dc[o0 + t] = sc[a0 + L + j];
        j++;
      }
    }
  }
  __syncthreads();
}

// Sorts P keys with counts (P a power of two in [32, 4096]) held in buffer 0
// (k0, c0), using buffer 1 (k1, c1) as well: runs of P / W keys sorted by W
// warps in registers, then merged pairwise.  Returns the buffer that holds
// the result.
template <int NT, typename CT>
GKC_DEV int block_merge_sort(uint64_t *k0, CT *c0, uint64_t *k1, CT *c1, uint32_t P) {
  const uint32_t W = min((uint32_t)NT / 32, P / 32), C = P / W, w = threadIdx.x >> 5;
  if (w < W) {
    switch (C / 32) {
      case 1: warp_sort_run<1, CT>(k0 + w * C, c0 + w * C); break;
      case 2: warp_sort_run<2, CT>(k0 + w * C, c0 + w * C); break;
      case 4: warp_sort_run<4, CT>(k0 + w * C, c0 + w * C); break;
      default: warp_sort_run<8, CT>(k0 + w * C, c0 + w * C); break;
    }
  }
  __syncthreads();
  int src = 0;
  for (uint32_t L = C; L < P; L <<= 1) {
    if (src == 0) merge_round<NT, CT>(k0, c0, k1, c1, P, L);
    else merge_round<NT, CT>(k1, c1, k0, c0, P, L);
    src ^= 1;
  }
  return src;
}

// ---- hash path (8-byte keys): a bucket's keys aggregated in a shared-memory
// table first, so that only its distinct keys are sorted, by comparisons
// (keys of a minimizer bin are far from uniform in their leading bases:
// those holding the minimizer near their start share them, so digit splits
// of a bucket can be very uneven).  The keys are read from global memory, so
// a bucket of any size with few enough distinct keys takes this path.  The
// table lives in the upper half of the key area (keys) and in the run-count
// area (counts); the distinct keys go to the lower half of the key area,
// their counts to the per-sub-bucket array, and are merge-sorted with the
// table's two areas as the second buffer.  The slices of a bucket too large
// for the table are counted the same way.
constexpr uint32_t HT_SLOTS = 4096;
constexpr uint32_t HT_MAX_DISTINCT = 3072;  // 3/4 full: beyond it the bucket takes the sub-bucket path
constexpr uint64_t HT_MAX_KEYS = 65535;     // counts of the sorted pairs are 16-bit
constexpr uint32_t HT_MAX_PROBE = 64;       // a longer probe chain also abandons the table
constexpr uint64_t HT_EMPTY = ~0ull;        // never a canonical key: the reverse complement of all-T is all-A

GKC_DEV uint32_t ht_slot(uint64_t x) { return (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> 52); }

template <int NT, typename K>
GKC_DEV bool hash_count(CountSmem<K> &, const SortCountArgs &, const K *, uint64_t, uint64_t) {
  return false;  // 16-byte keys: no 128-bit compare-and-swap in shared memory here
}

// Counts the n keys src[0, n) (read from global memory; n < 2^16, so counts
// fit 16 bits) through the table and writes their sorted runs to the staging
// arrays at `out_at`; their number is left in S.hfill.  Returns false, with
// nothing written, when there are more than HT_MAX_DISTINCT distinct keys
// (the caller then takes another path).  Uses the key area, the run-count
// area and the per-sub-bucket array only (S.cnt is left as it is).  Not
// inlined: its registers are then not added to the count kernel's.
template <int NT>
__device__ __noinline__ bool hash_count(CountSmem<uint64_t> &S, const SortCountArgs &a, const uint64_t *src,
                                        uint64_t n, uint64_t out_at) {
  static_assert(2 * HT_SLOTS <= (uint32_t)CountShape<uint64_t>::CAP, "table and sorted keys share the key area");
  static_assert(sizeof(S.C) >= HT_SLOTS * 4, "table counts fit the run-count area");
  static_assert(sizeof(S.w.dc) >= HT_SLOTS * 2, "sorted counts fit the per-sub-bucket array");
  constexpr uint32_t SPT = HT_SLOTS / NT;
  constexpr int U = 8;  // keys in flight per thread
  if (n > HT_MAX_KEYS) return false;
  volatile uint64_t *T = S.u.A + HT_SLOTS;
  uint32_t *TC = reinterpret_cast<uint32_t *>(S.C);
  uint64_t *B = S.u.A;
  uint16_t *BC = S.w.dc;
  const int tid = threadIdx.x;
  for (uint32_t i = tid; i < HT_SLOTS; i += NT) {
    T[i] = HT_EMPTY;
    TC[i] = 0;
  }
  if (tid == 0) {
    S.hfill = 0;
    S.flag = 0;
  }
  __syncthreads();
  for (uint64_t i0 = tid; i0 < n; i0 += (uint64_t)U * NT) {
    if (*(volatile int *)&S.flag) break;
    uint64_t xs[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t i = i0 + (uint64_t)u * NT;
      xs[u] = i < n ? __ldg(reinterpret_cast<const unsigned long long *>(src) + i) : HT_EMPTY;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t x = xs[u];
      if (i0 + (uint64_t)u * NT >= n || *(volatile int *)&S.flag) break;
      uint32_t h = ht_slot(x);
      for (uint32_t probe = 0;; probe++) {
        if (probe == HT_MAX_PROBE) {  // a long chain: the table is too full, give up
          S.flag = 1;
          break;
        }
        uint64_t cur = T[h];
        if (cur == HT_EMPTY) {
          cur = atomicCAS((unsigned long long *)(S.u.A + HT_SLOTS + h), (unsigned long long)HT_EMPTY,
                          (unsigned long long)x);
          if (cur == HT_EMPTY) {
            atomicAdd(&TC[h], 1u);
            if (atomicAdd(&S.hfill, 1u) + 1 > HT_MAX_DISTINCT) S.flag = 1;
            break;
          }
        }
        if (cur == x) {
          atomicAdd(&TC[h], 1u);
          break;
        }
        h = (h + 1) & (HT_SLOTS - 1);
      }
    }
  }
  __syncthreads();
  if (S.flag) return false;
  const uint32_t D = S.hfill;
  // the distinct keys, in slot order, to B[0, D), their counts to BC; the
  // rest of the power of two above D holds the largest key
  uint32_t own = 0;
#pragma unroll
  for (int q = 0; q < (int)SPT; q++) own += T[q * NT + tid] != HT_EMPTY ? 1u : 0u;
  uint32_t tot;
  uint32_t pos = block_exclusive_scan<NT>(own, S.tmp, &tot);
#pragma unroll
  for (int q = 0; q < (int)SPT; q++) {
    const uint32_t slot = q * NT + tid;
    const uint64_t x = T[slot];
    if (x != HT_EMPTY) {
      B[pos] = x;
      BC[pos] = (uint16_t)TC[slot];  // <= n < 2^16
      pos++;
    }
  }
  uint32_t P = 32;
  while (P < D) P <<= 1;
  for (uint32_t i = D + tid; i < P; i += NT) {
    B[i] = HT_EMPTY;
    BC[i] = 0;
  }
  __syncthreads();
  // the table is free now: its two areas are the sort's second buffer
  uint64_t *B1 = S.u.A + HT_SLOTS;
  uint16_t *BC1 = S.C;
  const int res = block_merge_sort<NT, uint16_t>(B, BC, B1, BC1, P);
  const uint64_t *RK = res ? B1 : B;
  const uint16_t *RC = res ? BC1 : BC;
  uint64_t *out = reinterpret_cast<uint64_t *>(a.stage_keys);
  for (uint32_t i = tid; i < D; i += NT) {
    if (out_at + i < a.stage_cap) {
      out[out_at + i] = RK[i];
      a.stage_counts[out_at + i] = RC[i];
    } else {
      atomicOr(a.err, ERR_CAPACITY);
    }
  }
  __syncthreads();
  return true;
}

// Counts the m <= CAP keys src[0, m) in shared memory and stages their runs
// at out_at; returns their number.  The keys are counting-sorted by the
// sub-bucket digit that follows the common prefix of their smallest and
// largest key, then each sub-bucket is reduced to runs (slice_runs).  Not
// inlined: it is called for whole buckets and for the slices of large ones.
template <typename K, int NT, int KPT>
__device__ __noinline__ uint32_t smem_count(CountSmem<K> &S, const SortCountArgs &a, const K *src, uint32_t m,
                                            uint64_t out_at) {
  const int tid = threadIdx.x;
  K xs[KPT];
  K lo = ~(K)0, hi = 0;
#pragma unroll
  for (int u = 0; u < KPT; u++) {
    const uint32_t i = u * NT + tid;
    if (i < m) {
      xs[u] = src[i];
      lo = xs[u] < lo ? xs[u] : lo;
      hi = xs[u] > hi ? xs[u] : hi;
    }
  }
  block_minmax<K, NT>(S, lo, hi);
  int cp, sb;
  prefix_split<K>(lo, hi, m, CC_SB_MAX, &cp, &sb);
  const uint32_t nsub = 1u << sb;
  for (uint32_t jj = tid; jj < nsub; jj += NT) S.cnt[jj] = 0;
  __syncthreads();
  uint32_t rk[(KPT + 1) / 2];
#pragma unroll
  for (int u = 0; u < (KPT + 1) / 2; u++) rk[u] = 0;
#pragma unroll
  for (int u = 0; u < KPT; u++) {
    const uint32_t i = u * NT + tid;
    if (i < m) rk[u / 2] |= atomicAdd(&S.cnt[prefix_digit<K>(xs[u], cp, sb)], 1u) << (16 * (u & 1));
  }
  __syncthreads();
  scan_sub<K, NT>(S, nsub);
#pragma unroll
  for (int u = 0; u < KPT; u++) {
    const uint32_t i = u * NT + tid;
    if (i < m) S.u.A[S.cnt[prefix_digit<K>(xs[u], cp, sb)] + ((rk[u / 2] >> (16 * (u & 1))) & 0xFFFFu)] = xs[u];
  }
  __syncthreads();
  const uint32_t D = slice_runs<K, NT>(S, m, 0, nsub, 0);
  write_runs<K, NT>(S, a, D, out_at);
  __syncthreads();
  return D;
}

template <typename K>
__global__ void __launch_bounds__(CountShape<K>::NT, 2) k_bucket_count(SortCountArgs a) {
  constexpr int NT = CountShape<K>::NT, CAP = CountShape<K>::CAP, KPT = CAP / NT;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  CountSmem<K> &S = *reinterpret_cast<CountSmem<K> *>(smem_raw);
  const K *keys = reinterpret_cast<const K *>(a.keys);
  K *tmp = reinterpret_cast<K *>(a.scratch);
  const int tid = threadIdx.x;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ | ERR_BIN_TOO_LARGE)) return;
  const uint64_t n_buckets = a.bucket_base[a.nbins];
  int hash_skip = 0;                // the same in every thread of the block
  int slice_skip = 0;               // the same, for the slices of large buckets
  uint64_t t_next = 0, t_end = 0;   // thread 0: the rest of its batch of tickets
  bool big_phase = true;            // thread 0: the large buckets first, so none is left for the end
  while (true) {
    if (tid == 0) {
      uint64_t gg = n_buckets;
      if (big_phase) {
        const unsigned long long bi = atomicAdd(a.big_ticket, 1ull);
        if (bi < *a.big_count) gg = a.big_list[bi];
        else big_phase = false;
      }
      if (!big_phase) {
        while (true) {
          if (t_next == t_end) {
            t_next = atomicAdd(a.ticket, (unsigned long long)CC_TICKETS);
            t_end = t_next + CC_TICKETS;
          }
          gg = t_next++;
          if (gg >= n_buckets || a.bucket_size[gg] < a.big_min) break;  // a large one: taken from the list
        }
      }
      S.g = gg;
      if (gg < n_buckets) {
        S.b = a.bucket_bin[gg];
        S.start = a.bucket_start[gg];
        S.n = a.bucket_size[gg];
      }
      // the next bucket of the batch, if it is a regular one
      S.pf_n = 0;
      if (!big_phase && t_next < t_end && t_next < n_buckets) {
        const uint64_t nn = a.bucket_size[t_next];
        if (nn < a.big_min) {
          S.pf_start = a.bucket_start[t_next];
          S.pf_n = nn;
        }
      }
    }
    __syncthreads();
    const uint64_t g = S.g;
    if (g >= n_buckets) break;
    const uint64_t start = S.start, n = S.n;
    {
      constexpr int KPL = 128 / (int)sizeof(K);
      const uint64_t ps = S.pf_start, pe = ps + S.pf_n;
      for (uint64_t i = ps + (uint64_t)tid * KPL; i < pe; i += (uint64_t)NT * KPL) prefetch_l2(keys + i);
    }
    // distinct keys through the table first, unless the last bucket that
    // tried it had too many (then skip it for a few buckets)
    if (n <= HT_MAX_KEYS) {
      if (hash_skip == 0) {
        if (hash_count<NT>(S, a, keys + start, n, start)) {
          if (tid == 0) a.bucket_d[g] = S.hfill;
          __syncthreads();
          continue;
        }
        hash_skip = 8;
      } else {
        hash_skip--;
      }
    }
    if (n <= (uint64_t)CAP) {
      // ---- the whole bucket in shared memory; the runs go to the staging
      // arrays at the bucket's own key range (its keys are all on chip by
      // then), and a later pass moves them to their final place
      const uint32_t D = smem_count<K, NT, KPT>(S, a, keys + start, (uint32_t)n, start);
      if (tid == 0) a.bucket_d[g] = D;
      continue;
    }

    // ---- oversized bucket: placed by sub-bucket in the scratch area, then
    // counted in slices of at most CAP keys in key order
    K lo = ~(K)0, hi = 0;
    for (uint64_t i = tid; i < n; i += NT) {
      const K x = keys[start + i];
      lo = x < lo ? x : lo;
      hi = x > hi ? x : hi;
    }
    block_minmax<K, NT>(S, lo, hi);
    int cp, sb;
    prefix_split<K>(lo, hi, n, CC_SB_MAX, &cp, &sb);
    const uint32_t nsub = 1u << sb;
    for (uint32_t jj = tid; jj < nsub; jj += NT) S.cnt[jj] = 0;
    __syncthreads();
    // the bucket's own key range of the scratch array (the result's key
    // array, written only after this kernel)
    K *place = tmp + start;
    for (uint64_t i = tid; i < n; i += NT) atomicAdd(&S.cnt[prefix_digit<K>(keys[start + i], cp, sb)], 1u);
    __syncthreads();
    scan_sub<K, NT>(S, nsub);
    static_assert(sizeof(S.C) / 4 >= CC_NSUB_MAX, "cursors fit in C");
    uint32_t *cur = reinterpret_cast<uint32_t *>(S.C);
    for (uint32_t jj = tid; jj < nsub; jj += NT) cur[jj] = S.cnt[jj];
    __syncthreads();
    for (uint64_t i = tid; i < n; i += NT) {
      const K x = keys[start + i];
      place[atomicAdd(&cur[prefix_digit<K>(x, cp, sb)], 1u)] = x;
    }
    // the sub-bucket starts go to this CTA's global area: the slices are
    // counted with the shared-memory counters
    uint32_t *gst = a.slice_starts + (uint64_t)blockIdx.x * (CC_NSUB_MAX + 1);
    for (uint32_t jj = tid; jj < nsub; jj += NT) gst[jj] = S.cnt[jj];
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
      const uint32_t s0 = gst[jlo];
      uint32_t lo = jlo + 1, hi = nsub;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        const uint64_t e = mid < nsub ? gst[mid] : n;
        if (e - s0 <= (uint64_t)CAP) lo = mid; else hi = mid - 1;
      }
      const uint32_t jhi = lo;
      const uint64_t se = jhi < nsub ? gst[jhi] : n;
      const uint64_t ns = se - s0;
      if (ns <= (uint64_t)CAP) {
        uint32_t D;
        bool hashed = false;
        if (slice_skip == 0) {
          hashed = hash_count<NT>(S, a, place + s0, ns, S.out_base + S.run);
          if (!hashed) slice_skip = 8;
        } else {
          slice_skip--;
        }
        if (hashed) D = S.hfill;
        else D = smem_count<K, NT, KPT>(S, a, place + s0, (uint32_t)ns, S.out_base + S.run);
        __syncthreads();
        if (tid == 0) S.run += D;
        __syncthreads();
      } else if (hash_count<NT>(S, a, place + s0, ns, S.out_base + S.run)) {
        // one sub-bucket larger than a slice with few distinct keys
        if (tid == 0) S.run += S.hfill;
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
template __global__ void k_bucket_hist<uint64_t>(ExpandArgs);
template __global__ void k_bucket_hist<u128>(ExpandArgs);
template __global__ void k_bucket_scatter<uint64_t>(ExpandArgs);
template __global__ void k_bucket_scatter<u128>(ExpandArgs);
template __global__ void k_bucket_count<uint64_t>(SortCountArgs);
template __global__ void k_bucket_count<u128>(SortCountArgs);

}  // namespace gkc
