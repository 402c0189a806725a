// Canonical k-mer counting from bin-grouped superkmers (batched path).
//
// Semantics follow kmc_counting_GPU (kmer_counting.cu:95-191): every k-mer of
// every superkmer of a bin, canonicalised as min(x, revcomp(x)), sorted
// ascending, run-length counted (count clamped to 2^32-1), per bin.
//
// Device layout:
//   1. k_coarse_hist    - each chunk of a bin's k-mer stream (load-balanced:
//                         every thread expands the same number of k-mers)
//                         histograms the top `bin_bits[b]` bits of the
//                         canonical keys; counts go to a (bin, digit, chunk)
//                         matrix whose exclusive scan gives every chunk its
//                         write offset per digit -- no global atomics;
//   2. k_coarse_scatter - re-expands and writes each key into its coarse
//                         bucket (bin, top bits);
//   3. k_coarse_count   - persistent, one coarse bucket per iteration: a
//                         sub-histogram of the next bits plans slices; each
//                         slice is aggregated in an order-preserving shared
//                         memory hash table (duplicates meet in one slot, a
//                         left-to-right scan is ascending once collision
//                         clusters are sorted) and written as sorted
//                         (k-mer, count) runs to a staging area;
//   4. k_compact        - moves each coarse bucket's runs to its final offset.
#include "common.cuh"
#include "kernels.h"
#include "sortsmem.cuh"

namespace gkc {

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

// ----------------------------------------------------------------- expansion

// The 2k bits of bases [o, o+k) of a packed superkmer starting at byte `off`
// (2 bits per base, first base in the top bits of its byte).
template <typename K>
GKC_DEV K extract_kmer(const uint8_t *packed, uint64_t off, uint32_t o, int k);

template <>
GKC_DEV uint64_t extract_kmer<uint64_t>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  const uint8_t *p = packed + off + (o >> 2);
  const int sh = 2 * (o & 3);
  uint64_t hi = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) hi = (hi << 8) | __ldg(p + i);
  const uint32_t nx = __ldg(p + 8);
  const uint64_t v = sh ? ((hi << sh) | (nx >> (8 - sh))) : hi;
  return v >> (64 - 2 * k);
}

template <>
GKC_DEV u128 extract_kmer<u128>(const uint8_t *packed, uint64_t off, uint32_t o, int k) {
  const uint8_t *p = packed + off + (o >> 2);
  const int sh = 2 * (o & 3);
  u128 hi = 0;
#pragma unroll
  for (int i = 0; i < 16; i++) hi = (hi << 8) | (u128)__ldg(p + i);
  const uint32_t nx = __ldg(p + 16);
  const u128 v = sh ? ((hi << sh) | (u128)(nx >> (8 - sh))) : hi;
  return v >> (128 - 2 * k);
}

// Calls f(canonical key) for the k-mers with global indices [q0, q1) of the
// bin-ordered superkmer stream (superkmers [s_lo, s_hi) hold them; koff is
// the exclusive prefix of their k-mer counts).  The first k-mer of each
// superkmer segment is extracted whole and reverse-complemented; the rest roll
// in one base at a time (kmer_counting.cu:99-112, canonical form :33-44).
template <typename K, typename F>
GKC_DEV void expand_range(const uint64_t *desc, const uint64_t *koff, const uint8_t *packed,
                          uint64_t s_lo, uint64_t s_hi, uint64_t q0, uint64_t q1, int k, F &&f) {
  if (q0 >= q1) return;
  uint64_t lo = s_lo, hi = s_hi - 1;
  while (lo < hi) {
    uint64_t mid = (lo + hi + 1) >> 1;
    if (koff[mid] <= q0) lo = mid; else hi = mid - 1;
  }
  uint64_t s = lo;
  const K mask = kmer_mask<K>(k);
  const int top = 2 * k - 2;
  while (q0 < q1 && s < s_hi) {
    const uint64_t kb = koff[s], ke = koff[s + 1];
    if (q0 >= ke) {
      s++;
      continue;
    }
    const uint64_t off = desc[s] >> 24;
    const uint32_t o = (uint32_t)(q0 - kb);
    const uint32_t cnt = (uint32_t)(min(q1, ke) - q0);
    K x = extract_kmer<K>(packed, off, o, k);
    K r = revcomp_k<K>(x, k);
    f(x < r ? x : r);
    const uint8_t *src = packed + off;
    uint32_t j = o + (uint32_t)k;
    uint32_t byte = cnt > 1 ? __ldg(src + (j >> 2)) : 0u;
    for (uint32_t t = 1; t < cnt; t++, j++) {
      if ((j & 3u) == 0) byte = __ldg(src + (j >> 2));
      const uint32_t c = (byte >> (6 - 2 * (j & 3u))) & 3u;
      x = ((x << 2) | (K)c) & mask;
      r = (r >> 2) | ((K)(3u - c) << top);
      f(x < r ? x : r);
    }
    q0 += cnt;
    s++;
  }
}

GKC_DEV uint32_t find_bin(const uint64_t *base, uint32_t nbins, uint64_t c) {
  uint32_t lo = 0, hi = nbins - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (base[mid] <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

constexpr int EX_NT = 256;

struct ChunkInfo {
  uint32_t b, nbits;
  uint64_t j, nch, q0, q1, s_lo, s_hi;
};

GKC_DEV ChunkInfo chunk_info(const ExpandArgs &a, uint64_t c) {
  ChunkInfo ci;
  ci.b = find_bin(a.chunk_base, a.nbins, c);
  ci.j = c - a.chunk_base[ci.b];
  ci.nch = a.chunk_base[ci.b + 1] - a.chunk_base[ci.b];
  ci.nbits = a.bin_bits[ci.b];
  const uint64_t k0 = a.bin_kstart[ci.b] + ci.j * a.chunk_kmers;
  const uint64_t k1 = min(k0 + a.chunk_kmers, a.bin_kstart[ci.b + 1]);
  const uint64_t per = (k1 - k0 + EX_NT - 1) / EX_NT;
  ci.q0 = min(k0 + per * threadIdx.x, k1);
  ci.q1 = min(ci.q0 + per, k1);
  ci.s_lo = a.bin_start[ci.b];
  ci.s_hi = a.bin_start[ci.b + 1];
  return ci;
}

template <typename K>
__global__ void __launch_bounds__(EX_NT) k_coarse_hist(ExpandArgs a) {
  extern __shared__ uint32_t hist[];  // 1 << max bits
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ)) return;
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const ChunkInfo ci = chunk_info(a, c);
    const uint32_t nd = 1u << ci.nbits;
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT) hist[d] = 0;
    __syncthreads();
    expand_range<K>(a.desc, a.koff, a.packed, ci.s_lo, ci.s_hi, ci.q0, ci.q1, a.k, [&](K key) {
      atomicAdd(&hist[key_digit<K>(key, key_bits, 0, (int)ci.nbits)], 1u);
    });
    __syncthreads();
    unsigned long long *row = a.chunk_hist + a.hist_base[ci.b] + ci.j;
    for (uint32_t d = threadIdx.x; d < nd; d += EX_NT) row[(uint64_t)d * ci.nch] = hist[d];
    __syncthreads();
  }
}

// Writes every k-mer key at its (bin, coarse digit, chunk) slot.  A chunk is
// processed in sub-chunks of SctSub<K> k-mers: expanded into shared memory
// (with a digit histogram), permuted there into digit order, then written out
// linearly, so that consecutive threads store consecutive keys of one digit's
// run and global writes come in whole sectors instead of scattered words.
template <typename K>
__global__ void __launch_bounds__(SCT_NT) k_coarse_scatter(ExpandArgs a) {
  constexpr int SUB = SctSub<K>::value;
  extern __shared__ __align__(16) uint8_t sct_raw[];
  K *stage = reinterpret_cast<K *>(sct_raw);
  K *sorted = stage + SUB;
  unsigned long long *gbase = reinterpret_cast<unsigned long long *>(sorted + SUB);
  uint32_t *cursor = reinterpret_cast<uint32_t *>(gbase + (1u << a.max_bits));
  uint32_t *hstart = cursor + (1u << a.max_bits);
  __shared__ uint32_t tmp[64];
  __shared__ uint64_t s_first, s_last;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ)) return;
  K *keys = reinterpret_cast<K *>(a.keys);
  const uint64_t n_chunks = a.chunk_base[a.nbins];
  const int key_bits = 2 * a.k;
  const int tid = threadIdx.x;
  for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const uint32_t b = find_bin(a.chunk_base, a.nbins, c);
    const uint64_t j = c - a.chunk_base[b];
    const uint64_t nch = a.chunk_base[b + 1] - a.chunk_base[b];
    const uint32_t nbits = a.bin_bits[b], nd = 1u << nbits;
    const uint64_t k0 = a.bin_kstart[b] + j * a.chunk_kmers;
    const uint64_t k1 = min(k0 + a.chunk_kmers, a.bin_kstart[b + 1]);
    const uint64_t s_lo = a.bin_start[b], s_hi = a.bin_start[b + 1];
    const uint64_t *row = a.chunk_off + a.hist_base[b] + j;
    for (uint32_t d = tid; d < nd; d += SCT_NT) gbase[d] = row[(uint64_t)d * nch];
    for (uint64_t q0s = k0; q0s < k1; q0s += SUB) {
      const uint64_t q1s = min(q0s + SUB, k1);
      const uint32_t m = (uint32_t)(q1s - q0s);
      // the superkmers holding k-mers [q0s, q1s): last with koff <= q0s, last with koff < q1s
      if (tid < 2) {
        const uint64_t target = tid == 0 ? q0s : q1s - 1;
        uint64_t lo = s_lo, hi = s_hi - 1;
        while (lo < hi) {
          const uint64_t mid = (lo + hi + 1) >> 1;
          if (a.koff[mid] <= target) lo = mid; else hi = mid - 1;
        }
        if (tid == 0) s_first = lo; else s_last = lo;
      }
      for (uint32_t d = tid; d < nd; d += SCT_NT) cursor[d] = 0;
      __syncthreads();
      // expand into the stage in k-mer order, counting digits
      const uint32_t per = (m + SCT_NT - 1) / SCT_NT;
      const uint32_t p0 = min(m, (uint32_t)tid * per), p1 = min(m, p0 + per);
      uint32_t p = p0;
      expand_range<K>(a.desc, a.koff, a.packed, s_first, s_last + 1, q0s + p0, q0s + p1, a.k, [&](K key) {
        stage[p++] = key;
        atomicAdd(&cursor[key_digit<K>(key, key_bits, 0, (int)nbits)], 1u);
      });
      __syncthreads();
      // digit starts inside the sub-chunk (nd <= SCT_NT: one digit per thread)
      {
        const uint32_t v = (uint32_t)tid < nd ? cursor[tid] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan<SCT_NT>(v, tmp, &total);
        if ((uint32_t)tid < nd) {
          hstart[tid] = ex;
          cursor[tid] = ex;
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < m; i += SCT_NT) {
        const K x = stage[i];
        sorted[atomicAdd(&cursor[key_digit<K>(x, key_bits, 0, (int)nbits)], 1u)] = x;
      }
      __syncthreads();
      for (uint32_t i = tid; i < m; i += SCT_NT) {
        const K x = sorted[i];
        const uint32_t d = key_digit<K>(x, key_bits, 0, (int)nbits);
        const uint64_t slot = gbase[d] + (i - hstart[d]);
        if (slot < a.keys_cap) keys[slot] = x;
        else atomicOr(a.err, ERR_CAPACITY);
      }
      __syncthreads();
      for (uint32_t d = tid; d < nd; d += SCT_NT) gbase[d] += cursor[d] - hstart[d];
      __syncthreads();
    }
  }
}

template <typename K> size_t coarse_scatter_smem_bytes(uint32_t max_bits) {
  return 2 * (size_t)SctSub<K>::value * sizeof(K) + ((size_t)1 << max_bits) * 16;
}
template size_t coarse_scatter_smem_bytes<uint64_t>(uint32_t);
template size_t coarse_scatter_smem_bytes<u128>(uint32_t);

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

// ------------------------------------------- coarse bucket: hash-aggregate sort

// Order-preserving shared-memory hash table: a key's home slot is a monotone
// function of the key (piecewise linear over the slice's sub-buckets, each
// given slots in proportion to its keys), so duplicates meet in one slot and a
// left-to-right scan is ascending once each run of occupied slots (a
// collision cluster) is sorted: every key of a cluster has its home inside
// it, so clusters are mutually ordered.
template <typename K> struct SliceTab;
template <> struct SliceTab<uint64_t> { static constexpr int TS = 16384, OVF = 512; };
template <> struct SliceTab<u128> { static constexpr int TS = 8192, OVF = 512; };
constexpr int CC_SUB_BITS = 11;        // sub-histogram inside a coarse bucket
constexpr int CC_NSUB = 1 << CC_SUB_BITS;
constexpr int SL_PROBE_LIMIT = 256;
constexpr int SL_CLUSTER_LIMIT = 512;
constexpr int SL_LOW_BITS = 20;
constexpr int kSliceStack = 32;  // > 2 * log2(CC_NSUB) + 1: splits halve a slice's keys
// clusters longer than CW_MIN slots are sorted by a warp (up to CW_LIST a slice)
constexpr int CW_MIN = 16;
constexpr int CW_LIST = 128;
static_assert(SL_CLUSTER_LIMIT < 1024, "cluster lengths are packed in 10 bits");

template <typename K>
struct CoarseSmem {
  static constexpr int TSO = SliceTab<K>::TS + SliceTab<K>::OVF;
  union {
    struct {
      K key[TSO];
      uint32_t cnt[TSO];
    } t;
    SortSmem<K> s;  // fallback sort layout
  } u;
  uint32_t sub[CC_NSUB + 2];        // sub-bucket counts, then first placed keys
  uint32_t slot_base[CC_NSUB + 1];
  uint16_t slo[CC_NSUB + 1];        // first sub-bucket of each slice
  uint32_t tmp[64];
  uint64_t g, start, n, run;
  uint32_t b, nsl, cursor;
  int overflow;
  int sp;                    // slice stack: (first << 16) | end sub-bucket
  uint32_t stk[kSliceStack];
  uint64_t tot_n, tot_d;     // keys and distinct keys of this CTA's slices so far
  int sort_mode;
  int dirty;                 // the table memory was reused by a sort
  uint32_t occ[(TSO + 31) / 32];  // occupied table slots
  unsigned long long ph[8];  // phase cycles (profiling only)
  uint32_t nbig;             // long clusters: (first slot << 10) | length
  uint32_t bigl[CW_LIST];
};

template <typename K> size_t coarse_smem_bytes() { return sizeof(CoarseSmem<K>); }
template size_t coarse_smem_bytes<uint64_t>();
template size_t coarse_smem_bytes<u128>();

template <typename K> GKC_DEV K empty_key() { return ~(K)0; }

GKC_DEV uint64_t smem_cas(uint64_t *p, uint64_t cmp, uint64_t val) {
  return atomicCAS((unsigned long long *)p, (unsigned long long)cmp, (unsigned long long)val);
}
GKC_DEV u128 smem_cas(u128 *p, u128 cmp, u128 val) {
  // 16-byte compare-and-swap on shared memory (sm_90+)
  uint64_t clo = (uint64_t)cmp, chi = (uint64_t)(cmp >> 64);
  uint64_t vlo = (uint64_t)val, vhi = (uint64_t)(val >> 64);
  uint64_t rlo, rhi;
  unsigned addr = (unsigned)__cvta_generic_to_shared(p);
  asm volatile(
      "{\n\t.reg .b128 c, v, r;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 v, {%4, %5};\n\t"
      "atom.shared.cas.b128 r, [%6], c, v;\n\t"
      "mov.b128 {%0, %1}, r;\n\t}"
      : "=l"(rlo), "=l"(rhi)
      : "l"(clo), "l"(chi), "l"(vlo), "l"(vhi), "r"(addr)
      : "memory");
  return ((u128)rhi << 64) | rlo;
}

template <typename K>
GKC_DEV K volatile_load(const K *p) {
  return *(const volatile K *)p;
}

GKC_DEV void set_overflow(int *f) { *(volatile int *)f = 1; }

GKC_DEV uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded spin lock (thread 0 of a CTA): false if the wait ran out.
GKC_DEV bool acquire_lock(unsigned long long *lock, uint32_t *err) {
  const uint64_t t0 = globaltimer_ns();
  uint32_t it = 0;
  while (atomicCAS(lock, 0ull, 1ull) != 0ull) {
    if (++it > (1u << 24) || globaltimer_ns() - t0 > 10000000000ull) {
      atomicOr(err, ERR_SPIN_TIMEOUT);
      return false;
    }
    nanosleep_backoff(it);
  }
  __threadfence();
  return true;
}

// Records the first failed bounds check (code, index, limit); the caller
// skips the access.
GKC_DEV bool in_bounds(const SortCountArgs &a, int code, uint64_t idx, uint64_t lim) {
  if (idx < lim) return true;
  if (atomicCAS(a.dbg, 0ull, (unsigned long long)code) == 0ull) {
    a.dbg[1] = idx;
    a.dbg[2] = lim;
  }
  atomicOr(a.err, ERR_BOUNDS);
  return false;
}
GKC_DEV int get_overflow(const int *f) { return *(const volatile int *)f; }

// Oversized slice fallback: MSD passes through global scratch, depth first in
// key order; sub-ranges that fit are finished in shared memory.  Input: n keys
// in scratch half 0.  Output runs are appended at S.out.
template <typename K>
GKC_DEV void scratch_sort(SortSmem<K> &S, const SortCountArgs &a, uint64_t n, int skip0,
                          K *out_keys, uint32_t *out_counts) {
  const int key_bits = 2 * a.k;
  const int CAP = SortCap<K>::value;
  K *half[2] = {reinterpret_cast<K *>(a.scratch), reinterpret_cast<K *>(a.scratch) + a.scratch_keys};
  if (threadIdx.x == 0) {
    S.depth = 0;
    S.fr[0] = {0, n, skip0, 0, 0, 0, 0};
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
        if (in_bounds(a, 2, off + pos, a.scratch_keys)) half[1 - src][off + pos] = x;
      }
      __syncthreads();
      if (!in_bounds(a, 3, dep, 24)) return;
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
    if (threadIdx.x == 0) {
      // next action: a run of consecutive children that fits in shared memory
      // is sorted together (it is contiguous and in key order); a single child
      // too large to fit is split further, or emitted whole if all its bits
      // are consumed (all keys equal)
      S.act = 0;
      auto &F = S.fr[dep];
      const uint32_t nd = 1u << F.d;
      while (F.cursor < nd) {
        uint32_t j = F.cursor;
        uint64_t s0 = j ? gc[j - 1] : 0, e = gc[j];
        if (e == s0) {
          F.cursor++;
          continue;
        }
        if (e - s0 > (uint64_t)CAP) {
          F.cursor++;
          S.c_off = F.off + s0;
          S.c_len = e - s0;
          S.c_skip = F.skip + F.d;
          S.c_src = 1 - F.src;
          S.act = (S.c_skip >= key_bits) ? 2 : 3;
          break;
        }
        uint32_t jn = j + 1;
        while (jn < nd && gc[jn] - s0 <= (uint64_t)CAP) jn++;
        F.cursor = jn;
        S.c_off = F.off + s0;
        S.c_len = gc[jn - 1] - s0;
        S.c_skip = F.skip;  // the run shares only the parent's prefix
        S.c_src = 1 - F.src;
        S.act = 1;
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
      if (!in_bounds(a, 4, m, (uint64_t)CAP + 1) || !in_bounds(a, 5, S.c_off + m, a.scratch_keys + 1)) return;
      load_keys<K>(S.A, half[S.c_src] + S.c_off, m);
      __syncthreads();
      smem_sort<K>(S, m, key_bits, S.c_skip);
      uint32_t D = smem_runs<K>(S, m);
      if (!in_bounds(a, 6, S.out + D, a.tmp_cap + 1)) return;
      write_runs<K>(S, D, out_keys, out_counts, S.out);
      __syncthreads();
      if (threadIdx.x == 0) S.out += D;
    } else if (act == 2) {
      if (threadIdx.x == 0 && in_bounds(a, 7, S.out, a.tmp_cap)) {
        out_keys[S.out] = half[S.c_src][S.c_off];
        out_counts[S.out] = S.c_len > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)S.c_len;
        S.out += 1;
      }
    }
    __syncthreads();
  }
}

// In-place ascending sort of m (key, count) pairs by one warp: a bitonic
// network in the form where every comparator puts the smaller key at the
// lower index, so positions >= m act as +infinity.
template <typename K>
GKC_DEV void warp_sort_pairs(K *key, uint32_t *cnt, uint32_t m) {
  uint32_t P = 1;
  while (P < m) P <<= 1;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t size = 2; size <= P; size <<= 1) {
    const uint32_t half = size >> 1;
    for (uint32_t i = lane; i < P / 2; i += 32) {
      const uint32_t blk = i / half, off = i % half;
      const uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
      if (hi < m && key[hi] < key[lo]) {
        const K x = key[lo];
        key[lo] = key[hi];
        key[hi] = x;
        const uint32_t c = cnt[lo];
        cnt[lo] = cnt[hi];
        cnt[hi] = c;
      }
    }
    __syncwarp();
    for (uint32_t stride = size >> 2; stride >= 1; stride >>= 1) {
      for (uint32_t i = lane; i < P / 2; i += 32) {
        const uint32_t blk = i / stride, off = i % stride;
        const uint32_t lo = blk * 2 * stride + off, hi = lo + stride;
        if (hi < m && key[hi] < key[lo]) {
          const K x = key[lo];
          key[lo] = key[hi];
          key[hi] = x;
          const uint32_t c = cnt[lo];
          cnt[lo] = cnt[hi];
          cnt[hi] = c;
        }
      }
      __syncwarp();
    }
  }
}

template <typename K>
__global__ void __launch_bounds__(SC_NT, 1) k_coarse_count(SortCountArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  CoarseSmem<K> &S = *reinterpret_cast<CoarseSmem<K> *>(smem_raw);
  constexpr int TS = SliceTab<K>::TS, TSO = CoarseSmem<K>::TSO;
  const K *keys = reinterpret_cast<const K *>(a.keys);
  K *tkeys = reinterpret_cast<K *>(a.tmp_keys);
  const int key_bits = 2 * a.k;
  const int tid = threadIdx.x;
  if (*a.err & (ERR_CAPACITY | ERR_BAD_READ)) return;  // keys incomplete: the host re-runs
  const uint64_t n_buckets = a.bucket_base[a.nbins];
  if (tid == 0) {
    S.tot_n = 0;
    S.tot_d = 0;
    S.dirty = 1;  // the table starts uncleared
  }
  // optional phase profile (cycles of thread 0 between marks, per phase)
  const bool prof = a.prof != nullptr;
  if (tid < 8) S.ph[tid] = 0;
  long long tph = 0;
#define PHASE(i)                                       \
  if (prof && tid == 0) {                              \
    const long long _t = clock64();                    \
    S.ph[i] += (unsigned long long)(_t - tph);         \
    tph = _t;                                          \
  }
  while (true) {
    if (tid == 0) {
      S.g = atomicAdd(a.ticket, 1ull);
      if (S.g < n_buckets) {
        const uint32_t b = find_bin(a.bucket_base, a.nbins, S.g);
        const uint64_t d = S.g - a.bucket_base[b];
        const uint64_t nch = a.chunk_base[b + 1] - a.chunk_base[b];
        const uint64_t hb = a.hist_base[b];
        S.b = b;
        S.start = a.chunk_off[hb + d * nch];
        S.n = a.chunk_off[hb + (d + 1) * nch] - S.start;
      }
      S.run = 0;
      // Mostly distinct keys gain little from the table (and near-equal ones
      // make long probe chains): when this CTA's slices so far were more
      // than 55% distinct, the bucket's slices are sorted directly instead.
      S.sort_mode = S.tot_n > 0 && S.tot_d * 20 > S.tot_n * 11;
    }
    __syncthreads();
    const bool sort_mode = S.sort_mode;
    const uint32_t target = sort_mode ? (uint32_t)SortCap<K>::value : (uint32_t)(SliceTab<K>::TS / 2);
    const uint64_t g = S.g;
    if (g >= n_buckets) break;
    const uint64_t start = S.start, n = S.n;
    if (prof && tid == 0) tph = clock64();
    const int cb = (int)a.bin_bits[S.b];
    const int SB = min(CC_SUB_BITS, key_bits - cb);
    const uint32_t nsub = 1u << SB;
    const int lbits = min(SL_LOW_BITS, key_bits - cb - SB);
    if (n == 0) {
      if (tid == 0) {
        a.coarse_start[g] = start;
        a.coarse_d[g] = 0;
      }
      __syncthreads();
      continue;
    }
    // Sub-bucket counts at sub[1 + j]; their exclusive scan is the cursor of
    // sub-bucket j while the keys are placed in sub-bucket order in the
    // bucket's own range of tmp_keys (where they stay in L2), after which
    // sub[j] is the first placed key of sub-bucket j.  A slice then reads only
    // its own keys.  Its runs are written at or before its first key, after
    // all of its keys were read, so the placed keys of later slices survive.
    K *placed = tkeys + start;
    if (!in_bounds(a, 11, start + n, a.tmp_cap + 1)) return;
    for (uint32_t j = tid; j <= nsub; j += SC_NT) S.sub[j] = 0;
    __syncthreads();
    {
      constexpr int U = 8;
      for (uint64_t i0 = 0; i0 < n; i0 += (uint64_t)SC_NT * U) {
        K xs[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint64_t i = i0 + (uint64_t)u * SC_NT + tid;
          xs[u] = i < n ? keys[start + i] : (K)0;
        }
#pragma unroll
        for (int u = 0; u < U; u++)
          if (i0 + (uint64_t)u * SC_NT + tid < n) atomicAdd(&S.sub[1 + key_digit<K>(xs[u], key_bits, cb, SB)], 1u);
      }
      __syncthreads();
      scan_counters(S.sub + 1, nsub, S.tmp);
      for (uint64_t i0 = 0; i0 < n; i0 += (uint64_t)SC_NT * U) {
        K xs[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint64_t i = i0 + (uint64_t)u * SC_NT + tid;
          xs[u] = i < n ? keys[start + i] : (K)0;
        }
#pragma unroll
        for (int u = 0; u < U; u++)
          if (i0 + (uint64_t)u * SC_NT + tid < n) {
            const uint32_t pos = atomicAdd(&S.sub[1 + key_digit<K>(xs[u], key_bits, cb, SB)], 1u);
            if (in_bounds(a, 12, pos, n)) placed[pos] = xs[u];
          }
      }
    }
    __syncthreads();
    PHASE(0)
    // slices: runs of sub-buckets whose exclusive start falls in the same
    // multiple of `target` (a slice holds < target keys plus one sub-bucket)
    {
      const uint32_t per = (nsub + SC_NT - 1) / SC_NT, j0 = tid * per;
      uint32_t cnt = 0;
      for (uint32_t j = j0; j < j0 + per && j < nsub; j++)
        cnt += (j == 0 || S.sub[j] / target != S.sub[j - 1] / target);
      uint32_t total;
      uint32_t idx = block_exclusive_scan<SC_NT>(cnt, S.tmp, &total);
      for (uint32_t j = j0; j < j0 + per && j < nsub; j++)
        if (j == 0 || S.sub[j] / target != S.sub[j - 1] / target) S.slo[idx++] = (uint16_t)j;
      if (tid == 0) S.nsl = total;
      __syncthreads();
    }
    const uint32_t nsl = S.nsl;
    for (uint32_t sl = 0; sl < nsl; sl++) {
      // A slice that overflows the table is split at its key midpoint and the
      // halves retried, the left one first (a stack), so that the output
      // stays in key order; only a single sub-bucket falls back to sorting.
      if (tid == 0) {
        S.stk[0] = ((uint32_t)S.slo[sl] << 16) | ((sl + 1 < nsl) ? (uint32_t)S.slo[sl + 1] : nsub);
        S.sp = 1;
      }
     while (true) {
      __syncthreads();
      const int sp = S.sp;
      if (sp == 0) break;
      const uint32_t top = S.stk[sp - 1];
      __syncthreads();  // every thread has read the top before it is popped
      if (tid == 0) S.sp = sp - 1;
      const uint32_t j_lo = top >> 16;
      const uint32_t j_hi = top & 0xFFFFu;
      const uint32_t base_cnt = S.sub[j_lo];
      const uint32_t ns = S.sub[j_hi] - base_cnt;
      if (ns == 0) continue;
      if (!in_bounds(a, 13, (uint64_t)base_cnt + ns, n + 1)) continue;  // slice inside its bucket
      for (uint32_t j = j_lo + tid; j < j_hi; j += SC_NT)
        S.slot_base[j - j_lo] = (uint32_t)(((uint64_t)(S.sub[j] - base_cnt) * TS) / ns);
      if (tid == 0) {
        S.slot_base[j_hi - j_lo] = TS;
        S.overflow = 0;
        S.nbig = 0;
      }
      // slices of a sort-mode bucket that fit the shared-memory sort go there
      // directly; larger ones (one heavy sub-bucket) still use the table
      const bool direct_sort = sort_mode && ns <= (uint32_t)SortCap<K>::value;
      if (!direct_sort) {  // aggregate in the table
      // The occupancy bitmap (a bit per slot, set when an insert claims the
      // slot) lets the cluster walk, the output and the clearing touch only
      // occupied slots; the whole table is cleared only after a sort reused
      // its memory.
      constexpr int NW = (TSO + 31) / 32;
      static_assert(NW <= SC_NT, "one bitmap word per thread");
      if (S.dirty) {
        for (int s = tid; s < TSO; s += SC_NT) {
          S.u.t.key[s] = empty_key<K>();
          S.u.t.cnt[s] = 0;
        }
        for (int w = tid; w < NW; w += SC_NT) S.occ[w] = 0;
        __syncthreads();
        if (tid == 0) S.dirty = 0;
      }
      __syncthreads();
      for (uint32_t i = tid; i < ns; i += SC_NT) {
        const K x = placed[base_cnt + i];
        const uint32_t j = key_digit<K>(x, key_bits, cb, SB) - j_lo;
        const uint32_t low = key_digit<K>(x, key_bits, cb + SB, lbits);
        const uint32_t w = S.slot_base[j + 1] - S.slot_base[j];
        int slot = (int)(S.slot_base[j] + (uint32_t)(((uint64_t)low * w) >> lbits));
        int probes = 0;
        while (true) {
          if (slot >= TSO || probes > a.probe_limit) {
            set_overflow(&S.overflow);
            break;
          }
          // 8-byte keys are read atomically; 16-byte keys only through the CAS
          K cur = sizeof(K) == 8 ? volatile_load<K>(&S.u.t.key[slot]) : empty_key<K>();
          if (cur == x) {
            atomicAdd(&S.u.t.cnt[slot], 1u);
            break;
          }
          if (cur == empty_key<K>()) {
            K prev = smem_cas(&S.u.t.key[slot], empty_key<K>(), x);
            if (prev == empty_key<K>()) {
              atomicOr(&S.occ[slot >> 5], 1u << (slot & 31));
              atomicAdd(&S.u.t.cnt[slot], 1u);
              break;
            }
            if (prev == x) {
              atomicAdd(&S.u.t.cnt[slot], 1u);
              break;
            }
          }
          slot++;
          probes++;
        }
        if (get_overflow(&S.overflow)) break;
      }
      __syncthreads();
      PHASE(1)
      // clusters: runs of occupied slots; the owner of a cluster's first slot
      // sorts a short one, long ones go to warps
      const int w = tid;
      const uint32_t wbits = w < NW ? S.occ[w] : 0u;
      uint32_t occ = __popc(wbits);
      if (!S.overflow && wbits) {
        uint32_t bits = wbits;
        while (bits) {
          const int q = __ffs(bits) - 1;
          bits &= bits - 1;
          const int s = w * 32 + q;
          const bool prev_occ = q > 0 ? ((wbits >> (q - 1)) & 1u) != 0 : (w > 0 && (S.occ[w - 1] >> 31) != 0);
          if (prev_occ) continue;  // not a cluster start
          int e = s + 1;
          for (int ww = e >> 5; ww < NW; ww++) {  // first free slot after s
            const uint32_t inv = ~S.occ[ww] & (0xFFFFFFFFu << (ww == (e >> 5) ? (e & 31) : 0));
            if (inv) {
              e = ww * 32 + __ffs(inv) - 1;
              break;
            }
            e = (ww + 1) * 32;
            if (e - s > SL_CLUSTER_LIMIT) break;
          }
          e = min(e, TSO);
          if (e - s > SL_CLUSTER_LIMIT) {
            set_overflow(&S.overflow);
            break;
          }
          if (e - s > CW_MIN) {  // long: sorted by a warp below
            const uint32_t t = atomicAdd(&S.nbig, 1u);
            if (t < (uint32_t)CW_LIST) {
              S.bigl[t] = ((uint32_t)s << 10) | (uint32_t)(e - s);
              continue;
            }
          }
          for (int qq = s + 1; qq < e; qq++) {  // insertion sort of (key, count)
            K x = S.u.t.key[qq];
            uint32_t c = S.u.t.cnt[qq];
            int r = qq;
            while (r > s && x < S.u.t.key[r - 1]) {
              S.u.t.key[r] = S.u.t.key[r - 1];
              S.u.t.cnt[r] = S.u.t.cnt[r - 1];
              r--;
            }
            S.u.t.key[r] = x;
            S.u.t.cnt[r] = c;
          }
        }
      }
      __syncthreads();
      if (!S.overflow) {
        const uint32_t nbl = min(S.nbig, (uint32_t)CW_LIST);
        for (uint32_t t = threadIdx.x >> 5; t < nbl; t += SC_NT / 32)
          warp_sort_pairs<K>(S.u.t.key + (S.bigl[t] >> 10), S.u.t.cnt + (S.bigl[t] >> 10), S.bigl[t] & 1023u);
      }
      __syncthreads();
      PHASE(2)
      const bool ok = !S.overflow;
      if (ok) {
        uint32_t D;
        const uint32_t pos = block_exclusive_scan<SC_NT>(occ, S.tmp, &D);
        const uint64_t base = start + S.run + pos;
        uint32_t o = 0, bits = wbits;
        while (bits) {
          const int s = w * 32 + __ffs(bits) - 1;
          bits &= bits - 1;
          if (!in_bounds(a, 8, base + o, a.tmp_cap)) break;
          tkeys[base + o] = S.u.t.key[s];
          a.tmp_counts[base + o] = S.u.t.cnt[s];
          o++;
        }
        __syncthreads();
        if (tid == 0) {
          S.run += D;
          S.tot_n += ns;
          S.tot_d += D;
        }
      }
      // empty the occupied slots and the bitmap (after an overflow too: the
      // bitmap marks exactly the slots inserts claimed)
      {
        uint32_t bits = wbits;
        while (bits) {
          const int s = w * 32 + __ffs(bits) - 1;
          bits &= bits - 1;
          S.u.t.key[s] = empty_key<K>();
          S.u.t.cnt[s] = 0;
        }
        if (w < NW) S.occ[w] = 0;
      }
      __syncthreads();
      PHASE(3)
      if (ok) continue;
      if (j_hi - j_lo > 1 && sp + 1 <= kSliceStack) {
        if (tid == 0) {  // split: smallest mid in [j_lo+1, j_hi-1] with half the keys before it
          const uint32_t half = base_cnt + ns / 2;
          uint32_t lo = j_lo + 1, hi = j_hi - 1;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (S.sub[mid] >= half) hi = mid; else lo = mid + 1;
          }
          S.stk[sp - 1] = (lo << 16) | j_hi;  // the popped entry's place, then one more
          S.stk[sp] = (j_lo << 16) | lo;
          S.sp = sp + 1;
          if (a.prof) atomicAdd(a.prof + 6, 1ull);
        }
        continue;
      }
      }  // table
      // ---- gather the slice's keys and sort them (this reuses the table) ----
      if (tid == 0) S.dirty = 1;
      if (tid == 0 && a.prof) atomicAdd(a.prof + (direct_sort ? 7 : 5), 1ull);
      const uint32_t fh = j_hi - 1;
      const int skip = (j_lo == fh) ? cb + SB : cb + SB - (32 - __clz(j_lo ^ fh));
      SortSmem<K> &T = S.u.s;
      if (tid == 0) S.cursor = 0;
      __syncthreads();
      const bool fits = ns <= (uint32_t)SortCap<K>::value;
      if (!fits && ns > a.scratch_keys) {
        if (tid == 0) atomicOr(a.err, ERR_OVERSIZE_SCRATCH);
        __syncthreads();
        continue;
      }
      if (!fits) {
        // the global scratch area is shared by all CTAs: one user at a time
        if (tid == 0) S.overflow = acquire_lock(a.scratch_lock, a.err) ? 0 : 1;
        __syncthreads();
        if (S.overflow) continue;  // wait ran out: reported through the error word
      }
      K *dst = fits ? T.A : reinterpret_cast<K *>(a.scratch);
      for (uint32_t i = tid; i < ns; i += SC_NT) dst[i] = placed[base_cnt + i];
      if (tid == 0) T.out = start + S.run;
      __syncthreads();
      if (fits) {
        smem_sort<K>(T, ns, key_bits, skip);
        const uint32_t D = smem_runs<K>(T, ns);
        if (!in_bounds(a, 10, T.out + D, a.tmp_cap + 1)) {
          __syncthreads();
          continue;
        }
        write_runs<K>(T, D, tkeys, a.tmp_counts, T.out);
        __syncthreads();
        if (tid == 0) {
          S.run += D;
          S.tot_n += ns;
          S.tot_d += D;
        }
      } else {
        __threadfence_block();
        scratch_sort<K>(T, a, ns, skip, tkeys, a.tmp_counts);
        if (tid == 0) S.run = T.out - start;
        // release the scratch area (all threads are past their last access)
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicExch(a.scratch_lock, 0ull);
      }
      __syncthreads();
      PHASE(4)
     }
    }
    if (tid == 0) {
      a.coarse_start[g] = start;
      a.coarse_d[g] = S.run;
    }
    __syncthreads();
  }
  if (prof && tid == 0)
    for (int i = 0; i < 8; i++) atomicAdd(a.prof + 16 + i, S.ph[i]);
#undef PHASE
}

// Moves each coarse bucket's sorted runs to its final offset.
template <typename K>
__global__ void k_compact(const K *tkeys, const uint32_t *tcounts, const uint64_t *coarse_start,
                          const unsigned long long *coarse_d, const uint64_t *coarse_out,
                          const uint64_t *bucket_base, uint32_t nbins, K *out_keys,
                          uint32_t *out_counts) {
  const uint64_t nb = bucket_base[nbins];
  for (uint64_t g = blockIdx.x; g < nb; g += gridDim.x) {
    const uint64_t s = coarse_start[g], d = coarse_d[g], o = coarse_out[g];
    for (uint64_t i = threadIdx.x; i < d; i += blockDim.x) {
      out_keys[o + i] = tkeys[s + i];
      out_counts[o + i] = tcounts[s + i];
    }
  }
}

// bin_out[b] = output offset of the first coarse bucket of bin b.
__global__ void k_bin_out_offsets(const uint64_t *coarse_out, const uint64_t *bucket_base,
                                  uint32_t nbins, uint64_t *bin_out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins; b += gridDim.x * blockDim.x)
    bin_out[b] = coarse_out[bucket_base[b]];
}

template __global__ void k_coarse_hist<uint64_t>(ExpandArgs);
template __global__ void k_coarse_hist<u128>(ExpandArgs);
template __global__ void k_coarse_scatter<uint64_t>(ExpandArgs);
template __global__ void k_coarse_scatter<u128>(ExpandArgs);
template __global__ void k_coarse_count<uint64_t>(SortCountArgs);
template __global__ void k_coarse_count<u128>(SortCountArgs);
template __global__ void k_compact<uint64_t>(const uint64_t *, const uint32_t *, const uint64_t *,
                                             const unsigned long long *, const uint64_t *,
                                             const uint64_t *, uint32_t, uint64_t *, uint32_t *);
template __global__ void k_compact<u128>(const u128 *, const uint32_t *, const uint64_t *,
                                         const unsigned long long *, const uint64_t *,
                                         const uint64_t *, uint32_t, u128 *, uint32_t *);

}  // namespace gkc
