// Superkmer partitioning on the device.
//
// Semantics follow the reference's GPU_GenMinimizer / GPU_GenSKM /
// SKMStore::add_skms (gkc_cuda.cu:234-324, superkmers.hpp:167-186):
//   * every k-window of a read gets a canonical minimizer: the smallest
//     forward or reverse-complement p-mer that passes the filter, else 4^p-1;
//     windows touching a byte outside ACGTU follow the reference's exact
//     per-window update rule (including its 255-code smear);
//   * a superkmer is a maximal run of windows with equal minimizer value; its
//     bases are packed 2 bits per base, MSB first, N as T, byte aligned;
//   * its bin is minimizer % nbins.
// Reads shorter than k produce nothing.
//
// The fused kernel is persistent and tiled over the concatenated read bytes:
// each tile of PT_T window positions (+ halo) is loaded with 16-byte vector
// loads into shared memory, minimizers are computed with a sliding-window
// minimum over per-position filtered p-mer values, superkmer breaks are
// compacted with a block scan, and the packed bytes are written as coalesced
// 32-bit words.
#include "common.cuh"
#include "kernels.h"
#include "minimizer.cuh"

namespace gkc {

constexpr int PT_NT = 512;
constexpr int PT_T = 4096;                       // core windows per tile
constexpr int PT_H = 512;                        // halo windows to find superkmer ends
constexpr int PT_PRE = 64;                       // local index of the first core window
constexpr int PT_NLOC = PT_PRE + PT_T + PT_H + 64;  // bytes held per tile (k <= 64)
constexpr int PT_NW = PT_T + PT_H;               // windows with break flags
constexpr int PT_WORDS = PT_NLOC / 32;
constexpr int PT_PER_THREAD = PT_NW / PT_NT;     // 9 contiguous windows per thread
constexpr int PT_PT = 9;                         // positions per rolling p-mer task
constexpr int PT_STG = 6144;                     // packed bytes of a tile staged in shared memory
static_assert(PT_NW % PT_NT == 0, "windows per thread");
static_assert(PT_NLOC % 64 == 0, "tile alignment");

struct PartSmem {
  uint8_t cd[PT_NLOC];             // 2-bit code, or 255
  uint32_t badw[PT_WORDS];         // bit i: byte i is not ACGTU
  uint32_t rsw[PT_WORDS];          // bit i: a read starts at byte i
  uint32_t validw[PT_WORDS];       // bit l: window l lies inside one read
  uint32_t touchw[PT_WORDS];       // bit l: window l covers a byte that is not ACGTU
  union {
    uint32_t g[PT_NLOC];           // filtered p-mer minimum per position, then suffix minima
    uint32_t boff[PT_NLOC];        // per superkmer: byte offset in the tile
  } a;
  union {
    uint32_t pre[PT_NLOC];         // prefix minima
    uint32_t smm[PT_T + 1];        // minimizer of each core superkmer (after the window pass)
  } b;
  uint32_t pk[PT_NLOC / 16 + 1];   // the tile's bases, 2 bits each, first base in the top bits
  alignas(16) uint8_t stg[PT_STG]; // the tile's packed superkmers before they are written out (read as uint4)
  uint8_t code_tab[256];           // byte -> 2-bit code or 255
  uint16_t brk[PT_NW + 1];         // local positions of breaks, ascending
  uint16_t skm[PT_T + 1];          // break index of each core superkmer start
  uint32_t scan_tmp[64];
  uint64_t red_tmp[32];
  int ext_end;                     // local end window of an extended last superkmer
  int use_stg;                     // the tile's superkmers are packed through stg
  uint32_t n_brk, n_skm, n_bytes;
  unsigned long long base_skm, base_byte;
};

// Filtered p-mer minimum of every tile position (forward and reverse
// complement), rolling over tasks of PT_PT consecutive positions; an odd
// stride between threads keeps their shared-memory accesses in different
// banks.  The filter is fixed per instantiation so the inner loop holds no
// branch on it.
template <int FILT>
GKC_DEV void pmer_minima(PartSmem &S, int p, uint32_t M, int tid) {
  const int npos = PT_NLOC - p + 1;
  const int ntask = (npos + PT_PT - 1) / PT_PT;
  for (int task = tid; task < ntask; task += PT_NT) {
    int a0 = task * PT_PT;
    uint32_t f = 0, r = 0;
    for (int j = 0; j < p - 1; j++) {
      uint32_t c = S.cd[a0 + j] & 3u;
      f = (f << 2) | c;
      r = (r >> 2) | ((3u - c) << (2 * p - 2));
    }
    int e = min(a0 + PT_PT, npos);
    for (int i = a0; i < e; i++) {
      uint32_t c = S.cd[i + p - 1] & 3u;
      f = ((f << 2) | c) & M;
      r = (r >> 2) | ((3u - c) << (2 * p - 2));
      uint32_t vf = mm_filter(f, p, FILT) ? f : M;
      uint32_t vr = mm_filter(r, p, FILT) ? r : M;
      S.a.g[i] = vf < vr ? vf : vr;
    }
  }
}

GKC_DEV bool bit_at(const uint32_t *w, int i) { return (w[i >> 5] >> (i & 31)) & 1u; }

// Any bit set in [a, b] (inclusive), b - a < 96.
GKC_DEV bool any_bits(const uint32_t *w, int a, int b) {
  if (a > b) return false;
  int wa = a >> 5, wb = b >> 5;
  if (wa == wb) {
    uint32_t m = (0xFFFFFFFFu >> (31 - (b & 31))) & (0xFFFFFFFFu << (a & 31));
    return (w[wa] & m) != 0u;
  }
  if (w[wa] & (0xFFFFFFFFu << (a & 31))) return true;
  for (int x = wa + 1; x < wb; x++)
    if (w[x]) return true;
  return (w[wb] & (0xFFFFFFFFu >> (31 - (b & 31)))) != 0u;
}

// Bit i (0..31) of the result = OR of bits i .. i+n-1 of the 96-bit value
// (x2:x1:x0), for 1 <= n <= 64: a sliding OR built by doubling shifts.
GKC_DEV uint32_t span_or(uint32_t x0, uint32_t x1, uint32_t x2, int n) {
  uint64_t lo = (uint64_t)x0 | ((uint64_t)x1 << 32);
  uint64_t hi = x2;
  int m = 1;
  while (2 * m <= n) {  // lo:hi now holds the OR over m consecutive bits
    lo |= (lo >> m) | (hi << (64 - m));
    hi |= hi >> m;
    m *= 2;
  }
  const int r = n - m;  // 0 <= r < m: cover the remaining bits with an overlapping shift
  if (r > 0) lo |= (lo >> r) | (hi << (64 - r));
  return (uint32_t)lo;
}

__global__ void __launch_bounds__(PT_NT, 3) k_partition(PartArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  PartSmem &S = *reinterpret_cast<PartSmem *>(smem_raw);
  const int tid = threadIdx.x;
  const int k = a.k, p = a.p, omega = a.k - a.p + 1;
  const uint32_t M = 0xFFFFFFFFu >> (32 - 2 * p);
  if (a.nbytes_dev) a.nbytes = *a.nbytes_dev;
  const uint64_t n_tiles = (a.nbytes + PT_T - 1) / PT_T;

  // per-CTA bin histograms (small bin counts only)
  unsigned long long *h_km = reinterpret_cast<unsigned long long *>(smem_raw + sizeof(PartSmem));
  uint32_t *h_skm = reinterpret_cast<uint32_t *>(h_km + a.nbins_smem);
  for (int i = tid; i < a.nbins_smem; i += PT_NT) {
    h_skm[i] = 0;
    h_km[i] = 0;
  }
  for (int i = tid; i < 256; i += PT_NT) S.code_tab[i] = (uint8_t)code_of_byte((uint32_t)i);
  __syncthreads();

  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t ts = (int64_t)tile * PT_T;
    const int64_t G0 = ts - PT_PRE;  // global position of local 0 (64-aligned)

    // ---- load bytes -> codes (16 per thread, one 16-byte store), bad-code
    //      bitmap (lane pairs combine their 16-bit halves), read-start bitmap ----
    static_assert(PT_NLOC % 16 == 0 && PT_NLOC / 16 <= PT_NT, "one 16-byte group per thread");
    if ((tid & ~31) * 16 < PT_NLOC) {  // warps with at least one group
      const int q = tid * 16;
      const bool act = q < PT_NLOC;
      uint32_t cw[4] = {0u, 0u, 0u, 0u};
      uint32_t bad16 = 0, pkw = 0;
      if (act) {
        const int64_t g = G0 + q;
        const bool fast = g >= 0 && (uint64_t)(g + 16) <= a.nbytes && a.aligned16;
        if (fast) {
          const uint4 v = __ldg(reinterpret_cast<const uint4 *>(a.reads + g));
          const uint32_t vw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const uint32_t c = S.code_tab[(vw[t >> 2] >> (8 * (t & 3))) & 0xFFu];
            cw[t >> 2] |= c << (8 * (t & 3));
            bad16 |= (c >> 7) << t;
            pkw |= (c & 3u) << (30 - 2 * t);
          }
        } else {
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const uint32_t c = global_code(a.reads, a.nbytes, g + t);
            cw[t >> 2] |= c << (8 * (t & 3));
            bad16 |= (c >> 7) << t;
            pkw |= (c & 3u) << (30 - 2 * t);
          }
        }
        *reinterpret_cast<uint4 *>(S.cd + q) = make_uint4(cw[0], cw[1], cw[2], cw[3]);
        S.pk[q >> 4] = pkw;
      }
      const uint32_t other = __shfl_xor_sync(0xffffffffu, bad16, 1);
      if (act && (tid & 1) == 0) S.badw[q >> 5] = bad16 | (other << 16);
    }
    for (int w = tid; w < PT_WORDS; w += PT_NT) {
      int64_t gw = (G0 >> 5) + w;  // G0 is a multiple of 64
      S.rsw[w] = (gw >= 0 && (uint64_t)gw < a.rs_words) ? a.rs_bits[gw] : 0u;
      S.validw[w] = 0u;
    }
    if (tid == 0) S.pk[PT_NLOC / 16] = 0u;
    __syncthreads();
    // Windows are valid when no read starts inside them (after their first
    // byte) and they lie inside the data; they touch a bad byte when one of
    // their k bytes is not ACGTU.  32 windows per word, by sliding ORs.
    for (int w = tid; w < PT_WORDS; w += PT_NT) {
      const uint32_t r0 = S.rsw[w], r1 = w + 1 < PT_WORDS ? S.rsw[w + 1] : 0u,
                     r2 = w + 2 < PT_WORDS ? S.rsw[w + 2] : 0u;
      // read starts at window bytes 1 .. k-1: shift the span right by one
      const uint32_t hit = k > 1 ? span_or((r0 >> 1) | (r1 << 31), (r1 >> 1) | (r2 << 31), r2 >> 1, k - 1) : 0u;
      const uint32_t b0 = S.badw[w], b1 = w + 1 < PT_WORDS ? S.badw[w + 1] : 0u,
                     b2 = w + 2 < PT_WORDS ? S.badw[w + 2] : 0u;
      S.touchw[w] = span_or(b0, b1, b2, k);
      // windows inside the data: G0 + l >= 0 and G0 + l + k <= nbytes
      const int64_t s0 = G0 + 32 * (int64_t)w;
      const int64_t ilo = s0 < 0 ? -s0 : 0;
      const int64_t ihi = (int64_t)a.nbytes - k - s0;
      uint32_t range = 0u;
      if (ihi >= 0 && ilo <= 31) {
        const int lo_i = (int)ilo, hi_i = (int)(ihi > 31 ? 31 : ihi);
        if (hi_i >= lo_i) range = (0xFFFFFFFFu >> (31 - hi_i)) & (0xFFFFFFFFu << lo_i);
      }
      S.validw[w] = ~hit & range;
    }

    // ---- filtered p-mer minimum per position ----
    switch (a.filter) {
      case FILTER_ALL: pmer_minima<FILTER_ALL>(S, p, M, tid); break;
      case FILTER_NEW: pmer_minima<FILTER_NEW>(S, p, M, tid); break;
      case FILTER_SIGNATURE: pmer_minima<FILTER_SIGNATURE>(S, p, M, tid); break;
      default: pmer_minima<FILTER_NEW2>(S, p, M, tid); break;
    }
    __syncthreads();

    // ---- van Herk / Gil-Werman: prefix and suffix minima in blocks of omega ----
    {
      const int npos = PT_NLOC - p + 1;
      const int nblk = (npos + omega - 1) / omega;
      for (int blk = tid; blk < nblk; blk += PT_NT) {
        int b0 = blk * omega, b1 = min(b0 + omega, npos);
        uint32_t m = 0xFFFFFFFFu;
        for (int i = b0; i < b1; i++) {
          m = min(m, S.a.g[i]);
          S.b.pre[i] = m;
        }
        m = 0xFFFFFFFFu;
        for (int i = b1 - 1; i >= b0; i--) {
          m = min(m, S.a.g[i]);
          S.a.g[i] = m;  // suffix minima in place
        }
      }
    }
    __syncthreads();

    // ---- window minimizers and breaks, thread-contiguous: windows
    //      [lw0 - 1, lw0 + 9), the first only for the comparison ----
    uint32_t nb_local = 0, ns_local = 0;
    uint32_t brkbits = 0, startbits = 0;
    const int lw0 = PT_PRE + tid * PT_PER_THREAD;
    uint32_t mmv[PT_PER_THREAD + 1];
    uint32_t vbits, tbits, rbits;  // bit j: window lw0 - 1 + j
    {
      const int l0 = lw0 - 1, w0 = l0 >> 5, sh = l0 & 31;
      auto bits10 = [&](const uint32_t *arr) -> uint32_t {
        const uint64_t v = (uint64_t)arr[w0] | ((uint64_t)(w0 + 1 < PT_WORDS ? arr[w0 + 1] : 0u) << 32);
        return (uint32_t)(v >> sh) & 0x3FFu;
      };
      vbits = bits10(S.validw);
      tbits = bits10(S.touchw);
      rbits = bits10(S.rsw);
#pragma unroll
      for (int j = 0; j <= PT_PER_THREAD; j++) {
        const int l = l0 + j;
        mmv[j] = 0xFFFFFFFFu;
        if ((vbits >> j) & 1u) {
          if (!((tbits >> j) & 1u)) {
            mmv[j] = min(S.a.g[l], S.b.pre[l + omega - 1]);
          } else {
            const uint8_t *cw = S.cd + l;
            mmv[j] = exact_window_minimizer([&](int i) { return (uint32_t)cw[i]; }, k, p, a.filter);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < PT_PER_THREAD; j++) {
      const int l = lw0 + j;
      const bool valid = (vbits >> (j + 1)) & 1u;
      const bool start = valid && (((rbits >> (j + 1)) & 1u) || mmv[j + 1] != mmv[j] || !((vbits >> j) & 1u));
      const bool brk = !valid || start;
      brkbits |= (brk ? 1u : 0u) << j;
      const bool core_start = start && l < PT_PRE + PT_T;
      startbits |= (core_start ? 1u : 0u) << j;
      nb_local += brk;
      ns_local += core_start;
    }
    uint32_t tot;
    uint32_t excl = block_exclusive_scan<PT_NT>(nb_local | (ns_local << 16), S.scan_tmp, &tot);
    {
      uint32_t bi = excl & 0xFFFFu, si = excl >> 16;
#pragma unroll
      for (int j = 0; j < PT_PER_THREAD; j++) {
        if ((brkbits >> j) & 1u) {
          if ((startbits >> j) & 1u) {
            S.b.smm[si] = mmv[j + 1];  // pre[] is no longer read: the scan above ended with a barrier
            S.skm[si++] = (uint16_t)bi;
          }
          S.brk[bi++] = (uint16_t)(lw0 + j);
        }
      }
    }
    if (tid == 0) {
      S.n_brk = tot & 0xFFFFu;
      S.n_skm = tot >> 16;
      S.ext_end = -1;
    }
    __syncthreads();
    const uint32_t n_brk = S.n_brk, n_skm = S.n_skm;

    // ---- the last core superkmer may run past the halo: extend it ----
    if (n_skm > 0 && tid == 0) {
      uint32_t jlast = S.skm[n_skm - 1];
      if (jlast + 1 >= n_brk) {
        uint32_t mv = S.b.smm[n_skm - 1];
        uint64_t w = (uint64_t)(G0 + PT_PRE + PT_NW);
        // walk windows beyond the halo with the exact rule until a break
        while (w < a.nbytes) {
          if (global_rs(a.rs_bits, w) || !global_window_valid(a.rs_bits, a.nbytes, w, k)) break;
          uint32_t v = exact_window_minimizer(
              [&](int i) { return global_code(a.reads, a.nbytes, (int64_t)w + i); }, k, p, a.filter);
          if (v != mv) break;
          w++;
        }
        S.ext_end = (int)((int64_t)w - G0);
      }
    }
    __syncthreads();

    // ---- superkmer sizes -> byte offsets (contiguous chunks of 8 per thread) ----
    uint32_t my_bytes = 0;
    const int sk0 = tid * 8;
    for (int i = sk0; i < sk0 + 8 && i < (int)n_skm; i++) {
      uint32_t j = S.skm[i];
      int l = S.brk[j];
      int e = (j + 1 < n_brk) ? S.brk[j + 1] : S.ext_end;
      uint32_t len = (uint32_t)(e - l) + k - 1;
      my_bytes += (len + 3) / 4;
    }
    uint32_t tile_bytes;
    uint32_t boff = block_exclusive_scan<PT_NT>(my_bytes, S.scan_tmp, &tile_bytes);
    // S.a.g is no longer needed: reuse it for per-superkmer byte offsets
    for (int i = sk0; i < sk0 + 8 && i < (int)n_skm; i++) {
      uint32_t j = S.skm[i];
      int l = S.brk[j];
      int e = (j + 1 < n_brk) ? S.brk[j + 1] : S.ext_end;
      uint32_t len = (uint32_t)(e - l) + k - 1;
      S.a.boff[i] = boff;
      boff += (len + 3) / 4;
    }
    if (tid == 0) {
      S.n_bytes = tile_bytes;
      uint32_t rounded = (tile_bytes + 15u) & ~15u;
      // the staged packing needs every superkmer's bases in the tile's data
      S.use_stg = rounded <= (uint32_t)PT_STG && (S.ext_end < 0 || S.ext_end + k - 1 <= PT_NLOC);
      S.base_skm = n_skm ? atomicAdd(a.cursors + 0, (unsigned long long)n_skm) : 0ull;
      S.base_byte = rounded ? atomicAdd(a.cursors + 1, (unsigned long long)rounded) : 0ull;
      if (S.base_skm + n_skm > a.cap_skm || S.base_byte + rounded > a.cap_bytes)
        atomicOr(a.err, ERR_CAPACITY);
    }
    __syncthreads();
    const unsigned long long base_skm = S.base_skm, base_byte = S.base_byte;
    const bool fits = base_skm + n_skm <= a.cap_skm && base_byte + ((tile_bytes + 15u) & ~15u) <= a.cap_bytes;

    // ---- descriptors, bin histograms ----
    for (int i = tid; i < (int)n_skm; i += PT_NT) {
      uint32_t j = S.skm[i];
      int l = S.brk[j];
      int e = (j + 1 < n_brk) ? S.brk[j + 1] : S.ext_end;
      uint32_t nk = (uint32_t)(e - l);
      uint32_t len = nk + k - 1;
      uint32_t mv = S.b.smm[i];
      uint32_t bin = mv % (uint32_t)a.nbins;
      if (len > 0xFFFFFFu) atomicOr(a.err, ERR_BAD_READ);
      if (fits && len <= 0xFFFFFFu) {
        uint64_t off = base_byte + S.a.boff[i];
        a.skm_desc[base_skm + i] = (off << 24) | (uint64_t)len;
        a.skm_mm[base_skm + i] = mv;
        if (a.skm_gpos) a.skm_gpos[base_skm + i] = (uint64_t)(G0 + l);
      }
      if (bin < (uint32_t)a.nbins_smem) {
        atomicAdd(&h_skm[bin], 1u);
        atomicAdd(&h_km[bin], (unsigned long long)nk);
      } else {
        atomicAdd(&a.bin_nskm[bin], 1ull);
        atomicAdd(&a.bin_nkmers[bin], (unsigned long long)nk);
      }
    }

    // ---- packed bytes: each superkmer's bases cut from the tile's 2-bit
    //      stream into the staging area, then written out in 16-byte pieces ----
    if (fits && S.use_stg) {
      for (int i = tid; i < (int)n_skm; i += PT_NT) {
        const uint32_t j = S.skm[i];
        const int l = S.brk[j];
        const int e = (j + 1 < n_brk) ? S.brk[j + 1] : S.ext_end;
        const uint32_t len = (uint32_t)(e - l) + k - 1, nb = (len + 3) / 4;
        uint8_t *dst = S.stg + S.a.boff[i];
        for (uint32_t m = 0; 16 * m < len; m++) {
          const uint32_t B = (uint32_t)l + 16 * m, w = B >> 4, sh = 2 * (B & 15u);
          uint32_t v = sh ? (S.pk[w] << sh) | (S.pk[w + 1] >> (32 - sh)) : S.pk[w];
          const uint32_t rem = len - 16 * m;
          if (rem < 16) v &= 0xFFFFFFFFu << (32 - 2 * rem);  // zero padding after the last base
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (4 * m + u < nb) dst[4 * m + u] = (uint8_t)(v >> (24 - 8 * u));
        }
      }
      if (tid < 16 && tile_bytes + tid < ((tile_bytes + 15u) & ~15u)) S.stg[tile_bytes + tid] = 0;
      __syncthreads();
      const uint32_t n16 = (tile_bytes + 15u) / 16u;
      uint4 *dst16 = reinterpret_cast<uint4 *>(a.packed + base_byte);
      const uint4 *src16 = reinterpret_cast<const uint4 *>(S.stg);
      for (uint32_t v = tid; v < n16; v += PT_NT) dst16[v] = src16[v];
    } else if (fits) {
      const uint32_t nwords = (tile_bytes + 3) / 4;
      uint32_t *dst = reinterpret_cast<uint32_t *>(a.packed + base_byte);
      for (uint32_t w = tid; w < nwords; w += PT_NT) {
        uint32_t word = 0;
        // superkmer holding the word's first byte: last i with boff[i] <= 4w
        int lo = 0;
        {
          int hi = (int)n_skm - 1;
          while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (S.a.boff[mid] <= w * 4) lo = mid; else hi = mid - 1;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          uint32_t q = w * 4 + u;
          if (q >= tile_bytes) break;
          while (lo + 1 < (int)n_skm && S.a.boff[lo + 1] <= q) lo++;
          uint32_t j = S.skm[lo];
          int l = S.brk[j];
          int e = (j + 1 < n_brk) ? S.brk[j + 1] : S.ext_end;
          uint32_t len = (uint32_t)(e - l) + k - 1;
          uint32_t bb = q - S.a.boff[lo];
          uint32_t byte = 0;
#pragma unroll
          for (int t = 0; t < 4; t++) {
            uint32_t bi = bb * 4 + t;
            uint32_t c = 0;
            if (bi < len) {
              int lp = l + (int)bi;
              c = (lp < PT_NLOC) ? (S.cd[lp] & 3u) : (global_code(a.reads, a.nbytes, G0 + lp) & 3u);
            }
            byte = (byte << 2) | c;
          }
          word |= byte << (8 * u);
        }
        dst[w] = word;
      }
    }
    __syncthreads();
  }

  // flush bin histograms
  for (int i = tid; i < a.nbins_smem; i += PT_NT) {
    if (h_skm[i]) atomicAdd(&a.bin_nskm[i], (unsigned long long)h_skm[i]);
    if (h_km[i]) atomicAdd(&a.bin_nkmers[i], h_km[i]);
  }
}

size_t partition_smem_bytes(int nbins_smem) {
  return sizeof(PartSmem) + (size_t)nbins_smem * (sizeof(uint32_t) + sizeof(unsigned long long)) + 16;
}

// Read-start bitmap: bit offs[r]-offs[0] for every read, plus bit nbytes as
// the end-of-data sentinel.
__global__ void k_read_start_bits(const uint64_t *offs, uint64_t n_reads, uint32_t *bits) {
  uint64_t base = offs[0];
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= n_reads;
       r += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t pos = offs[r] - base;
    atomicOr(&bits[pos >> 5], 1u << (pos & 31));
  }
}

// Counting sort of superkmer descriptors by bin, with warp-aggregated atomics
// on the per-bin fill counters.
__global__ void k_bin_scatter(const unsigned long long *n_skm_ptr, const uint64_t *desc,
                              const uint32_t *mm, uint32_t nbins, const uint64_t *bin_start,
                              unsigned long long *bin_fill, uint64_t *out_desc, uint32_t *out_mm,
                              const uint64_t *gpos, uint64_t *out_gpos, const uint32_t *err) {
  if (*err & (ERR_CAPACITY | ERR_BAD_READ)) return;  // outputs incomplete: the host re-runs
  const uint64_t n = *n_skm_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x; i0 < n; i0 += stride) {
    uint64_t i = i0 + threadIdx.x;
    bool act = i < n;
    uint32_t active = __ballot_sync(0xffffffffu, act);
    if (!act) continue;
    uint32_t m = mm[i];
    uint32_t b = m % nbins;
    uint32_t peers = __match_any_sync(active, b);
    int leader = __ffs(peers) - 1;
    uint32_t rank = __popc(peers & ((1u << lane_id()) - 1u));
    unsigned long long base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(&bin_fill[b], (unsigned long long)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    uint64_t slot = bin_start[b] + base + rank;
    out_desc[slot] = desc[i];
    out_mm[slot] = m;
    if (gpos) out_gpos[slot] = gpos[i];
  }
}

// Bin placement without global atomics, for nbins <= kBinPlaceMaxBins.
// k_bin_count: superkmers per (bin, chunk of kBinChunk superkmers), stored
// bin-major (mat[b * nch_cap + c]) so that one exclusive scan gives every
// (bin, chunk) its first slot in bin order; k_bin_place then moves each
// chunk's superkmers with shared-memory cursors per bin.
__global__ void k_bin_count(const unsigned long long *n_skm_ptr, const uint32_t *mm, uint32_t nbins,
                            uint64_t nch_cap, unsigned long long *mat, const uint32_t *err) {
  extern __shared__ uint32_t hcnt[];
  if (*err & (ERR_CAPACITY | ERR_BAD_READ)) return;
  const uint64_t n = *n_skm_ptr;
  for (uint64_t c = blockIdx.x; c < nch_cap; c += gridDim.x) {
    for (uint32_t b = threadIdx.x; b < nbins; b += blockDim.x) hcnt[b] = 0;
    __syncthreads();
    const uint64_t i1 = min(n, (c + 1) * (uint64_t)kBinChunk);
    for (uint64_t i = c * (uint64_t)kBinChunk + threadIdx.x; i < i1; i += blockDim.x)
      atomicAdd(&hcnt[mm[i] % nbins], 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nbins; b += blockDim.x) mat[(uint64_t)b * nch_cap + c] = hcnt[b];
    __syncthreads();
  }
}

// Each chunk is placed in sub-rounds of kBinRound superkmers: counted per
// bin in shared memory, grouped by bin there, then written out so that each
// bin's superkmers leave as a run of consecutive slots.
__global__ void __launch_bounds__(kBinPlaceThreads, 2) k_bin_place(const unsigned long long *n_skm_ptr,
                                                                const uint64_t *desc, const uint32_t *mm,
                                                                uint32_t nbins, uint64_t nch_cap,
                                                                const uint64_t *off, uint64_t *out_desc,
                                                                uint32_t *out_mm, const uint32_t *err) {
  extern __shared__ __align__(16) uint8_t bp_raw[];
  uint64_t *st_desc = reinterpret_cast<uint64_t *>(bp_raw);               // kBinRound
  uint32_t *st_mm = reinterpret_cast<uint32_t *>(st_desc + kBinRound);   // kBinRound
  uint64_t *cur = reinterpret_cast<uint64_t *>(st_mm + kBinRound);       // nbins: next global slot
  uint32_t *cnt = reinterpret_cast<uint32_t *>(cur + nbins);             // nbins: counts, then cursors
  uint32_t *lst = cnt + nbins;                                            // nbins: starts in the round
  __shared__ uint32_t tmp[64];
  if (*err & (ERR_CAPACITY | ERR_BAD_READ)) return;
  const uint64_t n = *n_skm_ptr;
  const uint64_t nch = min(nch_cap, (n + kBinChunk - 1) / kBinChunk);
  const int tid = threadIdx.x;
  for (uint64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    for (uint32_t b = tid; b < nbins; b += kBinPlaceThreads) cur[b] = off[(uint64_t)b * nch_cap + c];
    const uint64_t c1 = min(n, (c + 1) * (uint64_t)kBinChunk);
    for (uint64_t r0 = c * (uint64_t)kBinChunk; r0 < c1; r0 += kBinRound) {
      const uint32_t m = (uint32_t)min((uint64_t)kBinRound, c1 - r0);
      for (uint32_t b = tid; b < nbins; b += kBinPlaceThreads) cnt[b] = 0;
      __syncthreads();
      constexpr int PER = kBinRound / kBinPlaceThreads;
      uint64_t dv[PER];
      uint32_t mv[PER], rk[PER];
#pragma unroll
      for (int u = 0; u < PER; u++) {
        const uint32_t i = u * kBinPlaceThreads + tid;
        if (i < m) {
          dv[u] = desc[r0 + i];
          mv[u] = mm[r0 + i];
          rk[u] = atomicAdd(&cnt[mv[u] % nbins], 1u);
        }
      }
      __syncthreads();
      // exclusive scan of the bin counts (thread-contiguous groups)
      {
        const uint32_t per = (nbins + kBinPlaceThreads - 1) / kBinPlaceThreads, b0 = tid * per;
        uint32_t s = 0;
        for (uint32_t b = b0; b < b0 + per && b < nbins; b++) s += cnt[b];
        uint32_t tot;
        uint32_t run = block_exclusive_scan<kBinPlaceThreads>(s, tmp, &tot);
        for (uint32_t b = b0; b < b0 + per && b < nbins; b++) {
          lst[b] = run;
          run += cnt[b];
        }
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < PER; u++) {
        const uint32_t i = u * kBinPlaceThreads + tid;
        if (i < m) {
          const uint32_t p = lst[mv[u] % nbins] + rk[u];
          st_desc[p] = dv[u];
          st_mm[p] = mv[u];
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < m; i += kBinPlaceThreads) {
        const uint32_t v = st_mm[i], b = v % nbins;
        const uint64_t slot = cur[b] + (i - lst[b]);
        out_desc[slot] = st_desc[i];
        out_mm[slot] = v;
      }
      __syncthreads();
      for (uint32_t b = tid; b < nbins; b += kBinPlaceThreads) cur[b] += cnt[b];
      __syncthreads();
    }
  }
}

size_t bin_place_smem_bytes(uint32_t nbins) {
  return (size_t)kBinRound * 12 + (size_t)nbins * 16;
}

// Exclusive scans of the per-bin counters (one thread; nbins is small).
__global__ void k_bin_prefix(const unsigned long long *bin_nskm, const unsigned long long *bin_nkmers,
                             uint32_t nbins, uint64_t *bin_start, uint64_t *bin_kstart) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t cs = 0, ck = 0;
  for (uint32_t b = 0; b < nbins; b++) {
    bin_start[b] = cs;
    bin_kstart[b] = ck;
    cs += bin_nskm[b];
    ck += bin_nkmers[b];
  }
  bin_start[nbins] = cs;
  bin_kstart[nbins] = ck;
}

}  // namespace gkc
