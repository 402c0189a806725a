// Seeded synthetic read generators, shared by host loops and device kernels.
//
// Every base is a pure function of (seed, stream, index) through a counter-based
// splitmix64 mix, so a host loop and a CUDA kernel produce byte-identical reads
// in any order.  The workloads follow the shapes of the benchmark configs:
//   * i.i.d. short reads with a per-base N rate;
//   * a random genome with 1-5 kbp segment copies (1% divergence) placed at
//     other loci, sampled as fixed-length reads on both strands with i.i.d.
//     substitution errors;
//   * long reads (lengths supplied by the host) with substitutions and
//     homopolymer-biased insertions / deletions.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GKC_HD __host__ __device__ __forceinline__
#else
#define GKC_HD static inline
#endif

enum {
  GKC_S_IID = 1,
  GKC_S_GENOME = 2,
  GKC_S_SEG = 3,
  GKC_S_SEGMUT = 4,
  GKC_S_READPOS = 5,
  GKC_S_READERR = 6,
  GKC_S_LONGLEN = 7,
  GKC_S_LONGPOS = 8,
  GKC_S_LONGERR = 9,
};

// splitmix64 output function (Steele, Lea & Flood, OOPSLA 2014).
GKC_HD uint64_t gkc_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

GKC_HD uint64_t gkc_rng(uint64_t seed, uint64_t stream, uint64_t idx) {
  uint64_t base = gkc_mix64(seed * 0x9E3779B97F4A7C15ULL + stream);
  return gkc_mix64(base + idx * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL);
}

GKC_HD char gkc_code_char(uint32_t c) { return "ACGT"[c & 3]; }

// Probability p as a 32-bit threshold on the top half of a 64-bit draw.
GKC_HD uint32_t gkc_prob32(double p) {
  double t = p * 4294967296.0;
  return t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
}

// ---- config 1: i.i.d. uniform ACGT, each base N with probability n_thr/2^32 ----
GKC_HD char gkc_iid_base(uint64_t seed, uint64_t read, uint32_t pos, uint32_t read_len,
                         uint32_t n_thr) {
  uint64_t h = gkc_rng(seed, GKC_S_IID, read * (uint64_t)read_len + pos);
  if ((uint32_t)(h >> 32) < n_thr) return 'N';
  return gkc_code_char((uint32_t)h);
}

// ---- genome with segment copies ----
// Segment s of n_seg copies bases [src, src+len) of the i.i.d. genome to
// [dst, dst+len); destinations lie in disjoint slots of length G/n_seg, so the
// copies never overlap and can be applied in parallel.
typedef struct {
  uint64_t genome_len;
  uint64_t n_seg;
  uint64_t slot;
} gkc_genome_desc;

GKC_HD gkc_genome_desc gkc_genome_describe(uint64_t genome_len, double seg_fraction) {
  gkc_genome_desc d;
  d.genome_len = genome_len;
  uint64_t n = (uint64_t)(seg_fraction * (double)genome_len / 3000.0 + 0.5);
  d.n_seg = (genome_len >= 4096 && n > 0) ? n : 0;
  d.slot = d.n_seg ? genome_len / d.n_seg : 0;
  return d;
}

GKC_HD uint32_t gkc_genome_iid_code(uint64_t seed, uint64_t i) {
  return (uint32_t)gkc_rng(seed, GKC_S_GENOME, i) & 3u;
}

GKC_HD void gkc_genome_segment(uint64_t seed, const gkc_genome_desc* d, uint64_t s,
                               uint64_t* src, uint64_t* dst, uint64_t* len) {
  uint64_t l = 1000 + gkc_rng(seed, GKC_S_SEG, 3 * s) % 4001;
  if (l + 1 >= d->slot) l = d->slot / 2;
  uint64_t room = d->slot - l;
  *dst = s * d->slot + gkc_rng(seed, GKC_S_SEG, 3 * s + 1) % room;
  *src = gkc_rng(seed, GKC_S_SEG, 3 * s + 2) % (d->genome_len - l);
  *len = l;
}

// Base code of a copied segment position (1% substitution divergence).
GKC_HD uint32_t gkc_segment_code(uint64_t seed, uint64_t src_pos, uint64_t dst_pos,
                                 uint32_t div_thr) {
  uint32_t b = gkc_genome_iid_code(seed, src_pos);
  uint64_t h = gkc_rng(seed, GKC_S_SEGMUT, dst_pos);
  if ((uint32_t)(h >> 32) < div_thr) b = (b + 1 + (uint32_t)((h & 0xFFFF) % 3)) & 3u;
  return b;
}

// ---- fixed-length reads sampled on both strands with substitution errors ----
GKC_HD void gkc_short_read_origin(uint64_t seed, uint64_t read, uint64_t genome_len,
                                  uint32_t read_len, uint64_t* pos, uint32_t* strand) {
  *pos = gkc_rng(seed, GKC_S_READPOS, 2 * read) % (genome_len - read_len + 1);
  *strand = (uint32_t)gkc_rng(seed, GKC_S_READPOS, 2 * read + 1) & 1u;
}

GKC_HD char gkc_short_read_base(uint64_t seed, const uint8_t* genome, uint64_t pos,
                                uint32_t strand, uint64_t read, uint32_t j,
                                uint32_t read_len, uint32_t err_thr) {
  uint32_t g = strand ? 3u - genome[pos + read_len - 1 - j] : genome[pos + j];
  uint64_t e = gkc_rng(seed, GKC_S_READERR, read * (uint64_t)read_len + j);
  if ((uint32_t)(e >> 32) < err_thr) g = (g + 1 + (uint32_t)((e & 0xFFFF) % 3)) & 3u;
  return gkc_code_char(g);
}

// ---- long reads with homopolymer-biased indels ----
// Error model per emitted step: substitution 2%; insertion and deletion 1%
// each outside homopolymer runs and 3% each inside them (overall about 5%,
// split roughly 40/30/30).  The walk wraps around the genome ends.
typedef struct {
  uint32_t t_sub, t_ins_lo, t_ins_hi, t_del_lo, t_del_hi;  // thresholds on 24-bit draws
} gkc_longerr;

GKC_HD gkc_longerr gkc_longerr_default(void) {
  gkc_longerr e;
  e.t_sub = (uint32_t)(0.02 * 16777216.0);
  e.t_ins_lo = (uint32_t)(0.01 * 16777216.0);
  e.t_ins_hi = (uint32_t)(0.03 * 16777216.0);
  e.t_del_lo = e.t_ins_lo;
  e.t_del_hi = e.t_ins_hi;
  return e;
}

GKC_HD uint32_t gkc_genome_at(const uint8_t* genome, uint64_t G, int64_t g) {
  int64_t m = g % (int64_t)G;
  if (m < 0) m += (int64_t)G;
  return genome[m];
}

GKC_HD void gkc_long_read(uint64_t seed, const uint8_t* genome, uint64_t G, uint64_t read,
                          uint32_t len, char* out) {
  gkc_longerr e = gkc_longerr_default();
  uint64_t h0 = gkc_rng(seed, GKC_S_LONGPOS, read);
  int64_t g = (int64_t)(h0 % G);
  int strand = (int)((h0 >> 63) & 1);
  int64_t dir = strand ? -1 : 1;
  uint64_t step = 0;
  uint32_t o = 0;
  uint64_t rstream = GKC_S_LONGERR + (read << 8);
  while (o < len) {
    uint64_t h = gkc_rng(seed, rstream, step++);
    uint32_t b = gkc_genome_at(genome, G, g);
    uint32_t prev = gkc_genome_at(genome, G, g - dir);
    int hp = (b == prev);
    uint32_t u = (uint32_t)(h >> 40);
    uint32_t t_ins = hp ? e.t_ins_hi : e.t_ins_lo;
    uint32_t t_del = hp ? e.t_del_hi : e.t_del_lo;
    uint32_t bc = strand ? 3u - b : b;
    if (u < e.t_sub) {
      out[o++] = gkc_code_char((bc + 1 + (uint32_t)((h & 0xFFFF) % 3)) & 3u);
      g += dir;
    } else if (u < e.t_sub + t_ins) {
      out[o++] = gkc_code_char((uint32_t)(h >> 16));
    } else if (u < e.t_sub + t_ins + t_del) {
      g += dir;
    } else {
      out[o++] = gkc_code_char(bc);
      g += dir;
    }
  }
}
