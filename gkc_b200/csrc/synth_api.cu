// C ABI for the synthetic workload generators.
#include <cmath>
#include <cstring>

#include "../../include/gkc/gkc.h"
#include "synth.h"
#include "synth_core.h"

using namespace gkc;

static gkc_status sync_status() {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return GKC_ERR_CUDA;
  }
  return GKC_OK;
}

gkc_status gkc_synth_iid_reads(int on_device, uint64_t seed, uint64_t n_reads, uint32_t read_len,
                               double n_rate, char *out, uint64_t *offs) {
  if (!out || !offs) return GKC_ERR_INVALID_ARG;
  if (on_device) {
    synth_iid_reads_dev(seed, n_reads, read_len, n_rate, out, offs, 0);
    return sync_status();
  }
  uint32_t thr = gkc_prob32(n_rate);
  for (uint64_t r = 0; r < n_reads; r++)
    for (uint32_t j = 0; j < read_len; j++) out[r * read_len + j] = gkc_iid_base(seed, r, j, read_len, thr);
  for (uint64_t r = 0; r <= n_reads; r++) offs[r] = r * read_len;
  return GKC_OK;
}

gkc_status gkc_synth_genome(int on_device, uint64_t seed, uint64_t genome_len, double seg_fraction,
                            double divergence, uint8_t *g) {
  if (!g) return GKC_ERR_INVALID_ARG;
  if (on_device) {
    synth_genome_dev(seed, genome_len, seg_fraction, divergence, g, 0);
    return sync_status();
  }
  for (uint64_t i = 0; i < genome_len; i++) g[i] = (uint8_t)gkc_genome_iid_code(seed, i);
  gkc_genome_desc d = gkc_genome_describe(genome_len, seg_fraction);
  uint32_t thr = gkc_prob32(divergence);
  for (uint64_t s = 0; s < d.n_seg; s++) {
    uint64_t src, dst, len;
    gkc_genome_segment(seed, &d, s, &src, &dst, &len);
    for (uint64_t j = 0; j < len; j++) g[dst + j] = (uint8_t)gkc_segment_code(seed, src + j, dst + j, thr);
  }
  return GKC_OK;
}

gkc_status gkc_synth_short_reads(int on_device, uint64_t seed, const uint8_t *g, uint64_t G,
                                 uint64_t first_read, uint64_t n_reads, uint32_t read_len,
                                 double err_rate, char *out, uint64_t *offs) {
  if (!g || !out || G < read_len) return GKC_ERR_INVALID_ARG;
  if (on_device) {
    synth_short_reads_dev(seed, g, G, first_read, n_reads, read_len, err_rate, out, offs, 0);
    return sync_status();
  }
  uint32_t thr = gkc_prob32(err_rate);
  for (uint64_t rr = 0; rr < n_reads; rr++) {
    uint64_t r = first_read + rr, pos;
    uint32_t strand;
    gkc_short_read_origin(seed, r, G, read_len, &pos, &strand);
    for (uint32_t j = 0; j < read_len; j++)
      out[rr * read_len + j] = gkc_short_read_base(seed, g, pos, strand, r, j, read_len, thr);
  }
  if (offs)
    for (uint64_t r = 0; r <= n_reads; r++) offs[r] = r * read_len;
  return GKC_OK;
}

uint64_t gkc_synth_long_read_offsets(uint64_t seed, double median, double sigma, uint32_t min_len,
                                     uint32_t max_len, uint64_t total_bases, uint64_t max_reads,
                                     uint64_t *offs) {
  // lognormal by Box-Muller on two 53-bit uniforms (host libm only)
  uint64_t n = 0, sum = 0;
  if (offs) offs[0] = 0;
  while (sum < total_bases && n < max_reads) {
    double u1 = ((gkc_rng(seed, GKC_S_LONGLEN, 2 * n) >> 11) + 1) * (1.0 / 9007199254740993.0);
    double u2 = (gkc_rng(seed, GKC_S_LONGLEN, 2 * n + 1) >> 11) * (1.0 / 9007199254740992.0);
    double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    double len = median * std::exp(sigma * z);
    uint32_t L = len < min_len ? min_len : (len > max_len ? max_len : (uint32_t)(len + 0.5));
    sum += L;
    n++;
    if (offs) offs[n] = sum;
  }
  return n;
}

gkc_status gkc_synth_long_reads(int on_device, uint64_t seed, const uint8_t *g, uint64_t G,
                                uint64_t n_reads, const uint64_t *offs, char *out) {
  if (!g || !offs || !out) return GKC_ERR_INVALID_ARG;
  if (on_device) {
    synth_long_reads_dev(seed, g, G, n_reads, offs, out, 0);
    return sync_status();
  }
  for (uint64_t r = 0; r < n_reads; r++)
    gkc_long_read(seed, g, G, r, (uint32_t)(offs[r + 1] - offs[r]), out + offs[r]);
  return GKC_OK;
}
