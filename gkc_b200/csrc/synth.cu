// Device generators for the synthetic workloads (same bytes as the host
// loops in synth_host.cpp and the numpy mirror gkc_b200/synth.py).
#include "common.cuh"
#include "synth_core.h"
#include "synth.h"

namespace gkc {

__global__ void k_iid_reads(uint64_t seed, uint64_t n_reads, uint32_t read_len, uint32_t n_thr,
                            char *out) {
  uint64_t total = n_reads * read_len;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = i / read_len;
    uint32_t j = (uint32_t)(i - r * read_len);
    out[i] = gkc_iid_base(seed, r, j, read_len, n_thr);
  }
}

__global__ void k_genome_iid(uint64_t seed, uint64_t G, uint8_t *g) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < G;
       i += (uint64_t)gridDim.x * blockDim.x)
    g[i] = (uint8_t)gkc_genome_iid_code(seed, i);
}

__global__ void k_genome_segments(uint64_t seed, gkc_genome_desc d, uint32_t div_thr, uint8_t *g) {
  for (uint64_t s = blockIdx.x; s < d.n_seg; s += gridDim.x) {
    uint64_t src, dst, len;
    gkc_genome_segment(seed, &d, s, &src, &dst, &len);
    for (uint64_t j = threadIdx.x; j < len; j += blockDim.x)
      g[dst + j] = (uint8_t)gkc_segment_code(seed, src + j, dst + j, div_thr);
  }
}

__global__ void k_short_reads(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t first_read,
                              uint64_t n_reads, uint32_t read_len, uint32_t err_thr, char *out) {
  uint64_t total = n_reads * read_len;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t rr = i / read_len;
    uint32_t j = (uint32_t)(i - rr * read_len);
    uint64_t r = first_read + rr;
    uint64_t pos;
    uint32_t strand;
    gkc_short_read_origin(seed, r, G, read_len, &pos, &strand);
    out[i] = gkc_short_read_base(seed, genome, pos, strand, r, j, read_len, err_thr);
  }
}

__global__ void k_long_reads(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t n_reads,
                             const uint64_t *offs, char *out) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads;
       r += (uint64_t)gridDim.x * blockDim.x)
    gkc_long_read(seed, genome, G, r, (uint32_t)(offs[r + 1] - offs[r]), out + offs[r]);
}

__global__ void k_fixed_offsets(uint64_t n_reads, uint32_t read_len, uint64_t *offs) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= n_reads;
       r += (uint64_t)gridDim.x * blockDim.x)
    offs[r] = r * read_len;
}

void synth_iid_reads_dev(uint64_t seed, uint64_t n_reads, uint32_t read_len, double n_rate,
                         char *out, uint64_t *offs, cudaStream_t st) {
  k_iid_reads<<<4096, 256, 0, st>>>(seed, n_reads, read_len, gkc_prob32(n_rate), out);
  k_fixed_offsets<<<1024, 256, 0, st>>>(n_reads, read_len, offs);
}

void synth_genome_dev(uint64_t seed, uint64_t G, double seg_fraction, double divergence,
                      uint8_t *genome, cudaStream_t st) {
  k_genome_iid<<<4096, 256, 0, st>>>(seed, G, genome);
  gkc_genome_desc d = gkc_genome_describe(G, seg_fraction);
  if (d.n_seg) k_genome_segments<<<1024, 256, 0, st>>>(seed, d, gkc_prob32(divergence), genome);
}

void synth_short_reads_dev(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t first_read,
                           uint64_t n_reads, uint32_t read_len, double err_rate, char *out,
                           uint64_t *offs, cudaStream_t st) {
  k_short_reads<<<4096, 256, 0, st>>>(seed, genome, G, first_read, n_reads, read_len,
                                      gkc_prob32(err_rate), out);
  if (offs) k_fixed_offsets<<<1024, 256, 0, st>>>(n_reads, read_len, offs);
}

void synth_long_reads_dev(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t n_reads,
                          const uint64_t *offs, char *out, cudaStream_t st) {
  k_long_reads<<<(unsigned)((n_reads + 127) / 128), 128, 0, st>>>(seed, genome, G, n_reads, offs, out);
}

}  // namespace gkc
