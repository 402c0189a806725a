// Synthetic workload generators (device launchers and host loops).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gkc {
void synth_iid_reads_dev(uint64_t seed, uint64_t n_reads, uint32_t read_len, double n_rate,
                         char *out, uint64_t *offs, cudaStream_t st);
void synth_genome_dev(uint64_t seed, uint64_t G, double seg_fraction, double divergence,
                      uint8_t *genome, cudaStream_t st);
void synth_short_reads_dev(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t first_read,
                           uint64_t n_reads, uint32_t read_len, double err_rate, char *out,
                           uint64_t *offs, cudaStream_t st);
void synth_long_reads_dev(uint64_t seed, const uint8_t *genome, uint64_t G, uint64_t n_reads,
                          const uint64_t *offs, char *out, cudaStream_t st);
}  // namespace gkc
