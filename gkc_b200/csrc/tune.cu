// Launch-shape tuner for the batched pipeline.
//
// The reference fixes its launch shape by hand (NUM_BLOCKS_PER_GRID x
// NUM_THREADS_PER_BLOCK and the stream count, experiment.cpp:234-238).  Here
// the shapes of the count stage that do not need a rebuild are chosen per
// device and workload class by measurement: the mean keys per count bucket
// (the coarse digit width follows from it), the k-mers per histogram chunk,
// and the count kernel's CTAs per SM.  A search times the count stages of the
// graph-captured pipeline on a sample of the caller's reads for each
// candidate, one dimension at a time from the defaults, and keeps the
// fastest.  The sample runs with its bin count scaled down so that its bins
// hold as many bases as the full run's (digit counts, bucket sizes and the
// scatter's working set follow the bin size).  Choices are cached per (SM
// count, key width, read-length class, bin count, bin-size class: bases per
// bin in factors of 4) for the process and can be saved to and loaded from a
// file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/gkc/gkc.h"
#include "common.cuh"
#include "ctx.h"
#include "kernels.h"

namespace {

struct TuneKey {
  int sms, key_words, long_reads, nbins, bin_class;
  bool operator<(const TuneKey &o) const {
    return std::tie(sms, key_words, long_reads, nbins, bin_class) <
           std::tie(o.sms, o.key_words, o.long_reads, o.nbins, o.bin_class);
  }
};

std::mutex g_mu;
std::map<TuneKey, gkc_tune_params> g_cache;

TuneKey key_for(int sms, const gkc_params *prm, uint64_t n_bases, uint64_t n_reads) {
  const uint64_t mean = n_reads ? n_bases / n_reads : 0;
  const uint64_t per_bin = std::max<uint64_t>(1, n_bases / (uint64_t)std::max(prm->nbins, 1));
  int lg = 0;
  while ((per_bin >> lg) > 1) lg++;
  return TuneKey{sms, prm->k <= 32 ? 1 : 2, mean > 1000 ? 1 : 0, prm->nbins, lg / 2};
}

gkc_tune_params defaults() {
  gkc_tune_params d;
  d.coarse_target = gkc::kCoarseTarget;
  d.chunk_kmers = (uint32_t)gkc::kChunkKmers;
  d.count_ctas_per_sm = 2;
  d.reserved = 0;
  return d;
}

bool valid(const gkc_tune_params &p) {
  const bool pow2 = p.chunk_kmers && (p.chunk_kmers & (p.chunk_kmers - 1)) == 0;
  return p.coarse_target >= 256 && p.coarse_target <= 65536 && pow2 && p.chunk_kmers >= 4096 &&
         p.chunk_kmers <= (1u << 22) && p.count_ctas_per_sm >= 1 && p.count_ctas_per_sm <= 4;
}

}  // namespace

gkc_status gkc_tune_get(const gkc_ctx *c, gkc_tune_params *out) {
  if (!c || !out) return GKC_ERR_INVALID_ARG;
  gkc_tune_params d = defaults();
  out->coarse_target = c->tune.coarse_target ? c->tune.coarse_target : d.coarse_target;
  out->chunk_kmers = c->tune.chunk_kmers ? c->tune.chunk_kmers : d.chunk_kmers;
  out->count_ctas_per_sm = c->tune.count_ctas ? c->tune.count_ctas : d.count_ctas_per_sm;
  out->reserved = 0;
  return GKC_OK;
}

gkc_status gkc_tune_set(gkc_ctx *c, const gkc_tune_params *p) {
  if (!c) return GKC_ERR_INVALID_ARG;
  gkc_tune_params v = p ? *p : defaults();
  const gkc_tune_params d = defaults();
  if (!v.coarse_target) v.coarse_target = d.coarse_target;
  if (!v.chunk_kmers) v.chunk_kmers = d.chunk_kmers;
  if (!v.count_ctas_per_sm) v.count_ctas_per_sm = d.count_ctas_per_sm;
  if (!valid(v)) return ctx_fail(c, GKC_ERR_INVALID_ARG, "tuning parameters out of range");
  if (v.coarse_target != c->tune.coarse_target || v.chunk_kmers != c->tune.chunk_kmers ||
      v.count_ctas_per_sm != c->tune.count_ctas) {
    c->tune.coarse_target = v.coarse_target;
    c->tune.chunk_kmers = v.chunk_kmers;
    c->tune.count_ctas = v.count_ctas_per_sm;
    graphs_invalidate(c);  // the captured pipeline holds the old shapes
  }
  return GKC_OK;
}

gkc_status gkc_tune_cache_lookup(int sms, const gkc_params *prm, uint64_t n_bases, uint64_t n_reads,
                                 gkc_tune_params *out) {
  if (!prm || !out) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key_for(sms, prm, n_bases, n_reads));
  if (it == g_cache.end()) return GKC_ERR_NOT_FOUND;
  *out = it->second;
  return GKC_OK;
}

gkc_status gkc_tune_cache_store(int sms, const gkc_params *prm, uint64_t n_bases, uint64_t n_reads,
                                const gkc_tune_params *p) {
  if (!prm || !p || !valid(*p)) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache[key_for(sms, prm, n_bases, n_reads)] = *p;
  return GKC_OK;
}

void gkc_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.clear();
}

// One line per entry:
// "gkc-tune 2 sms key_words long_reads nbins bin_class coarse_target chunk_kmers ctas".
gkc_status gkc_tune_cache_save(const char *path) {
  if (!path) return GKC_ERR_INVALID_ARG;
  FILE *f = fopen(path, "w");
  if (!f) return GKC_ERR_NOT_FOUND;
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto &kv : g_cache)
    fprintf(f, "gkc-tune 2 %d %d %d %d %d %u %u %u\n", kv.first.sms, kv.first.key_words, kv.first.long_reads,
            kv.first.nbins, kv.first.bin_class, kv.second.coarse_target, kv.second.chunk_kmers,
            kv.second.count_ctas_per_sm);
  return fclose(f) == 0 ? GKC_OK : GKC_ERR_INTERNAL;
}

gkc_status gkc_tune_cache_load(const char *path) {
  if (!path) return GKC_ERR_INVALID_ARG;
  FILE *f = fopen(path, "r");
  if (!f) return GKC_ERR_NOT_FOUND;
  char line[256];
  std::vector<std::pair<TuneKey, gkc_tune_params>> got;
  gkc_status st = GKC_OK;
  while (fgets(line, sizeof(line), f)) {
    TuneKey k{};
    gkc_tune_params p{};
    int ver = 0;
    if (sscanf(line, "gkc-tune %d %d %d %d %d %d %u %u %u", &ver, &k.sms, &k.key_words, &k.long_reads, &k.nbins,
               &k.bin_class, &p.coarse_target, &p.chunk_kmers, &p.count_ctas_per_sm) != 9 ||
        ver != 2 || !valid(p)) {
      st = GKC_ERR_INVALID_ARG;
      break;
    }
    got.emplace_back(k, p);
  }
  fclose(f);
  if (st != GKC_OK) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto &e : got) g_cache[e.first] = e.second;
  return GKC_OK;
}

// Device time of the count stages (k-mer offsets through the count kernel)
// of the captured pipeline on the sample, median of `reps` replays.
static gkc_status time_count_stages(gkc_ctx *c, const gkc_params *prm, const char *d_reads, uint64_t nb,
                                    const uint64_t *d_offs, uint64_t nr, int reps, float *ms) {
  std::vector<float> t;
  for (int r = 0; r < reps + 1; r++) {  // the first call captures the graph
    gkc_status s = gkc_pipeline_device(c, prm, GKC_MODE_BATCHED, d_reads, nb, d_offs, nr, nullptr, nullptr);
    if (s != GKC_OK) return s;
    if (r == 0) continue;
    float sum = 0;
    for (int i = 3; i <= 5; i++) sum += c->tm.stage_ms[i];
    t.push_back(sum);
  }
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return GKC_OK;
}

gkc_status gkc_autotune_device(gkc_ctx *c, const gkc_params *prm, const char *d_reads, uint64_t n_bytes,
                               const uint64_t *d_offs, uint64_t n_reads, int force, gkc_tune_report *out) {
  if (!c || !prm || (n_reads && (!d_reads || !d_offs))) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  gkc_tune_report rep;
  memset(&rep, 0, sizeof(rep));
  rep.defaults = defaults();
  if (!force && gkc_tune_cache_lookup(c->n_sms, prm, n_bytes, n_reads, &rep.chosen) == GKC_OK) {
    rep.from_cache = 1;
    if (out) *out = rep;
    return gkc_tune_set(c, &rep.chosen);
  }
  // the sample: the first reads, up to about 2^30 bases
  uint64_t ns = n_reads;
  uint64_t nb = n_bytes;
  const uint64_t want = 1ull << 30;
  if (n_bytes > want && n_reads > 1) {
    ns = std::max<uint64_t>(1, (uint64_t)((double)n_reads * ((double)want / (double)n_bytes)));
    if (cudaMemcpy(&nb, d_offs + ns, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
      return ctx_cuda(c, cudaGetLastError(), "reading the sample's size");
  }
  rep.sample_bases = nb;
  // bins of the sample as large as the full run's
  gkc_params ps = *prm;
  if (nb < n_bytes)
    ps.nbins = std::max(1, (int)((double)prm->nbins * (double)nb / (double)n_bytes + 0.5));
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, prm->k <= 32 ? (const void *)gkc::k_bucket_count<uint64_t> : (const void *)gkc::k_bucket_count<u128>,
      gkc::kBucketCountThreads,
      prm->k <= 32 ? gkc::bucket_count_smem_bytes<uint64_t>() : gkc::bucket_count_smem_bytes<u128>());
  gkc_tune_params cur = rep.defaults;
  if (occ < 2) cur.count_ctas_per_sm = 1;
  const gkc_tune_params saved = {c->tune.coarse_target, c->tune.chunk_kmers, c->tune.count_ctas, 0};
  float best_ms = 0;
  gkc_status s = gkc_tune_set(c, &cur);
  if (s == GKC_OK) s = time_count_stages(c, &ps, d_reads, nb, d_offs, ns, 3, &best_ms);
  if (s != GKC_OK) {
    gkc_tune_set(c, &saved);
    return s;
  }
  rep.default_ms = best_ms;
  rep.candidates = 1;
  const uint32_t ctas[] = {1, 2};
  const uint32_t targets[] = {4096, 8192, 16384};
  const uint32_t chunks[] = {32768, 65536, 131072};
  for (int dim = 0; dim < 3; dim++) {
    const uint32_t *vals = dim == 0 ? ctas : dim == 1 ? targets : chunks;
    const int nv = dim == 0 ? 2 : dim == 1 ? 3 : 3;
    gkc_tune_params best = cur;
    for (int i = 0; i < nv; i++) {
      gkc_tune_params cand = cur;
      uint32_t *field = dim == 0 ? &cand.count_ctas_per_sm : dim == 1 ? &cand.coarse_target : &cand.chunk_kmers;
      if (*field == vals[i]) continue;
      if (dim == 0 && vals[i] > (uint32_t)std::max(occ, 1)) continue;
      *field = vals[i];
      float ms = 0;
      s = gkc_tune_set(c, &cand);
      if (s == GKC_OK) s = time_count_stages(c, &ps, d_reads, nb, d_offs, ns, 3, &ms);
      if (s != GKC_OK) {
        gkc_tune_set(c, &saved);
        return s;
      }
      rep.candidates++;
      if (ms < best_ms) {
        best_ms = ms;
        best = cand;
      }
    }
    cur = best;
  }
  rep.chosen = cur;
  rep.tuned_ms = best_ms;
  gkc_tune_cache_store(c->n_sms, prm, n_bytes, n_reads, &cur);
  if (out) *out = rep;
  return gkc_tune_set(c, &cur);
}
