// C ABI: contexts, device workspaces, and the partition / count pipelines.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gkc/gkc.h"
#include "common.cuh"
#include "ctx.h"
#include "kernels.h"

using namespace gkc;

// ------------------------------------------------------------------ helpers

const char *gkc_status_string(gkc_status s) {
  switch (s) {
    case GKC_OK: return "ok";
    case GKC_ERR_INVALID_ARG: return "invalid argument";
    case GKC_ERR_CUDA: return "CUDA error";
    case GKC_ERR_NO_DEVICE: return "no CUDA device";
    case GKC_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GKC_ERR_BUDGET: return "HBM budget exceeded";
    case GKC_ERR_CAPACITY: return "capacity exceeded";
    case GKC_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case GKC_ERR_NOT_READY: return "not ready";
    case GKC_ERR_CANCELLED: return "cancelled";
    case GKC_ERR_NOT_FOUND: return "not found";
    default: return "internal error";
  }
}

int gkc_abi_version(void) { return GKC_ABI_VERSION; }

// Stages of the batched pipeline, bounded by events sev[i] .. sev[i+1].
static const char *kStageNames[] = {"prepare", "partition", "bin_scatter", "coarse_hist",
                                    "coarse_scatter", "coarse_count", "finish"};
constexpr int kNumStages = 7;
const char *gkc_stage_name(int i) { return (i >= 0 && i < kNumStages) ? kStageNames[i] : ""; }

// Records stage boundary i on the context stream (as a graph node while capturing).
static void stage_mark(gkc_ctx *c, int i) {
  if (c->capturing) cudaEventRecordWithFlags(c->sev[i], c->st, cudaEventRecordExternal);
  else cudaEventRecord(c->sev[i], c->st);
}

static void read_stage_times(gkc_ctx *c) {
  c->tm.n_stages = kNumStages;
  for (int i = 0; i < kNumStages; i++) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, c->sev[i], c->sev[i + 1]) != cudaSuccess) {
      cudaGetLastError();
      ms = -1;
    }
    c->tm.stage_ms[i] = ms;
  }
}

gkc_status ctx_fail(gkc_ctx *c, gkc_status s, const std::string &msg) {
  if (c) c->err = msg;
  return s;
}

gkc_status ctx_cuda(gkc_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return GKC_OK;
  cudaGetLastError();
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return ctx_fail(c, e == cudaErrorMemoryAllocation ? GKC_ERR_OUT_OF_MEMORY : GKC_ERR_CUDA, m);
}

#define CK(call)                                                  \
  do {                                                            \
    gkc_status _s = ctx_cuda(c, (call), #call);                   \
    if (_s != GKC_OK) return _s;                                  \
  } while (0)
#define LAUNCHED(c)                                               \
  do {                                                            \
    (c)->launches++;                                              \
    cudaError_t _e = cudaPeekAtLastError();                       \
    if (_e != cudaSuccess) return ctx_cuda((c), _e, "kernel launch"); \
  } while (0)

// Workspaces come from one stream-ordered memory pool per device, owned by
// the library: allocations and frees are ordered on the context's stream and
// do not synchronise the device, and freed blocks stay cached in the pool for
// the next request (from any context) until a context is destroyed or its
// workspace released through the public call, which trims the pool.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64];

static cudaMemPool_t device_pool(int dev, cudaError_t *err) {
  *err = cudaSuccess;
  if (dev < 0 || dev >= 64) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    *err = cudaMemPoolCreate(&pool, &props);
    if (*err != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[dev] = pool;
  }
  return g_pool[dev];
}

static void trim_pool(int dev) {
  cudaError_t e;
  cudaMemPool_t pool = device_pool(dev, &e);
  if (pool) cudaMemPoolTrimTo(pool, 0);
}

// A buffer from the device pool outside any context (ordered on st).
cudaError_t result_alloc(int dev, void **p, size_t bytes, cudaStream_t st) {
  cudaError_t e;
  cudaMemPool_t pool = device_pool(dev, &e);
  if (!pool) return e;
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

void *ws_get(gkc_ctx *c, const char *name, size_t bytes, gkc_status *st) {
  *st = GKC_OK;
  if (bytes == 0) bytes = 16;
  bytes = (bytes + 255) & ~(size_t)255;
  auto it = c->bufs.find(name);
  if (it != c->bufs.end() && it->second.bytes >= bytes) return it->second.p;
  if (c->capturing) {  // the capture pass repeats the sizing pass: nothing may grow
    *st = ctx_fail(c, GKC_ERR_INTERNAL, std::string("workspace '") + name + "' grew during capture");
    return nullptr;
  }
  size_t old = 0;
  if (it != c->bufs.end()) {
    old = it->second.bytes;
    cudaFreeAsync(it->second.p, c->st);
    c->used -= old;
    c->bufs.erase(it);
    graphs_invalidate(c);
  }
  size_t want = std::max(bytes, old + old / 4);
  if (c->budget && c->used + want > c->budget) want = bytes;
  if (c->budget && c->used + want > c->budget) {
    *st = ctx_fail(c, GKC_ERR_BUDGET, std::string("workspace '") + name + "' needs " +
                                          std::to_string(bytes) + " bytes beyond the HBM budget");
    return nullptr;
  }
  cudaError_t e;
  cudaMemPool_t pool = device_pool(c->dev, &e);
  void *p = nullptr;
  if (pool) e = cudaMallocFromPoolAsync(&p, want, pool, c->st);
  if (e != cudaSuccess) {
    *st = ctx_cuda(c, e, (std::string("allocating ") + name).c_str());
    return nullptr;
  }
  c->used += want;
  c->bufs[name] = DevBuf{p, want};
  if (old) graphs_invalidate(c);  // captured graphs may hold the freed buffer; a new one is in none
  return p;
}

// Frees every workspace of c into the pool (ordered on c's stream).
void ws_release_all(gkc_ctx *c) {
  cudaStreamSynchronize(c->st);
  for (auto &g : c->graphs)
    if (g.exec) {
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  for (auto &kv : c->bufs) cudaFreeAsync(kv.second.p, c->st);
  cudaStreamSynchronize(c->st);
  c->bufs.clear();
  c->used = 0;
  graphs_invalidate(c);
  c->have_part = c->have_count = false;
}

#define WS(ptr, type, name, count)                                      \
  type *ptr;                                                            \
  do {                                                                  \
    gkc_status _s;                                                      \
    ptr = (type *)ws_get(c, name, sizeof(type) * (size_t)(count), &_s); \
    if (_s != GKC_OK) return _s;                                        \
  } while (0)

// ------------------------------------------------------------------ context

static cudaError_t set_dyn_smem_limit(const void *f, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, f);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

gkc_status gkc_ctx_create(int device_id, uint64_t hbm_budget_bytes, gkc_ctx **out) {
  if (!out) return GKC_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return GKC_ERR_NO_DEVICE;
  }
  if (device_id < 0 || device_id >= n) return GKC_ERR_INVALID_ARG;
  gkc_ctx *c = new gkc_ctx();
  c->dev = device_id;
  c->budget = hbm_budget_bytes;
  if (cudaSetDevice(device_id) != cudaSuccess) {
    delete c;
    return GKC_ERR_CUDA;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device_id);
  c->n_sms = prop.multiProcessorCount;
  c->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
  // The dynamic shared-memory limit of a kernel is process-wide: set it to
  // the device maximum (less the kernel's static shared memory) once, here,
  // and never per launch, where one thread could lower it between another
  // thread's setting and launch.
  if (set_dyn_smem_limit((const void *)k_partition, c->max_smem_optin) != cudaSuccess ||
      set_dyn_smem_limit((const void *)k_bin_place, c->max_smem_optin) != cudaSuccess ||
      set_dyn_smem_limit((const void *)k_bucket_count<uint64_t>, c->max_smem_optin) != cudaSuccess ||
      set_dyn_smem_limit((const void *)k_bucket_count<u128>, c->max_smem_optin) != cudaSuccess ||
      set_dyn_smem_limit((const void *)k_bucket_scatter<uint64_t>, c->max_smem_optin) != cudaSuccess ||
      set_dyn_smem_limit((const void *)k_bucket_scatter<u128>, c->max_smem_optin) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return GKC_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&c->h_tots[0], 2 * sizeof(DevTotals)) != cudaSuccess) {
    delete c;
    return GKC_ERR_CUDA;
  }
  c->h_tots[1] = c->h_tots[0] + 1;
  c->h_tot = c->h_tots[0];
  c->own_stream = true;
  for (int i = 0; i < 4; i++) cudaEventCreate(&c->ev[i]);
  for (int i = 0; i <= GKC_MAX_STAGES; i++) cudaEventCreate(&c->sev[i]);
  *out = c;
  return GKC_OK;
}

void gkc_ctx_destroy(gkc_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  ws_release_all(c);
  trim_pool(c->dev);
  for (int i = 0; i < 4; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  for (int i = 0; i <= GKC_MAX_STAGES; i++)
    if (c->sev[i]) cudaEventDestroy(c->sev[i]);
  if (c->h_tots[0]) cudaFreeHost(c->h_tots[0]);
  if (c->st_up) cudaStreamDestroy(c->st_up);
  if (c->st_dl) cudaStreamDestroy(c->st_dl);
  for (int i = 0; i < 2; i++) {
    if (c->ev_up[i]) cudaEventDestroy(c->ev_up[i]);
    if (c->ev_comp[i]) cudaEventDestroy(c->ev_comp[i]);
  }
  for (int i = 0; i < 4; i++)
    if (c->ev_dl[i]) cudaEventDestroy(c->ev_dl[i]);
  if (c->own_stream && c->st) cudaStreamDestroy(c->st);
  delete c;
}

const char *gkc_ctx_last_error(const gkc_ctx *c) { return c ? c->err.c_str() : "no context"; }

gkc_status gkc_ctx_set_filter(gkc_ctx *c, int filter) {
  if (!c) return GKC_ERR_INVALID_ARG;
  if (filter < GKC_FILTER_NEW2 || filter > GKC_FILTER_SIGNATURE)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "unknown minimizer filter");
  if (filter != c->filter) {
    c->filter = filter;
    graphs_invalidate(c);
    c->have_part = c->have_count = false;
  }
  return GKC_OK;
}

gkc_status gkc_ctx_set_stream(gkc_ctx *c, void *stream) {
  if (!c) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->st);
  if (c->own_stream) cudaStreamDestroy(c->st);
  c->st = (cudaStream_t)stream;
  c->own_stream = false;
  graphs_invalidate(c);
  return GKC_OK;
}

gkc_status gkc_ctx_synchronize(gkc_ctx *c) {
  if (!c) return GKC_ERR_INVALID_ARG;
  CK(cudaStreamSynchronize(c->st));
  return GKC_OK;
}

uint64_t gkc_ctx_device_bytes(const gkc_ctx *c) { return c ? c->used : 0; }

gkc_status gkc_ctx_release_workspace(gkc_ctx *c) {
  if (!c) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  ws_release_all(c);
  trim_pool(c->dev);
  return GKC_OK;
}

gkc_status gkc_last_timings(const gkc_ctx *c, gkc_timings *out) {
  if (!c || !out) return GKC_ERR_INVALID_ARG;
  *out = c->tm;
  return GKC_OK;
}

// ------------------------------------------------------------- validation

static gkc_status check_params(gkc_ctx *c, const gkc_params *prm) {
  if (!prm) return ctx_fail(c, GKC_ERR_INVALID_ARG, "params is NULL");
  if (prm->k < 1 || prm->k > 64) return ctx_fail(c, GKC_ERR_INVALID_ARG, "k must be in [1, 64]");
  if (prm->p < 3 || prm->p > 16 || prm->p > prm->k)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "p must be in [3, 16] and <= k");
  if (prm->nbins < 1 || prm->nbins > (1 << 20))
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "nbins must be in [1, 2^20]");
  return GKC_OK;
}

// --------------------------------------------------------------- totals

__global__ void k_finalize(DevTotals *t, const unsigned long long *cursors, const uint32_t *err,
                           const uint64_t *bin_kstart, uint32_t nbins, const uint64_t *n_bytes_dev,
                           const uint64_t *bin_out) {
  t->n_skm = cursors[0];
  t->n_packed = cursors[1];
  t->err = *err;
  t->n_kmers = bin_kstart ? bin_kstart[nbins] : 0;
  t->n_bytes = n_bytes_dev ? *n_bytes_dev : 0;
  t->n_distinct = bin_out ? bin_out[nbins] : 0;
}

// ------------------------------------------------------------- partition

// Capacity estimates for the superkmer outputs (exact sizes are re-derived
// from the device cursors when a run overflows them).
static void partition_caps(const gkc_params *prm, uint64_t n_bytes, uint64_t n_reads,
                           uint64_t *cap_skm, uint64_t *cap_bytes) {
  const double omega = prm->k - prm->p + 1;
  uint64_t w = n_bytes;
  uint64_t s = (uint64_t)((double)w * 3.0 / (omega + 1.0)) + n_reads + 4096;
  if (s > w + 16) s = w + 16;
  uint64_t tiles = n_bytes / kPartTile + 2;
  *cap_skm = s;
  *cap_bytes = (w + s * (uint64_t)(prm->k - 1)) / 4 + s + tiles * 16 + 64;
}

// Device bytes one pipeline run over n_bases bases in n_reads reads needs:
// the workspaces the batched pipeline sizes for it (reads uploaded from the
// host, optional HPC copies, the read-start bitmap, superkmers in tile and bin
// order, k-mer offsets, coarse-bucket matrices, keys, runs, counts, sort
// scratch) plus a fixed allowance for the small per-bin arrays.
uint64_t gkc_job_hbm_estimate(const gkc_params *prm, uint64_t n_bases, uint64_t n_reads) {
  if (!prm || prm->k < 1 || prm->k > 64 || prm->nbins < 1) return 0;
  const uint64_t B = n_bases, R = n_reads, w = prm->k <= 32 ? 8 : 16;
  uint64_t cap_skm, cap_bytes;
  partition_caps(prm, B, R, &cap_skm, &cap_bytes);
  uint64_t e = (B + 64) + 8 * (R + 1);                                  // reads, offsets
  if (prm->hpc) e += 8 * (R + 1) + 8 * (R + 2) + (B + 64) + 4 * (B + 16);  // HPC copies
  e += (B + 1) / 8 + 16;                                                 // read starts
  e += cap_skm * (8 + 4 + 8 + 4) + cap_bytes;                            // superkmers
  e += cap_skm * 16;                                                     // k-mer offsets
  if ((uint32_t)prm->nbins <= (uint32_t)kBinPlaceMaxBins)                // bin placement matrices
    e += 17 * ((cap_skm + kBinChunk - 1) / kBinChunk) * (uint64_t)prm->nbins;
  const uint64_t kc = std::max<uint64_t>(B, 16);
  uint32_t max_bits = kCoarseMaxBits;
  while (max_bits > 0 && ((uint64_t)prm->nbins << max_bits) > (1ull << 20)) max_bits--;
  const uint64_t chunks = kc / 32768 + prm->nbins + 1;  // the smallest chunk the tuner picks
  e += 4 * (chunks << max_bits) + 8 * chunks;                            // chunk matrix, first superkmers
  e += w * kc * 2 + 4 * kc * 2;                                          // keys, output keys, staged and output counts
  e += ((uint64_t)prm->nbins << max_bits) * (8 * 5 + 4 * 2);             // bucket starts, sizes, distinct counts,
                                                                         // offsets, scan; bins, large-bucket list
  e += 8ull << 20;                                                       // count kernel's per-CTA slice starts
  return e + (64ull << 20);
}

// Enqueues HPC (optional), partition and bin scatter on c->st.
static gkc_status enqueue_partition(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                    uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                    uint64_t cap_skm, uint64_t cap_bytes) {
  const uint32_t nbins = (uint32_t)prm->nbins;
  const uint8_t *src = reinterpret_cast<const uint8_t *>(d_reads);
  const uint64_t *offs = d_offs;
  const uint64_t *nbytes_dev = nullptr;
  WS(tot, unsigned long long, "cursors", 4);
  WS(err, uint32_t, "err", 4);
  stage_mark(c, 0);
  CK(cudaMemsetAsync(tot, 0, 4 * sizeof(unsigned long long), c->st));
  CK(cudaMemsetAsync(err, 0, 4 * sizeof(uint32_t), c->st));
  c->part_hpc_reads = nullptr;
  c->part_hpc_offs = nullptr;
  c->part_hpc_orig = nullptr;
  if (prm->hpc) {
    WS(runlen, unsigned long long, "hpc_runlen", n_reads + 1);
    WS(hoffs, uint64_t, "hpc_offs", n_reads + 2);
    WS(hreads, uint8_t, "hpc_reads", n_bytes + 64);
    WS(horig, int32_t, "hpc_orig", n_bytes + 16);
    WS(stmp, uint64_t, "scan_tmp", scan_u64_tmp_words(n_reads + 1) + 8);
    k_hpc_count<<<c->n_sms * 8, 256, 0, c->st>>>(src, offs, n_reads, runlen);
    LAUNCHED(c);
    scan_u64(runlen, hoffs, n_reads, stmp, c->st);
    c->launches += 4;
    k_hpc_write<<<c->n_sms * 8, 256, 0, c->st>>>(src, offs, n_reads, hoffs, hreads, horig);
    LAUNCHED(c);
    src = hreads;
    offs = hoffs;
    nbytes_dev = hoffs + n_reads;
    c->part_hpc_reads = (const char *)hreads;
    c->part_hpc_offs = hoffs;
    c->part_hpc_orig = horig;
  }
  const uint64_t rs_words = (n_bytes + 1 + 31) / 32 + 2;
  WS(rs, uint32_t, "rs_bits", rs_words);
  CK(cudaMemsetAsync(rs, 0, rs_words * 4, c->st));
  k_read_start_bits<<<(unsigned)std::min<uint64_t>((n_reads + 256) / 256, 65535), 256, 0, c->st>>>(
      offs, n_reads, rs);
  LAUNCHED(c);

  WS(desc, uint64_t, "skm_desc_tile", cap_skm);
  WS(mm, uint32_t, "skm_mm_tile", cap_skm);
  WS(packed, uint8_t, "packed", cap_bytes);
  WS(bin_nskm, unsigned long long, "bin_nskm", nbins + 1);
  WS(bin_nkm, unsigned long long, "bin_nkmers", nbins + 1);
  CK(cudaMemsetAsync(bin_nskm, 0, (nbins + 1) * 8, c->st));
  CK(cudaMemsetAsync(bin_nkm, 0, (nbins + 1) * 8, c->st));

  PartArgs a;
  memset(&a, 0, sizeof(a));
  a.filter = c->filter;
  a.reads = src;
  a.nbytes = n_bytes;
  a.nbytes_dev = nbytes_dev;
  a.aligned16 = ((uintptr_t)src % 16) == 0;
  a.rs_bits = rs;
  a.rs_words = rs_words;
  a.k = prm->k;
  a.p = prm->p;
  a.nbins = (int)nbins;
  a.nbins_smem = nbins <= 1024 ? (int)((nbins + 1) & ~1u) : 0;
  a.skm_desc = desc;
  a.skm_mm = mm;
  a.skm_gpos = nullptr;
  a.packed = packed;
  a.cursors = tot;
  a.cap_skm = cap_skm;
  a.cap_bytes = cap_bytes;
  a.bin_nskm = bin_nskm;
  a.bin_nkmers = bin_nkm;
  a.err = err;
  size_t smem = partition_smem_bytes(a.nbins_smem);
  if ((int)smem > c->max_smem_optin) return ctx_fail(c, GKC_ERR_INVALID_ARG, "too many bins for shared memory");
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_partition, kPartThreads, smem));
  uint64_t tiles = (n_bytes + kPartTile - 1) / kPartTile;
  unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)c->n_sms * std::max(occ, 1)));
  stage_mark(c, 1);
  k_partition<<<grid, kPartThreads, smem, c->st>>>(a);
  LAUNCHED(c);
  stage_mark(c, 2);

  WS(bin_start, uint64_t, "bin_start", nbins + 1);
  WS(bin_kstart, uint64_t, "bin_kstart", nbins + 1);
  k_bin_prefix<<<1, 32, 0, c->st>>>(bin_nskm, bin_nkm, nbins, bin_start, bin_kstart);
  LAUNCHED(c);
  WS(bdesc, uint64_t, "skm_desc_bin", cap_skm);
  WS(bmm, uint32_t, "skm_mm_bin", cap_skm);
  if (nbins <= (uint32_t)kBinPlaceMaxBins) {
    // (bin, chunk) counts, one scan, then placement: no global atomics
    const uint64_t nch_cap = (cap_skm + kBinChunk - 1) / kBinChunk;
    const uint64_t cells = nch_cap * nbins;
    WS(bmat, unsigned long long, "bin_chunk_cnt", cells + 1);
    WS(boff, uint64_t, "bin_chunk_off", cells + 2);
    WS(btmp, uint64_t, "bin_chunk_scan", scan_u64_tmp_words(cells + 1) + 8);
    const unsigned g = (unsigned)std::min<uint64_t>(nch_cap, (uint64_t)c->n_sms * 8);
    k_bin_count<<<g, 256, nbins * 4, c->st>>>(tot, mm, nbins, nch_cap, bmat, err);
    LAUNCHED(c);
    scan_u64(bmat, boff, cells, btmp, c->st);
    c->launches += 4;
    k_bin_place<<<(unsigned)std::min<uint64_t>(nch_cap, (uint64_t)c->n_sms * 2), kBinPlaceThreads,
                  bin_place_smem_bytes(nbins), c->st>>>(tot, desc, mm, nbins, nch_cap, boff, bdesc, bmm, err);
    LAUNCHED(c);
  } else {
    WS(bfill, unsigned long long, "bin_fill", nbins + 1);
    CK(cudaMemsetAsync(bfill, 0, (nbins + 1) * 8, c->st));
    k_bin_scatter<<<c->n_sms * 8, 256, 0, c->st>>>(tot, desc, mm, nbins, bin_start, bfill, bdesc,
                                                   bmm, nullptr, nullptr, err);
    LAUNCHED(c);
  }
  c->part_packed = packed;  // descriptors point into the tile-order bases

  c->part_cap_skm = cap_skm;
  c->part_cap_bytes = cap_bytes;
  c->part_nbytes_dev = nbytes_dev;
  return GKC_OK;
}

static gkc_status fill_partition_view(gkc_ctx *c, const gkc_params *prm, uint64_t n_reads,
                                      uint64_t n_bytes) {
  gkc_partition_view &v = c->pv;
  memset(&v, 0, sizeof(v));
  v.n_reads = n_reads;
  v.n_bases = prm->hpc ? c->h_tot->n_bytes : n_bytes;
  v.n_superkmers = c->h_tot->n_skm;
  v.n_packed_bytes = c->h_tot->n_packed;
  v.n_kmers = c->h_tot->n_kmers;
  v.nbins = (uint32_t)prm->nbins;
  v.bin_skm_off = (const uint64_t *)c->bufs["bin_start"].p;
  v.bin_kmer_off = (const uint64_t *)c->bufs["bin_kstart"].p;
  v.skm_desc = (const uint64_t *)c->bufs["skm_desc_bin"].p;
  v.skm_minimizer = (const uint32_t *)c->bufs["skm_mm_bin"].p;
  v.packed = c->part_packed;
  v.hpc_reads = c->part_hpc_reads;
  v.hpc_offs = c->part_hpc_offs;
  v.hpc_orig_pos = c->part_hpc_orig;
  c->pp = *prm;
  c->have_part = true;
  return GKC_OK;
}

static gkc_status read_totals(gkc_ctx *c, bool with_count, uint32_t nbins) {
  const uint64_t *bk = (const uint64_t *)c->bufs["bin_kstart"].p;
  const uint64_t *bo = with_count ? (const uint64_t *)c->bufs[slot_name(c, "bin_out")].p : nullptr;
  WS(dt, DevTotals, "totals", 1);
  k_finalize<<<1, 1, 0, c->st>>>(dt, (const unsigned long long *)c->bufs["cursors"].p,
                                 (const uint32_t *)c->bufs["err"].p, bk, nbins, c->part_nbytes_dev, bo);
  LAUNCHED(c);
  CK(cudaMemcpyAsync(c->h_tot, dt, sizeof(DevTotals), cudaMemcpyDeviceToHost, c->st));
  stage_mark(c, 7);
  return GKC_OK;
}

static gkc_status check_device_err(gkc_ctx *c) {
  uint32_t e = c->h_tot->err;
  if (e & ERR_BIN_TOO_LARGE)
    return ctx_fail(c, GKC_ERR_CAPACITY, "a bin holds 2^32 or more k-mers: use more bins");
  if (e & ERR_BOUNDS) return ctx_fail(c, GKC_ERR_INTERNAL, "device bounds check failed");
  if (e & ERR_SPIN_TIMEOUT) return ctx_fail(c, GKC_ERR_DEVICE_TIMEOUT, "device look-back wait timed out");
  if (e & ERR_BAD_READ) return ctx_fail(c, GKC_ERR_INVALID_ARG, "read longer than supported");
  return GKC_OK;
}

gkc_status partition_device_impl(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                 uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads) {
  uint64_t cap_skm, cap_bytes;
  partition_caps(prm, n_bytes, n_reads, &cap_skm, &cap_bytes);
  for (int attempt = 0; attempt < 2; attempt++) {
    graphs_invalidate(c);
    gkc_status s = enqueue_partition(c, prm, d_reads, n_bytes, d_offs, n_reads, cap_skm, cap_bytes);
    if (s != GKC_OK) return s;
    s = read_totals(c, false, (uint32_t)prm->nbins);
    if (s != GKC_OK) return s;
    CK(cudaStreamSynchronize(c->st));
    if (!(c->h_tot->err & ERR_CAPACITY)) break;
    cap_skm = c->h_tot->n_skm + 16;
    cap_bytes = c->h_tot->n_packed + 64;
    if (attempt == 1) return ctx_fail(c, GKC_ERR_CAPACITY, "partition capacity");
  }
  gkc_status s = check_device_err(c);
  if (s != GKC_OK) return s;
  return fill_partition_view(c, prm, n_reads, n_bytes);
}

gkc_status gkc_partition_device(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                gkc_partition_view *out) {
  if (!c) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  if (n_bytes > 0 && (!d_reads || !d_offs)) return ctx_fail(c, GKC_ERR_INVALID_ARG, "null input");
  cudaSetDevice(c->dev);
  c->launches = 0;
  CK(cudaEventRecord(c->ev[0], c->st));
  s = partition_device_impl(c, prm, d_reads, n_bytes, d_offs, n_reads);
  if (s != GKC_OK) return s;
  CK(cudaEventRecord(c->ev[1], c->st));
  CK(cudaEventSynchronize(c->ev[1]));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  c->tm = gkc_timings{};
  c->tm.partition_ms = ms;
  c->tm.total_ms = ms;
  c->tm.launches = c->launches;
  if (out) *out = c->pv;
  return GKC_OK;
}

// ------------------------------------------------------------------ count

template <typename K>
static gkc_status enqueue_count_batched(gkc_ctx *c, const gkc_params *prm, uint64_t keys_cap,
                                        uint64_t) {
  const uint32_t nbins = (uint32_t)prm->nbins;
  uint32_t max_bits = kCoarseMaxBits;
  while (max_bits > 0 && ((uint64_t)nbins << max_bits) > (1ull << 20)) max_bits--;
  const uint64_t max_buckets = (uint64_t)nbins << max_bits;
  const uint64_t cap_skm = std::max<uint64_t>(c->part_cap_skm, 1);
  WS(err, uint32_t, "err", 4);
  const unsigned long long *n_skm_dev = (const unsigned long long *)c->bufs["cursors"].p;
  const uint64_t *desc = (const uint64_t *)c->bufs["skm_desc_bin"].p;
  const uint64_t *bin_start = (const uint64_t *)c->bufs["bin_start"].p;
  const uint64_t *bin_kstart = (const uint64_t *)c->bufs["bin_kstart"].p;

  // k-mer offset of every bin-ordered superkmer
  stage_mark(c, 3);
  WS(nk, unsigned long long, "skm_nk", cap_skm + 1);
  WS(koff, uint64_t, "skm_koff", cap_skm + 2);
  WS(stmp, uint64_t, "scan_tmp2", scan_u64_tmp_words(cap_skm + 1) + 8);
  k_skm_nk<<<c->n_sms * 8, 256, 0, c->st>>>(desc, n_skm_dev, prm->k, nk);
  LAUNCHED(c);
  scan_u64_dev(nk, koff, cap_skm, (const uint64_t *)n_skm_dev, stmp, c->st);
  c->launches += 4;

  WS(bin_bits, uint32_t, "bin_bits", nbins + 1);
  WS(bucket_base, uint64_t, "bucket_base", nbins + 1);
  WS(chunk_base, uint64_t, "chunk_base", nbins + 1);
  WS(hist_base, uint64_t, "hist_base", nbins + 1);
  CountPlan pl;
  pl.nbins = nbins;
  pl.bin_start = bin_start;
  pl.bin_kstart = bin_kstart;
  pl.coarse_target = c->tune.coarse_target ? c->tune.coarse_target : kCoarseTarget;
  pl.max_bits = max_bits;
  const uint64_t chunk_kmers = c->tune.chunk_kmers ? c->tune.chunk_kmers : kChunkKmers;
  pl.chunk_kmers = chunk_kmers;
  pl.k = prm->k;
  pl.err = err;
  pl.bin_bits = bin_bits;
  pl.bucket_base = bucket_base;
  pl.chunk_base = chunk_base;
  pl.hist_base = hist_base;
  k_count_plan<<<1, 32, 0, c->st>>>(pl);
  LAUNCHED(c);

  // chunks: at most keys_cap / kChunkKmers + nbins; histogram cells: chunks << max_bits
  const uint64_t max_chunks = keys_cap / chunk_kmers + nbins + 1;
  WS(chunk_s0, uint64_t, "chunk_s0", max_chunks);
  WS(hist, uint32_t, "bucket_hist", max_chunks << max_bits);
  WS(keys, K, "keys", keys_cap);
  // the result's key array holds the k-mer-order keys until the count stage is done with them
  WS(out_keys, K, slot_name(c, "out_keys").c_str(), keys_cap);
  WS(bstart, uint64_t, "bucket_start", max_buckets + 1);
  WS(bsize, uint64_t, "bucket_size", max_buckets + 1);
  ExpandArgs ea;
  memset(&ea, 0, sizeof(ea));
  ea.desc = desc;
  ea.koff = koff;
  ea.packed = c->part_packed;
  ea.nbins = nbins;
  ea.bin_start = bin_start;
  ea.bin_kstart = bin_kstart;
  ea.chunk_base = chunk_base;
  ea.hist_base = hist_base;
  ea.bucket_base = bucket_base;
  ea.bin_bits = bin_bits;
  ea.chunk_kmers = chunk_kmers;
  ea.k = prm->k;
  ea.chunk_s0 = chunk_s0;
  ea.hist = hist;
  ea.keys = keys;
  ea.flat = out_keys;
  ea.keys_cap = keys_cap;
  ea.err = err;
  k_chunk_first<<<(unsigned)std::min<uint64_t>((max_chunks + 255) / 256, 65535), 256, 0, c->st>>>(ea);
  LAUNCHED(c);
  k_bucket_hist<K><<<c->n_sms * 8, kBucketHistThreads, 0, c->st>>>(ea);
  LAUNCHED(c);
  WS(bbin, uint32_t, "bucket_bin", max_buckets + 1);
  WS(big_list, uint32_t, "big_list", max_buckets + 1);
  // [0] bucket ticket, [1] unused, [2] large buckets listed, [3] their ticket
  WS(ticket, unsigned long long, "count_ticket", 4);
  CK(cudaMemsetAsync(ticket, 0, 32, c->st));
  ea.big_list = big_list;
  ea.big_count = ticket + 2;
  ea.big_min = bucket_count_cap<K>();
  k_bucket_scan<<<std::min<uint32_t>(nbins, 65535), kBucketScanThreads, 0, c->st>>>(ea, bstart, bsize, bbin);
  LAUNCHED(c);
  stage_mark(c, 4);
  const size_t sct_smem = bucket_scatter_smem_bytes<K>();
  if ((int)sct_smem > c->max_smem_optin) return ctx_fail(c, GKC_ERR_INTERNAL, "scatter tile exceeds shared memory");
  k_bucket_scatter<K><<<c->n_sms, kBucketScatterThreads, sct_smem, c->st>>>(ea);
  LAUNCHED(c);

  // counting: buckets independently, each bucket's runs staged over its own
  // keys (counts beside them), then moved to the scan of the distinct counts;
  // oversized buckets are placed at their own key range of the result's key
  // array (free between the scatter and the compaction)
  WS(stage_counts, uint32_t, "stage_counts", keys_cap);
  WS(bucket_d, unsigned long long, "bucket_d", max_buckets + 1);
  WS(bucket_out, uint64_t, "bucket_out", max_buckets + 2);
  WS(dtmp, uint64_t, "scan_tmp3", scan_u64_tmp_words(max_buckets + 1) + 8);
  SortCountArgs sa;
  memset(&sa, 0, sizeof(sa));
  sa.nbins = nbins;
  sa.k = prm->k;
  sa.bucket_base = bucket_base;
  sa.bin_bits = bin_bits;
  sa.bucket_start = bstart;
  sa.bucket_size = bsize;
  sa.bucket_bin = bbin;
  sa.keys = keys;
  sa.scratch = out_keys;
  sa.stage_keys = keys;
  sa.stage_counts = stage_counts;
  sa.stage_cap = keys_cap;
  sa.bucket_d = bucket_d;
  sa.ticket = ticket;
  sa.big_list = big_list;
  sa.big_count = ticket + 2;
  sa.big_ticket = ticket + 3;
  sa.big_min = ea.big_min;
  sa.err = err;
  const size_t smem = bucket_count_smem_bytes<K>();
  if ((int)smem > c->max_smem_optin) return ctx_fail(c, GKC_ERR_INTERNAL, "count tables exceed shared memory");
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bucket_count<K>, kBucketCountThreads, smem));
  stage_mark(c, 5);
  // persistent, buckets taken by ticket
  const int ctas = std::max(1, std::min(occ, c->tune.count_ctas ? (int)c->tune.count_ctas : 2));
  WS(sstarts, uint32_t, "slice_starts", (uint64_t)c->n_sms * ctas * 4097);
  sa.slice_starts = sstarts;
  k_bucket_count<K><<<c->n_sms * ctas, kBucketCountThreads, smem, c->st>>>(sa);
  LAUNCHED(c);
  stage_mark(c, 6);
  // final offsets: the exclusive scan of the distinct counts (the bucket count is read on the device)
  scan_u64_dev(bucket_d, bucket_out, max_buckets, bucket_base + nbins, dtmp, c->st);
  c->launches += 4;
  WS(out_counts, uint32_t, slot_name(c, "counts").c_str(), keys_cap);
  WS(bin_out, uint64_t, slot_name(c, "bin_out").c_str(), nbins + 1);
  k_compact_runs<K><<<c->n_sms * 8, 256, 0, c->st>>>(keys, stage_counts, bstart, bucket_d, bucket_out, bucket_base,
                                                      nbins, out_keys, out_counts, bin_out, err);
  LAUNCHED(c);
  c->count_keys_cap = keys_cap;
  return GKC_OK;
}

static gkc_status enqueue_count(gkc_ctx *c, const gkc_params *prm, uint64_t keys_cap) {
  if (prm->k <= 32) return enqueue_count_batched<uint64_t>(c, prm, keys_cap, 0);
  return enqueue_count_batched<u128>(c, prm, keys_cap, 0);
}

static void fill_count_view(gkc_ctx *c, const gkc_params *prm) {
  gkc_count_view &v = c->cv;
  memset(&v, 0, sizeof(v));
  v.n_distinct = c->h_tot->n_distinct;
  v.n_kmers = c->h_tot->n_kmers;
  v.nbins = (uint32_t)prm->nbins;
  v.key_words = prm->k <= 32 ? 1 : 2;
  v.bin_off = (const uint64_t *)c->bufs[slot_name(c, "bin_out")].p;
  v.keys = (const uint64_t *)c->bufs[slot_name(c, "out_keys")].p;
  v.counts = (const uint32_t *)c->bufs[slot_name(c, "counts")].p;
  c->ck = prm->k;
  c->have_count = true;
  c->count_gen++;
}

gkc_status count_device_impl(gkc_ctx *c, const gkc_params *prm, gkc_mode mode) {
  if (!c->have_part) return ctx_fail(c, GKC_ERR_INVALID_ARG, "no partition in the context");
  if (mode == GKC_MODE_PLAIN) return count_plain_impl(c, prm);
  uint64_t n_kmers = c->pv.n_kmers;
  uint64_t keys_cap = n_kmers + 16;
  CK(cudaMemsetAsync(c->bufs["err"].p, 0, 16, c->st));
  gkc_status s = enqueue_count(c, prm, keys_cap);
  if (s != GKC_OK) return s;
  s = read_totals(c, true, (uint32_t)prm->nbins);
  if (s != GKC_OK) return s;
  CK(cudaStreamSynchronize(c->st));
  if (c->h_tot->err & ERR_CAPACITY) return ctx_fail(c, GKC_ERR_CAPACITY, "key capacity");
  if (c->h_tot->err & ERR_BOUNDS) return check_device_err(c);
  s = check_device_err(c);
  if (s != GKC_OK) return s;
  fill_count_view(c, prm);
  return GKC_OK;
}

gkc_status gkc_count_device(gkc_ctx *c, const gkc_params *prm, gkc_mode mode, gkc_count_view *out) {
  if (!c) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  if (c->have_part && (prm->k != c->pp.k || prm->nbins != c->pp.nbins))
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "params differ from the partition's");
  cudaSetDevice(c->dev);
  c->launches = 0;
  CK(cudaEventRecord(c->ev[0], c->st));
  s = count_device_impl(c, prm, mode);
  if (s != GKC_OK) return s;
  CK(cudaEventRecord(c->ev[1], c->st));
  CK(cudaEventSynchronize(c->ev[1]));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  c->tm = gkc_timings{};
  c->tm.count_ms = ms;
  c->tm.total_ms = ms;
  c->tm.launches = c->launches;
  if (out) *out = c->cv;
  return GKC_OK;
}

// -------------------------------------------------------------- pipeline

// Batched: the whole partition -> count pipeline is enqueued once under
// stream capture and replayed as a CUDA graph while inputs and parameters are
// unchanged (one graph per buffer slot).  All sizes the kernels need are read
// on the device.  With `async`, a replay is only enqueued: its totals land in
// the slot's pinned totals and are checked by the caller after the stream.
static gkc_status pipeline_batched(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                   uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                                   bool async = false) {
  GraphKey key{d_reads, d_offs, n_bytes, n_reads, prm->k, prm->p, prm->hpc, prm->nbins, c->filter};
  SlotGraph &G = c->graphs[c->slot];
  uint64_t cap_skm, cap_bytes;
  partition_caps(prm, n_bytes, n_reads, &cap_skm, &cap_bytes);
  const bool have = G.valid && G.key == key && G.exec;
  if (have) {
    cap_skm = c->part_cap_skm;
    cap_bytes = c->part_cap_bytes;
  }
  uint64_t keys_cap = std::max<uint64_t>(n_bytes, 16);
  if (have) keys_cap = c->count_keys_cap;
  for (int attempt = 0; attempt < 3; attempt++) {
    if (G.valid && G.key == key && G.exec) {
      CK(cudaGraphLaunch(G.exec, c->st));
      c->tm.graph_replayed = 1;
      c->launches = G.launches;
      if (async) return GKC_OK;
    } else {
      // allocate every workspace outside capture: one dry enqueue sizes them
      c->launches = 0;
      CK(cudaStreamSynchronize(c->st));
      if (G.exec) {
        cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
      }
      cudaStreamCaptureStatus cs;
      CK(cudaStreamIsCapturing(c->st, &cs));
      if (cs != cudaStreamCaptureStatusNone) return ctx_fail(c, GKC_ERR_INVALID_ARG, "stream already capturing");
      // size pass: plain enqueue (not captured) so that allocation happens now
      gkc_status s = enqueue_partition(c, prm, d_reads, n_bytes, d_offs, n_reads, cap_skm, cap_bytes);
      if (s == GKC_OK) s = enqueue_count(c, prm, keys_cap);
      if (s == GKC_OK) s = read_totals(c, true, (uint32_t)prm->nbins);
      if (s != GKC_OK) return s;
      CK(cudaStreamSynchronize(c->st));
      if (c->one_shot && !(c->h_tot->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH))) {
        c->tm.graph_replayed = 0;
        break;
      }
      if (!(c->h_tot->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH))) {
        // capture the same sequence into a graph for later replays
        G.valid = true;
        uint32_t launches = c->launches;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        c->launches = 0;
        s = enqueue_partition(c, prm, d_reads, n_bytes, d_offs, n_reads, cap_skm, cap_bytes);
        if (s == GKC_OK) s = enqueue_count(c, prm, keys_cap);
        if (s == GKC_OK) s = read_totals(c, true, (uint32_t)prm->nbins);
        cudaError_t e = cudaStreamEndCapture(c->st, &g);
        c->capturing = false;
        if (s != GKC_OK) return s;
        CK(e);
        if (!G.valid) {  // a workspace moved during capture: do not keep it
          cudaGraphDestroy(g);
        } else {
          CK(cudaGraphInstantiate(&G.exec, g, 0));
          cudaGraphDestroy(g);
          G.key = key;
          G.launches = c->launches;
        }
        c->launches = launches;
        c->tm.graph_replayed = 0;
        break;
      }
    }
    CK(cudaStreamSynchronize(c->st));
    if (!(c->h_tot->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH))) break;
    // grow to the sizes the device reported and retry
    graphs_invalidate(c);
    cap_skm = std::max<uint64_t>(cap_skm, c->h_tot->n_skm + 16);
    cap_bytes = std::max<uint64_t>(cap_bytes, c->h_tot->n_packed + 64);
    keys_cap = std::max<uint64_t>(keys_cap, c->h_tot->n_kmers + 16);
    if (attempt == 2) return ctx_fail(c, GKC_ERR_CAPACITY, "pipeline capacity");
  }
  CK(cudaStreamSynchronize(c->st));
  if (c->h_tot->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH)) {
    graphs_invalidate(c);
    return ctx_fail(c, GKC_ERR_CAPACITY, "pipeline capacity");
  }
  gkc_status s = check_device_err(c);
  if (s != GKC_OK) return s;
  read_stage_times(c);
  fill_partition_view(c, prm, n_reads, n_bytes);
  fill_count_view(c, prm);
  return GKC_OK;
}

gkc_status gkc_pipeline_device(gkc_ctx *c, const gkc_params *prm, gkc_mode mode,
                               const char *d_reads, uint64_t n_bytes, const uint64_t *d_offs,
                               uint64_t n_reads, gkc_partition_view *part, gkc_count_view *cnt) {
  if (!c) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  if (n_bytes > 0 && (!d_reads || !d_offs)) return ctx_fail(c, GKC_ERR_INVALID_ARG, "null input");
  cudaSetDevice(c->dev);
  c->tm = gkc_timings{};
  CK(cudaEventRecord(c->ev[0], c->st));
  if (mode == GKC_MODE_BATCHED) {
    s = pipeline_batched(c, prm, d_reads, n_bytes, d_offs, n_reads);
  } else {
    c->launches = 0;
    s = partition_plain_impl(c, prm, d_reads, n_bytes, d_offs, n_reads);
    if (s == GKC_OK) {
      CK(cudaEventRecord(c->ev[2], c->st));
      s = count_plain_impl(c, prm);
    }
  }
  if (s != GKC_OK) return s;
  CK(cudaEventRecord(c->ev[1], c->st));
  CK(cudaEventSynchronize(c->ev[1]));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  c->tm.total_ms = ms;
  c->tm.launches = c->launches;
  if (part) *part = c->pv;
  if (cnt) *cnt = c->cv;
  return GKC_OK;
}

// Host entry: H2D of reads and rebased offsets, then the device pipeline.
gkc_status upload_reads(gkc_ctx *c, const char *reads, const uint64_t *offs, uint64_t n_reads,
                        char **d_reads, uint64_t **d_offs, uint64_t *n_bytes) {
  const uint64_t base = n_reads ? offs[0] : 0;
  const uint64_t nb = n_reads ? offs[n_reads] - base : 0;
  WS(dr, char, slot_name(c, "in_reads").c_str(), nb + 64);
  WS(doffs, uint64_t, slot_name(c, "in_offs").c_str(), n_reads + 1);
  if (nb) CK(cudaMemcpyAsync(dr, reads + base, nb, cudaMemcpyHostToDevice, c->st));
  if (base == 0) {
    CK(cudaMemcpyAsync(doffs, offs, (n_reads + 1) * 8, cudaMemcpyHostToDevice, c->st));
  } else {
    c->offs_tmp.resize(n_reads + 1);
    for (uint64_t r = 0; r <= n_reads; r++) c->offs_tmp[r] = offs[r] - base;
    CK(cudaMemcpyAsync(doffs, c->offs_tmp.data(), (n_reads + 1) * 8, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  *d_reads = dr;
  *d_offs = doffs;
  *n_bytes = nb;
  return GKC_OK;
}

gkc_status gkc_partition_host(gkc_ctx *c, const gkc_params *prm, const char *reads,
                              const uint64_t *offs, uint64_t n_reads, gkc_partition_view *out) {
  if (!c || (n_reads && (!reads || !offs))) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  cudaSetDevice(c->dev);
  char *dr;
  uint64_t *doffs, nb;
  s = upload_reads(c, reads, offs, n_reads, &dr, &doffs, &nb);
  if (s != GKC_OK) return s;
  return gkc_partition_device(c, prm, dr, nb, doffs, n_reads, out);
}

gkc_status gkc_pipeline_host(gkc_ctx *c, const gkc_params *prm, gkc_mode mode, const char *reads,
                             const uint64_t *offs, uint64_t n_reads, gkc_count_view *cnt) {
  if (!c || (n_reads && (!reads || !offs))) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  cudaSetDevice(c->dev);
  CK(cudaEventRecord(c->ev[3], c->st));
  char *dr;
  uint64_t *doffs, nb;
  s = upload_reads(c, reads, offs, n_reads, &dr, &doffs, &nb);
  if (s != GKC_OK) return s;
  s = gkc_pipeline_device(c, prm, mode, dr, nb, doffs, n_reads, nullptr, cnt);
  if (s != GKC_OK) return s;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[3], c->ev[0]);
  c->tm.h2d_ms = ms;
  return GKC_OK;
}

// ------------------------------------------------------ streaming host form

// offs[i] -= offs[0] (offsets of a batch cut from a larger CSR); one CTA
__global__ void k_rebase_offs(uint64_t *offs, uint64_t n) {
  const uint64_t base = offs[0];
  __syncthreads();  // every thread has read offs[0]
  for (uint64_t i = threadIdx.x + 1; i <= n; i += blockDim.x) offs[i] -= base;
  __syncthreads();
  if (threadIdx.x == 0) offs[0] = 0;
}
// The download of a streaming call: once its pipeline is done, its totals
// (copied to page-locked memory inside the captured pipeline) give the exact
// sizes, and three DMA copies on the download stream move the bin offsets,
// keys and counts into the caller's page-locked buffers while the next call
// computes.  Blocks until the call's pipeline is done.  rec: the call's
// record (ticket & 3); its slot is ticket & 1.
static gkc_status issue_download(gkc_ctx *c, int rec) {
  StreamCall &sc = c->calls[rec];
  if (sc.dl_issued) return GKC_OK;
  const int slot = (int)(sc.ticket & 1);
  CK(cudaEventSynchronize(c->ev_comp[slot]));
  sc.tot = *c->h_tots[slot];  // the slot's next call overwrites them
  const DevTotals *h = &sc.tot;
  const bool bad = (h->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH | ERR_BIN_TOO_LARGE | ERR_SPIN_TIMEOUT | ERR_BOUNDS |
                              ERR_BAD_READ)) != 0;
  if (!bad) {
    const uint64_t nd = std::min<uint64_t>(h->n_distinct, sc.capacity);
    if (sc.h_bin_off)
      CK(cudaMemcpyAsync(sc.h_bin_off, sc.d_bin_off, 8 * ((uint64_t)sc.nbins + 1), cudaMemcpyDeviceToHost, c->st_dl));
    if (sc.h_keys && nd)
      CK(cudaMemcpyAsync(sc.h_keys, sc.d_keys, nd * 8 * (uint64_t)sc.key_words, cudaMemcpyDeviceToHost, c->st_dl));
    if (sc.h_counts && nd)
      CK(cudaMemcpyAsync(sc.h_counts, sc.d_counts, nd * 4, cudaMemcpyDeviceToHost, c->st_dl));
  }
  CK(cudaEventRecord(c->ev_dl[rec], c->st_dl));
  sc.dl_issued = true;
  return GKC_OK;
}

static bool host_visible(const void *p) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost && a.devicePointer != nullptr;
}

gkc_status gkc_stream_submit(gkc_ctx *c, const gkc_params *prm, const char *reads, const uint64_t *offs,
                             uint64_t n_reads, uint64_t *bin_off, uint64_t *keys, uint32_t *counts,
                             uint64_t capacity, uint64_t *ticket) {
  if (!c || !ticket || (n_reads && (!reads || !offs))) return GKC_ERR_INVALID_ARG;
  gkc_status s = check_params(c, prm);
  if (s != GKC_OK) return s;
  if (!host_visible(reads) || !host_visible(offs) || !host_visible(bin_off) || !host_visible(keys) ||
      !host_visible(counts))
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "streaming buffers must be page-locked host memory");
  cudaSetDevice(c->dev);
  if (!c->st_up) {
    CK(cudaStreamCreateWithFlags(&c->st_up, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->st_dl, cudaStreamNonBlocking));
    for (int i = 0; i < 2; i++) {
      CK(cudaEventCreateWithFlags(&c->ev_up[i], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->ev_comp[i], cudaEventDisableTiming));
    }
    for (int i = 0; i < 4; i++) CK(cudaEventCreateWithFlags(&c->ev_dl[i], cudaEventDisableTiming));
  }
  const uint64_t t = c->next_ticket;
  const int slot = (int)(t & 1), rec = (int)(t & 3);
  if (!c->calls[rec].waited)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "four calls await their wait: wait for the oldest first");
  // the slot's previous call must have its download enqueued before its
  // buffers are reused
  const int prev = (int)((t + 2) & 3);  // record of call t - 2
  if (t >= 2) {
    s = issue_download(c, prev);
    if (s != GKC_OK) return s;
  }
  // the slot's input buffers; growing them waits for everything in flight
  const uint64_t base = n_reads ? offs[0] : 0, nb = n_reads ? offs[n_reads] - base : 0;
  c->slot = slot;
  c->h_tot = c->h_tots[slot];
  struct SlotReset {  // every return leaves the context on slot 0
    gkc_ctx *c;
    ~SlotReset() {
      c->slot = 0;
      c->h_tot = c->h_tots[0];
    }
  } reset{c};
  const std::string rn = slot_name(c, "in_reads"), on = slot_name(c, "in_offs");
  auto fits = [&](const std::string &n, size_t bytes) {
    auto it = c->bufs.find(n);
    return it != c->bufs.end() && it->second.bytes >= bytes;
  };
  if (!fits(rn, nb + 64) || !fits(on, 8 * (n_reads + 1))) {
    CK(cudaStreamSynchronize(c->st_up));
    CK(cudaStreamSynchronize(c->st_dl));
    CK(cudaStreamSynchronize(c->st));
  }
  WS(dr, char, rn.c_str(), nb + 64);
  WS(doffs, uint64_t, on.c_str(), n_reads + 1);
  // inputs of the slot's previous call must have been read before they are replaced
  if (t >= 2) CK(cudaStreamWaitEvent(c->st_up, c->ev_comp[slot], 0));
  if (nb) CK(cudaMemcpyAsync(dr, reads + base, nb, cudaMemcpyHostToDevice, c->st_up));
  CK(cudaMemcpyAsync(doffs, offs, 8 * (n_reads + 1), cudaMemcpyHostToDevice, c->st_up));
  CK(cudaEventRecord(c->ev_up[slot], c->st_up));
  CK(cudaStreamWaitEvent(c->st, c->ev_up[slot], 0));
  // and its outputs must have been copied out before they are recomputed
  if (t >= 2) CK(cudaStreamWaitEvent(c->st, c->ev_dl[prev], 0));
  if (base) {
    k_rebase_offs<<<1, 1024, 0, c->st>>>(doffs, n_reads);
    LAUNCHED(c);
  }
  c->tm = gkc_timings{};
  s = pipeline_batched(c, prm, dr, nb, doffs, n_reads, true);
  if (s != GKC_OK) return s;
  CK(cudaEventRecord(c->ev_comp[slot], c->st));
  StreamCall sc;
  sc.ticket = t;
  sc.capacity = capacity;
  sc.nbins = (uint32_t)prm->nbins;
  sc.key_words = prm->k <= 32 ? 1 : 2;
  sc.h_bin_off = bin_off;
  sc.h_keys = keys;
  sc.h_counts = counts;
  sc.d_bin_off = c->bufs[slot_name(c, "bin_out")].p;
  sc.d_keys = c->bufs[slot_name(c, "out_keys")].p;
  sc.d_counts = c->bufs[slot_name(c, "counts")].p;
  sc.dl_issued = false;
  sc.waited = false;
  c->calls[rec] = sc;
  c->next_ticket = t + 1;
  *ticket = t;
  // the previous call (the other slot), if its pipeline is already done:
  // start its download now
  if (t >= 1) {
    const int last = (int)((t + 3) & 3);
    if (!c->calls[last].dl_issued && cudaEventQuery(c->ev_comp[slot ^ 1]) == cudaSuccess) {
      s = issue_download(c, last);
      if (s != GKC_OK) return s;
    }
  }
  return GKC_OK;
}

gkc_status gkc_stream_wait(gkc_ctx *c, uint64_t ticket, uint64_t *n_distinct, uint64_t *n_kmers) {
  if (!c) return GKC_ERR_INVALID_ARG;
  const int rec = (int)(ticket & 3);
  StreamCall &sc = c->calls[rec];
  if (sc.ticket != ticket || sc.waited) return ctx_fail(c, GKC_ERR_NOT_FOUND, "no call in flight with this ticket");
  cudaSetDevice(c->dev);
  gkc_status s = issue_download(c, rec);
  if (s != GKC_OK) return s;
  CK(cudaEventSynchronize(c->ev_dl[rec]));
  sc.waited = true;
  const DevTotals *h = &sc.tot;
  if (n_distinct) *n_distinct = h->n_distinct;
  if (n_kmers) *n_kmers = h->n_kmers;
  if (h->err & (ERR_CAPACITY | ERR_OVERSIZE_SCRATCH))
    return ctx_fail(c, GKC_ERR_CAPACITY, "the call's input outgrew the captured pipeline: run it with gkc_pipeline_host");
  if (h->err & ERR_BIN_TOO_LARGE) return ctx_fail(c, GKC_ERR_CAPACITY, "a bin holds 2^32 or more k-mers");
  if (h->err & ERR_SPIN_TIMEOUT) return ctx_fail(c, GKC_ERR_DEVICE_TIMEOUT, "device look-back wait timed out");
  if (h->err & (ERR_BOUNDS | ERR_BAD_READ)) return ctx_fail(c, GKC_ERR_INTERNAL, "device check failed");
  if (h->n_distinct > sc.capacity)
    return ctx_fail(c, GKC_ERR_CAPACITY, "result larger than the output capacity (bin offsets and the first entries copied)");
  return GKC_OK;
}

// --------------------------------------------------------------- copy out

gkc_status gkc_partition_copy_out(gkc_ctx *c, uint64_t *bin_skm_off, uint32_t *skm_len,
                                  uint64_t *skm_byte_off, uint8_t *packed, uint32_t *minimizer) {
  if (!c || !c->have_part) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const gkc_partition_view &v = c->pv;
  if (bin_skm_off)
    CK(cudaMemcpyAsync(bin_skm_off, v.bin_skm_off, (v.nbins + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  if (minimizer && v.n_superkmers) {
    if (v.skm_minimizer)
      CK(cudaMemcpyAsync(minimizer, v.skm_minimizer, v.n_superkmers * 4, cudaMemcpyDeviceToHost, c->st));
    else  // an imported partition carries no minimizers
      memset(minimizer, 0xFF, v.n_superkmers * 4);
  }
  if (packed && v.n_packed_bytes)
    CK(cudaMemcpyAsync(packed, v.packed, v.n_packed_bytes, cudaMemcpyDeviceToHost, c->st));
  if ((skm_len || skm_byte_off) && v.n_superkmers) {
    c->desc_tmp.resize(v.n_superkmers);
    CK(cudaMemcpyAsync(c->desc_tmp.data(), v.skm_desc, v.n_superkmers * 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (uint64_t i = 0; i < v.n_superkmers; i++) {
      if (skm_len) skm_len[i] = (uint32_t)(c->desc_tmp[i] & 0xFFFFFFu);
      if (skm_byte_off) skm_byte_off[i] = c->desc_tmp[i] >> 24;
    }
  }
  CK(cudaStreamSynchronize(c->st));
  return GKC_OK;
}

// The partition kernels already hold, per bin, the superkmer prefix and the
// k-mer prefix; a superkmer of w k-mers has w + k - 1 bases, so the bases of
// bin b are its k-mers plus (k - 1) per superkmer.  Only the two prefix
// arrays (nbins + 1 words each) cross to the host.
gkc_status gkc_partition_balance(gkc_ctx *c, uint64_t *bin_bases, uint32_t capacity,
                                 gkc_balance_stats *st) {
  if (!c || !c->have_part) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const gkc_partition_view &v = c->pv;
  const uint32_t nb = v.nbins;
  if (bin_bases && capacity < nb)
    return ctx_fail(c, GKC_ERR_CAPACITY, "bin_bases holds " + std::to_string(capacity) + " entries, the partition has " +
                                             std::to_string(nb) + " bins");
  std::vector<uint64_t> so(nb + 1), ko(nb + 1);
  CK(cudaMemcpyAsync(so.data(), v.bin_skm_off, (nb + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(ko.data(), v.bin_kmer_off, (nb + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const uint64_t km1 = (uint64_t)(c->pp.k - 1);
  gkc_balance_stats s{};
  s.min = ~0ull;
  std::vector<uint64_t> sz(nb);
  for (uint32_t b = 0; b < nb; b++) {
    sz[b] = (ko[b + 1] - ko[b]) + km1 * (so[b + 1] - so[b]);
    s.total += sz[b];
    s.max = std::max(s.max, sz[b]);
    s.min = std::min(s.min, sz[b]);
  }
  s.mean = nb ? s.total / nb : 0;
  double acc = 0.0;
  for (uint32_t b = 0; b < nb; b++) {
    const uint64_t d = sz[b] - s.mean;  // wraps below the mean; the square is the same mod 2^64
    acc += (double)(d * d);
  }
  s.variance = nb ? acc / nb : 0.0;
  s.stdev = std::sqrt(s.variance);
  s.cv = s.stdev / (double)s.mean;
  if (bin_bases) std::copy(sz.begin(), sz.end(), bin_bases);
  if (st) *st = s;
  return GKC_OK;
}

gkc_status gkc_count_copy_out(gkc_ctx *c, uint64_t *bin_off, uint64_t *keys, uint32_t *counts) {
  if (!c || !c->have_count) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const gkc_count_view &v = c->cv;
  CK(cudaEventRecord(c->ev[2], c->st));
  // cudaMemcpyDefault: each destination may be host or device memory
  if (bin_off)
    CK(cudaMemcpyAsync(bin_off, v.bin_off, (v.nbins + 1) * 8, cudaMemcpyDefault, c->st));
  if (keys && v.n_distinct)
    CK(cudaMemcpyAsync(keys, v.keys, v.n_distinct * 8 * v.key_words, cudaMemcpyDefault, c->st));
  if (counts && v.n_distinct)
    CK(cudaMemcpyAsync(counts, v.counts, v.n_distinct * 4, cudaMemcpyDefault, c->st));
  CK(cudaEventRecord(c->ev[3], c->st));
  CK(cudaStreamSynchronize(c->st));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
  c->tm.d2h_ms = ms;
  return GKC_OK;
}

// One bin of packed superkmers from the host (kmc_counting_GPU drop-in).
gkc_status gkc_count_superkmers_host(gkc_ctx *c, int k, const uint32_t *skm_len,
                                     const uint8_t *packed, uint64_t n_skm, gkc_mode mode,
                                     uint64_t *n_distinct) {
  if (!c || k < 1 || k > 64 || (n_skm && (!skm_len || !packed))) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  std::vector<uint64_t> desc(n_skm);
  uint64_t off = 0, nk = 0;
  for (uint64_t i = 0; i < n_skm; i++) {
    if (skm_len[i] > 0xFFFFFFu) return ctx_fail(c, GKC_ERR_INVALID_ARG, "superkmer too long");
    desc[i] = (off << 24) | skm_len[i];
    off += (skm_len[i] + 3) / 4;
    if (skm_len[i] >= (uint32_t)k) nk += skm_len[i] - k + 1;
  }
  WS(dd, uint64_t, "skm_desc_bin", n_skm + 1);
  WS(dp, uint8_t, "packed_bin", off + 16);
  WS(dmm, uint32_t, "skm_mm_bin", n_skm + 1);
  WS(bs, uint64_t, "bin_start", 2);
  WS(bk, uint64_t, "bin_kstart", 2);
  WS(cur, unsigned long long, "cursors", 4);
  WS(err, uint32_t, "err", 4);
  if (n_skm) CK(cudaMemcpyAsync(dd, desc.data(), n_skm * 8, cudaMemcpyHostToDevice, c->st));
  if (off) CK(cudaMemcpyAsync(dp, packed, off, cudaMemcpyHostToDevice, c->st));
  c->part_packed = dp;
  uint64_t hb[4] = {0, n_skm, 0, nk};
  CK(cudaMemcpyAsync(bs, hb, 16, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(bk, hb + 2, 16, cudaMemcpyHostToDevice, c->st));
  unsigned long long hc[4] = {n_skm, off, 0, 0};
  CK(cudaMemcpyAsync(cur, hc, 32, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(err, 0, 16, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->pv = gkc_partition_view{};
  c->pv.n_superkmers = n_skm;
  c->pv.n_packed_bytes = off;
  c->pv.n_kmers = nk;
  c->pv.nbins = 1;
  c->pv.bin_skm_off = bs;
  c->pv.bin_kmer_off = bk;
  c->pv.skm_desc = dd;
  c->pv.skm_minimizer = dmm;
  c->pv.packed = dp;
  c->part_nbytes_dev = nullptr;
  // the count path sizes its per-superkmer arrays from the partition's
  // capacities, which a fresh context has not set
  c->part_cap_skm = n_skm + 1;
  c->part_cap_bytes = off + 16;
  c->have_part = true;
  gkc_params prm{k, 3, 0, 1};
  c->pp = prm;
  graphs_invalidate(c);
  gkc_status s = gkc_count_device(c, &prm, mode, nullptr);
  if (s != GKC_OK) return s;
  if (n_distinct) *n_distinct = c->cv.n_distinct;
  return GKC_OK;
}
