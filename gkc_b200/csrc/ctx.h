// Context state shared by the host-side translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gkc/gkc.h"

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

// Small summary of a run, written on the device and read back once.
struct DevTotals {
  unsigned long long n_skm, n_packed;
  uint32_t err, pad;
  uint64_t n_kmers, n_bytes, n_distinct;
};

struct GraphKey {
  const void *reads, *offs;
  uint64_t n_bytes, n_reads;
  int k, p, hpc, nbins, filter;
  bool operator==(const GraphKey &o) const {
    return reads == o.reads && offs == o.offs && n_bytes == o.n_bytes && n_reads == o.n_reads &&
           k == o.k && p == o.p && hpc == o.hpc && nbins == o.nbins && filter == o.filter;
  }
};

// Launch shapes picked per device and workload class (the tuner's choices;
// zero means the built-in default).
struct TuneChoice {
  uint32_t coarse_target = 0;  // largest mean keys per count bucket
  uint32_t chunk_kmers = 0;    // k-mers per histogram chunk (a power of two)
  uint32_t count_ctas = 0;     // count kernel CTAs per SM
};

// A captured batched pipeline for one buffer slot.
struct SlotGraph {
  bool valid = false;  // captured against the current workspaces and parameters
  GraphKey key{};
  cudaGraphExec_t exec = nullptr;
  uint32_t launches = 0;
};

// A call of the streaming host form in flight on a slot.
struct StreamCall {
  uint64_t ticket = ~0ull;
  uint64_t capacity = 0;
  uint32_t nbins = 0;
  int key_words = 1;
  // the caller's page-locked outputs and the slot's device results
  uint64_t *h_bin_off = nullptr, *h_keys = nullptr;
  uint32_t *h_counts = nullptr;
  const void *d_bin_off = nullptr, *d_keys = nullptr, *d_counts = nullptr;
  bool dl_issued = true;  // the download has been enqueued (ev_dl of the record recorded)
  bool waited = true;     // the record is free for a new call
  DevTotals tot{};        // the call's totals, copied when its download is enqueued
};

struct gkc_ctx {
  int dev = 0;
  TuneChoice tune;
  int filter = 0;  // minimizer filter (gkc_filter)
  int n_sms = 148;
  int max_smem_optin = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  uint64_t budget = 0, used = 0;
  std::string err;
  std::unordered_map<std::string, DevBuf> bufs;
  DevTotals *h_tots[2] = {nullptr, nullptr};  // pinned, one per slot
  DevTotals *h_tot = nullptr;                 // the current slot's
  int slot = 0;  // buffer set of the inputs and outputs in use (streaming form: 0 or 1)
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t sev[GKC_MAX_STAGES + 1] = {};  // stage boundaries of the batched pipeline
  bool capturing = false;
  uint32_t launches = 0;
  gkc_timings tm{};
  // partition state
  gkc_params pp{};
  bool have_part = false;
  gkc_partition_view pv{};
  uint64_t part_cap_skm = 0, part_cap_bytes = 0;
  const uint8_t *part_packed = nullptr;  // packed bases the partition's descriptors point into
  const uint64_t *part_nbytes_dev = nullptr;
  const char *part_hpc_reads = nullptr;
  const uint64_t *part_hpc_offs = nullptr;
  const int32_t *part_hpc_orig = nullptr;
  // count state
  bool have_count = false;
  uint64_t count_gen = 0;  // bumped by every new count result
  // gkc_count_output cache
  bool have_out = false;
  uint32_t out_min = 0, out_max = 0, out_nbins = 0;
  int out_merged = 0;
  uint64_t out_n = 0, out_gen = 0;
  int ck = 0;
  gkc_count_view cv{};
  uint64_t count_keys_cap = 0;
  bool one_shot = false;      // inputs are not run again: no graph capture
  // graphs of the batched pipeline, one per slot
  SlotGraph graphs[2];
  // streaming host form: upload and download streams, events per slot
  cudaStream_t st_up = nullptr, st_dl = nullptr;
  // streaming: inputs and outputs in two slots (ticket & 1), call records
  // with their download events in four (ticket & 3): up to four calls may
  // await their wait
  cudaEvent_t ev_up[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr};
  cudaEvent_t ev_dl[4] = {nullptr, nullptr, nullptr, nullptr};
  StreamCall calls[4];
  uint64_t next_ticket = 0;
  // host scratch
  std::vector<uint64_t> offs_tmp, desc_tmp;
};

inline void graphs_invalidate(gkc_ctx *c) { c->graphs[0].valid = c->graphs[1].valid = false; }
// Workspace name of the current slot's copy of a per-slot buffer.
inline std::string slot_name(const gkc_ctx *c, const char *n) { return c->slot ? std::string(n) + "#1" : std::string(n); }

gkc_status ctx_fail(gkc_ctx *c, gkc_status s, const std::string &msg);
gkc_status ctx_cuda(gkc_ctx *c, cudaError_t e, const char *what);
void *ws_get(gkc_ctx *c, const char *name, size_t bytes, gkc_status *st);
void ws_release_all(gkc_ctx *c);
cudaError_t result_alloc(int dev, void **p, size_t bytes, cudaStream_t st);  // from the device pool  // workspaces back to the device pool, which keeps them
gkc_status partition_plain_impl(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads);
gkc_status count_plain_impl(gkc_ctx *c, const gkc_params *prm);
gkc_status partition_device_impl(gkc_ctx *c, const gkc_params *prm, const char *d_reads,
                                 uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads);
gkc_status count_device_impl(gkc_ctx *c, const gkc_params *prm, gkc_mode mode);
gkc_status upload_reads(gkc_ctx *c, const char *reads, const uint64_t *offs, uint64_t n_reads,
                        char **d_reads, uint64_t **d_offs, uint64_t *n_bytes);
