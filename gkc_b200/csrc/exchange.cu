// Superkmer exchange for bin sharding over several GPUs.
//
// Reads are independent and so are bins: every GPU partitions its own reads,
// then each bin's superkmers move to the GPU that owns the bin, which counts
// them (the one exchange step of the path; the reference runs on one GPU and
// has no counterpart).  Owners hold contiguous bin ranges, so a sender's
// bin-ordered descriptors are already grouped by destination.
//
//   gkc_exchange_pack     sender side: per destination, one run of
//                         descriptors and one run of packed bytes, each
//                         descriptor's byte offset relative to its run
//   gkc_partition_import  receiver side: the runs of all senders, in sender
//                         order, become the context's partition in local bin
//                         order (bin-major, then sender), ready to count
//
// The transfer between them is the caller's (an all-to-all over NCCL: two
// calls, one for descriptors, one for bytes, with the split sizes returned
// by the pack).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "kernels.h"

namespace gkc {

// Largest index i in [0, n) with a[i] <= x (a ascending, a[0] <= x).
GKC_DEV uint32_t last_le(const uint64_t *a, uint32_t n, uint64_t x) {
  uint32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_xchg_nbytes(const uint64_t *desc, uint64_t n, unsigned long long *nb) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    nb[i] = ((desc[i] & 0xFFFFFFull) + 3) >> 2;
}

// seg[r] = first superkmer of destination r (n_dest + 1 entries, seg[n_dest] = n).
__global__ void k_xchg_pack(const uint64_t *desc, const uint8_t *packed, uint64_t n, const uint64_t *off,
                            const uint64_t *seg, uint32_t n_dest, uint64_t *out_desc, uint8_t *out_bytes) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = desc[i];
    const uint64_t len = d & 0xFFFFFFull, src = d >> 24, dst = off[i];
    const uint64_t nb = (len + 3) >> 2;
    const uint32_t r = last_le(seg, n_dest + 1, i);
    out_desc[i] = ((dst - off[seg[r]]) << 24) | len;
    for (uint64_t j = 0; j < nb; j++) out_bytes[dst + j] = packed[src + j];
  }
}

// Received descriptor j of sender s (its run starts at e[s]) lies in local
// bin b of that run (run-relative bin starts q[s*(nbl+1) + b]); it goes to
// p[s*nbl + b] + its index inside the bin, its bytes rebased by dbyte[s].
__global__ void k_xchg_import(const uint64_t *in_desc, uint64_t n, const uint64_t *e, uint32_t n_src,
                              const uint64_t *dbyte, const uint64_t *q, const uint64_t *p, uint32_t nbl,
                              uint64_t *out_desc) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = last_le(e, n_src + 1, j);
    const uint64_t t = j - e[s];
    const uint64_t *qs = q + (uint64_t)s * (nbl + 1);
    const uint32_t b = last_le(qs, nbl + 1, t);
    const uint64_t d = in_desc[j];
    out_desc[p[(uint64_t)s * nbl + b] + (t - qs[b])] = (((d >> 24) + dbyte[s]) << 24) | (d & 0xFFFFFFull);
  }
}

}  // namespace gkc

using namespace gkc;

#define CK(call)                                \
  do {                                          \
    gkc_status _s = ctx_cuda(c, (call), #call); \
    if (_s != GKC_OK) return _s;                \
  } while (0)
#define WS(ptr, type, name, count)                                      \
  type *ptr;                                                            \
  do {                                                                  \
    gkc_status _s;                                                      \
    ptr = (type *)ws_get(c, name, sizeof(type) * (size_t)(count), &_s); \
    if (_s != GKC_OK) return _s;                                        \
  } while (0)

static unsigned grid_for(const gkc_ctx *c, uint64_t n) {
  const uint64_t want = (n + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)c->n_sms * 16));
}

gkc_status gkc_exchange_pack(gkc_ctx *c, uint32_t n_dest, const uint32_t *bin_lo, uint64_t *d_send_desc,
                             uint64_t desc_capacity, uint8_t *d_send_bytes, uint64_t bytes_capacity,
                             uint64_t *skm_split, uint64_t *byte_split, uint64_t *bin_skm, uint64_t *bin_kmers) {
  if (!c || !c->have_part || n_dest < 1 || !bin_lo || !skm_split || !byte_split) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const gkc_partition_view &v = c->pv;
  const uint32_t nb = v.nbins;
  if (bin_lo[0] != 0 || bin_lo[n_dest] != nb)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "bin ranges must start at 0 and end at the partition's bin count");
  for (uint32_t r = 0; r < n_dest; r++)
    if (bin_lo[r] > bin_lo[r + 1]) return ctx_fail(c, GKC_ERR_INVALID_ARG, "bin ranges must not decrease");
  const uint64_t n = v.n_superkmers;
  c->launches = 0;
  if (n > desc_capacity || (n && !d_send_desc))
    return ctx_fail(c, GKC_ERR_CAPACITY, "send descriptors hold " + std::to_string(desc_capacity) +
                                             " entries, the partition has " + std::to_string(n) + " superkmers");
  std::vector<uint64_t> so(nb + 1), ko(nb + 1);
  CK(cudaMemcpyAsync(so.data(), v.bin_skm_off, (nb + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(ko.data(), v.bin_kmer_off, (nb + 1) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  std::vector<uint64_t> seg(n_dest + 1);
  for (uint32_t r = 0; r <= n_dest; r++) seg[r] = so[bin_lo[r]];
  WS(nbytes, unsigned long long, "xchg_nbytes", n + 1);
  WS(off, uint64_t, "xchg_off", n + 2);
  WS(stmp, uint64_t, "xchg_scan_tmp", scan_u64_tmp_words(n + 1) + 8);
  WS(dseg, uint64_t, "xchg_seg", n_dest + 1);
  std::vector<uint64_t> hoff(n_dest + 1, 0);
  if (n) {
    k_xchg_nbytes<<<grid_for(c, n), 256, 0, c->st>>>(v.skm_desc, n, nbytes);
    scan_u64(nbytes, off, n, stmp, c->st);
    CK(cudaPeekAtLastError());
    c->launches += 5;  // the byte-length kernel and the scan's four
    // byte offset of every destination's first superkmer (and the total)
    for (uint32_t r = 0; r <= n_dest; r++)
      CK(cudaMemcpyAsync(&hoff[r], off + seg[r], 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (hoff[n_dest] > bytes_capacity || (hoff[n_dest] && !d_send_bytes))
    return ctx_fail(c, GKC_ERR_CAPACITY, "send bytes hold " + std::to_string(bytes_capacity) + ", " +
                                             std::to_string(hoff[n_dest]) + " needed");
  if (n) {
    CK(cudaMemcpyAsync(dseg, seg.data(), (n_dest + 1) * 8, cudaMemcpyHostToDevice, c->st));
    k_xchg_pack<<<grid_for(c, n), 256, 0, c->st>>>(v.skm_desc, v.packed, n, off, dseg, n_dest, d_send_desc,
                                                   d_send_bytes);
    CK(cudaPeekAtLastError());
    c->launches++;
  }
  for (uint32_t r = 0; r < n_dest; r++) {
    skm_split[r] = seg[r + 1] - seg[r];
    byte_split[r] = hoff[r + 1] - hoff[r];
  }
  for (uint32_t b = 0; b < nb; b++) {
    if (bin_skm) bin_skm[b] = so[b + 1] - so[b];
    if (bin_kmers) bin_kmers[b] = ko[b + 1] - ko[b];
  }
  CK(cudaStreamSynchronize(c->st));
  c->tm = gkc_timings{};
  c->tm.launches = c->launches;
  return GKC_OK;
}

gkc_status gkc_partition_import(gkc_ctx *c, const gkc_params *prm, uint32_t n_src, const uint64_t *seg_bin_skm,
                                const uint64_t *seg_bin_kmers, const uint64_t *seg_bytes, const uint64_t *d_desc,
                                const uint8_t *d_bytes, gkc_partition_view *out) {
  if (!c || !prm || n_src < 1 || !seg_bin_skm || !seg_bin_kmers || !seg_bytes) return GKC_ERR_INVALID_ARG;
  if (prm->k < 1 || prm->k > 64 || prm->nbins < 1 || prm->nbins > (1 << 20)) return GKC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const uint32_t nbl = (uint32_t)prm->nbins;
  // host plan: run starts e, byte bases, run-relative bin starts q, targets p
  std::vector<uint64_t> e(n_src + 1, 0), dby(n_src + 1, 0), q((uint64_t)n_src * (nbl + 1)),
      p((uint64_t)n_src * nbl), bs(nbl + 1, 0), bk(nbl + 1, 0);
  for (uint32_t s = 0; s < n_src; s++) {
    uint64_t t = 0;
    for (uint32_t b = 0; b < nbl; b++) {
      q[(uint64_t)s * (nbl + 1) + b] = t;
      t += seg_bin_skm[(uint64_t)s * nbl + b];
    }
    q[(uint64_t)s * (nbl + 1) + nbl] = t;
    e[s + 1] = e[s] + t;
    dby[s + 1] = dby[s] + seg_bytes[s];
  }
  for (uint32_t b = 0; b < nbl; b++) {
    uint64_t ns = 0, nk = 0;
    for (uint32_t s = 0; s < n_src; s++) {
      p[(uint64_t)s * nbl + b] = bs[b] + ns;
      ns += seg_bin_skm[(uint64_t)s * nbl + b];
      nk += seg_bin_kmers[(uint64_t)s * nbl + b];
    }
    bs[b + 1] = bs[b] + ns;
    bk[b + 1] = bk[b] + nk;
  }
  const uint64_t n = e[n_src], nbytes = dby[n_src];
  if ((n && !d_desc) || (nbytes && !d_bytes)) return GKC_ERR_INVALID_ARG;
  // descriptors keep the byte offset in 40 bits, rebased over all runs
  if (nbytes >> 40) return ctx_fail(c, GKC_ERR_INVALID_ARG, "received bytes exceed 2^40");
  WS(dd, uint64_t, "skm_desc_bin", n + 1);
  WS(dp, uint8_t, "packed_bin", nbytes + 16);
  WS(dbs, uint64_t, "bin_start", nbl + 1);
  WS(dbk, uint64_t, "bin_kstart", nbl + 1);
  WS(cur, unsigned long long, "cursors", 4);
  WS(err, uint32_t, "err", 4);
  const uint64_t plan_words = (n_src + 1) + (n_src + 1) + q.size() + p.size();
  WS(plan, uint64_t, "import_plan", plan_words);
  std::vector<uint64_t> hp;
  hp.reserve(plan_words);
  hp.insert(hp.end(), e.begin(), e.end());
  hp.insert(hp.end(), dby.begin(), dby.end());
  hp.insert(hp.end(), q.begin(), q.end());
  hp.insert(hp.end(), p.begin(), p.end());
  CK(cudaMemcpyAsync(plan, hp.data(), plan_words * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dbs, bs.data(), (nbl + 1) * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dbk, bk.data(), (nbl + 1) * 8, cudaMemcpyHostToDevice, c->st));
  unsigned long long hc[4] = {n, nbytes, 0, 0};
  CK(cudaMemcpyAsync(cur, hc, 32, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(err, 0, 16, c->st));
  if (nbytes) CK(cudaMemcpyAsync(dp, d_bytes, nbytes, cudaMemcpyDeviceToDevice, c->st));
  if (n) {
    const uint64_t *pe = plan, *pd = plan + (n_src + 1), *pq = pd + (n_src + 1), *pp = pq + q.size();
    k_xchg_import<<<grid_for(c, n), 256, 0, c->st>>>(d_desc, n, pe, n_src, pd, pq, pp, nbl, dd);
    CK(cudaPeekAtLastError());
  }
  c->tm = gkc_timings{};
  c->tm.launches = n ? 1 : 0;
  CK(cudaStreamSynchronize(c->st));  // the host plan arrays end with this call
  gkc_partition_view &v = c->pv;
  v = gkc_partition_view{};
  v.n_superkmers = n;
  v.n_packed_bytes = nbytes;
  v.n_kmers = bk[nbl];
  v.nbins = nbl;
  v.bin_skm_off = dbs;
  v.bin_kmer_off = dbk;
  v.skm_desc = dd;
  v.skm_minimizer = nullptr;  // minimizers do not travel
  v.packed = dp;
  c->part_packed = dp;
  c->part_nbytes_dev = nullptr;
  c->part_hpc_reads = nullptr;
  c->part_hpc_offs = nullptr;
  c->part_hpc_orig = nullptr;
  c->part_cap_skm = n + 1;
  c->part_cap_bytes = nbytes + 16;
  c->pp = *prm;
  c->have_part = true;
  c->have_count = false;
  graphs_invalidate(c);
  if (out) *out = v;
  return GKC_OK;
}
