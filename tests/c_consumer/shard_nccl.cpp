// The bin-sharded count driven from C++ over NCCL, through the C ABI only:
// what a native caller with one process (or thread) per GPU writes in place
// of gkc_b200/shard.py.  Compiled (not run) by tests/test_lib.py.
//
// Every rank: partition its reads, pack its superkmers by bin owner, exchange
// run sizes and per-bin counts, then descriptors and bytes, with grouped
// ncclSend / ncclRecv; import the received runs and count the owned bins
// [bin_lo[rank], bin_lo[rank+1]).
#include <cuda_runtime.h>
#include <nccl.h>

#include <cstdint>
#include <vector>

#include "gkc/gkc.h"

namespace {

// Device memory owned by the caller, freed on every return path.
struct DeviceBuffer {
  void *p = nullptr;
  explicit DeviceBuffer(size_t bytes) {
    if (cudaMalloc(&p, bytes) != cudaSuccess) p = nullptr;
  }
  ~DeviceBuffer() {
    if (p) cudaFree(p);
  }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// One all-to-all of byte runs: send[d] bytes from sbuf + soff[d] to rank d,
// recv[s] bytes from rank s into rbuf + roff[s].
ncclResult_t all_to_all_bytes(const uint8_t *sbuf, const std::vector<uint64_t> &send,
                              const std::vector<uint64_t> &soff, uint8_t *rbuf,
                              const std::vector<uint64_t> &recv, const std::vector<uint64_t> &roff,
                              ncclComm_t comm, cudaStream_t st) {
  const int world = (int)send.size();
  ncclResult_t r = ncclGroupStart();
  for (int p = 0; p < world && r == ncclSuccess; p++) {
    if (send[p]) r = ncclSend(sbuf + soff[p], send[p], ncclUint8, p, comm, st);
    if (r == ncclSuccess && recv[p]) r = ncclRecv(rbuf + roff[p], recv[p], ncclUint8, p, comm, st);
  }
  ncclResult_t e = ncclGroupEnd();
  return r != ncclSuccess ? r : e;
}

std::vector<uint64_t> prefix(const std::vector<uint64_t> &v) {
  std::vector<uint64_t> o(v.size() + 1, 0);
  for (size_t i = 0; i < v.size(); i++) o[i + 1] = o[i] + v[i];
  return o;
}

}  // namespace

// Returns GKC_OK with the owned bins counted in ctx (gkc_count_copy_out),
// or the first failing status (GKC_ERR_CUDA for NCCL and CUDA failures).
gkc_status sharded_count(gkc_ctx *ctx, ncclComm_t comm, int rank, int world, const gkc_params *prm,
                         const char *d_reads, uint64_t n_bytes, const uint64_t *d_offs, uint64_t n_reads,
                         cudaStream_t st, gkc_count_view *out) {
  if (prm->nbins < world) return GKC_ERR_INVALID_ARG;
  gkc_status s = gkc_ctx_set_stream(ctx, st);
  if (s != GKC_OK) return s;
  gkc_partition_view pv;
  if ((s = gkc_partition_device(ctx, prm, d_reads, n_bytes, d_offs, n_reads, &pv)) != GKC_OK) return s;

  std::vector<uint32_t> bin_lo(world + 1);
  for (int r = 0; r <= world; r++) bin_lo[r] = (uint32_t)((uint64_t)r * prm->nbins / world);
  const uint32_t nbl = bin_lo[rank + 1] - bin_lo[rank];

  // the caller owns the exchange buffers
  DeviceBuffer send_desc(8 * (pv.n_superkmers + 1)), send_bytes(pv.n_packed_bytes + 16);
  if (!send_desc.p || !send_bytes.p) return GKC_ERR_OUT_OF_MEMORY;
  uint64_t *d_desc = send_desc.as<uint64_t>();
  uint8_t *d_bytes = send_bytes.as<uint8_t>();
  std::vector<uint64_t> skm_split(world), byte_split(world), bin_skm(prm->nbins), bin_kmers(prm->nbins);
  s = gkc_exchange_pack(ctx, (uint32_t)world, bin_lo.data(), d_desc, pv.n_superkmers, d_bytes,
                        pv.n_packed_bytes, skm_split.data(), byte_split.data(), bin_skm.data(), bin_kmers.data());
  if (s != GKC_OK) return s;

  // metadata: to rank d, [superkmers, bytes, per owned bin: superkmers, k-mers]
  std::vector<uint64_t> meta, msend(world), moff(world);
  for (int d = 0; d < world; d++) {
    moff[d] = meta.size() * 8;
    meta.push_back(skm_split[d]);
    meta.push_back(byte_split[d]);
    for (uint32_t b = bin_lo[d]; b < bin_lo[d + 1]; b++) meta.push_back(bin_skm[b]);
    for (uint32_t b = bin_lo[d]; b < bin_lo[d + 1]; b++) meta.push_back(bin_kmers[b]);
    msend[d] = meta.size() * 8 - moff[d];
  }
  const uint64_t run = 8 * (2 + 2 * (uint64_t)nbl);
  std::vector<uint64_t> mrecv(world, run), mroff(world);
  for (int p = 0; p < world; p++) mroff[p] = p * run;
  DeviceBuffer meta_buf(meta.size() * 8 + world * run);
  if (!meta_buf.p) return GKC_ERR_OUT_OF_MEMORY;
  uint64_t *d_meta = meta_buf.as<uint64_t>();
  uint8_t *d_mrecv = meta_buf.as<uint8_t>() + meta.size() * 8;
  if (cudaMemcpyAsync(d_meta, meta.data(), meta.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return GKC_ERR_CUDA;
  if (all_to_all_bytes(reinterpret_cast<uint8_t *>(d_meta), msend, moff, d_mrecv, mrecv, mroff, comm, st) !=
      ncclSuccess)
    return GKC_ERR_CUDA;
  std::vector<uint64_t> rmeta(world * (2 + 2 * nbl));
  if (cudaMemcpyAsync(rmeta.data(), d_mrecv, world * run, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return GKC_ERR_CUDA;

  std::vector<uint64_t> seg_skm(world), seg_bytes(world), seg_bin_skm(world * nbl), seg_bin_kmers(world * nbl);
  for (int p = 0; p < world; p++) {
    const uint64_t *m = rmeta.data() + p * (2 + 2 * nbl);
    seg_skm[p] = m[0];
    seg_bytes[p] = m[1];
    for (uint32_t b = 0; b < nbl; b++) {
      seg_bin_skm[p * nbl + b] = m[2 + b];
      seg_bin_kmers[p * nbl + b] = m[2 + nbl + b];
    }
  }

  // descriptors (as bytes, 8 per superkmer) and packed bytes
  std::vector<uint64_t> dsend(world), drecv(world);
  for (int p = 0; p < world; p++) {
    dsend[p] = 8 * skm_split[p];
    drecv[p] = 8 * seg_skm[p];
  }
  const std::vector<uint64_t> dsoff = prefix(dsend), droff = prefix(drecv);
  const std::vector<uint64_t> bsoff = prefix(byte_split), broff = prefix(seg_bytes);
  DeviceBuffer recv_desc(droff[world] + 8), recv_bytes(broff[world] + 16);
  if (!recv_desc.p || !recv_bytes.p) return GKC_ERR_OUT_OF_MEMORY;
  uint64_t *d_rdesc = recv_desc.as<uint64_t>();
  uint8_t *d_rbytes = recv_bytes.as<uint8_t>();
  if (all_to_all_bytes(reinterpret_cast<uint8_t *>(d_desc), dsend, dsoff, reinterpret_cast<uint8_t *>(d_rdesc),
                       drecv, droff, comm, st) != ncclSuccess ||
      all_to_all_bytes(d_bytes, byte_split, bsoff, d_rbytes, seg_bytes, broff, comm, st) != ncclSuccess)
    return GKC_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GKC_ERR_CUDA;

  gkc_params local = *prm;
  local.nbins = (int)nbl;
  s = gkc_partition_import(ctx, &local, (uint32_t)world, seg_bin_skm.data(), seg_bin_kmers.data(),
                           seg_bytes.data(), d_rdesc, d_rbytes, nullptr);
  if (s != GKC_OK) return s;
  return gkc_count_device(ctx, &local, GKC_MODE_BATCHED, out);
}
