// Drop-in definitions of GKC's GPU entry points over the gkc-b200 C ABI.
//
// A GKC build compiles this file (C++14, with GKC's own headers on the
// include path) in place of its gkc_cuda.cu and kmer_counting.cu, and links
// libgkc_b200.so.  It defines what those two files define and gkc_cuda.hpp /
// kmer_counting.hpp declare:
//   PinnedCSR (gkc_cuda.hpp:33-46; gkc_cuda.cu:103-143), GPUReset
//   (gkc_cuda.cu:367-373), CalcSKMPartSize_instream (gkc_cuda.cu:350-365),
//   GenSuperkmerGPU (gkc_cuda.hpp:58-61; gkc_cuda.cu:376-541) and
//   kmc_counting_GPU (kmer_counting.hpp:9-12; kmer_counting.cu:59-199).
// Behaviour kept from the reference:
//   * GenSuperkmerGPU hands process_func one T_h_data per batch of
//     NUM_BLOCKS_PER_GRID * NUM_THREADS_PER_BLOCK reads, in read order, on the
//     calling thread, valid only during the call: `reads` points into the
//     caller's CSR (with HPC, each read's compressed bases are written over
//     the start of its own bytes), `reads_offs` into the caller's offsets
//     (not rebased), `minimizers[i]` is the minimizer of the window starting
//     at batch byte i, and each read's slice of `superkmer_offs` lists its
//     superkmer starts, then the end (read length - k + 1), then 0
//     (gkc_cuda.cu:298-324).  `read_len` holds the (HPC) read lengths and
//     `hpc_orig_pos` each kept base's original position in its read.
//   * kmc_counting_GPU drains and deletes the store and returns the bin's
//     distinct canonical k-mers (k <= 32).
//   * Any error prints a message and exits the process, as CUDA_CHECK does
//     (gkc_cuda.hpp:4-9).
// Differences: all reads of a call go through the GPU in one pass (the
// batches only shape the callbacks); windows past a read's last k-mer hold
// minimizer 0xFFFFFFFF where the reference leaves them unset; a read
// shorter than k lists no superkmer (the reference's list for it starts with
// a non-positive end, gkc_cuda.cu:320); kmc_counting_GPU also fills
// kmc_result_curthread with the (k-mer, count) pairs whose counts lie in
// [kmer_min_freq, kmer_max_freq] (the filter the reference declares but
// leaves commented out, kmer_counting.cu:188-190), while its return value is
// the unfiltered distinct count, as the reference's is.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "gkc_cuda.hpp"
#include "kmer_counting.hpp"

#include "gkc/gkc.h"

namespace {

[[noreturn]] void die(const char *what, const std::string &detail) {
  std::fprintf(stderr, "gkc-b200: %s failed: %s\n", what, detail.c_str());
  std::exit(1);
}

void cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(what, cudaGetErrorString(e));
}

// One context per concurrent caller: the reference calls both entry points
// from several threads at once (read_loader.hpp:473,494; experiment.cpp:197).
std::mutex g_mu;
std::vector<std::pair<int, gkc_ctx *>> g_idle;

gkc_ctx *acquire(int dev) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (size_t i = 0; i < g_idle.size(); i++)
      if (g_idle[i].first == dev) {
        gkc_ctx *c = g_idle[i].second;
        g_idle.erase(g_idle.begin() + (long)i);
        return c;
      }
  }
  gkc_ctx *c = nullptr;
  const gkc_status s = gkc_ctx_create(dev, 0, &c);
  if (s != GKC_OK) die("gkc_ctx_create", gkc_status_string(s));
  return c;
}

void release(int dev, gkc_ctx *c) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_idle.emplace_back(dev, c);
}

void check(gkc_ctx *c, gkc_status s, const char *what) {
  if (s != GKC_OK) die(what, std::string(gkc_status_string(s)) + ": " + gkc_ctx_last_error(c));
}

template <typename T>
T *dev_alloc(size_t n) {
  void *p = nullptr;
  cuda_ok(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
  return static_cast<T *>(p);
}

}  // namespace

// ------------------------------------------------------------- PinnedCSR

PinnedCSR::PinnedCSR(vector<string> &reads) {
  n_reads = (T_read_cnt)reads.size();
  size_capacity = 0;
  for (const string &r : reads) size_capacity += r.size();
  cuda_ok(cudaHostAlloc((void **)&reads_offs, (n_reads + 1) * sizeof(T_CSR_cap), cudaHostAllocDefault),
          "cudaHostAlloc");
  cuda_ok(cudaHostAlloc((void **)&reads_CSR, size_capacity + 1, cudaHostAllocDefault), "cudaHostAlloc");
  T_CSR_cap o = 0;
  reads_offs[0] = 0;
  for (T_read_cnt i = 0; i < n_reads; i++) {
    std::memcpy(reads_CSR + o, reads[i].data(), reads[i].size());
    o += reads[i].size();
    reads_offs[i + 1] = o;
  }
}

PinnedCSR::PinnedCSR(vector<ReadPtr> &reads, bool keep_original) {
  (void)keep_original;
  n_reads = (T_read_cnt)reads.size();
  size_capacity = 0;
  for (const ReadPtr &r : reads) size_capacity += (T_CSR_cap)r.len;
  cuda_ok(cudaHostAlloc((void **)&reads_offs, (n_reads + 1) * sizeof(T_CSR_cap), cudaHostAllocDefault),
          "cudaHostAlloc");
  cuda_ok(cudaHostAlloc((void **)&reads_CSR, size_capacity + 1, cudaHostAllocDefault), "cudaHostAlloc");
  T_CSR_cap o = 0;
  reads_offs[0] = 0;
  for (T_read_cnt i = 0; i < n_reads; i++) {
    std::memcpy(reads_CSR + o, reads[i].read, (size_t)reads[i].len);
    o += (T_CSR_cap)reads[i].len;
    reads_offs[i + 1] = o;
  }
}

PinnedCSR::~PinnedCSR() {
  cudaFreeHost(reads_offs);
  cudaFreeHost(reads_CSR);
}

// ------------------------------------------------------------- helpers

void GPUReset(int did) {
  cuda_ok(cudaSetDevice(did), "cudaSetDevice");
  cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
}

// Bases of each bin's superkmers, each with its k-1 overlap, added up.
void CalcSKMPartSize_instream(T_read_cnt reads_cnt, T_read_len *superkmer_offs, T_CSR_cap *reads_offs,
                              T_minimizer *minimizers, int n_partitions, int k, atomic<size_t> part_sizes[]) {
  const T_CSR_cap base = reads_offs[0];
  for (T_read_cnt r = 0; r < reads_cnt; r++) {
    const T_CSR_cap ro = reads_offs[r] - base;
    for (T_CSR_cap j = ro + 1; superkmer_offs[j] != 0; j++) {
      const T_read_len s = superkmer_offs[j - 1];
      part_sizes[minimizers[ro + (T_CSR_cap)s] % (T_minimizer)n_partitions] +=
          (size_t)(superkmer_offs[j] - s + k - 1);
    }
  }
}

// ------------------------------------------------------- GenSuperkmerGPU

void GenSuperkmerGPU(PinnedCSR &pinned_reads, int K_kmer, int P_minimizer, bool HPC, CUDAParams gpars,
                     CountTask task, int SKM_partitions, std::function<void(T_h_data)> process_func) {
  (void)task;            // the reference handles every task alike (SaveSKMs_instream is empty)
  (void)SKM_partitions;  // bins are the callback's business (SKMStore::add_skms)
  const T_read_cnt n = pinned_reads.n_reads;
  if (n <= 0) return;
  cuda_ok(cudaSetDevice(gpars.device_id), "cudaSetDevice");
  gkc_ctx *c = acquire(gpars.device_id);
  gkc_ctx_set_filter(c, GKC_FILTER_NEW2);
  const T_CSR_cap *offs = pinned_reads.reads_offs;
  const uint64_t base = offs[0], nb = offs[n] - base;
  std::vector<uint64_t> h_offs((size_t)n + 1);
  for (T_read_cnt r = 0; r <= n; r++) h_offs[r] = offs[r] - base;

  char *d_reads = dev_alloc<char>(nb + 64);
  uint64_t *d_offs = dev_alloc<uint64_t>((size_t)n + 1);
  uint32_t *d_mm = dev_alloc<uint32_t>(nb + 1);
  cuda_ok(cudaMemcpy(d_reads, pinned_reads.reads_CSR + base, nb, cudaMemcpyHostToDevice), "cudaMemcpy");
  cuda_ok(cudaMemcpy(d_offs, h_offs.data(), 8 * ((size_t)n + 1), cudaMemcpyHostToDevice), "cudaMemcpy");

  std::vector<T_read_len> read_len((size_t)n);
  std::vector<T_read_len> orig;
  std::vector<uint32_t> mm(nb + 1);
  gkc_params prm{K_kmer, P_minimizer, 0, 1};
  if (HPC) {
    // compressed reads in a CSR of their own, mapped back below
    char *d_h = dev_alloc<char>(nb + 64);
    uint64_t *d_hoffs = dev_alloc<uint64_t>((size_t)n + 1);
    int32_t *d_orig = dev_alloc<int32_t>(nb + 1);
    check(c, gkc_hpc_device(c, d_reads, nb, d_offs, (uint64_t)n, d_h, d_hoffs, d_orig), "gkc_hpc_device");
    std::vector<uint64_t> ho((size_t)n + 1);
    cuda_ok(cudaMemcpy(ho.data(), d_hoffs, 8 * ((size_t)n + 1), cudaMemcpyDeviceToHost), "cudaMemcpy");
    const uint64_t hnb = ho[n];
    check(c, gkc_minimizers_device(c, &prm, d_h, hnb, d_hoffs, (uint64_t)n, d_mm, nullptr, nullptr),
          "gkc_minimizers_device");
    std::vector<char> hr(hnb + 1);
    std::vector<uint32_t> hmm(hnb + 1);
    std::vector<int32_t> hor(hnb + 1);
    cuda_ok(cudaMemcpy(hr.data(), d_h, hnb, cudaMemcpyDeviceToHost), "cudaMemcpy");
    cuda_ok(cudaMemcpy(hmm.data(), d_mm, 4 * hnb, cudaMemcpyDeviceToHost), "cudaMemcpy");
    cuda_ok(cudaMemcpy(hor.data(), d_orig, 4 * hnb, cudaMemcpyDeviceToHost), "cudaMemcpy");
    orig.assign(nb + 1, 0);
    char *csr = pinned_reads.reads_CSR + base;
    for (T_read_cnt r = 0; r < n; r++) {
      const uint64_t L = ho[r + 1] - ho[r];
      read_len[r] = (T_read_len)L;
      std::memcpy(csr + h_offs[r], hr.data() + ho[r], L);
      std::memcpy(mm.data() + h_offs[r], hmm.data() + ho[r], 4 * L);
      for (uint64_t j = 0; j < L; j++) orig[h_offs[r] + j] = hor[ho[r] + j];
    }
    cudaFree(d_h);
    cudaFree(d_hoffs);
    cudaFree(d_orig);
  } else {
    check(c, gkc_minimizers_device(c, &prm, d_reads, nb, d_offs, (uint64_t)n, d_mm, nullptr, nullptr),
          "gkc_minimizers_device");
    cuda_ok(cudaMemcpy(mm.data(), d_mm, 4 * nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (T_read_cnt r = 0; r < n; r++) read_len[r] = (T_read_len)(h_offs[r + 1] - h_offs[r]);
  }
  cudaFree(d_reads);
  cudaFree(d_offs);
  cudaFree(d_mm);
  release(gpars.device_id, c);

  // superkmer starts per read: a new superkmer wherever the minimizer value
  // changes between neighbouring windows, then the end, then 0
  std::vector<T_read_len> skm(nb + 3, 0);
  for (T_read_cnt r = 0; r < n; r++) {
    T_read_len *s = skm.data() + h_offs[r];
    const uint32_t *m = mm.data() + h_offs[r];
    const T_read_len L = read_len[r];
    s[0] = 0;
    if (L < K_kmer) {
      s[1] = 0;
      continue;
    }
    T_read_len cnt = 0;
    for (T_read_len i = 1; i <= L - K_kmer; i++)
      if (m[i] != m[i - 1]) s[++cnt] = i;
    s[cnt + 1] = L - K_kmer + 1;
    s[cnt + 2] = 0;
  }

  const T_read_cnt per = std::max(1, gpars.NUM_BLOCKS_PER_GRID * gpars.NUM_THREADS_PER_BLOCK);
  for (T_read_cnt b = 0; b < n; b += per) {
    const T_read_cnt e = std::min(n, b + per);
    const uint64_t o = h_offs[b];
    T_h_data hd;
    hd.reads_cnt = e - b;
    hd.reads = pinned_reads.reads_CSR + base + o;
    hd.reads_offs = pinned_reads.reads_offs + b;
    hd.read_len = read_len.data() + b;
    hd.hpc_orig_pos = HPC ? orig.data() + o : nullptr;
    hd.minimizers = mm.data() + o;
    hd.superkmer_offs = skm.data() + o;
    process_func(hd);
  }
}

// ------------------------------------------------------- kmc_counting_GPU

size_t kmc_counting_GPU(T_kvalue k, SKMStore &skms_store, int gpuid, unsigned short kmer_min_freq,
                        unsigned short kmer_max_freq, vector<T_kmc> &kmc_result_curthread) {
  if (k < 1 || k > 32) die("kmc_counting_GPU", "k must be in [1, 32] (64-bit k-mers)");
  std::vector<uint32_t> lens;
  std::vector<uint8_t> packed;
  {
    const size_t BULK = 10000;
    std::vector<CRead<T_skm_len>> bulk(BULK);
    size_t got;
    while ((got = skms_store.try_pop_skm_bulk(bulk.data(), BULK)) != 0) {
      for (size_t i = 0; i < got; i++) {
        const size_t nbyte = CRead<T_skm_len>::compressed_length(bulk[i].len);
        lens.push_back(bulk[i].len);
        const uint8_t *p = reinterpret_cast<const uint8_t *>(bulk[i].compressed_read.get());
        packed.insert(packed.end(), p, p + nbyte);
      }
    }
  }
  delete &skms_store;  // the reference takes the store over (kmer_counting.cu:197)
  if (lens.empty()) return 0;
  cuda_ok(cudaSetDevice(gpuid), "cudaSetDevice");
  gkc_ctx *c = acquire(gpuid);
  uint64_t nd = 0;
  check(c, gkc_count_superkmers_host(c, k, lens.data(), packed.data(), lens.size(), GKC_MODE_BATCHED, &nd),
        "gkc_count_superkmers_host");
  std::vector<uint64_t> keys(nd + 1), bin_off(2);
  std::vector<uint32_t> counts(nd + 1);
  check(c, gkc_count_copy_out(c, bin_off.data(), keys.data(), counts.data()), "gkc_count_copy_out");
  release(gpuid, c);
  for (uint64_t i = 0; i < nd; i++)
    if (counts[i] >= kmer_min_freq && counts[i] <= kmer_max_freq) kmc_result_curthread.push_back(T_kmc{keys[i], counts[i]});
  return (size_t)nd;
}
