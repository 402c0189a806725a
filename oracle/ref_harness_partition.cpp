// Reference harness, partition half.  TEST INFRASTRUCTURE (oracle/_ref).
// Drives the reference's kernels the way GenSuperkmerGPU does
// (gkc_cuda.cu:403-470) and feeds SKMStore::add_skms (superkmers.hpp:167-186)
// as process_reads_count does (experiment.cpp:85-88).
#include "ref_shim.h"

using std::atomic;  // CalcSKMPartSize_instream's signature names atomic<size_t>
#include "ref_kernels.inc"  // generated from the reference by extract_ref.py

#include <cassert>
#include <memory>
#include <mutex>
#include <thread>

#include "superkmers.hpp"
#include "thread_pool.hpp"
#include "ref_harness.h"

namespace {

// One batch through the reference kernels; the superkmers go to the stores,
// or, with part_sizes set, only their bases per bin to CalcSKMPartSize_instream
// (the process_func of process_reads_v2, experiment.cpp:51).
void run_batch(const char *reads, const uint64_t *offs, int64_t beg, int64_t end, int k, int p,
               bool hpc, std::vector<SKMStore *> &stores, std::atomic<size_t> *part_sizes = nullptr,
               int nbins = 0) {
  T_read_cnt cnt = (T_read_cnt)(end - beg);
  size_t bsize = offs[end] - offs[beg];
  std::vector<char> d_reads(reads + offs[beg], reads + offs[end]);
  d_reads.push_back(0);
  std::vector<T_CSR_cap> d_offs(offs + beg, offs + end + 1);
  std::vector<T_read_len> d_len(cnt), d_hpc(bsize + 1), d_mm_len(1);
  std::vector<T_minimizer> d_mm(bsize + 1, 0);
  std::vector<T_read_len> d_skm(bsize + 3, 0);
  MoveOffset(cnt, d_offs.data(), 0);
  if (hpc) {
    // One "grid" per read: the kernel's start index uses the thread id
    // (gkc_cuda.cu:180), which is the read id only for a grid of >= reads.
    for (T_read_cnt r = 0; r < cnt; r++)
      GPU_HPCEncoding(1, &d_len[r], d_reads.data(), &d_offs[r], true, d_hpc.data());
  } else {
    GPU_HPCEncoding(cnt, d_len.data(), d_reads.data(), d_offs.data(), false, nullptr);
  }
  GPU_GenMinimizer(cnt, d_len.data(), d_reads.data(), d_offs.data(), d_mm.data(), k, p);
  GPU_GenSKM(cnt, d_len.data(), d_offs.data(), d_mm.data(), d_skm.data(), k, p);
  if (part_sizes) {
    CalcSKMPartSize_instream(cnt, d_skm.data(), d_offs.data(), d_mm.data(), nbins, k, part_sizes);
    return;
  }
  SKMStore::add_skms(stores, (T_kvalue)k, cnt, d_reads.data(), d_offs.data(), d_skm.data(),
                     d_mm.data());
}

int partition_into(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int hpc,
                   int batch_reads, int n_threads, std::vector<SKMStore *> &stores) {
  if (batch_reads < 1) batch_reads = 2048;
  if (n_threads < 1) n_threads = 1;
  ThreadPool<void> tp(n_threads);
  for (int64_t b = 0; b < n_reads; b += batch_reads) {
    int64_t e = std::min<int64_t>(n_reads, b + batch_reads);
    tp.commit_task([=, &stores]() { run_batch(reads, offs, b, e, k, p, hpc != 0, stores); });
  }
  tp.finish();
  return 0;
}

}  // namespace

extern "C" int ref_partition(const char *reads, const uint64_t *offs, int64_t n_reads, int k,
                             int p, int hpc, int nbins, int batch_reads, int n_threads,
                             ref_skms *out) {
  std::memset(out, 0, sizeof(*out));
  std::vector<SKMStore *> stores;
  for (int i = 0; i < nbins; i++) stores.push_back(new SKMStore());
  partition_into(reads, offs, n_reads, k, p, hpc, batch_reads, n_threads, stores);
  std::vector<uint32_t> bin, len;
  std::vector<uint64_t> boff;
  std::vector<uint8_t> bytes;
  for (int b = 0; b < nbins; b++) {
    CRead<T_skm_len> c;
    while (stores[b]->skms.try_dequeue(c)) {
      size_t nb = CRead<T_skm_len>::compressed_length(c.len);
      bin.push_back((uint32_t)b);
      len.push_back(c.len);
      boff.push_back(bytes.size());
      bytes.insert(bytes.end(), c.compressed_read.get(), c.compressed_read.get() + nb);
    }
    delete stores[b];
  }
  out->n_skm = bin.size();
  out->n_bytes = bytes.size();
  out->bin = (uint32_t *)malloc(sizeof(uint32_t) * (bin.size() + 1));
  out->len = (uint32_t *)malloc(sizeof(uint32_t) * (bin.size() + 1));
  out->byte_off = (uint64_t *)malloc(sizeof(uint64_t) * (bin.size() + 1));
  out->bytes = (uint8_t *)malloc(bytes.size() + 1);
  std::copy(bin.begin(), bin.end(), out->bin);
  std::copy(len.begin(), len.end(), out->len);
  std::copy(boff.begin(), boff.end(), out->byte_off);
  std::copy(bytes.begin(), bytes.end(), out->bytes);
  return 0;
}

extern "C" int ref_partition_sizes(const char *reads, const uint64_t *offs, int64_t n_reads, int k,
                                   int p, int hpc, int nbins, int batch_reads, int n_threads,
                                   uint64_t *sizes) {
  if (nbins < 1 || nbins > 512) return 1;  // experiment.cpp:57 holds 512 counters
  std::atomic<size_t> part[512];
  for (int i = 0; i < nbins; i++) part[i] = 0;
  if (batch_reads < 1) batch_reads = 2048;
  std::vector<SKMStore *> none;
  {
    ThreadPool<void> tp(n_threads < 1 ? 1 : n_threads);
    for (int64_t b = 0; b < n_reads; b += batch_reads) {
      int64_t e = std::min<int64_t>(n_reads, b + batch_reads);
      tp.commit_task([=, &none, &part]() { run_batch(reads, offs, b, e, k, p, hpc != 0, none, part, nbins); });
    }
    tp.finish();
  }
  for (int i = 0; i < nbins; i++) sizes[i] = part[i];
  return 0;
}

extern "C" void ref_skms_free(ref_skms *s) {
  free(s->bin);
  free(s->len);
  free(s->byte_off);
  free(s->bytes);
  std::memset(s, 0, sizeof(*s));
}

// Declared in the count half.
size_t ref_count_store(int k, SKMStore *store, std::vector<uint64_t> *keys,
                       std::vector<uint64_t> *runs);

extern "C" int ref_pipeline(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                            int hpc, int nbins, int batch_reads, int n_threads,
                            uint64_t *distinct_out, uint64_t *kmers_out) {
  std::vector<SKMStore *> stores;
  for (int i = 0; i < nbins; i++) stores.push_back(new SKMStore());
  partition_into(reads, offs, n_reads, k, p, hpc, batch_reads, n_threads, stores);
  uint64_t kmers = 0;  // sum over superkmers of (len - k + 1)
  for (int b = 0; b < nbins; b++)
    kmers += stores[b]->tot_size - stores[b]->skms.size_approx() * (uint64_t)(k - 1);
  // Phase 2 as gen_skm_and_count_with_TP (experiment.cpp:189-208).
  ThreadPool<size_t> tp(n_threads < 1 ? 1 : n_threads);
  std::vector<std::future<size_t>> fut(nbins);
  for (int b = 0; b < nbins; b++)
    fut[b] = tp.commit_task([=, &stores]() { return ref_count_store(k, stores[b], nullptr, nullptr); });
  tp.finish();
  uint64_t distinct = 0;
  for (int b = 0; b < nbins; b++) distinct += fut[b].get();
  *distinct_out = distinct;
  *kmers_out = kmers;
  return 0;
}

// The same CPU path with the sorted (k-mer, count) lists kept: per bin, the
// sorted keys and run lengths kmc_counting_GPU computes (captured as in
// ref_count_bins), for comparing a GPU run on the same reads.
extern "C" int ref_pipeline_counts(const char *reads, const uint64_t *offs, int64_t n_reads, int k,
                                   int p, int hpc, int nbins, int batch_reads, int n_threads,
                                   uint64_t *kmers_out, ref_counts *out) {
  std::memset(out, 0, sizeof(*out));
  if (k < 1 || k > 32) return -1;
  std::vector<SKMStore *> stores;
  for (int i = 0; i < nbins; i++) stores.push_back(new SKMStore());
  partition_into(reads, offs, n_reads, k, p, hpc, batch_reads, n_threads, stores);
  uint64_t kmers = 0;
  for (int b = 0; b < nbins; b++)
    kmers += stores[b]->tot_size - stores[b]->skms.size_approx() * (uint64_t)(k - 1);
  std::vector<std::vector<uint64_t>> keys(nbins), runs(nbins);
  std::vector<size_t> ret(nbins, 0);
  {
    ThreadPool<size_t> tp(n_threads < 1 ? 1 : n_threads);
    std::vector<std::future<size_t>> fut(nbins);
    for (int b = 0; b < nbins; b++)
      fut[b] = tp.commit_task([=, &stores, &keys, &runs]() { return ref_count_store(k, stores[b], &keys[b], &runs[b]); });
    tp.finish();
    for (int b = 0; b < nbins; b++) ret[b] = fut[b].get();
  }
  uint64_t total = 0;
  for (int b = 0; b < nbins; b++) total += ret[b];
  out->nbins = (uint32_t)nbins;
  out->n_distinct = total;
  out->bin_off = (uint64_t *)malloc(sizeof(uint64_t) * (nbins + 1));
  out->keys = (uint64_t *)malloc(sizeof(uint64_t) * (total + 1));
  out->counts = (uint32_t *)malloc(sizeof(uint32_t) * (total + 1));
  out->returned = (uint64_t *)malloc(sizeof(uint64_t) * (nbins + 1));
  uint64_t w = 0;
  for (int b = 0; b < nbins; b++) {
    out->bin_off[b] = w;
    out->returned[b] = ret[b];
    for (size_t i = 0; i < ret[b]; i++) {
      out->keys[w] = keys[b][i];
      const uint64_t r = runs[b][i];
      out->counts[w] = r > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)r;
      w++;
    }
    std::vector<uint64_t>().swap(keys[b]);
    std::vector<uint64_t>().swap(runs[b]);
  }
  out->bin_off[nbins] = w;
  *kmers_out = kmers;
  return 0;
}
