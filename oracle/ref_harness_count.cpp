// Reference harness, count half.  TEST INFRASTRUCTURE (oracle/_ref).
// Compiles the reference's kmer_counting.cu against Thrust's host (CPP)
// backend.  kmc_counting_GPU computes the sorted k-mer array and the run
// starts (kmer_counting.cu:135,174-175) but drops them; the MAX_KMER_CNT
// macro below is expanded at kmer_counting.cu:185, inside its count loop,
// where it records (sorted_kmers_h[idx_h[i]], run length) before yielding
// the reference's clamp value.
#define THRUST_DEVICE_SYSTEM THRUST_DEVICE_SYSTEM_CPP
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/remove.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/transform.h>

// The reference's functors are marked __host__ __device__ for nvcc.
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif

#include <cstdint>
#include <cstring>
#include <future>
#include <vector>

#include "types.h"

struct ref_capture_buf {
  std::vector<uint64_t> *keys;
  std::vector<uint64_t> *runs;
};
static thread_local ref_capture_buf ref_cap = {nullptr, nullptr};

static inline int ref_capture(unsigned long long key, long long run, long long i) {
  if (ref_cap.keys) {
    if ((size_t)i >= ref_cap.keys->size()) {
      ref_cap.keys->resize(i + 1);
      ref_cap.runs->resize(i + 1);
    }
    (*ref_cap.keys)[i] = key;
    (*ref_cap.runs)[i] = (uint64_t)run;
  }
  return 0;
}

#define MAX_KMER_CNT                                                                       \
  (ref_capture(sorted_kmers_h[idx_h[i]], (long long)(idx_h[i + 1] - idx_h[i]), (long long)i), \
   (T_kmer_cnt)0xFFFFFFFFu)

#include "kmer_counting.cu"

#undef MAX_KMER_CNT

#include "thread_pool.hpp"
#include "ref_harness.h"

size_t ref_count_store(int k, SKMStore *store, std::vector<uint64_t> *keys,
                       std::vector<uint64_t> *runs) {
  if (store->tot_size == 0) {  // kmc_counting_GPU returns before its delete (:74)
    delete store;
    return 0;
  }
  ref_cap.keys = keys;
  ref_cap.runs = runs;
  std::vector<T_kmc> unused;
  size_t nd = kmc_counting_GPU((T_kvalue)k, *store, 0, 1, 1000, unused);
  ref_cap.keys = nullptr;
  ref_cap.runs = nullptr;
  return nd;
}

extern "C" int ref_count_bins(const ref_skms *s, int k, int nbins, int n_threads,
                              ref_counts *out) {
  std::memset(out, 0, sizeof(*out));
  if (k < 1 || k > 32) return -1;
  std::vector<std::vector<uint64_t>> idx(nbins);
  for (uint64_t i = 0; i < s->n_skm; i++) idx[s->bin[i]].push_back(i);
  std::vector<std::vector<uint64_t>> keys(nbins), runs(nbins);
  std::vector<size_t> ret(nbins, 0);
  {
    ThreadPool<size_t> tp(n_threads < 1 ? 1 : n_threads);
    std::vector<std::future<size_t>> fut(nbins);
    for (int b = 0; b < nbins; b++) {
      fut[b] = tp.commit_task([&, b]() {
        SKMStore *st = new SKMStore();
        for (uint64_t i : idx[b]) {
          st->skms.enqueue(CRead<T_skm_len>((T_skm_len)s->len[i], s->bytes + s->byte_off[i]));
          st->tot_size += s->len[i];
        }
        return ref_count_store(k, st, &keys[b], &runs[b]);
      });
    }
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
      uint64_t r = runs[b][i];
      out->counts[w] = r > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)r;
      w++;
    }
  }
  out->bin_off[nbins] = w;
  return 0;
}

extern "C" void ref_counts_free(ref_counts *c) {
  free(c->bin_off);
  free(c->keys);
  free(c->counts);
  free(c->returned);
  std::memset(c, 0, sizeof(*c));
}
