// Test driver for the GKC drop-in (gkc_b200/compat/gkc_compat.cpp), written
// the way GKC's own driver uses its two GPU entry points
// (process_reads_count and gen_skm_and_count_with_TP, experiment.cpp:76-89,
// 156-219): reads into a PinnedCSR, GenSuperkmerGPU with SKMStore::add_skms
// as the callback, then kmc_counting_GPU per bin from a pool of threads.
//
// usage: compat_driver reads.bin k p hpc nbins threads out.bin
//   reads.bin: uint64 n_reads, uint64 offs[n_reads + 1], the bytes
//   out.bin:   per bin: uint64 n_superkmers, then (uint32 len, bytes) each;
//              then per bin: uint64 returned distinct count, uint64 n_pairs,
//              then (uint64 k-mer, uint32 count) each
#include <cstdio>
#include <cstdlib>
#include <future>
#include <thread>
#include <vector>

#include "gkc_cuda.hpp"
#include "kmer_counting.hpp"

int main(int argc, char **argv) {
  if (argc != 8) {
    std::fprintf(stderr, "usage: compat_driver reads.bin k p hpc nbins threads out.bin\n");
    return 2;
  }
  const int k = std::atoi(argv[2]), p = std::atoi(argv[3]), hpc = std::atoi(argv[4]);
  const int nbins = std::atoi(argv[5]), threads = std::atoi(argv[6]);
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  uint64_t n = 0;
  if (std::fread(&n, 8, 1, f) != 1) return 3;
  std::vector<uint64_t> offs(n + 1);
  if (std::fread(offs.data(), 8, n + 1, f) != n + 1) return 3;
  std::vector<char> bytes(offs[n] + 1);
  if (offs[n] && std::fread(bytes.data(), 1, offs[n], f) != offs[n]) return 3;
  std::fclose(f);

  std::vector<ReadPtr> reads(n);
  for (uint64_t r = 0; r < n; r++) reads[r] = ReadPtr{bytes.data() + offs[r], (T_read_len)(offs[r + 1] - offs[r])};
  PinnedCSR pinned(reads);
  std::vector<SKMStore *> stores;
  for (int b = 0; b < nbins; b++) stores.push_back(new SKMStore());
  CUDAParams gpars;
  gpars.device_id = 0;
  gpars.n_streams = 6;
  gpars.NUM_BLOCKS_PER_GRID = 8;
  gpars.NUM_THREADS_PER_BLOCK = 256;
  std::function<void(T_h_data)> add = [&stores, k](T_h_data hd) {
    SKMStore::add_skms(stores, (T_kvalue)k, hd.reads_cnt, hd.reads, hd.reads_offs, hd.superkmer_offs,
                       hd.minimizers);
  };
  GenSuperkmerGPU(pinned, k, p, hpc != 0, gpars, CountTask::SKMPartition, nbins, add);

  FILE *o = std::fopen(argv[7], "wb");
  if (!o) return 4;
  // the partition: each store drained, written, and refilled for counting
  for (int b = 0; b < nbins; b++) {
    std::vector<CRead<T_skm_len>> got;
    CRead<T_skm_len> c;
    while (stores[b]->skms.try_dequeue(c)) got.push_back(c);
    uint64_t cnt = got.size();
    std::fwrite(&cnt, 8, 1, o);
    for (auto &x : got) {
      uint32_t len = x.len;
      std::fwrite(&len, 4, 1, o);
      std::fwrite(x.compressed_read.get(), 1, CRead<T_skm_len>::compressed_length(x.len), o);
      stores[b]->skms.enqueue(x);
    }
  }
  // counting per bin from a pool of threads, as gen_skm_and_count_with_TP does
  std::vector<std::vector<T_kmc>> res(nbins);
  std::vector<size_t> ret(nbins, 0);
  std::vector<std::thread> pool;
  std::atomic<int> next{0};
  for (int t = 0; t < (threads < 1 ? 1 : threads); t++)
    pool.emplace_back([&]() {
      for (int b; (b = next++) < nbins;) ret[b] = kmc_counting_GPU((T_kvalue)k, *stores[b], 0, 1, 65535, res[b]);
    });
  for (auto &th : pool) th.join();
  for (int b = 0; b < nbins; b++) {
    uint64_t r = ret[b], m = res[b].size();
    std::fwrite(&r, 8, 1, o);
    std::fwrite(&m, 8, 1, o);
    for (auto &x : res[b]) {
      uint64_t key = x.kmer;
      uint32_t cnt = x.cnt;
      std::fwrite(&key, 8, 1, o);
      std::fwrite(&cnt, 4, 1, o);
    }
  }
  std::fclose(o);
  return 0;
}
