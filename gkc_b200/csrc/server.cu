// Serving: continuous batching of counting jobs on one GPU.
//
// A server owns `max_running` worker slots.  Each slot is a thread with its
// own context (its own non-blocking stream and its own resident workspaces),
// so jobs admitted to different slots run on the device at the same time.
// A job is admitted when a slot is free and its HBM estimate
// (gkc_job_hbm_estimate plus its generated inputs) fits in what the budget
// has left; the slot's context is capped at that amount for the job.  The
// queue is served in arrival order, except that up to kMaxBypass later jobs
// that fit may start ahead of a head job that does not; after that the head
// waits alone until memory frees up.  A finished job's workspaces go back to
// the library's device memory pool, which keeps them for the next job of any
// slot (no allocation or free synchronises the device).  A finished job's
// result stays in device memory (copied out of the slot's workspaces, so the
// slot can take the next job at once) and counts against the budget until
// the job is released; gkc_server_copy_result copies it to host buffers.
//
// The reference has no serving layer; its driver counts one batch of reads at
// a time (process_reads_count, experiment.cpp:76-89).
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gkc/gkc.h"
#include "ctx.h"
#include "synth.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kMaxBypass = 8;

struct Job {
  uint64_t id = 0;
  gkc_params prm{};
  bool synth = false;
  int generator = 0;
  uint64_t seed = 0;
  std::vector<char> reads;
  std::vector<uint64_t> offs;  // host jobs: read offsets; long-read jobs: generated lengths
  uint64_t n_reads = 0, n_bases = 0;
  uint64_t est = 0;
  bool cancel = false;
  int bypassed = 0;
  gkc_job_info info{};
  // the result, in device memory from the library's pool until released:
  // bin offsets (nbins+1), keys (n_distinct * key_words), counts (n_distinct)
  void *d_res = nullptr;
  uint64_t res_bytes = 0;
};

struct Slot {
  gkc_ctx *ctx = nullptr;
  uint64_t charged = 0;  // HBM counted against the budget for this slot
  bool busy = false;
};

// Synthetic job shapes (the generators of the benchmark configurations).
constexpr uint32_t kShortLen = 150;
constexpr double kLongMedian = 8000.0, kLongSigma = 0.5;
constexpr uint32_t kLongMin = 1000, kLongMax = 50000;

uint64_t synth_genome_len(int gen, uint64_t n_bases) {
  if (gen == 2) return std::max<uint64_t>(n_bases / 30, 4 * kShortLen);  // 30x coverage
  if (gen == 3) return std::max<uint64_t>(n_bases / 20, 2 * kLongMax);   // 20x coverage
  return 0;
}

}  // namespace

struct gkc_server {
  int dev = 0;
  uint64_t budget = 0;
  int max_running = 1;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job *> queue;
  std::unordered_map<uint64_t, Job *> jobs;
  std::vector<Slot> slots;
  std::vector<std::thread> workers;
  int ready = 0;
  gkc_status init_status = GKC_OK;
  uint64_t next_id = 1, committed = 0;
  uint64_t held = 0;  // device bytes of finished jobs' results (in `committed`)
  bool stop = false;
  Clock::time_point t0 = Clock::now();

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  static bool finished(const Job *j) {
    return j->info.state == GKC_JOB_DONE || j->info.state == GKC_JOB_FAILED ||
           j->info.state == GKC_JOB_CANCELLED;
  }

  // Picks a queued job for idle slot `me` (lock held), or null.
  Job *pick(Slot &me) {
    const size_t limit = std::min<size_t>(queue.size(), kMaxBypass + 1);
    for (size_t i = 0; i < limit; i++) {
      if (i > 0 && queue[0]->bypassed >= kMaxBypass) break;
      Job *j = queue[i];
      const uint64_t need = std::max<uint64_t>(j->est, me.charged);
      if (committed - me.charged + need > budget) continue;
      for (size_t q = 0; q < i; q++) queue[q]->bypassed++;
      queue.erase(queue.begin() + i);
      committed = committed - me.charged + need;
      me.charged = need;
      return j;
    }
    return nullptr;
  }


  bool any_busy() const {
    for (const Slot &s : slots)
      if (s.busy) return true;
    return false;
  }

  void fail_head_if_impossible() {
    // a job that alone exceeds the budget can never start
    while (!queue.empty() && queue.front()->est > budget) {
      Job *j = queue.front();
      queue.pop_front();
      j->info.state = GKC_JOB_FAILED;
      j->info.status = GKC_ERR_BUDGET;
      j->info.end_s = now();
    }
  }

  void worker(int i);
  gkc_status run(gkc_ctx *c, Job *j, double *t_gen, double *t_pipe);
};

gkc_status gkc_server::run(gkc_ctx *c, Job *j, double *t_gen, double *t_pipe) {
  gkc_count_view cv{};
  gkc_status s;
  const double t0 = now();
  if (!j->synth) {
    s = gkc_pipeline_host(c, &j->prm, GKC_MODE_BATCHED, j->reads.data(), j->offs.data(), j->n_reads, &cv);
  } else {
    const uint64_t G = synth_genome_len(j->generator, j->n_bases);
    const uint64_t R = j->n_reads, nb = j->n_bases;
    char *reads = (char *)ws_get(c, "srv_reads", nb + 64, &s);
    if (s != GKC_OK) return s;
    uint64_t *offs = (uint64_t *)ws_get(c, "srv_offs", 8 * (R + 1), &s);
    if (s != GKC_OK) return s;
    uint8_t *genome = nullptr;
    if (G) {
      genome = (uint8_t *)ws_get(c, "srv_genome", G + 64, &s);
      if (s != GKC_OK) return s;
      gkc::synth_genome_dev(j->seed, G, 0.05, 0.01, genome, c->st);
    }
    if (j->generator == 1) {
      gkc::synth_iid_reads_dev(j->seed, R, kShortLen, 0.001, reads, offs, c->st);
    } else if (j->generator == 2) {
      gkc::synth_short_reads_dev(j->seed, genome, G, 0, R, kShortLen, 0.005, reads, offs, c->st);
    } else {
      if (cudaMemcpyAsync(offs, j->offs.data(), 8 * (R + 1), cudaMemcpyHostToDevice, c->st) != cudaSuccess)
        return ctx_cuda(c, cudaGetLastError(), "upload long-read offsets");
      gkc::synth_long_reads_dev(j->seed, genome, G, R, offs, reads, c->st);
    }
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return ctx_cuda(c, e, "synthetic reads");
    if (t_gen) {
      cudaStreamSynchronize(c->st);
      *t_gen = now() - t0;
    }
    s = gkc_pipeline_device(c, &j->prm, GKC_MODE_BATCHED, reads, nb, offs, R, nullptr, &cv);
  }
  if (t_pipe) *t_pipe = now() - t0;
  if (s != GKC_OK) return s;
  j->info.n_kmers = cv.n_kmers;
  j->info.n_distinct = cv.n_distinct;
  j->info.nbins = cv.nbins;
  j->info.key_words = cv.key_words;
  const uint64_t b_bo = 8 * (cv.nbins + 1), b_keys = 8 * cv.n_distinct * cv.key_words,
                 b_cnt = 4 * cv.n_distinct;
  j->res_bytes = (b_bo + b_keys + b_cnt + 511) & ~511ull;
  cudaError_t e = result_alloc(c->dev, &j->d_res, j->res_bytes, c->st);
  if (e != cudaSuccess) return ctx_cuda(c, e, "result buffer");
  char *r = static_cast<char *>(j->d_res);
  e = cudaMemcpyAsync(r, cv.bin_off, b_bo, cudaMemcpyDeviceToDevice, c->st);
  if (e == cudaSuccess && b_keys) e = cudaMemcpyAsync(r + b_bo, cv.keys, b_keys, cudaMemcpyDeviceToDevice, c->st);
  if (e == cudaSuccess && b_cnt)
    e = cudaMemcpyAsync(r + b_bo + b_keys, cv.counts, b_cnt, cudaMemcpyDeviceToDevice, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return ctx_cuda(c, e, "result copy");
  return GKC_OK;
}

void gkc_server::worker(int i) {
  gkc_ctx *c = nullptr;
  gkc_status s = gkc_ctx_create(dev, 0, &c);
  if (s == GKC_OK) c->one_shot = true;  // every job is a new input
  const bool debug = getenv("GKC_SERVER_DEBUG") != nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    slots[i].ctx = c;
    if (s != GKC_OK) init_status = s;
    ready++;
  }
  cv.notify_all();
  if (s != GKC_OK) return;
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    Job *j = nullptr;
    while (!stop) {
      fail_head_if_impossible();
      j = pick(slots[i]);
      if (j) break;
      cv.notify_all();  // waiters on failed jobs
      cv.wait(lk);
    }
    if (!j) break;
    slots[i].busy = true;
    j->info.state = GKC_JOB_RUNNING;
    j->info.start_s = now();
    j->info.hbm_bytes = slots[i].charged;
    c->budget = slots[i].charged;
    lk.unlock();
    const double t_run = now();
    double t_gen = 0, t_pipe = 0;
    gkc_status st = run(c, j, debug ? &t_gen : nullptr, debug ? &t_pipe : nullptr);
    if (debug)
      fprintf(stderr,
              "gkc server: job %llu slot %d bases %llu k %d hpc %d status %d (%s) run %.3f s gen %.3f pipe %.3f "
              "distinct %llu hbm %.2f GB\n",
              (unsigned long long)j->id, i, (unsigned long long)j->n_bases, j->prm.k, j->prm.hpc, (int)st,
              st == GKC_OK ? "" : gkc_ctx_last_error(c), now() - t_run, t_gen, t_pipe,
              (unsigned long long)j->info.n_distinct, slots[i].charged / 1e9);
    lk.lock();
    j->reads.clear();
    j->reads.shrink_to_fit();
    ws_release_all(c);  // the memory stays in the device pool for the next job
    if (st != GKC_OK || j->cancel) {
      if (j->d_res) cudaFreeAsync(j->d_res, c->st);
      j->d_res = nullptr;
      j->res_bytes = 0;
    }
    held += j->res_bytes;
    committed += j->res_bytes;
    j->info.end_s = now();
    j->info.status = st;
    j->info.state = j->cancel ? GKC_JOB_CANCELLED : (st == GKC_OK ? GKC_JOB_DONE : GKC_JOB_FAILED);
    const uint64_t resident = gkc_ctx_device_bytes(c);
    committed = committed - slots[i].charged + resident;
    slots[i].charged = resident;
    slots[i].busy = false;
    cv.notify_all();
  }
  slots[i].ctx = nullptr;
  lk.unlock();
  gkc_ctx_destroy(c);
}

extern "C" {

gkc_status gkc_server_create(int device_id, uint64_t hbm_budget_bytes, int max_running,
                             gkc_server **out) {
  if (!out || max_running < 1 || max_running > 64) return GKC_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return GKC_ERR_NO_DEVICE;
  }
  if (device_id < 0 || device_id >= n) return GKC_ERR_INVALID_ARG;
  if (hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    cudaSetDevice(device_id);
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return GKC_ERR_CUDA;
    hbm_budget_bytes = (uint64_t)(fr * 0.9);
  }
  gkc_server *S = new gkc_server();
  S->dev = device_id;
  S->budget = hbm_budget_bytes;
  S->max_running = max_running;
  S->slots.resize(max_running);
  for (int i = 0; i < max_running; i++) S->workers.emplace_back([S, i] { S->worker(i); });
  gkc_status st;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv.wait(lk, [S] { return S->ready == S->max_running; });
    st = S->init_status;
  }
  if (st != GKC_OK) {
    gkc_server_destroy(S);
    return st;
  }
  *out = S;
  return GKC_OK;
}

void gkc_server_destroy(gkc_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  for (auto &t : S->workers) t.join();
  cudaSetDevice(S->dev);
  for (auto &kv : S->jobs) {
    if (kv.second->d_res) cudaFreeAsync(kv.second->d_res, 0);
    delete kv.second;
  }
  cudaDeviceSynchronize();
  delete S;
}

static gkc_status enqueue(gkc_server *S, Job *j, uint64_t *job_id) {
  std::lock_guard<std::mutex> lk(S->mu);
  j->id = S->next_id++;
  j->info.state = GKC_JOB_QUEUED;
  j->info.status = GKC_OK;
  j->info.n_bases = j->n_bases;
  j->info.submit_s = S->now();
  S->jobs[j->id] = j;
  S->queue.push_back(j);
  *job_id = j->id;
  S->cv.notify_all();
  return GKC_OK;
}

static bool params_ok(const gkc_params *p) {
  return p && p->k >= 1 && p->k <= 64 && p->p >= 3 && p->p <= 16 && p->p <= p->k && p->nbins >= 1;
}

gkc_status gkc_server_submit(gkc_server *S, const gkc_params *prm, const char *reads,
                             const uint64_t *offs, uint64_t n_reads, uint64_t *job_id) {
  if (!S || !job_id || !params_ok(prm) || !offs || (n_reads && !reads)) return GKC_ERR_INVALID_ARG;
  Job *j = new Job();
  j->prm = *prm;
  const uint64_t base = offs[0], nb = offs[n_reads] - base;
  j->reads.assign(reads + base, reads + base + nb);
  j->offs.resize(n_reads + 1);
  for (uint64_t r = 0; r <= n_reads; r++) j->offs[r] = offs[r] - base;
  j->n_reads = n_reads;
  j->n_bases = nb;
  j->est = gkc_job_hbm_estimate(prm, nb, n_reads);
  return enqueue(S, j, job_id);
}

gkc_status gkc_server_submit_device_synth(gkc_server *S, const gkc_params *prm, int generator,
                                          uint64_t seed, uint64_t n_bases, uint64_t *job_id) {
  if (!S || !job_id || !params_ok(prm) || generator < 1 || generator > 3) return GKC_ERR_INVALID_ARG;
  Job *j = new Job();
  j->prm = *prm;
  j->synth = true;
  j->generator = generator;
  j->seed = seed;
  if (generator == 3) {
    const uint64_t max_reads = n_bases / kLongMin + 2;
    j->offs.resize(max_reads + 1);
    j->n_reads = gkc_synth_long_read_offsets(seed, kLongMedian, kLongSigma, kLongMin, kLongMax, n_bases,
                                             max_reads, j->offs.data());
    j->offs.resize(j->n_reads + 1);
    j->n_bases = j->offs[j->n_reads];
  } else {
    j->n_reads = std::max<uint64_t>(n_bases / kShortLen, 1);
    j->n_bases = j->n_reads * kShortLen;
  }
  const uint64_t G = synth_genome_len(generator, j->n_bases);
  j->est = gkc_job_hbm_estimate(prm, j->n_bases, j->n_reads) + j->n_bases + 64 + 8 * (j->n_reads + 1) +
           (G ? G + 64 : 0);
  return enqueue(S, j, job_id);
}

gkc_status gkc_server_poll(gkc_server *S, uint64_t id, gkc_job_info *info) {
  if (!S || !info) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return GKC_ERR_NOT_FOUND;
  *info = it->second->info;
  return GKC_OK;
}

gkc_status gkc_server_wait(gkc_server *S, uint64_t id, double timeout_s, gkc_job_info *info) {
  if (!S) return GKC_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return GKC_ERR_NOT_FOUND;
  Job *j = it->second;
  auto done = [j] { return gkc_server::finished(j); };
  if (timeout_s < 0) {
    S->cv.wait(lk, done);
  } else if (!S->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    if (info) *info = j->info;
    return GKC_ERR_NOT_READY;
  }
  if (info) *info = j->info;
  return GKC_OK;
}

gkc_status gkc_server_cancel(gkc_server *S, uint64_t id) {
  if (!S) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return GKC_ERR_NOT_FOUND;
  Job *j = it->second;
  if (j->info.state == GKC_JOB_QUEUED) {
    for (auto q = S->queue.begin(); q != S->queue.end(); ++q)
      if (*q == j) {
        S->queue.erase(q);
        break;
      }
    j->info.state = GKC_JOB_CANCELLED;
    j->info.status = GKC_ERR_CANCELLED;
    j->info.end_s = S->now();
    S->cv.notify_all();
  } else if (j->info.state == GKC_JOB_RUNNING) {
    j->cancel = true;  // the result is dropped when the run ends
  }
  return GKC_OK;
}

gkc_status gkc_server_copy_result(gkc_server *S, uint64_t id, uint64_t *bin_off, uint64_t *keys,
                                  uint32_t *counts) {
  if (!S) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return GKC_ERR_NOT_FOUND;
  Job *j = it->second;
  if (j->info.state != GKC_JOB_DONE) return j->info.state == GKC_JOB_FAILED ? j->info.status : GKC_ERR_NOT_READY;
  const uint64_t b_bo = 8 * (j->info.nbins + 1), b_keys = 8 * j->info.n_distinct * j->info.key_words,
                 b_cnt = 4 * j->info.n_distinct;
  const char *r = static_cast<const char *>(j->d_res);
  cudaSetDevice(S->dev);
  cudaError_t e = cudaSuccess;
  if (bin_off) e = cudaMemcpy(bin_off, r, b_bo, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && keys && b_keys) e = cudaMemcpy(keys, r + b_bo, b_keys, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && counts && b_cnt) e = cudaMemcpy(counts, r + b_bo + b_keys, b_cnt, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return GKC_ERR_CUDA;
  }
  return GKC_OK;
}

gkc_status gkc_server_release(gkc_server *S, uint64_t id) {
  if (!S) return GKC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return GKC_ERR_NOT_FOUND;
  Job *j = it->second;
  if (!gkc_server::finished(j)) return GKC_ERR_NOT_READY;  // cancel it first
  if (j->d_res) {
    cudaSetDevice(S->dev);
    cudaFreeAsync(j->d_res, 0);
    S->held -= j->res_bytes;
    S->committed -= j->res_bytes;
    S->cv.notify_all();
  }
  delete j;
  S->jobs.erase(it);
  return GKC_OK;
}

}  // extern "C"
