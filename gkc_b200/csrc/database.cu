// On-disk k-mer database in the style of KMC's (a prefix lookup table and
// fixed-width suffix + counter records), written from the merged count list
// and read back on the host.  The reference has no on-disk output; its
// README (README.md:17) names KMC3's partitioned counting as the use case.
//
// Layout (all integers little-endian unless stated):
//   <path>.gkc_pre  "GKCP" u32 version=1
//                   u32 k, u32 lut_prefix_len l, u32 suffix_bytes, u32 counter_bytes,
//                   u32 min_count, u32 max_count, u64 n_records, u64 total_count
//                   u64 lut[4^l + 1]   lut[p] = first record whose key >> 2(k-l) is p
//                   "GKCP"
//   <path>.gkc_suf  "GKCS"
//                   n_records x (suffix: the low 2(k-l) bits of the key, big-endian
//                   in suffix_bytes bytes; counter: counter_bytes bytes, little-endian)
//                   "GKCS"
// Records are in ascending key order, one per canonical k-mer (the merged
// list, with the min/max frequency filter applied), so a lookup is one
// table read and a binary search over one prefix's records.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"

namespace gkc {

constexpr uint32_t kDbVersion = 1;
constexpr int kDbMaxLut = 13;  // 4^13 + 1 table entries, 512 MB

template <typename K>
GKC_DEV uint64_t key_prefix(K key, int shift) {
  return (uint64_t)(key >> shift);
}

// lut[q] = first index i with keys[i] >> shift >= q (keys ascending).
template <typename K>
__global__ void k_db_lut(const K *keys, uint64_t n, int shift, uint64_t n_lut, uint64_t *lut) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n_lut; q += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (key_prefix(keys[mid], shift) < q) lo = mid + 1;
      else hi = mid;
    }
    lut[q] = lo;
  }
}

// Largest count and sum of counts (out[0] max, out[1] sum; zeroed before).
__global__ void k_db_stats(const uint32_t *counts, uint64_t n, unsigned long long *out) {
  uint32_t mx = 0;
  unsigned long long sum = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = counts[i];
    mx = c > mx ? c : mx;
    sum += c;
  }
  for (int o = 16; o; o >>= 1) {
    const uint32_t m2 = __shfl_down_sync(0xFFFFFFFFu, mx, o);
    mx = m2 > mx ? m2 : mx;
    sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)mx);
    atomicAdd(out + 1, sum);
  }
}

// One record per key: the low `shift` bits big-endian in sbytes bytes, the
// count little-endian in cbytes bytes.
template <typename K>
__global__ void k_db_encode(const K *keys, const uint32_t *counts, uint64_t n, int shift, int sbytes, int cbytes,
                            uint8_t *out) {
  const int rec = sbytes + cbytes;
  const K mask = (((K)1) << shift) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const K key = keys[i] & mask;
    uint8_t *o = out + i * rec;
    for (int j = 0; j < sbytes; j++) o[j] = (uint8_t)(key >> (8 * (sbytes - 1 - j)));
    const uint32_t c = counts[i];
    for (int j = 0; j < cbytes; j++) o[sbytes + j] = (uint8_t)(c >> (8 * j));
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

namespace {

struct DbHeader {
  uint32_t k, lut_len, sbytes, cbytes, min_count, max_count;
  uint64_t n, total;
};

int auto_lut(uint64_t n, int k) {
  int l = 1;
  while (l < kDbMaxLut && (1ull << (2 * (l + 1))) * 8 <= n) l++;  // about 8 records per table entry
  return std::min(l, k - 1);  // 0 for k = 1: a two-entry table
}

bool put(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }

}  // namespace

template <typename K>
static gkc_status db_write_t(gkc_ctx *c, const char *path, uint32_t min_count, uint32_t max_count, int lut_len,
                             uint64_t n) {
  const int k = c->ck;
  const K *keys = (const K *)c->bufs["flt_keys"].p;
  const uint32_t *counts = (const uint32_t *)c->bufs["flt_counts"].p;
  const unsigned grid = c->n_sms * 16;
  // counter width: the smallest that holds the largest count
  WS(stats, unsigned long long, "db_stats", 2);
  CK(cudaMemsetAsync(stats, 0, 16, c->st));
  if (n) k_db_stats<<<grid, 256, 0, c->st>>>(counts, n, stats);
  CK(cudaPeekAtLastError());
  unsigned long long hs[2] = {0, 0};
  CK(cudaMemcpyAsync(hs, stats, 16, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const uint32_t cmax = (uint32_t)hs[0];
  const uint64_t total = hs[1];
  const int cbytes = cmax < 256u ? 1 : cmax < 65536u ? 2 : cmax < (1u << 24) ? 3 : 4;
  const int shift = 2 * (k - lut_len);
  const int sbytes = (shift + 7) / 8;
  const uint64_t n_lut = (1ull << (2 * lut_len)) + 1;
  WS(lut, uint64_t, "db_lut", n_lut);
  k_db_lut<K><<<grid, 256, 0, c->st>>>(keys, n, shift, n_lut, lut);
  CK(cudaPeekAtLastError());
  std::vector<uint64_t> hl(n_lut);
  CK(cudaMemcpyAsync(hl.data(), lut, 8 * n_lut, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));

  const std::string pre = std::string(path) + ".gkc_pre", suf = std::string(path) + ".gkc_suf";
  FILE *f = fopen(pre.c_str(), "wb");
  if (!f) return ctx_fail(c, GKC_ERR_NOT_FOUND, "cannot create " + pre);
  DbHeader h{(uint32_t)k, (uint32_t)lut_len, (uint32_t)sbytes, (uint32_t)cbytes, min_count, max_count, n, total};
  bool ok = put(f, "GKCP", 4) && put(f, &kDbVersion, 4) && put(f, &h.k, 4) && put(f, &h.lut_len, 4) &&
            put(f, &h.sbytes, 4) && put(f, &h.cbytes, 4) && put(f, &h.min_count, 4) && put(f, &h.max_count, 4) &&
            put(f, &h.n, 8) && put(f, &h.total, 8) && put(f, hl.data(), 8 * n_lut) && put(f, "GKCP", 4);
  ok = (fclose(f) == 0) && ok;
  if (!ok) return ctx_fail(c, GKC_ERR_INTERNAL, "writing " + pre + " failed");

  // records: encoded on the device in slices, copied out and appended
  f = fopen(suf.c_str(), "wb");
  if (!f) return ctx_fail(c, GKC_ERR_NOT_FOUND, "cannot create " + suf);
  ok = put(f, "GKCS", 4);
  const int rec = sbytes + cbytes;
  const uint64_t slice = std::max<uint64_t>(1, (256ull << 20) / rec);
  WS(enc, uint8_t, "db_records", std::min<uint64_t>(slice, std::max<uint64_t>(n, 1)) * rec);
  std::vector<uint8_t> host(std::min<uint64_t>(slice, std::max<uint64_t>(n, 1)) * rec);
  gkc_status st = GKC_OK;
  for (uint64_t s = 0; ok && st == GKC_OK && s < n; s += slice) {
    const uint64_t m = std::min(slice, n - s);
    k_db_encode<K><<<grid, 256, 0, c->st>>>(keys + s, counts + s, m, shift, sbytes, cbytes, enc);
    st = ctx_cuda(c, cudaPeekAtLastError(), "k_db_encode");
    if (st == GKC_OK) st = ctx_cuda(c, cudaMemcpyAsync(host.data(), enc, m * rec, cudaMemcpyDeviceToHost, c->st),
                                    "records to the host");
    if (st == GKC_OK) st = ctx_cuda(c, cudaStreamSynchronize(c->st), "records to the host");
    if (st == GKC_OK) ok = put(f, host.data(), m * rec);
  }
  if (st != GKC_OK) {
    fclose(f);
    return st;
  }
  ok = ok && put(f, "GKCS", 4);
  ok = (fclose(f) == 0) && ok;
  if (!ok) return ctx_fail(c, GKC_ERR_INTERNAL, "writing " + suf + " failed");
  return GKC_OK;
}

gkc_status gkc_db_write(gkc_ctx *c, const char *path, uint32_t min_count, uint32_t max_count, int lut_prefix_len) {
  if (!c || !path) return GKC_ERR_INVALID_ARG;
  if (!c->have_count) return ctx_fail(c, GKC_ERR_INVALID_ARG, "no count result in the context");
  const int k = c->ck;
  if (lut_prefix_len < 0 || lut_prefix_len > kDbMaxLut || lut_prefix_len >= k)
    return ctx_fail(c, GKC_ERR_INVALID_ARG, "lookup prefix length must be below k and at most 13");
  uint64_t n = 0;
  gkc_status s = gkc_count_output(c, min_count, max_count, 1, &n, nullptr, nullptr, nullptr);
  if (s != GKC_OK) return s;
  cudaSetDevice(c->dev);
  const int l = lut_prefix_len ? lut_prefix_len : auto_lut(n, k);
  return c->cv.key_words == 1 ? db_write_t<uint64_t>(c, path, min_count, max_count, l, n)
                              : db_write_t<u128>(c, path, min_count, max_count, l, n);
}

// ------------------------------------------------------------------ reader

struct gkc_db {
  DbHeader h{};
  std::vector<uint64_t> lut;
  const uint8_t *rec = nullptr;  // first record (mapped)
  void *map = nullptr;
  size_t map_bytes = 0;
};

static bool get(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

gkc_status gkc_db_open(const char *path, gkc_db **out) {
  if (!path || !out) return GKC_ERR_INVALID_ARG;
  *out = nullptr;
  const std::string pre = std::string(path) + ".gkc_pre", suf = std::string(path) + ".gkc_suf";
  FILE *f = fopen(pre.c_str(), "rb");
  if (!f) return GKC_ERR_NOT_FOUND;
  gkc_db *db = new gkc_db();
  char m[4];
  uint32_t ver = 0;
  DbHeader &h = db->h;
  bool ok = get(f, m, 4) && !memcmp(m, "GKCP", 4) && get(f, &ver, 4) && ver == kDbVersion && get(f, &h.k, 4) &&
            get(f, &h.lut_len, 4) && get(f, &h.sbytes, 4) && get(f, &h.cbytes, 4) && get(f, &h.min_count, 4) &&
            get(f, &h.max_count, 4) && get(f, &h.n, 8) && get(f, &h.total, 8);
  ok = ok && h.k >= 1 && h.k <= 64 && h.lut_len <= (uint32_t)kDbMaxLut && h.lut_len < h.k &&
       h.sbytes == (2 * (h.k - h.lut_len) + 7) / 8 && h.cbytes >= 1 && h.cbytes <= 4;
  if (ok) {
    db->lut.resize((1ull << (2 * h.lut_len)) + 1);
    ok = get(f, db->lut.data(), 8 * db->lut.size()) && get(f, m, 4) && !memcmp(m, "GKCP", 4) &&
         db->lut.back() == h.n;
  }
  fclose(f);
  if (ok) {
    const int fd = open(suf.c_str(), O_RDONLY);
    struct stat st;
    const size_t want = 8 + h.n * (size_t)(h.sbytes + h.cbytes);
    ok = fd >= 0 && fstat(fd, &st) == 0 && (size_t)st.st_size == want;
    if (ok) {
      db->map = mmap(nullptr, want, PROT_READ, MAP_PRIVATE, fd, 0);
      ok = db->map != MAP_FAILED;
      if (ok) {
        db->map_bytes = want;
        const uint8_t *b = (const uint8_t *)db->map;
        ok = !memcmp(b, "GKCS", 4) && !memcmp(b + want - 4, "GKCS", 4);
        db->rec = b + 4;
      } else {
        db->map = nullptr;
      }
    }
    if (fd >= 0) close(fd);
  }
  if (!ok) {
    gkc_db_close(db);
    return GKC_ERR_INVALID_ARG;
  }
  *out = db;
  return GKC_OK;
}

void gkc_db_close(gkc_db *db) {
  if (!db) return;
  if (db->map) munmap(db->map, db->map_bytes);
  delete db;
}

gkc_status gkc_db_get_info(const gkc_db *db, gkc_db_info *out) {
  if (!db || !out) return GKC_ERR_INVALID_ARG;
  out->k = db->h.k;
  out->lut_prefix_len = db->h.lut_len;
  out->suffix_bytes = db->h.sbytes;
  out->counter_bytes = db->h.cbytes;
  out->min_count = db->h.min_count;
  out->max_count = db->h.max_count;
  out->n_kmers = db->h.n;
  out->total_count = db->h.total;
  return GKC_OK;
}

static u128 rec_suffix(const gkc_db *db, uint64_t i) {
  const uint8_t *r = db->rec + i * (db->h.sbytes + db->h.cbytes);
  u128 s = 0;
  for (uint32_t j = 0; j < db->h.sbytes; j++) s = (s << 8) | r[j];
  return s;
}

static uint32_t rec_count(const gkc_db *db, uint64_t i) {
  const uint8_t *r = db->rec + i * (db->h.sbytes + db->h.cbytes) + db->h.sbytes;
  uint32_t v = 0;
  for (uint32_t j = 0; j < db->h.cbytes; j++) v |= (uint32_t)r[j] << (8 * j);
  return v;
}

static u128 key_at(const uint64_t *keys, uint64_t i, int kw) {
  return kw == 1 ? (u128)keys[i] : (((u128)keys[2 * i + 1]) << 64) | keys[2 * i];
}

gkc_status gkc_db_lookup(const gkc_db *db, const uint64_t *keys, uint64_t n, uint32_t *counts) {
  if (!db || (n && (!keys || !counts))) return GKC_ERR_INVALID_ARG;
  const int kw = db->h.k <= 32 ? 1 : 2;
  const int shift = 2 * (db->h.k - db->h.lut_len);
  const u128 smask = (((u128)1) << shift) - 1;
  for (uint64_t i = 0; i < n; i++) {
    const u128 key = key_at(keys, i, kw);
    const u128 p = key >> shift;
    counts[i] = 0;
    if (p >= (u128)(db->lut.size() - 1)) continue;  // beyond 4^k: not a k-mer
    uint64_t lo = db->lut[(size_t)p], hi = db->lut[(size_t)p + 1];
    const u128 want = key & smask;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (rec_suffix(db, mid) < want) lo = mid + 1;
      else hi = mid;
    }
    if (lo < db->lut[(size_t)p + 1] && rec_suffix(db, lo) == want) counts[i] = rec_count(db, lo);
  }
  return GKC_OK;
}

gkc_status gkc_db_read(const gkc_db *db, uint64_t first, uint64_t n, uint64_t *keys, uint32_t *counts) {
  if (!db || first > db->h.n || n > db->h.n - first) return GKC_ERR_INVALID_ARG;
  const int kw = db->h.k <= 32 ? 1 : 2;
  const int shift = 2 * (db->h.k - db->h.lut_len);
  // prefix of record i: the table entry whose range holds i
  uint64_t p = std::upper_bound(db->lut.begin(), db->lut.end(), first) - db->lut.begin() - 1;
  for (uint64_t i = first; i < first + n; i++) {
    while (db->lut[p + 1] <= i) p++;
    const u128 key = (((u128)p) << shift) | rec_suffix(db, i);
    if (keys) {
      if (kw == 1) keys[i - first] = (uint64_t)key;
      else {
        keys[2 * (i - first)] = (uint64_t)key;
        keys[2 * (i - first) + 1] = (uint64_t)(key >> 64);
      }
    }
    if (counts) counts[i - first] = rec_count(db, i);
  }
  return GKC_OK;
}
