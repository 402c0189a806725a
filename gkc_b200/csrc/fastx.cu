// FASTA / FASTQ ingest into the read CSR the pipeline takes (host code).
//
// The reference's loader (ReadLoader::_load_fastq / _load_fasta,
// read_loader.hpp:44-196, driven by load_file / work_while_loading_V2,
// :276-321, :470-520) reads fixed-size chunks on several threads and hands
// each chunk's incomplete last record to the next thread.  Here the whole
// file is read once, cut into one byte range per thread, and every thread
// parses the records that start in its range (a record start is found from
// the range's first line on), first counting and then copying, so that the
// reads land in file order in one CSR without hand-offs.
//
// Record rules, by default those of the reference:
//   format: FASTQ when the file name ends in 'q', else FASTA (load_file,
//          read_loader.hpp:285); GKC_FASTX_FORMAT_FROM_CONTENT decides by
//          the first byte ('@' or '>') instead;
//   FASTQ: '@' header line, sequence line, '+' line, quality line; the
//          sequence is the second line of the record (:110-122);
//   FASTA: '>' header line and the one line after it (:180-193: records of
//          two lines); with GKC_FASTX_JOIN_LINES the sequence is every line
//          up to the next line that starts with '>', joined.
//   A '\r' before a line end is dropped.  Bytes are kept as they are (the
//   pipeline maps A/C/G/T/U in either case and treats anything else as N).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/gkc/gkc.h"

namespace {

struct Range {
  size_t b, e;  // byte range [b, e) of the file whose record starts this thread owns
};

// Start of the first record that begins at or after `pos` (a line start).
size_t next_record(const char *d, size_t n, size_t pos, bool fastq) {
  if (pos > 0) {  // move to the next line start
    const void *nl = memchr(d + pos - 1, '\n', n - pos + 1);
    if (!nl) return n;
    pos = (const char *)nl - d + 1;
  }
  while (pos < n) {
    if (fastq) {
      // '@' at a line start is a header only if the line after the next one
      // starts with '+' (a quality line may start with '@')
      if (d[pos] == '@') {
        const char *l2 = (const char *)memchr(d + pos, '\n', n - pos);
        const char *l3 = l2 ? (const char *)memchr(l2 + 1, '\n', d + n - l2 - 1) : nullptr;
        if (l3 && l3 + 1 < d + n && l3[1] == '+') return pos;
        if (!l2) return n;
      }
    } else if (d[pos] == '>') {
      return pos;
    }
    const void *nl = memchr(d + pos, '\n', n - pos);
    if (!nl) return n;
    pos = (const char *)nl - d + 1;
  }
  return n;
}

size_t line_end(const char *d, size_t n, size_t pos) {  // index of '\n' or n
  const void *nl = memchr(d + pos, '\n', n - pos);
  return nl ? (size_t)((const char *)nl - d) : n;
}

// Walks the records starting in [r.b, r.e); calls emit(ptr, len) for every
// sequence piece (FASTA pieces of one record in order) and end() per record.
template <typename Piece, typename End>
void walk(const char *d, size_t n, Range r, bool fastq, bool join, Piece piece, End end) {
  size_t pos = r.b;
  while (pos < r.e && pos < n) {
    size_t h = line_end(d, n, pos);  // header line
    if (h >= n) break;
    size_t s = h + 1;
    if (fastq) {
      size_t se = line_end(d, n, s);
      size_t len = se - s;
      if (len && d[s + len - 1] == '\r') len--;
      piece(d + s, len);
      end();
      size_t plus = se < n ? line_end(d, n, se + 1) : n;       // '+' line
      size_t qual = plus < n ? line_end(d, n, plus + 1) : n;   // quality line
      pos = qual < n ? qual + 1 : n;
    } else if (!join) {
      // the line after the header; the rest of the record up to the next
      // header is skipped
      size_t se = line_end(d, n, s);
      size_t len = se - s;
      if (len && d[s + len - 1] == '\r') len--;
      piece(d + s, len);
      end();
      pos = next_record(d, n, se < n ? se + 1 : n, false);
    } else {
      size_t q = s;
      while (q < n && d[q] != '>') {
        size_t qe = line_end(d, n, q);
        size_t len = qe - q;
        if (len && d[q + len - 1] == '\r') len--;
        if (len) piece(d + q, len);
        q = qe < n ? qe + 1 : n;
      }
      end();
      pos = q;
    }
  }
}

}  // namespace

extern "C" gkc_status gkc_fastx_load_ex(const char *path, int n_threads, int pinned, int flags, char **reads,
                                        uint64_t **offs, uint64_t *n_reads) {
  if (!path || !reads || !offs || !n_reads || n_threads < 0) return GKC_ERR_INVALID_ARG;
  if (flags & ~(GKC_FASTX_JOIN_LINES | GKC_FASTX_FORMAT_FROM_CONTENT)) return GKC_ERR_INVALID_ARG;
  const bool join = (flags & GKC_FASTX_JOIN_LINES) != 0;
  *reads = nullptr;
  *offs = nullptr;
  *n_reads = 0;
  FILE *f = fopen(path, "rb");
  if (!f) return GKC_ERR_NOT_FOUND;
  std::vector<char> data;
  {
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + got);
  }
  fclose(f);
  const char *d = data.data();
  const size_t n = data.size();
  size_t first = 0;
  while (first < n && (d[first] == '\n' || d[first] == '\r')) first++;
  bool fastq;
  if (flags & GKC_FASTX_FORMAT_FROM_CONTENT) {
    if (first < n && d[first] != '>' && d[first] != '@') return GKC_ERR_INVALID_ARG;  // neither format
    fastq = first < n && d[first] == '@';
  } else {
    const size_t pl = strlen(path);
    fastq = pl > 0 && path[pl - 1] == 'q';
    if (first < n && d[first] != (fastq ? '@' : '>')) return GKC_ERR_INVALID_ARG;  // not the named format
  }
  int T = n_threads ? n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  T = (int)std::max<size_t>(1, std::min<size_t>((size_t)T, n / (1 << 20) + 1));
  // one byte range per thread, each starting at a record start
  std::vector<size_t> cut(T + 1, n);
  cut[0] = first;
  for (int t = 1; t < T; t++) cut[t] = std::max(cut[t - 1], next_record(d, n, first + (n - first) * t / T, fastq));
  std::vector<uint64_t> cnt_reads(T, 0), cnt_bytes(T, 0);
  auto run = [&](auto fn) {
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++) th.emplace_back(fn, t);
    for (auto &x : th) x.join();
  };
  run([&](int t) {
    walk(d, n, Range{cut[t], cut[t + 1]}, fastq, join, [&](const char *, size_t len) { cnt_bytes[t] += len; },
         [&] { cnt_reads[t]++; });
  });
  uint64_t R = 0, B = 0;
  std::vector<uint64_t> r0(T), b0(T);
  for (int t = 0; t < T; t++) {
    r0[t] = R;
    b0[t] = B;
    R += cnt_reads[t];
    B += cnt_bytes[t];
  }
  char *out = nullptr;
  uint64_t *o = nullptr;
  if (pinned) {
    if (cudaMallocHost((void **)&out, B + 64) != cudaSuccess ||
        cudaMallocHost((void **)&o, 8 * (R + 1)) != cudaSuccess) {
      cudaGetLastError();
      if (out) cudaFreeHost(out);
      return GKC_ERR_OUT_OF_MEMORY;
    }
  } else {
    out = (char *)malloc(B + 64);
    o = (uint64_t *)malloc(8 * (R + 1));
    if (!out || !o) {
      free(out);
      free(o);
      return GKC_ERR_OUT_OF_MEMORY;
    }
  }
  run([&](int t) {
    uint64_t r = r0[t], b = b0[t];
    o[r] = b;
    walk(d, n, Range{cut[t], cut[t + 1]}, fastq, join,
         [&](const char *p, size_t len) {
           memcpy(out + b, p, len);
           b += len;
         },
         [&] { o[++r] = b; });
  });
  o[0] = 0;
  o[R] = B;
  *reads = out;
  *offs = o;
  *n_reads = R;
  return GKC_OK;
}

extern "C" gkc_status gkc_fastx_load(const char *path, int n_threads, int pinned, char **reads, uint64_t **offs,
                                     uint64_t *n_reads) {
  return gkc_fastx_load_ex(path, n_threads, pinned, 0, reads, offs, n_reads);
}

extern "C" void gkc_fastx_free(char *reads, uint64_t *offs, int pinned) {
  if (pinned) {
    if (reads) cudaFreeHost(reads);
    if (offs) cudaFreeHost(offs);
  } else {
    free(reads);
    free(offs);
  }
}
