/* CPU restatement of GKC's partition-and-count path -- TEST INFRASTRUCTURE.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may use this
 * file, and only to check results.  Each function cites the reference lines it
 * restates (paths relative to the GKC project root).
 */
#include "gkc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

int orc_version(void) { return 1; }
void orc_free(void *p) { free(p); }

/* ASCII -> 2-bit code: A/a 0, C/c 1, G/g 2, T/t 3, U/u 0, anything else 255
 * (gkc_cuda.cu:25-58 d_basemap; superkmers.hpp:14-47 basemap).  Bytes >= 0x80
 * index the reference table with a negative signed char, which is undefined
 * there; they are treated like N here. */
static inline uint32_t code_of(uint8_t c) {
  switch (c) {
    case 'A': case 'a': case 'U': case 'u': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 255;
  }
}

/* Complement code: A 3, C 2, G 1, T 0, U 3, else 255 (gkc_cuda.cu:60-93). */
static inline uint32_t ccode_of(uint8_t c) {
  uint32_t x = code_of(c);
  if (x == 255) return 255;
  return 3 - x;
}

/* The minimizer filter (FILTER_KERNEL, gkc_cuda.cu:6; variants :196-227),
 * applied to the unmasked p-mer value as the reference does:
 *   0 new_filter2 (:214-216, the reference's choice): top three bases not
 *     AAA, ACA or AGA;  1 mm_filter (:196-209): every p-mer;
 *   2 new_filter (:211-213): 2nd and 3rd bases not both A;
 *   3 sign_filter (:218-227): no AA among the lowest p-1 bases, top three
 *     bases not AAA or ACA. */
static int g_filter = 0;
void orc_set_filter(int f) { g_filter = f; }

static inline int filt(uint32_t v, int p) {
  uint32_t t = v >> (2 * (p - 3));
  switch (g_filter) {
    case 1:
      return 1;
    case 2:
      return (((v >> (2 * (p - 2))) & 3u) + ((v >> (2 * (p - 3))) & 3u)) != 0;
    case 3: {
      uint32_t x = v;
      int ok = 1;
      for (int i = 0; i < p - 2; i++) {
        ok &= (x & 0xFu) != 0;
        x >>= 2;
      }
      return ok & (t != 0) & (t != 4u);
    }
    default:
      return (t != 0) & (t != 4u) & (t != 8u);
  }
}

/* GPU_HPCEncoding with the per-read start index (gkc_cuda.cu:178-190; the
 * reference indexes the start by thread id at :180, which equals the read id
 * whenever the grid covers all reads). */
void orc_hpc(const uint8_t *reads, const uint64_t *offs, int64_t n_reads,
             uint8_t *out_reads, int32_t *out_len, int32_t *orig_pos) {
  for (int64_t r = 0; r < n_reads; r++) {
    uint64_t b = offs[r], e = offs[r + 1];
    int32_t len = (int32_t)(e - b);
    if (len == 0) { out_len[r] = 0; continue; }
    int32_t n = 0;
    out_reads[b] = reads[b];
    orig_pos[b] = 0;
    n = 1;
    for (int32_t i = 1; i < len; i++) {
      if (reads[b + i] != reads[b + i - 1]) {
        out_reads[b + n] = reads[b + i];
        orig_pos[b + n] = i;
        n++;
      }
    }
    out_len[r] = n;
  }
}

/* GPU_GenMinimizer, one window at a time (gkc_cuda.cu:243-286). */
void orc_window_minimizers(const uint8_t *read, int32_t len, int k, int p, uint32_t *mm) {
  const uint32_t M = 0xFFFFFFFFu >> (32 - 2 * p);
  for (int32_t s = 0; s + k <= len; s++) {
    uint32_t f = 0, r = 0, m, mr, best;
    for (int j = s; j < s + p; j++) f = (f << 2) | code_of(read[j]);
    m = filt(f, p) ? f : M;
    for (int j = s + p - 1; j >= s; j--) r = (r << 2) | ccode_of(read[j]);
    mr = filt(r, p) ? r : M;
    best = (mr < m) ? mr : m;
    for (int j = s + p; j < s + k; j++) {
      f = ((f << 2) | code_of(read[j])) & M;
      r = (r >> 2) | (ccode_of(read[j]) << (2 * p - 2));
      if (filt(f, p)) m = f;
      if (filt(r, p)) mr = r;
      best = (best < m) ? best : m;
      best = (best < mr) ? best : mr;
    }
    mm[s] = best;
  }
}

/* Position/strand of the selected p-mer.  The reference declares these
 * outputs (gkc_cuda.cu:159-160, gkc_cuda.hpp:50) but never computes them.
 * Definition used here: the window's minimizer value mm (reference
 * semantics) is located at the RIGHTMOST p-mer position j whose passing
 * forward or passing reverse-complement p-mer equals mm (the reference's
 * ">=" updates at gkc_cuda.cu:283-284 let later candidates win ties).
 * strand = -1 if the p-mer at j is its own reverse complement, else 1 if the
 * reverse complement at j is the match, else 0.  With no passing p-mer:
 * position 255, strand 0. */
void orc_window_minimizer_pos(const uint8_t *read, int32_t len, int k, int p,
                              uint32_t *mm, uint8_t *pos, int8_t *strand) {
  orc_window_minimizers(read, len, k, p, mm);
  for (int32_t s = 0; s + k <= len; s++) {
    int bpos = 255, bstr = 0;
    for (int j = 0; j <= k - p; j++) {
      uint32_t f = 0, r = 0;
      for (int t = 0; t < p; t++) {
        f = (f << 2) | (code_of(read[s + j + t]) & 3);
        r = (r << 2) | (ccode_of(read[s + j + p - 1 - t]) & 3);
      }
      int mf = filt(f, p) && f == mm[s];
      int mr = filt(r, p) && r == mm[s];
      if (mf || mr) {
        bpos = j;
        bstr = (f == r) ? -1 : (mr ? 1 : 0);
      }
    }
    pos[s] = (uint8_t)bpos;
    strand[s] = (int8_t)bstr;
  }
}

/* --- partition: GPU_GenSKM (gkc_cuda.cu:308-321) + SKMStore::add_skms
 *     (superkmers.hpp:175-183) + CRead packing (superkmers.hpp:63-71). --- */

typedef struct {
  uint64_t n, cap;
  uint32_t *bin, *len, *start, *minimizer;
  uint64_t *byte_off, *read_id;
  uint64_t nb, bcap;
  uint8_t *bytes;
} skm_builder;

static int sb_push(skm_builder *b, uint32_t bin, uint32_t len, uint64_t read_id, uint32_t start,
                   uint32_t mmv, const uint8_t *bases) {
  if (b->n == b->cap) {
    uint64_t nc = b->cap ? b->cap * 2 : 1024;
    void *p;
#define GROW(field, T) p = realloc(b->field, nc * sizeof(T)); if (!p) return -1; b->field = (T *)p;
    GROW(bin, uint32_t) GROW(len, uint32_t) GROW(start, uint32_t) GROW(minimizer, uint32_t)
    GROW(byte_off, uint64_t) GROW(read_id, uint64_t)
#undef GROW
    b->cap = nc;
  }
  uint64_t nbytes = (len + 3) / 4;
  if (b->nb + nbytes > b->bcap) {
    uint64_t nc = b->bcap ? b->bcap * 2 : 4096;
    while (nc < b->nb + nbytes) nc *= 2;
    void *p = realloc(b->bytes, nc);
    if (!p) return -1;
    b->bytes = (uint8_t *)p;
    b->bcap = nc;
  }
  uint8_t *dst = b->bytes + b->nb;
  memset(dst, 0, nbytes);
  for (uint32_t i = 0; i < len; i++)
    dst[i / 4] = (uint8_t)((dst[i / 4] << 2) | (code_of(bases[i]) & 3));
  if (len % 4) dst[len / 4] = (uint8_t)(dst[len / 4] << (2 * (4 - len % 4)));
  b->bin[b->n] = bin;
  b->len[b->n] = len;
  b->start[b->n] = start;
  b->minimizer[b->n] = mmv;
  b->byte_off[b->n] = b->nb;
  b->read_id[b->n] = read_id;
  b->n++;
  b->nb += nbytes;
  return 0;
}

int orc_partition(const uint8_t *reads, const uint64_t *offs, int64_t n_reads, int k, int p,
                  int hpc, int nbins, orc_skms *out) {
  memset(out, 0, sizeof(*out));
  if (k < 1 || p < 3 || p > 16 || p > k || nbins < 1) return -1;
  skm_builder b;
  memset(&b, 0, sizeof(b));
  uint64_t total = offs[n_reads] - offs[0];
  uint8_t *hreads = NULL;
  int32_t *hlen = NULL, *horig = NULL;
  const uint8_t *base = reads;
  if (hpc) {
    hreads = (uint8_t *)malloc(total + 1);
    hlen = (int32_t *)malloc(sizeof(int32_t) * (n_reads + 1));
    horig = (int32_t *)malloc(sizeof(int32_t) * (total + 1));
    if (!hreads || !hlen || !horig) return -1;
    /* offsets are used relative to offs[0] */
    uint64_t *roffs = (uint64_t *)malloc(sizeof(uint64_t) * (n_reads + 1));
    for (int64_t r = 0; r <= n_reads; r++) roffs[r] = offs[r] - offs[0];
    orc_hpc(reads + offs[0], roffs, n_reads, hreads, hlen, horig);
    free(roffs);
    base = hreads;
  }
  uint32_t *mm = NULL;
  int32_t mmcap = 0;
  for (int64_t r = 0; r < n_reads; r++) {
    const uint8_t *read = hpc ? base + (offs[r] - offs[0]) : reads + offs[r];
    int32_t len = hpc ? hlen[r] : (int32_t)(offs[r + 1] - offs[r]);
    /* Reads shorter than k have no window; the reference reads unwritten
     * minimizer memory for them (gkc_cuda.cu:320 with len-K+1 <= 0), so they
     * are defined here to produce no superkmer. */
    if (len < k) continue;
    int32_t W = len - k + 1;
    if (W > mmcap) {
      free(mm);
      mmcap = W;
      mm = (uint32_t *)malloc(sizeof(uint32_t) * W);
    }
    orc_window_minimizers(read, len, k, p, mm);
    int32_t s0 = 0;
    for (int32_t i = 1; i <= W; i++) {
      if (i == W || mm[i] != mm[i - 1]) {
        uint32_t slen = (uint32_t)(i - s0 + k - 1);
        if (sb_push(&b, mm[s0] % (uint32_t)nbins, slen, (uint64_t)r, (uint32_t)s0, mm[s0],
                    read + s0))
          return -1;
        s0 = i;
      }
    }
  }
  free(mm);
  free(hreads);
  free(hlen);
  free(horig);
  out->n_skm = b.n;
  out->n_bytes = b.nb;
  out->bin = b.bin;
  out->len = b.len;
  out->byte_off = b.byte_off;
  out->read_id = b.read_id;
  out->start = b.start;
  out->minimizer = b.minimizer;
  out->bytes = b.bytes;
  return 0;
}

void orc_skms_free(orc_skms *s) {
  free(s->bin); free(s->len); free(s->byte_off); free(s->read_id);
  free(s->start); free(s->minimizer); free(s->bytes);
  memset(s, 0, sizeof(*s));
}

/* --- counting: expansion (kmer_counting.cu:95-113, superkmers.hpp:105-127),
 *     canonical form (kmer_counting.cu:33-44), sort (:134) and run-length
 *     count clamped to 2^32-1 (:174-191). --- */

static inline uint32_t get2(const uint8_t *b, uint64_t i) {
  return (b[i / 4] >> (2 * (3 - i % 4))) & 3u;
}

static inline u128 canon128(u128 x, int k) {
  u128 x1 = ~x, res = 0;
  for (int i = 0; i < k; i++) {
    res = (res << 2) | (x1 & 3);
    x1 >>= 2;
  }
  return res < x ? res : x;
}

static int cmp_u128(const void *a, const void *b) {
  u128 x = *(const u128 *)a, y = *(const u128 *)b;
  return x < y ? -1 : (x > y);
}

static int count_group(const uint32_t *len, const uint64_t *byte_off, const uint8_t *bytes,
                       const uint64_t *idx, uint64_t n, int k, u128 **keys_out,
                       uint32_t **cnt_out, uint64_t *nd_out) {
  uint64_t nk = 0;
  for (uint64_t t = 0; t < n; t++) {
    uint64_t i = idx ? idx[t] : t;
    if (len[i] >= (uint32_t)k) nk += len[i] - k + 1;
  }
  u128 *keys = (u128 *)malloc(sizeof(u128) * (nk ? nk : 1));
  if (!keys) return -1;
  const u128 mask = (k == 64) ? ~(u128)0 : (((u128)1 << (2 * k)) - 1);
  uint64_t w = 0;
  for (uint64_t t = 0; t < n; t++) {
    uint64_t i = idx ? idx[t] : t;
    if (len[i] < (uint32_t)k) continue;
    const uint8_t *sb = bytes + byte_off[i];
    u128 x = 0;
    for (int j = 0; j < k; j++) x = (x << 2) | get2(sb, j);
    keys[w++] = canon128(x & mask, k);
    for (uint32_t j = k; j < len[i]; j++) {
      x = ((x << 2) | get2(sb, j)) & mask;
      keys[w++] = canon128(x, k);
    }
  }
  qsort(keys, nk, sizeof(u128), cmp_u128);
  uint64_t nd = 0;
  uint32_t *cnt = (uint32_t *)malloc(sizeof(uint32_t) * (nk ? nk : 1));
  for (uint64_t i = 0; i < nk;) {
    uint64_t j = i;
    while (j < nk && keys[j] == keys[i]) j++;
    keys[nd] = keys[i];
    uint64_t c = j - i;
    cnt[nd] = c > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)c;
    nd++;
    i = j;
  }
  *keys_out = keys;
  *cnt_out = cnt;
  *nd_out = nd;
  return 0;
}

static int alloc_counts(orc_counts *c, uint32_t nbins, uint64_t cap, int wide) {
  memset(c, 0, sizeof(*c));
  c->nbins = nbins;
  c->bin_off = (uint64_t *)calloc(nbins + 1, sizeof(uint64_t));
  c->keys_lo = (uint64_t *)malloc(sizeof(uint64_t) * (cap ? cap : 1));
  c->keys_hi = wide ? (uint64_t *)malloc(sizeof(uint64_t) * (cap ? cap : 1)) : NULL;
  c->counts = (uint32_t *)malloc(sizeof(uint32_t) * (cap ? cap : 1));
  return (c->bin_off && c->keys_lo && c->counts && (!wide || c->keys_hi)) ? 0 : -1;
}

int orc_count_bins(const orc_skms *s, int k, int nbins, orc_counts *out) {
  if (k < 1 || k > 64) return -1;
  uint64_t *cnt_bin = (uint64_t *)calloc(nbins + 1, sizeof(uint64_t));
  for (uint64_t i = 0; i < s->n_skm; i++) cnt_bin[s->bin[i] + 1]++;
  for (int b = 0; b < nbins; b++) cnt_bin[b + 1] += cnt_bin[b];
  uint64_t *idx = (uint64_t *)malloc(sizeof(uint64_t) * (s->n_skm ? s->n_skm : 1));
  uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * nbins);
  for (int b = 0; b < nbins; b++) fill[b] = cnt_bin[b];
  for (uint64_t i = 0; i < s->n_skm; i++) idx[fill[s->bin[i]]++] = i;
  uint64_t total_k = 0;
  for (uint64_t i = 0; i < s->n_skm; i++)
    if (s->len[i] >= (uint32_t)k) total_k += s->len[i] - k + 1;
  if (alloc_counts(out, nbins, total_k, k > 32)) return -1;
  uint64_t w = 0;
  for (int b = 0; b < nbins; b++) {
    out->bin_off[b] = w;
    u128 *keys;
    uint32_t *cnt;
    uint64_t nd;
    if (count_group(s->len, s->byte_off, s->bytes, idx + cnt_bin[b], cnt_bin[b + 1] - cnt_bin[b],
                    k, &keys, &cnt, &nd))
      return -1;
    for (uint64_t i = 0; i < nd; i++) {
      out->keys_lo[w] = (uint64_t)keys[i];
      if (out->keys_hi) out->keys_hi[w] = (uint64_t)(keys[i] >> 64);
      out->counts[w] = cnt[i];
      w++;
    }
    free(keys);
    free(cnt);
  }
  out->bin_off[nbins] = w;
  out->n_distinct = w;
  free(cnt_bin);
  free(idx);
  free(fill);
  return 0;
}

int orc_count_packed(const uint32_t *len, const uint64_t *byte_off, const uint8_t *bytes,
                     uint64_t n_skm, int k, orc_counts *out) {
  if (k < 1 || k > 64) return -1;
  u128 *keys;
  uint32_t *cnt;
  uint64_t nd;
  if (count_group(len, byte_off, bytes, NULL, n_skm, k, &keys, &cnt, &nd)) return -1;
  if (alloc_counts(out, 1, nd, k > 32)) return -1;
  for (uint64_t i = 0; i < nd; i++) {
    out->keys_lo[i] = (uint64_t)keys[i];
    if (out->keys_hi) out->keys_hi[i] = (uint64_t)(keys[i] >> 64);
    out->counts[i] = cnt[i];
  }
  out->bin_off[0] = 0;
  out->bin_off[1] = nd;
  out->n_distinct = nd;
  free(keys);
  free(cnt);
  return 0;
}

void orc_counts_free(orc_counts *c) {
  free(c->bin_off); free(c->keys_lo); free(c->keys_hi); free(c->counts);
  memset(c, 0, sizeof(*c));
}

/* --- sub-sampled counting with position lists (no reference counterpart;
 *     README.md:16 names the use case). --- */

typedef struct {
  u128 key;
  uint32_t pos;
} keypos;

static int cmp_keypos(const void *a, const void *b) {
  const keypos *x = (const keypos *)a, *y = (const keypos *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

int orc_subsample_positions(const uint8_t *reads, const uint64_t *offs, int64_t n_reads,
                            int k, int p, uint32_t mod, orc_poslists *out) {
  memset(out, 0, sizeof(*out));
  if (k < 1 || k > 64 || mod == 0) return -1;
  const u128 mask = (k == 64) ? ~(u128)0 : (((u128)1 << (2 * k)) - 1);
  uint64_t cap = 1024, n = 0;
  keypos *kp = (keypos *)malloc(sizeof(keypos) * cap);
  uint32_t *mm = NULL;
  int32_t mmcap = 0;
  for (int64_t r = 0; r < n_reads; r++) {
    const uint8_t *read = reads + offs[r];
    int32_t len = (int32_t)(offs[r + 1] - offs[r]);
    if (len < k) continue;
    int32_t W = len - k + 1;
    if (W > mmcap) { free(mm); mmcap = W; mm = (uint32_t *)malloc(sizeof(uint32_t) * W); }
    orc_window_minimizers(read, len, k, p, mm);
    u128 x = 0;
    for (int j = 0; j < k - 1; j++) x = (x << 2) | (code_of(read[j]) & 3);
    for (int32_t s = 0; s < W; s++) {
      x = ((x << 2) | (code_of(read[s + k - 1]) & 3)) & mask;
      if (mm[s] % mod) continue;
      if (n == cap) { cap *= 2; kp = (keypos *)realloc(kp, sizeof(keypos) * cap); }
      kp[n].key = canon128(x, k);
      kp[n].pos = (uint32_t)(offs[r] + s);
      n++;
    }
  }
  free(mm);
  qsort(kp, n, sizeof(keypos), cmp_keypos);
  uint64_t nd = 0;
  for (uint64_t i = 0; i < n; i++) nd += (i == 0 || kp[i].key != kp[i - 1].key);
  out->n_distinct = nd;
  out->n_pos = n;
  out->keys_lo = (uint64_t *)malloc(sizeof(uint64_t) * (nd ? nd : 1));
  out->keys_hi = (uint64_t *)malloc(sizeof(uint64_t) * (nd ? nd : 1));
  out->pos_off = (uint64_t *)malloc(sizeof(uint64_t) * (nd + 1));
  out->pos = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint64_t d = 0;
  for (uint64_t i = 0; i < n; i++) {
    if (i == 0 || kp[i].key != kp[i - 1].key) {
      out->keys_lo[d] = (uint64_t)kp[i].key;
      out->keys_hi[d] = (uint64_t)(kp[i].key >> 64);
      out->pos_off[d] = i;
      d++;
    }
    out->pos[i] = kp[i].pos;
  }
  out->pos_off[nd] = n;
  free(kp);
  return 0;
}

void orc_poslists_free(orc_poslists *p) {
  free(p->keys_lo); free(p->keys_hi); free(p->pos_off); free(p->pos);
  memset(p, 0, sizeof(*p));
}

/* ---- partition balance ------------------------------------------------ */

/* CalcSKMPartSize_instream (gkc_cuda.cu:350-365): a superkmer between
 * boundaries s and e adds e - s + k - 1 bases, i.e. its length, to the bin
 * of its first minimizer. */
void orc_partition_sizes(const orc_skms *s, int nbins, uint64_t *sizes) {
  for (int b = 0; b < nbins; b++) sizes[b] = 0;
  for (uint64_t i = 0; i < s->n_skm; i++) sizes[s->bin[i]] += s->len[i];
}

/* calVarStdev (experiment.cpp:18-37): integer mean, then the squares of
 * size - mean in unsigned 64-bit arithmetic (a size below the mean wraps,
 * its square does not change mod 2^64), each converted to double and summed
 * in bin order; variance = sum / n, cv = stdev / mean.  The reference's
 * std::accumulate starts from an int, so its total wraps at 2^31; here the
 * total is the exact sum. */
void orc_balance_stats(const uint64_t *sizes, int n, orc_balance *out) {
  uint64_t sum = 0, mx = 0, mn = UINT64_MAX;
  for (int i = 0; i < n; i++) {
    sum += sizes[i];
    if (sizes[i] > mx) mx = sizes[i];
    if (sizes[i] < mn) mn = sizes[i];
  }
  const uint64_t mean = n ? sum / (uint64_t)n : 0;
  double acc = 0.0;
  for (int i = 0; i < n; i++) {
    uint64_t d = sizes[i] - mean;
    acc += (double)(d * d);
  }
  out->total = sum;
  out->mean = mean;
  out->max = mx;
  out->min = mn;
  out->variance = n ? acc / n : 0.0;
  out->stdev = sqrt(out->variance);
  out->cv = out->stdev / (double)mean;
}

/* --- digests for comparing large outputs without moving them twice (test
 *     infrastructure; not a reference algorithm).  Both are sums of mixed
 *     64-bit words, so they are fast and need one pass. --- */

static inline uint64_t dg_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Per bin: the sum over the bin's list of mix(key, count, index in bin); the
 * list's order enters through the index.  Returns the digest of all bins
 * (each bin's sum mixed with its number and length). */
uint64_t orc_counts_digest(const uint64_t *bin_off, uint32_t nbins, const uint64_t *keys_lo,
                           const uint64_t *keys_hi, const uint32_t *counts, uint64_t *bin_digest) {
  uint64_t total = 0;
  for (uint32_t b = 0; b < nbins; b++) {
    uint64_t h = 0;
    for (uint64_t i = bin_off[b]; i < bin_off[b + 1]; i++) {
      uint64_t j = i - bin_off[b] + 1;
      uint64_t e = dg_mix(keys_lo[i] ^ (0x9E3779B97F4A7C15ull * j));
      e += (keys_hi ? keys_hi[i] : 0) * 0xD1B54A32D192ED03ull + (uint64_t)counts[i] * 0x632BE59BD9B4E019ull;
      h += dg_mix(e);
    }
    if (bin_digest) bin_digest[b] = h;
    total += dg_mix(h + 0xA24BAED4963EE407ull * (b + 1) + (bin_off[b + 1] - bin_off[b]) * 0x9FB21C651E98DF25ull);
  }
  return total;
}

/* Multiset digest of a partition: per superkmer a hash of (length, packed
 * bytes), summed per bin, so the order of superkmers does not matter. */
uint64_t orc_skm_multiset_digest(const uint32_t *bin, const uint32_t *len, const uint64_t *byte_off,
                                 const uint8_t *bytes, uint64_t n_skm, uint32_t nbins,
                                 uint64_t *bin_digest, uint64_t *bin_count) {
  uint64_t *h = (uint64_t *)calloc(nbins, sizeof(uint64_t));
  uint64_t *n = (uint64_t *)calloc(nbins, sizeof(uint64_t));
  for (uint64_t i = 0; i < n_skm; i++) {
    const uint8_t *p = bytes + byte_off[i];
    const uint64_t nb = (len[i] + 3) / 4;
    uint64_t x = dg_mix(0x51AF0DE5ull + len[i]);
    for (uint64_t j = 0; j < nb; j += 8) {
      uint64_t w = 0;
      for (uint64_t t = 0; t < 8 && j + t < nb; t++) w |= (uint64_t)p[j + t] << (8 * t);
      x = dg_mix(x ^ w ^ (j << 56));
    }
    h[bin[i]] += x;
    n[bin[i]]++;
  }
  uint64_t total = 0;
  for (uint32_t b = 0; b < nbins; b++) {
    if (bin_digest) bin_digest[b] = h[b];
    if (bin_count) bin_count[b] = n[b];
    total += dg_mix(h[b] + 0xA24BAED4963EE407ull * (b + 1) + n[b] * 0x9FB21C651E98DF25ull);
  }
  free(h);
  free(n);
  return total;
}
