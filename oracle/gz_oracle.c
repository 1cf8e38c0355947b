/*
 * gz_oracle.c -- plain-C restatement of GraphZeppelin's CameoSketch ingest and Boruvka
 * query (see gz_oracle.h for the function-by-function reference citations).
 *
 * TEST INFRASTRUCTURE ONLY: the parity oracle. Never linked into the product library.
 * Single-threaded and written for clarity, not speed.
 */
#include "gz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <omp.h>
#include <string.h>

/* ---- xxHash XXH3, 8-byte input path (published algorithm, xxHash 0.8.x) ---------------- */

/* First 24 bytes of the XXH3 default secret (XXH3_kSecret); the 4..8-byte path reads the
 * little-endian u64 words at offsets 8 and 16. */
static const uint8_t kSecretHead[24] = {
    0xb8, 0xfe, 0x6c, 0x39, 0x23, 0xa4, 0x4b, 0xbe, 0x7c, 0x01, 0x81, 0x2c,
    0xf7, 0x21, 0xad, 0x1c, 0xde, 0xd4, 0x6d, 0xe9, 0x83, 0x90, 0x97, 0xdb};
#define GZO_PRIME_MX2 0x9FB21C651E98DF25ULL

static uint64_t read_le64(const uint8_t *p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}
static uint32_t read_le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint32_t bswap32(uint32_t x) {
  return (x >> 24) | ((x >> 8) & 0xff00u) | ((x << 8) & 0xff0000u) | (x << 24);
}
static uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

uint64_t gzo_xxh3_8b(uint64_t value, uint64_t seed) {
  /* XXH3_len_4to8_64b with len == 8 */
  uint8_t in[8];
  for (int i = 0; i < 8; ++i) in[i] = (uint8_t)(value >> (8 * i));
  seed ^= (uint64_t)bswap32((uint32_t)seed) << 32;
  uint32_t input1 = read_le32(in);
  uint32_t input2 = read_le32(in + 4);
  uint64_t bitflip = (read_le64(kSecretHead + 8) ^ read_le64(kSecretHead + 16)) - seed;
  uint64_t input64 = (uint64_t)input2 + ((uint64_t)input1 << 32);
  uint64_t h = input64 ^ bitflip;
  /* XXH3_rrmxmx(h, 8) */
  h ^= rotl64(h, 49) ^ rotl64(h, 24);
  h *= GZO_PRIME_MX2;
  h ^= (h >> 35) + 8;
  h *= GZO_PRIME_MX2;
  return h ^ (h >> 28);
}

/* ---- sizing ------------------------------------------------------------------------------ */

int gzo_params_alg(uint32_t V, double f, int cube, uint32_t *num_samples, uint32_t *cols_per_sample,
                   uint32_t *bkt_per_col) {
  if (V < 2) return -1;
  uint64_t vec_len = (uint64_t)ceil((double)V * (uint32_t)(V - 1) / 2);
  *bkt_per_col = (uint32_t)(ceil(log2((double)vec_len)) + 1);
  /* include/sketch.h:183-190: CubeSketch (L0_SAMPLING) takes 7 columns per sample and
   * num_samples_div = log2(3) - 1; CameoSketch 1 column and 1 - log2(2 - 0.8) */
  const double num_samples_div = cube ? log2(3) - 1 : 1 - log2(2 - 0.8);
  size_t s = (size_t)ceil(f * log2((double)V) / num_samples_div);
  *num_samples = (uint32_t)(s > 18 ? s : 18);
  *cols_per_sample = cube ? 7 : 1;
  return 0;
}

int gzo_params(uint32_t V, double f, uint32_t *num_columns, uint32_t *bkt_per_col) {
  if (V < 2) return -1;
  /* Sketch::calc_vector_length: ceil(double(V) * (V - 1) / 2), stored as vec_t */
  uint64_t vec_len = (uint64_t)ceil((double)V * (uint32_t)(V - 1) / 2);
  /* Sketch::calc_bkt_per_col(size_t n): ceil(log2(n)) + 1 */
  *bkt_per_col = (uint32_t)(ceil(log2((double)vec_len)) + 1);
  /* Sketch::calc_cc_samples with num_samples_div = 1 - log2(2 - 0.8) (CameoSketch) */
  const double num_samples_div = 1 - log2(2 - 0.8);
  size_t s = (size_t)ceil(f * log2((double)V) / num_samples_div);
  *num_columns = (uint32_t)(s > 18 ? s : 18);
  return 0;
}

uint64_t gzo_concat_pairing(uint32_t a, uint32_t b) {
  uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return ((uint64_t)lo << 32) | hi;
}

/* ---- bucket helpers (include/bucket.h) ---------------------------------------------------- */

static uint64_t bkt_alpha(const uint8_t *b) { return read_le64(b); }
static uint32_t bkt_gamma(const uint8_t *b) { return read_le32(b + 8); }
static void bkt_xor(uint8_t *b, uint64_t alpha, uint32_t gamma) {
  for (int i = 0; i < 8; ++i) b[i] ^= (uint8_t)(alpha >> (8 * i));
  for (int i = 0; i < 4; ++i) b[8 + i] ^= (uint8_t)(gamma >> (8 * i));
}
/* Bucket_Boruvka::is_good (include/bucket.h:65-67): gamma == (u32) hash(alpha, seed) */
static int bkt_good(const uint8_t *b, uint64_t seed) {
  return bkt_gamma(b) == (uint32_t)gzo_xxh3_8b(bkt_alpha(b), seed);
}

/* Sketch::update of the CubeSketch build (src/sketch.cpp:50-67): the deterministic bucket, then
 * in every column all buckets of depth 0..d (d < B). */
void gzo_sketch_update_cube(uint8_t *sk, uint32_t C, uint32_t B, uint64_t seed, uint64_t idx) {
  uint32_t checksum = (uint32_t)gzo_xxh3_8b(idx, seed);
  bkt_xor(sk + (size_t)C * B * 12, idx, checksum);
  for (uint32_t c = 0; c < C; ++c) {
    uint64_t h = gzo_xxh3_8b(idx, seed + 5ull * c) | (1ull << B);
    uint32_t depth = (uint32_t)__builtin_ctzll(h);
    if (depth < B)
      for (uint32_t j = 0; j <= depth; ++j) bkt_xor(sk + ((size_t)c * B + j) * 12, idx, checksum);
  }
}

void gzo_sketch_update(uint8_t *sk, uint32_t C, uint32_t B, uint64_t seed, uint64_t idx) {
  /* checksum = get_index_hash(idx, checksum_seed() == seed) truncated to vec_hash_t */
  uint32_t checksum = (uint32_t)gzo_xxh3_8b(idx, seed);
  /* deterministic bucket is the last one (num_buckets - 1 == C*B) */
  bkt_xor(sk + (size_t)C * B * 12, idx, checksum);
  for (uint32_t c = 0; c < C; ++c) {
    /* get_index_depth(idx, column_seed(c) = seed + 5c, B): ctz(hash | 1 << B) */
    uint64_t h = gzo_xxh3_8b(idx, seed + 5ull * c) | (1ull << B);
    uint32_t depth = (uint32_t)__builtin_ctzll(h);
    if (depth < B) bkt_xor(sk + ((size_t)c * B + depth) * 12, idx, checksum);
  }
}

int gzo_apply_records_alg(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                          const uint8_t *rec, size_t n, const uint8_t *filter, int cube) {
  const size_t sk_bytes = ((size_t)C * B + 1) * 12;
  void (*upd)(uint8_t *, uint32_t, uint32_t, uint64_t, uint64_t) =
      cube ? gzo_sketch_update_cube : gzo_sketch_update;
  int rc = 0;
  for (size_t i = 0; i < n; ++i, rec += 9) {
    uint32_t u = read_le32(rec + 1), v = read_le32(rec + 5);
    if (u >= V || v >= V) { rc = GZO_BAD_VERTEX; continue; }
    uint64_t idx = gzo_concat_pairing(u, v);
    if (!filter || filter[u]) upd(sketches + u * sk_bytes, C, B, seed, idx);
    if (!filter || filter[v]) upd(sketches + v * sk_bytes, C, B, seed, idx);
  }
  return rc;
}

int gzo_apply_records(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                      const uint8_t *rec, size_t n, const uint8_t *filter) {
  return gzo_apply_records_alg(sketches, V, C, B, seed, rec, n, filter, 0);
}

int gzo_apply_batch(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                    uint32_t src, const uint32_t *dsts, size_t n) {
  const size_t sk_bytes = ((size_t)C * B + 1) * 12;
  if (src >= V) return GZO_BAD_VERTEX;
  for (size_t i = 0; i < n; ++i) {
    if (dsts[i] >= V) return GZO_BAD_VERTEX;
    gzo_sketch_update(sketches + src * sk_bytes, C, B, seed, gzo_concat_pairing(src, dsts[i]));
  }
  return 0;
}

/* Sketch::sample (src/sketch.cpp:94-116) over cps consecutive columns of B buckets. */
static int sample_cols(const uint8_t *det, const uint8_t *col, uint32_t cps, uint32_t B, uint64_t seed,
                       uint64_t *idx) {
  *idx = 0;
  if (bkt_alpha(det) == 0 && bkt_gamma(det) == 0) return GZO_ZERO;
  if (bkt_good(det, seed)) { *idx = bkt_alpha(det); return GZO_GOOD; }
  for (uint32_t j = 0; j < cps * B; ++j)
    if (bkt_good(col + 12 * j, seed)) { *idx = bkt_alpha(col + 12 * j); return GZO_GOOD; }
  return GZO_FAIL;
}

int gzo_sample(const uint8_t *det, const uint8_t *col, uint32_t B, uint64_t seed, uint64_t *idx) {
  *idx = 0;
  if (bkt_alpha(det) == 0 && bkt_gamma(det) == 0) return GZO_ZERO;
  if (bkt_good(det, seed)) { *idx = bkt_alpha(det); return GZO_GOOD; }
  for (uint32_t j = 0; j < B; ++j)
    if (bkt_good(col + 12 * j, seed)) { *idx = bkt_alpha(col + 12 * j); return GZO_GOOD; }
  return GZO_FAIL;
}

/* ---- Boruvka ------------------------------------------------------------------------------ */

static uint32_t uf_find(uint32_t *p, uint32_t x) {
  while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
  return x;
}
/* deterministic link: smaller root id wins (partition is independent of the link rule) */
static int uf_union(uint32_t *p, uint32_t a, uint32_t b) {
  a = uf_find(p, a); b = uf_find(p, b);
  if (a == b) return 0;
  if (a < b) p[b] = a; else p[a] = b;
  return 1;
}

int gzo_boruvka_alg(const uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint32_t cps,
                    uint64_t seed, uint32_t *labels, uint32_t *rounds_out, gzo_trace_rec *trace,
                    size_t cap, size_t *trace_len) {
  const size_t sk_bytes = ((size_t)C * B + 1) * 12;
  const size_t acc_bytes = (size_t)(cps * B + 1) * 12; /* the round's columns, then the det bucket */
  const uint32_t num_samples = C / cps;
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * V);
  uint32_t *root = (uint32_t *)malloc(sizeof(uint32_t) * V);
  uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * V);
  uint8_t *acc = (uint8_t *)malloc(acc_bytes * V);
  size_t tl = 0;
  int rc = GZO_OK;
  uint32_t round = 0;
  for (uint32_t v = 0; v < V; ++v) parent[v] = v;
  for (;;) {
    if (round >= num_samples) { rc = GZO_OUT_OF_SAMPLES; break; }
    /* components fixed before this round (create_merge_instructions) */
    for (uint32_t v = 0; v < V; ++v) root[v] = uf_find(parent, v);
    for (uint32_t v = 0; v < V; ++v) key[v] = UINT32_MAX;
    for (uint32_t v = 0; v < V; ++v)
      if (key[root[v]] == UINT32_MAX) key[root[v]] = v;
    memset(acc, 0, acc_bytes * V);
    /* range_merge of sample `round` (columns round*cps .. +cps) and the deterministic bucket */
    for (uint32_t v = 0; v < V; ++v) {
      const uint8_t *sk = sketches + v * sk_bytes;
      uint8_t *a = acc + root[v] * acc_bytes;
      for (size_t j = 0; j < (size_t)cps * B * 12; ++j) a[j] ^= sk[(size_t)round * cps * B * 12 + j];
      for (size_t j = 0; j < 12; ++j) a[(size_t)cps * B * 12 + j] ^= sk[(size_t)C * B * 12 + j];
    }
    /* sample every component (iterating roots in key order gives a sorted trace) */
    int modified = 0;
    uint32_t n_good = 0;
    uint64_t *good = (uint64_t *)malloc(sizeof(uint64_t) * V);
    for (uint32_t k = 0; k < V; ++k) {
      uint32_t r = root[k];
      if (key[r] != k) continue; /* k is the smallest member of component r */
      uint64_t idx;
      uint8_t *a = acc + r * acc_bytes;
      int res = sample_cols(a + (size_t)cps * B * 12, a, cps, B, seed, &idx);
      if (trace && tl < cap) {
        trace[tl].round = round; trace[tl].key = k; trace[tl].result = (uint32_t)res;
        trace[tl].pad = 0; trace[tl].idx = idx;
      }
      ++tl;
      if (res == GZO_FAIL) modified = 1;
      else if (res == GZO_GOOD) good[n_good++] = idx;
    }
    for (uint32_t i = 0; i < n_good; ++i) {
      uint32_t a = (uint32_t)(good[i] >> 32), b = (uint32_t)good[i];
      if (a >= V || b >= V) { rc = GZO_BAD_VERTEX; continue; }
      if (uf_union(parent, a, b)) modified = 1;
    }
    free(good);
    if (rc != GZO_OK) break;
    if (!modified) break;
    ++round;
  }
  for (uint32_t v = 0; v < V; ++v) root[v] = uf_find(parent, v);
  for (uint32_t v = 0; v < V; ++v) key[v] = UINT32_MAX;
  for (uint32_t v = 0; v < V; ++v) {
    if (key[root[v]] == UINT32_MAX) key[root[v]] = v;
    labels[v] = key[root[v]];
  }
  *rounds_out = round;
  if (trace_len) *trace_len = tl;
  free(parent); free(root); free(key); free(acc);
  return rc;
}

int gzo_boruvka(const uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                uint32_t *labels, uint32_t *rounds_out, gzo_trace_rec *trace, size_t cap,
                size_t *trace_len) {
  return gzo_boruvka_alg(sketches, V, C, B, 1, seed, labels, rounds_out, trace, cap, trace_len);
}

/* ---- exact connected components over the final edge set ---------------------------------- */

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

uint32_t gzo_exact_cc(uint32_t V, const uint8_t *rec, size_t n, uint32_t *labels) {
  uint64_t *e = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * V);
  for (size_t i = 0; i < n; ++i) {
    uint32_t u = read_le32(rec + 9 * i + 1), v = read_le32(rec + 9 * i + 5);
    if (u >= V || v >= V) { free(e); free(parent); return 0; }
    e[i] = gzo_concat_pairing(u, v);
  }
  qsort(e, n, sizeof(uint64_t), cmp_u64);
  for (uint32_t v = 0; v < V; ++v) parent[v] = v;
  for (size_t i = 0; i < n;) {
    size_t j = i;
    while (j < n && e[j] == e[i]) ++j;
    if ((j - i) & 1) uf_union(parent, (uint32_t)(e[i] >> 32), (uint32_t)e[i]); /* odd => present */
    i = j;
  }
  uint32_t ncc = 0;
  for (uint32_t v = 0; v < V; ++v) {
    uint32_t r = uf_find(parent, v);
    labels[v] = r; /* smaller root wins in uf_union, so the root is the smallest member */
    if (r == v) ++ncc;
  }
  free(e); free(parent);
  return ncc;
}

/* The same answer for full-size streams, on `threads` host threads: the edge indices are
 * bucketed by their smaller endpoint, each bucket sorted on its own, the indices of odd
 * multiplicity (present after the stream's toggles) unioned; labels = smallest member id. */
static void sort_u64(uint64_t *a, size_t n) {
  /* LSD radix sort, 8 bits per pass through a scratch array; a byte that is the same in every
   * key is skipped (inside a bucket of smaller endpoints the top bytes are) */
  if (n < 2) return;
  uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * n);
  uint64_t *src = a, *dst = tmp;
  for (int pass = 0; pass < 8; ++pass) {
    const int sh = 8 * pass;
    size_t cnt[256] = {0};
    uint64_t all_or = 0, all_and = ~(uint64_t)0;
    for (size_t i = 0; i < n; ++i) { all_or |= src[i]; all_and &= src[i]; }
    if ((((all_or ^ all_and) >> sh) & 0xff) == 0) continue; /* this byte is constant */
    for (size_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xff]++;
    size_t run = 0;
    for (int b = 0; b < 256; ++b) { size_t c = cnt[b]; cnt[b] = run; run += c; }
    for (size_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xff]++] = src[i];
    uint64_t *t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, sizeof(uint64_t) * n);
  free(tmp);
}

uint32_t gzo_exact_cc_mt(uint32_t V, const uint8_t *rec, size_t n, uint32_t *labels, int threads) {
  if (threads < 1) threads = 1;
  const uint32_t nb = 4096;
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t *out = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
  size_t *cnt = (size_t *)calloc((size_t)threads * nb, sizeof(size_t));
  size_t *bstart = (size_t *)calloc(nb + 1, sizeof(size_t));
  size_t *bkeep = (size_t *)calloc(nb, sizeof(size_t));
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * (V ? V : 1));
  int bad = 0;
#pragma omp parallel num_threads(threads)
  {
    const int t = omp_get_thread_num(), T = omp_get_num_threads();
    const size_t i0 = n * (size_t)t / T, i1 = n * (size_t)(t + 1) / T;
    size_t *c = cnt + (size_t)t * nb;
    for (size_t i = i0; i < i1; ++i) {
      uint32_t u = read_le32(rec + 9 * i + 1), v = read_le32(rec + 9 * i + 5);
      if (u >= V || v >= V) { bad = 1; u = v = 0; }
      keys[i] = gzo_concat_pairing(u, v);
      c[(uint32_t)(((uint64_t)(u < v ? u : v) * nb) / V)]++;
    }
#pragma omp barrier
#pragma omp single
    {
      size_t run = 0;
      for (uint32_t b = 0; b < nb; ++b) {
        bstart[b] = run;
        for (int k = 0; k < T; ++k) {
          const size_t x = cnt[(size_t)k * nb + b];
          cnt[(size_t)k * nb + b] = run;
          run += x;
        }
      }
      bstart[nb] = run;
    }
    for (size_t i = i0; i < i1; ++i) {
      const uint32_t lo = (uint32_t)(keys[i] >> 32);
      out[c[(uint32_t)(((uint64_t)lo * nb) / V)]++] = keys[i];
    }
#pragma omp barrier
#pragma omp for schedule(dynamic, 16)
    for (uint32_t b = 0; b < nb; ++b) {
      uint64_t *e = out + bstart[b];
      const size_t m = bstart[b + 1] - bstart[b];
      sort_u64(e, m);
      size_t w = 0;
      for (size_t i = 0; i < m;) {
        size_t j = i;
        while (j < m && e[j] == e[i]) ++j;
        if ((j - i) & 1) e[w++] = e[i]; /* odd multiplicity => present */
        i = j;
      }
      bkeep[b] = w;
    }
  }
  uint32_t ncc = 0;
  if (!bad) {
    for (uint32_t v = 0; v < V; ++v) parent[v] = v;
    for (uint32_t b = 0; b < nb; ++b)
      for (size_t i = 0; i < bkeep[b]; ++i) {
        const uint64_t k = out[bstart[b] + i];
        uf_union(parent, (uint32_t)(k >> 32), (uint32_t)k);
      }
    for (uint32_t v = 0; v < V; ++v) {
      const uint32_t r = uf_find(parent, v);
      labels[v] = r;
      if (r == v) ++ncc;
    }
  }
  free(keys); free(out); free(cnt); free(bstart); free(bkeep); free(parent);
  return ncc;
}

/* Eager DSU, CCSketchAlg::pre_insert of the default build (src/cc_sketch_alg.cpp:87-102), run
 * over the records in stream order from a valid DSU of singletons. The forest-edge set is an
 * open-addressing table of (min << 32 | max) keys (a forest has at most V - 1 edges). */
size_t gzo_eager_dsu(uint32_t V, const uint8_t *rec, size_t n, uint32_t *labels) {
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * V);
  size_t cap = 16;
  while (cap < 2 * (size_t)V) cap <<= 1;
  uint64_t *set = (uint64_t *)calloc(cap, sizeof(uint64_t)); /* 0 = empty (idx 0 is (0,0): a self-loop, never a forest edge) */
  for (uint32_t v = 0; v < V; ++v) parent[v] = v;
  size_t pos = n;
  for (size_t i = 0; i < n; ++i) {
    uint32_t u = read_le32(rec + 9 * i + 1), v = read_le32(rec + 9 * i + 5);
    if (u >= V || v >= V) { free(parent); free(set); return (size_t)-1; }
    uint32_t a = u < v ? u : v, b = u < v ? v : u;
    uint64_t key = ((uint64_t)a << 32) | b;
    size_t h = (size_t)((key * 0x9E3779B97F4A7C15ull) >> 20) & (cap - 1);
    if (uf_union(parent, a, b)) {
      while (set[h] && set[h] != key) h = (h + 1) & (cap - 1);
      set[h] = key;
    } else {
      int found = 0;
      while (set[h]) {
        if (set[h] == key) { found = 1; break; }
        h = (h + 1) & (cap - 1);
      }
      if (found) { pos = i; break; }
    }
  }
  if (pos == n && labels)
    for (uint32_t v = 0; v < V; ++v) labels[v] = uf_find(parent, v);
  free(parent);
  free(set);
  return pos;
}
