/*
 * gz_gen.c -- fast, seeded generator of large synthetic update streams (host, OpenMP).
 *
 * Every output value is a pure function of (seed, index), built from the splitmix64 finaliser,
 * so the stream is identical for any thread count and on any machine. The shuffle is a
 * pseudo-random permutation of the record positions: a 4-round Feistel network on
 * [0, 2^bits) restricted to [0, n) by cycle walking.
 *
 * Used to build the benchmark's planted-partition streams (hundreds of millions of records).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GZG_API __attribute__((visibility("default")))

static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* uniform u64 keyed by (seed, stream, index) */
static inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) + i);
}

/* ---- planted partition edges --------------------------------------------------------------- */

/* Pair k of component c is an edge iff rnd(seed, 1 + c, k) < p * 2^64. */
static inline int pair_is_edge(uint64_t seed, uint32_t c, uint64_t k, uint64_t thresh) {
  return rnd(seed, 1 + (uint64_t)c, k) < thresh;
}

static inline uint64_t p_to_thresh(double p) {
  if (p >= 1.0) return UINT64_MAX;
  if (p <= 0.0) return 0;
  return (uint64_t)ldexp(p, 64);
}

static inline void tri_decode(uint64_t k, uint64_t *i, uint64_t *j) {
  uint64_t jj = (uint64_t)((1.0 + sqrt(1.0 + 8.0 * (double)k)) / 2.0);
  while (jj * (jj - 1) / 2 > k) --jj;
  while ((jj + 1) * jj / 2 <= k) ++jj;
  *j = jj;
  *i = k - jj * (jj - 1) / 2;
}

/*
 * members: vertex ids grouped by component; comp_off[c]..comp_off[c+1] is component c.
 * Pass out == NULL to count. Returns the number of edges (written as (min << 32) | max).
 */
GZG_API uint64_t gzg_planted_edges(const uint32_t *members, const uint64_t *comp_off,
                                   uint32_t K, double p, uint64_t seed, uint64_t *out) {
  const uint64_t thresh = p_to_thresh(p);
  const uint64_t BLK = 1ull << 20;
  /* global pair offsets per component */
  uint64_t *poff = (uint64_t *)malloc(sizeof(uint64_t) * (K + 1));
  poff[0] = 0;
  for (uint32_t c = 0; c < K; ++c) {
    uint64_t s = comp_off[c + 1] - comp_off[c];
    poff[c + 1] = poff[c] + s * (s - 1) / 2;
  }
  const uint64_t total = poff[K];
  const uint64_t nblk = (total + BLK - 1) / BLK;
  uint64_t *bcnt = (uint64_t *)calloc(nblk + 1, sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 4)
  for (uint64_t b = 0; b < nblk; ++b) {
    uint64_t g0 = b * BLK, g1 = g0 + BLK < total ? g0 + BLK : total, n = 0;
    uint32_t c = 0;
    { uint32_t lo = 0, hi = K; while (lo + 1 < hi) { uint32_t m = (lo + hi) / 2; if (poff[m] <= g0) lo = m; else hi = m; } c = lo; }
    for (uint64_t g = g0; g < g1; ++g) {
      while (g >= poff[c + 1]) ++c;
      n += pair_is_edge(seed, c, g - poff[c], thresh);
    }
    bcnt[b + 1] = n;
  }
  for (uint64_t b = 0; b < nblk; ++b) bcnt[b + 1] += bcnt[b];
  const uint64_t E = bcnt[nblk];
  if (out) {
#pragma omp parallel for schedule(dynamic, 4)
    for (uint64_t b = 0; b < nblk; ++b) {
      uint64_t g0 = b * BLK, g1 = g0 + BLK < total ? g0 + BLK : total, w = bcnt[b];
      uint32_t c = 0;
      { uint32_t lo = 0, hi = K; while (lo + 1 < hi) { uint32_t m = (lo + hi) / 2; if (poff[m] <= g0) lo = m; else hi = m; } c = lo; }
      for (uint64_t g = g0; g < g1; ++g) {
        while (g >= poff[c + 1]) ++c;
        uint64_t k = g - poff[c];
        if (!pair_is_edge(seed, c, k, thresh)) continue;
        uint64_t i, j;
        tri_decode(k, &i, &j);
        uint32_t a = members[comp_off[c] + i], bb = members[comp_off[c] + j];
        uint32_t lo = a < bb ? a : bb, hi = a < bb ? bb : a;
        out[w++] = ((uint64_t)lo << 32) | hi;
      }
    }
  }
  free(poff);
  free(bcnt);
  return E;
}

/*
 * count vertex pairs that are not planted edges (self-loops excluded): comp[v] = component,
 * pos[v] = index of v inside its component. Duplicates are possible; callers dedupe.
 */
GZG_API void gzg_planted_nonedges(uint32_t V, const uint32_t *comp, const uint32_t *pos, double p,
                                  uint64_t seed, uint64_t churn_seed, uint64_t count,
                                  uint64_t *out) {
  const uint64_t thresh = p_to_thresh(p);
  uint64_t t = 0;
  for (uint64_t n = 0; n < count;) {
    uint32_t u = (uint32_t)(rnd(churn_seed, 7, t) % V);
    uint32_t v = (uint32_t)(rnd(churn_seed, 8, t) % V);
    ++t;
    if (u == v) continue;
    if (comp[u] == comp[v]) {
      uint64_t i = pos[u], j = pos[v];
      if (i > j) { uint64_t x = i; i = j; j = x; }
      if (pair_is_edge(seed, comp[u], j * (j - 1) / 2 + i, thresh)) continue;
    }
    uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
    out[n++] = ((uint64_t)lo << 32) | hi;
  }
}

/* ---- shuffled stream ------------------------------------------------------------------------- */

typedef struct {
  uint64_t key;
  int half;
  uint64_t mask;
  uint64_t n;
} perm_t;

static perm_t perm_make(uint64_t n, uint64_t seed) {
  perm_t P;
  int bits = 2;
  while ((1ull << bits) < n) bits += 2;
  P.half = bits / 2;
  P.mask = (1ull << P.half) - 1;
  P.key = mix64(seed ^ 0x5851F42D4C957F2DULL);
  P.n = n;
  return P;
}
static inline uint64_t feistel_fwd(const perm_t *P, uint64_t x) {
  uint64_t L = x >> P->half, R = x & P->mask;
  for (int r = 0; r < 4; ++r) {
    uint64_t F = mix64(R ^ (P->key + (uint64_t)r * 0x9E3779B97F4A7C15ULL)) & P->mask;
    uint64_t nl = R, nr = L ^ F;
    L = nl;
    R = nr;
  }
  return (L << P->half) | R;
}
static inline uint64_t feistel_inv(const perm_t *P, uint64_t y) {
  uint64_t L = y >> P->half, R = y & P->mask;
  for (int r = 3; r >= 0; --r) {
    uint64_t F = mix64(L ^ (P->key + (uint64_t)r * 0x9E3779B97F4A7C15ULL)) & P->mask;
    uint64_t pr = L, pl = R ^ F;
    L = pl;
    R = pr;
  }
  return (L << P->half) | R;
}
static inline uint64_t perm_fwd(const perm_t *P, uint64_t x) {
  do x = feistel_fwd(P, x); while (x >= P->n);
  return x;
}
static inline uint64_t perm_inv(const perm_t *P, uint64_t y) {
  do y = feistel_inv(P, y); while (y >= P->n);
  return y;
}

/*
 * Write E + 2*nc packed 9-byte records: every edge inserted once, every churn pair inserted
 * and later deleted, all in pseudo-random order, each with a random endpoint order.
 * Record at position i is source j = perm(i): j < E edge j; j < E + nc the first copy of churn
 * pair j - E; otherwise the second copy. Whichever copy of a churn pair lands first is the
 * insert.
 */
GZG_API void gzg_shuffle_stream(const uint64_t *edges, uint64_t E, const uint64_t *churn,
                                uint64_t nc, uint64_t seed, uint8_t *out) {
  const uint64_t n = E + 2 * nc;
  if (n == 0) return;
  const perm_t P = perm_make(n, seed);
#pragma omp parallel for schedule(static, 65536)
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t j = perm_inv(&P, i);
    uint64_t idx;
    uint8_t type = 0;
    if (j < E) {
      idx = edges[j];
    } else {
      const uint64_t k = j < E + nc ? j - E : j - E - nc;
      const uint64_t partner = j < E + nc ? j + nc : j - nc;
      idx = churn[k];
      type = perm_fwd(&P, partner) < i ? 1 : 0;
    }
    uint32_t a = (uint32_t)(idx >> 32), b = (uint32_t)idx;
    if (rnd(seed, 3, i) & 1) { uint32_t t = a; a = b; b = t; }
    uint8_t *r = out + 9 * i;
    r[0] = type;
    memcpy(r + 1, &a, 4);
    memcpy(r + 5, &b, 4);
  }
}

/* ---- Chung-Lu power-law streams ----------------------------------------------------------- */

/* vertex drawn with probability proportional to its weight: cdf holds the normalised cumulative
 * weights (cdf[V-1] == 1); ids relabels weight ranks to vertex ids */
static inline uint32_t cl_draw(const double *cdf, const uint32_t *ids, uint32_t V, uint64_t r) {
  const double x = (double)(r >> 11) * 0x1.0p-53;
  uint32_t lo = 0, hi = V - 1;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (cdf[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  return ids[lo];
}

/* edge i of the stream: endpoints drawn independently from the weights, a repeat of the first
 * endpoint redrawn (up to 16 times, then its neighbour id) so there are no self-loops */
static inline void cl_edge(const double *cdf, const uint32_t *ids, uint32_t V, uint64_t seed,
                           uint64_t i, uint32_t *u, uint32_t *v) {
  *u = cl_draw(cdf, ids, V, rnd(seed, 101, i));
  uint32_t w = cl_draw(cdf, ids, V, rnd(seed, 102, i));
  for (uint32_t t = 0; w == *u && t < 16; ++t) w = cl_draw(cdf, ids, V, rnd(seed, 103 + t, i));
  if (w == *u) w = (*u + 1) % V;
  *v = w;
}

static inline void put_record(uint8_t *p, uint8_t type, uint32_t u, uint32_t v) {
  p[0] = type;
  memcpy(p + 1, &u, 4);
  memcpy(p + 5, &v, 4);
}

/*
 * A Chung-Lu stream of m edge inserts (i.i.d. weighted endpoints, so already in random order),
 * then deletions of nd = floor(del_frac * m) of them, then re-inserts of nr = floor(rein_frac * nd)
 * of the deleted ones, each phase in its own pseudo-random order. Writes m + nd + nr packed
 * 9-byte records to out (NULL: count only) and returns that number. An insert that repeats an
 * earlier edge toggles it, as any repeated update does.
 */
GZG_API uint64_t gzg_chung_lu_stream(const double *cdf, const uint32_t *ids, uint32_t V, uint64_t m,
                                     double del_frac, double rein_frac, uint64_t seed, uint8_t *out) {
  const uint64_t nd = (uint64_t)floor(del_frac * (double)m);
  const uint64_t nr = (uint64_t)floor(rein_frac * (double)nd);
  if (!out) return m + nd + nr;
  const perm_t Pd = perm_make(nd ? nd : 1, seed ^ 0xDE1E7Eull);
  const perm_t Pr = perm_make(nr ? nr : 1, seed ^ 0x4E1A5Eull);
#pragma omp parallel for schedule(static, 65536)
  for (uint64_t i = 0; i < m + nd + nr; ++i) {
    uint64_t e;
    uint8_t type = 0;
    if (i < m) {
      e = i;
    } else if (i < m + nd) {
      e = perm_fwd(&Pd, i - m); /* a deleted edge is one of the first nd inserted */
      type = 1;
    } else {
      e = perm_fwd(&Pr, i - m - nd); /* a re-inserted edge is one of the first nr deleted */
    }
    uint32_t u, v;
    cl_edge(cdf, ids, V, seed, e, &u, &v);
    put_record(out + 9 * i, type, u, v);
  }
  return m + nd + nr;
}
