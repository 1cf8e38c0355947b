/*
 * gz_oracle.h -- CPU restatement of GraphZeppelin's CameoSketch ingest and Boruvka
 * connected-components query, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle: tests/, the smoke check and the
 * bench's CPU-baseline leg use it to check the CUDA path. The product library
 * (graphzeppelin_b200/libgz_b200.so) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates. Byte layout of a sketch is the
 * reference's: num_columns * bkt_per_col packed 12-byte buckets {u64 alpha; u32 gamma}
 * (include/bucket.h:7-12), column-major (bucket col*B + depth), followed by one
 * deterministic bucket (src/sketch.cpp:13), so a dump of V sketches is directly comparable
 * with CCSketchAlg::write_binary's payload (src/cc_sketch_alg.cpp:614-623).
 */
#ifndef GZ_ORACLE_H
#define GZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sample result codes, same order as the reference enum SampleResult (include/sketch.h:20-24). */
enum { GZO_GOOD = 0, GZO_ZERO = 1, GZO_FAIL = 2 };

/* Return codes of gzo_boruvka. */
enum { GZO_OK = 0, GZO_OUT_OF_SAMPLES = 3, GZO_BAD_VERTEX = 5 };

/* XXH3_64bits_withSeed over one little-endian 8-byte input (xxHash 0.8.x, the len 4..8 path
 * XXH3_len_4to8_64b + XXH3_rrmxmx). The reference calls it through vec_hash / col_hash
 * (include/types.h:8-9) from include/bucket.h:56,62. */
uint64_t gzo_xxh3_8b(uint64_t value, uint64_t seed);

/* Sketch sizing for CCSketchAlg(V, seed, sketches_factor):
 *   vector_len  = ceil(V*(V-1)/2)                      include/sketch.h:62-64
 *   num_columns = max(18, ceil(f*log2(V)/(1-log2 1.2))) include/sketch.h:74-76, :188-190
 *   bkt_per_col = ceil(log2(vector_len)) + 1           include/sketch.h:181
 * Returns 0, or -1 when V < 2. */
int gzo_params(uint32_t num_vertices, double sketches_factor, uint32_t *num_columns,
               uint32_t *bkt_per_col);

/* concat_pairing_fn (src/util.cpp:45-51): (min << 32) | max. */
uint64_t gzo_concat_pairing(uint32_t a, uint32_t b);

/* Sketch::update, CameoSketch form (src/sketch.cpp:69-83) on one sketch of
 * (C*B+1)*12 bytes. */
void gzo_sketch_update(uint8_t *sketch, uint32_t C, uint32_t B, uint64_t seed, uint64_t idx);

/* Apply a stream of 9-byte records {u8 type, u32 src, u32 dst} to V sketches stored back to
 * back. Each record toggles index concat_pairing(src,dst) in both endpoint sketches; the type
 * byte is not consulted (CCSketchAlg::update, src/cc_sketch_alg.cpp:127-133; the driver
 * inserts both directions, include/graph_sketch_driver.h:169-172).
 * If vertex_filter is non-NULL only sketches with vertex_filter[v] != 0 are updated (lets a
 * test check a few vertices of a large graph cheaply). Returns 0 or GZO_BAD_VERTEX. */
int gzo_apply_records(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                      const uint8_t *records, size_t n_records, const uint8_t *vertex_filter);

/* CCSketchAlg::apply_update_batch (src/cc_sketch_alg.cpp:106-118): toggles
 * concat_pairing(src, dst_i) in src's sketch only. */
int gzo_apply_batch(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                    uint32_t src, const uint32_t *dsts, size_t n);

/* Sketch::sample for column `col` (src/sketch.cpp:94-116) over an explicit deterministic
 * bucket and the B buckets of that column. Returns GZO_GOOD/ZERO/FAIL; *idx gets the index. */
int gzo_sample(const uint8_t *det_bucket, const uint8_t *col_buckets, uint32_t B, uint64_t seed,
               uint64_t *idx);

/* One sampled component in a Boruvka trace. key = smallest member vertex id. */
typedef struct {
  uint32_t round;
  uint32_t key;
  uint32_t result;
  uint32_t pad;
  uint64_t idx;
} gzo_trace_rec;

/* boruvka_emulation (src/cc_sketch_alg.cpp:464-513) with the round structure of
 * perform_boruvka_round / run_round_zero / sample_supernode (:137-380): round r merges
 * column r and the deterministic bucket of every member of each current component
 * (Sketch::range_merge, src/sketch.cpp:156-179), samples it, unions every GOOD edge, and
 * stops after the first round in which no component FAILed and no union changed the
 * partition. Reaching round num_columns returns GZO_OUT_OF_SAMPLES (Sketch::sample throws
 * OutOfSamplesException, src/sketch.cpp:95-97).
 *   labels_out[v]  = smallest vertex id of v's component (canonical partition)
 *   rounds_out     = last_query_rounds
 *   trace          = optional; every sampled component of every round, sorted by (round,key)
 * Returns GZO_OK / GZO_OUT_OF_SAMPLES / GZO_BAD_VERTEX (a GOOD sample naming a vertex >= V). */
int gzo_boruvka(const uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                uint32_t *labels_out, uint32_t *rounds_out, gzo_trace_rec *trace,
                size_t trace_cap, size_t *trace_len);

/* CubeSketch (the reference built with -DL0_SAMPLING): sizing (include/sketch.h:183-190:
 * 7 columns per sample, num_samples_div = log2(3) - 1; cube = 0 gives CameoSketch), the update
 * (src/sketch.cpp:50-67: every depth 0..d of each column), and Boruvka whose round r merges and
 * scans the cps columns of sample r (src/sketch.cpp:94-116, 156-179). */
int gzo_params_alg(uint32_t num_vertices, double sketches_factor, int cube, uint32_t *num_samples,
                   uint32_t *cols_per_sample, uint32_t *bkt_per_col);
void gzo_sketch_update_cube(uint8_t *sketch, uint32_t C, uint32_t B, uint64_t seed, uint64_t idx);
int gzo_apply_records_alg(uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint64_t seed,
                          const uint8_t *records, size_t n_records, const uint8_t *vertex_filter,
                          int cube);
int gzo_boruvka_alg(const uint8_t *sketches, uint32_t V, uint32_t C, uint32_t B, uint32_t cps,
                    uint64_t seed, uint32_t *labels_out, uint32_t *rounds_out, gzo_trace_rec *trace,
                    size_t trace_cap, size_t *trace_len);

/* Ground truth: exact union-find over the final edge set of a record stream (edges toggled an
 * odd number of times), the role GraphVerifier's Kruskal plays in the reference
 * (test/util/graph_verifier.cpp). labels_out[v] = smallest vertex id of v's component.
 * Returns the number of components, or 0 on a bad vertex id. */
uint32_t gzo_exact_cc(uint32_t V, const uint8_t *records, size_t n_records, uint32_t *labels_out);
/* gzo_exact_cc on `threads` host threads (for full-size streams). */
uint32_t gzo_exact_cc_mt(uint32_t V, const uint8_t *records, size_t n_records, uint32_t *labels_out,
                         int threads);

/* Eager DSU of the default build: CCSketchAlg::pre_insert (src/cc_sketch_alg.cpp:87-102) over
 * the records in stream order, from a valid DSU of singletons. An update joining two sets merges
 * them and records (min, max) as a spanning-forest edge; an update whose endpoints are already
 * joined invalidates the DSU iff (min, max) is a recorded forest edge. Returns the index of the
 * invalidating record, or n_records if the DSU stays valid (then labels_out[v] = smallest member
 * of v's set); (size_t)-1 on a bad vertex id. */
size_t gzo_eager_dsu(uint32_t V, const uint8_t *records, size_t n_records, uint32_t *labels_out);

#ifdef __cplusplus
}
#endif
#endif
