/*
 * gz_b200.h -- C ABI of the B200-native GraphZeppelin sketch-ingest and Boruvka-query path.
 *
 * One opaque handle (gz_alg_t) stands for one CCSketchAlg (reference include/cc_sketch_alg.h:69)
 * whose V vertex sketches live in the HBM of the current CUDA device. Every entry point takes
 * plain pointers and sizes, returns a gz_status code, and never throws. Host buffers passed in
 * are borrowed for the duration of the call only; device buffers (the *_device entry points)
 * must stay valid until the next gz_flush / query on the same handle.
 *
 * Each entry point names the reference interface it replaces (file:line, paths relative to the
 * GraphZeppelin source tree). Semantics that the reference leaves to exceptions map to codes:
 *   OutOfSamplesException  (include/sketch.h:193-204)       -> GZ_ERR_OUT_OF_SAMPLES
 *   UpdateLockedException  (include/cc_sketch_alg.h:25-29)  -> GZ_ERR_LOCKED
 *
 * Thread safety: every call on a handle takes that handle's lock, so concurrent
 * gz_apply_update_batch calls from worker threads (the driver contract,
 * include/graph_sketch_driver.h:49-52) are safe; they are staged and applied in bulk.
 */
#ifndef GZ_B200_H
#define GZ_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GZ_API __attribute__((visibility("default")))
#else
#define GZ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gz_alg gz_alg_t;

/* Status codes. */
enum gz_status {
  GZ_OK = 0,
  GZ_ERR_INVALID = 1,        /* bad argument (null handle, V < 2, size mismatch ...) */
  GZ_ERR_CUDA = 2,           /* a CUDA runtime call failed; gz_last_error() has the text */
  GZ_ERR_OUT_OF_SAMPLES = 3, /* Boruvka needed more rounds than the sketch has columns */
  GZ_ERR_LOCKED = 4,         /* update while a query runs, or after a failed query */
  GZ_ERR_BAD_VERTEX = 5,     /* an update named a vertex id >= V (the update is dropped) */
  GZ_ERR_NOMEM = 6,          /* device or pinned host allocation failed */
  GZ_ERR_IO = 7,             /* file could not be read or written */
  GZ_ERR_TIMEOUT = 8,        /* a bounded device-side wait gave up (kernel returned early) */
  GZ_ERR_BAD_SAMPLE = 9,     /* a checksum-valid sample decoded to a vertex id >= V */
  GZ_ERR_NO_DEVICE = 10,     /* no usable CUDA device (there is no CPU fallback) */
  GZ_ERR_BUDGET = 11         /* a server's sketch-byte budget has no room for this tenant */
};

/* Query codes, reference enum QueryCode (include/cc_sketch_alg.h:60-63). */
enum gz_query_code { GZ_CONNECTIVITY = 0, GZ_KSPANNINGFORESTS = 1 };

/* Sketch algorithm: CameoSketch (the reference's default build) or CubeSketch (the reference
 * built with -DL0_SAMPLING: 7 columns per sample, every depth 0..d updated, include/sketch.h:183-190,
 * src/sketch.cpp:50-67). */
enum gz_sketch_algorithm { GZ_CAMEO_SKETCH = 0, GZ_CUBE_SKETCH = 1 };

/* Sample results, reference enum SampleResult (include/sketch.h:20-24). */
enum gz_sample_result { GZ_SAMPLE_GOOD = 0, GZ_SAMPLE_ZERO = 1, GZ_SAMPLE_FAIL = 2 };

/* Sizing and configuration of a handle. */
typedef struct gz_params {
  uint32_t num_vertices;        /* CCSketchAlg::get_num_vertices (include/cc_sketch_alg.h:255) */
  uint32_t num_columns;         /* Sketch::get_columns == calc_cc_samples(V, f) (include/sketch.h:74-76) */
  uint32_t bkt_per_col;         /* Sketch::calc_bkt_per_col(calc_vector_length(V)) (include/sketch.h:181) */
  uint32_t num_buckets;         /* num_columns * bkt_per_col + 1 (src/sketch.cpp:13) */
  uint64_t seed;                /* CCSketchAlg::get_seed (include/cc_sketch_alg.h:256) */
  uint64_t sketch_bytes;        /* Sketch::bucket_array_bytes (include/sketch.h:117) */
  uint64_t desired_updates_per_batch; /* include/cc_sketch_alg.h:146-150 */
  uint64_t max_rounds;          /* CCSketchAlg::max_rounds (include/cc_sketch_alg.h:257) */
  double sketches_factor;       /* CCAlgConfiguration::get_sketches_factor */
  double batch_factor;          /* CCAlgConfiguration::get_batch_factor */
  uint32_t vertices_per_tile;   /* device layout: sketches staged together in shared memory */
  uint32_t num_tiles;
  uint32_t vertices_per_bin;    /* device gutter: vertices sharing one gutter bin */
  uint32_t num_bins;
  uint32_t cols_per_sample;     /* Sketch::cols_per_sample: 1 (CameoSketch) or 7 (CubeSketch) */
  uint32_t sketch_algorithm;    /* enum gz_sketch_algorithm */
  uint32_t in_place;            /* 1: sketches too large to stage in shared memory are updated in HBM */
  uint32_t entry_form;          /* gutter entries of records: 1 = plain (hashed per endpoint where
                                   applied), 2 = coded (each record hashed once, bucket planes),
                                   3 = coded with 3-bit depth codes (larger graphs) */
} gz_params_t;

/* One sampled component of one Boruvka round (parity tracing). key = smallest member id. */
typedef struct gz_trace_rec {
  uint32_t round;
  uint32_t key;
  uint32_t result; /* enum gz_sample_result */
  uint32_t pad;
  uint64_t idx;    /* sampled edge index (min << 32) | max, 0 unless GOOD */
} gz_trace_rec_t;

/* Device time spent per phase since the last reset (CUDA events on the handle's stream). */
typedef struct gz_profile {
  double gutter_ms;        /* record parsing + counting sort into per-tile gutters */
  double sketch_update_ms; /* the sketch-update kernel (shared-memory XOR of every gutter entry) */
  double query_ms;         /* Boruvka rounds, labels included */
  uint64_t gutter_launches;
  uint64_t sketch_update_launches;
  uint64_t query_rounds;
  uint64_t entries_applied; /* endpoint updates folded into sketches */
  uint64_t kernel_launches; /* every kernel this handle launched */
} gz_profile_t;

/* ---- library ------------------------------------------------------------------------------ */

GZ_API const char *gz_version(void);
GZ_API const char *gz_status_string(int status);
/* Text of the last error raised on the calling thread (empty if none). */
GZ_API const char *gz_last_error(void);

/* ---- construction ------------------------------------------------------------------------- */

/* CCSketchAlg(num_vertices, seed, CCAlgConfiguration) -- src/cc_sketch_alg.cpp:11-28,
 * with CCAlgConfiguration::sketches_factor / batch_factor (src/cc_alg_configuration.cpp:10-26:
 * a factor <= 0 falls back to 1). Allocates V zeroed sketches on the current device. */
GZ_API int gz_create(uint32_t num_vertices, uint64_t seed, double sketches_factor, double batch_factor,
              gz_alg_t **out);

/* gz_create with the sketch algorithm chosen at run time (the reference chooses it when it is
 * compiled): GZ_CAMEO_SKETCH or GZ_CUBE_SKETCH. num_columns is then samples x cols_per_sample,
 * and a query can run max_rounds = samples rounds. */
GZ_API int gz_create_ex(uint32_t num_vertices, uint64_t seed, double sketches_factor,
                        double batch_factor, int sketch_algorithm, gz_alg_t **out);

/* CCSketchAlg::construct_from_serialized_data -- src/cc_sketch_alg.cpp:30-64. Reads a
 * write_binary file (u64 seed, u32 V, f64 sketches_factor, V sketches). The DSU starts invalid. */
GZ_API int gz_create_from_serialized(const char *path, double batch_factor, gz_alg_t **out);
/* Same, for a file written by a handle of the given sketch algorithm (the file format does not
 * record it). */
GZ_API int gz_create_from_serialized_ex(const char *path, double batch_factor, int sketch_algorithm,
                                        gz_alg_t **out);

/* ~CCSketchAlg -- src/cc_sketch_alg.cpp:66-77. */
GZ_API int gz_destroy(gz_alg_t *alg);

GZ_API int gz_get_params(const gz_alg_t *alg, gz_params_t *out);

/* Device gutter capacity in endpoint updates (default: V * desired_updates_per_batch, the
 * reference's total gutter size). A full gutter is applied to the sketches before more
 * updates are accepted. */
GZ_API int gz_set_gutter_capacity(gz_alg_t *alg, uint64_t endpoint_updates);

/* ---- ingest (the driver / algorithm contract, include/graph_sketch_driver.h:28-69) -------- */

/* CCSketchAlg::allocate_worker_memory -- include/cc_sketch_alg.h:161-169. Host staging only:
 * worker deltas are formed on the device, so this just records the worker count. */
GZ_API int gz_allocate_worker_memory(gz_alg_t *alg, size_t num_workers);

/* CCSketchAlg::pre_insert -- src/cc_sketch_alg.cpp:79-104 (NO_EAGER_DSU form: any update
 * invalidates the cached query answer). */
GZ_API int gz_pre_insert(gz_alg_t *alg, uint32_t src, uint32_t dst, int type, int thr_id);

/* Eager DSU, the reference's default build (without -DNO_EAGER_DSU): when enabled, gz_pre_insert,
 * gz_update and gz_ingest_records run CCSketchAlg::pre_insert (src/cc_sketch_alg.cpp:87-102) on
 * each update in order -- an update joining two components merges them and records a
 * spanning-forest edge; an update to a recorded forest edge invalidates the DSU -- so that while
 * the DSU stays valid, gz_has_cached_query is true and queries are answered from it without
 * Boruvka. Updates this cannot see (gz_ingest_records_device, gz_apply_raw_buckets_update)
 * invalidate it. Off by default (the NO_EAGER_DSU behaviour: every update invalidates the
 * cached answer). */
GZ_API int gz_set_eager_dsu(gz_alg_t *alg, int enable);

/* CCSketchAlg::apply_update_batch -- src/cc_sketch_alg.cpp:106-118: toggles edge index
 * concat_pairing_fn(src, dsts[i]) in src's sketch only. dsts is a host array. */
GZ_API int gz_apply_update_batch(gz_alg_t *alg, int thr_id, uint32_t src, const uint32_t *dsts,
                          size_t n);

/* CCSketchAlg::apply_raw_buckets_update -- src/cc_sketch_alg.cpp:120-123: XORs num_buckets
 * packed 12-byte buckets (host memory, Sketch layout) into src's sketch. */
GZ_API int gz_apply_raw_buckets_update(gz_alg_t *alg, uint32_t src, const void *raw_buckets);

/* CCSketchAlg::update -- src/cc_sketch_alg.cpp:127-133: one stream update, both endpoints. */
GZ_API int gz_update(gz_alg_t *alg, uint32_t src, uint32_t dst, int type);

/* Whole-stream ingest that replaces GraphSketchDriver::process_stream_until's reader threads
 * and the GutteringSystem (include/graph_sketch_driver.h:141-191): n_records packed 9-byte
 * records {u8 type, u32 src, u32 dst} (reference README "Binary Stream Format") in HOST
 * memory. Copies are pipelined against the device gutter; returns when the host buffer is no
 * longer needed. Both endpoints of every record are updated; the type byte is not consulted
 * (insert and delete are the same XOR toggle). */
GZ_API int gz_ingest_records(gz_alg_t *alg, const void *records, size_t n_records);

/* Same, records already in device memory of the handle's device (any byte alignment). */
GZ_API int gz_ingest_records_device(gz_alg_t *alg, const void *d_records, size_t n_records);

/* GraphSketchDriver::prep_query -- include/graph_sketch_driver.h:193-203: folds every buffered
 * update into the sketches and synchronizes. Reports deferred device errors (BAD_VERTEX). */
GZ_API int gz_flush(gz_alg_t *alg);

/* CCSketchAlg::has_cached_query -- include/cc_sketch_alg.h:184-190. */
GZ_API int gz_has_cached_query(const gz_alg_t *alg, int query_code, int *out);

/* Connectivity query on the state at submission: gz_query_submit queues every update so far
 * and then boruvka_emulation (src/cc_sketch_alg.cpp:464-513, every round on the device, with
 * its own query buffers) on the handle's stream, and returns at once; updates made after it are
 * queued behind the query, so the caller never waits for it and the answer is the state at
 * submission without a copy of the sketches (queries interleaved with ingest). Several tickets
 * may be in flight. gz_query_wait blocks until its query is done and returns parent_out (NULL or
 * V entries), the component count and the rounds, or GZ_ERR_OUT_OF_SAMPLES / GZ_ERR_BAD_SAMPLE.
 * Device errors of earlier updates are reported by the next flush. Ticket queries leave the
 * handle's cached answer and update lock alone. */
GZ_API int gz_query_submit(gz_alg_t *alg, uint64_t *ticket);
GZ_API int gz_query_wait(gz_alg_t *alg, uint64_t ticket, uint32_t *parent_out, uint32_t *num_cc,
                         size_t *rounds);

/* ---- queries ------------------------------------------------------------------------------ */

/* CCSketchAlg::connected_components -- src/cc_sketch_alg.cpp:515-557, returning the
 * ConnectedComponents payload (src/return_types.cpp:5-19): parent_out[v] = representative of
 * v's component (may be NULL), *num_cc = number of components. Runs device Boruvka unless the
 * cached answer is valid; flushes buffered updates first. */
GZ_API int gz_connected_components(gz_alg_t *alg, uint32_t *parent_out, uint32_t *num_cc);

/* CCSketchAlg::point_query -- src/cc_sketch_alg.cpp:570-612. */
GZ_API int gz_point_query(gz_alg_t *alg, uint32_t a, uint32_t b, int *out);

/* CCSketchAlg::last_query_rounds -- include/cc_sketch_alg.h:252. */
GZ_API int gz_last_query_rounds(const gz_alg_t *alg, size_t *out);

/* CCSketchAlg::calc_spanning_forest -- src/cc_sketch_alg.cpp:559-568: the edges whose union
 * changed the partition during the last Boruvka (runs one if the cache is invalid).
 * edges_out holds up to cap (src, dst) pairs with src < dst; *n_edges gets the count. */
GZ_API int gz_spanning_forest(gz_alg_t *alg, uint32_t *edges_out, size_t cap, size_t *n_edges);

/* ---- checkpoint ---------------------------------------------------------------------------- */

/* CCSketchAlg::write_binary -- src/cc_sketch_alg.cpp:614-623 (byte-identical format). */
GZ_API int gz_write_binary(gz_alg_t *alg, const char *path);

/* Sketch::zero_contents (src/sketch.cpp:86-92) on every vertex sketch, discarding buffered
 * updates: the handle holds the empty graph again (the cached answer is dropped). */
GZ_API int gz_clear(gz_alg_t *alg);

/* Copy the raw bucket bytes of all V sketches (V * sketch_bytes, reference layout) to a host
 * buffer; buffered updates are applied first. */
GZ_API int gz_dump_sketches(gz_alg_t *alg, void *host_buf, size_t bytes);

/* ---- ingest without allocation ------------------------------------------------------------------
 * No counterpart in the reference. For callers that may not allocate GPU memory: plugins inside
 * a host framework that owns all device memory through its own pool (a library cudaMalloc would
 * bypass its accounting), and latency-critical loops where cudaMalloc / cudaFree would
 * synchronize the device and stall other streams. Applies n_records packed 9-byte records (device
 * memory, any alignment) to the V sketches at d_sketches (caller-owned device memory,
 * V * sketch_bytes in the write_binary bucket layout, updated in place) for the sketch geometry
 * of (num_vertices, seed, sketches_factor), exactly as gz_ingest_records_device + gz_flush on a
 * handle would, and synchronizes `stream` (a cudaStream_t, NULL for the default stream).
 * It calls no cudaMalloc / cudaFree and no allocating library routine: its scratch is one fixed
 * file-scope device array of about 34 MiB that every GPU loading the library holds until the
 * process exits. Limits: at most 2,097,152 records per call and at most 4,194,304 vertices;
 * larger calls return GZ_ERR_INVALID without touching memory. The first call on each device looks
 * up the array's address (cudaGetSymbolAddress). Every call synchronizes `stream` before it
 * returns (and reads a status word back from the GPU), so it must not be called while `stream` is
 * being captured into a CUDA graph. Every call shares the array, which keeps the previous call's
 * contents (each call clears what must start at zero), so two calls whose GPU work overlapped
 * would race on it: the entry point therefore serializes its callers with a process-wide lock
 * that it holds until its GPU work is done, on success and on failure alike. On a failure after
 * the work was queued (a CUDA error, a timed-out device wait), the caller's sketches may be
 * partly updated. */
GZ_API int gz_ingest_records_noalloc(void *d_sketches, uint32_t num_vertices, uint64_t seed,
                                     double sketches_factor, const void *d_records,
                                     size_t n_records, void *stream);

/* ---- instrumentation ----------------------------------------------------------------------- */

/* Record every sampled component of every Boruvka round (for parity checks). */
GZ_API int gz_set_trace(gz_alg_t *alg, int enable);
GZ_API int gz_get_trace(gz_alg_t *alg, gz_trace_rec_t *out, size_t cap, size_t *len);

/* Per-phase device timings (CUDA events). enable != 0 starts a fresh accumulation. */
GZ_API int gz_set_profiling(gz_alg_t *alg, int enable);
GZ_API int gz_get_profile(gz_alg_t *alg, gz_profile_t *out);

/* The cudaStream_t (as void*) every kernel of this handle is launched on. */
GZ_API int gz_get_stream(gz_alg_t *alg, void **stream_out);

/* Peak rate of this GPU at the ingest's per-column hash: a register-only kernel evaluating the
 * 8-byte XXH3 of a column (the record's premixed input XOR the column's premixed seed constant,
 * the two rrmxmx multiplies and shifts) and the bucket-depth count-trailing-zeros, eight
 * independent chains per thread, each next input being the last one XOR its depth code. Timed
 * with CUDA events on the current device; *hashes_per_s gets the best of `repeats` launches. */
GZ_API int gz_measure_hash_rate(int repeats, double *hashes_per_s);

/* Peak rate of this GPU at the sketch update's shared-memory operation: bucket-slot updates of
 * the bucket planes, each two conflict-free 32-bit red.shared.xor (one entry = 32 slot steps,
 * 1024 threads per SM, no hashing, no global traffic). *updates_per_s gets the best of
 * `repeats` launches, in slot updates per second. */
GZ_API int gz_measure_update_rate(int repeats, double *updates_per_s);

/* Tuning knobs of the ingest kernels (0 picks the default): vertices per shared-memory tile
 * (power of two in [4, 64]; at most 32 with coded entries), threads per block of the
 * sketch-update kernel, tiles per gutter bin (power of two <= 64; 1 with coded entries), and the
 * gutter entry form for records: 1 = plain entries {vertex, neighbour} (hashed per endpoint by a
 * staged-tile sketch-update kernel), 2 = coded entries (each record hashed once in the gutter into
 * per-column depth codes, applied through bucket planes; CameoSketch with at most 31 columns and
 * at most 8192 gutter bins; 4-bit codes where they fit a 16-byte entry, else 3-bit codes),
 * 3 = coded entries with 3-bit codes (code 7 = depth 7 or more, hashed again where applied).
 * 0 picks coded entries where they apply. Buffered updates are applied first. */
GZ_API int gz_set_tuning(gz_alg_t *alg, uint32_t vertices_per_tile, uint32_t threads_per_block,
                         uint32_t tiles_per_bin, uint32_t entry_form);
/* Route of sparse tiles (one tile per gutter bin, plain CameoSketch entries): a tile holding
 * fewer entries than factor x (its sketch bytes / (32 (columns + 1))) -- the break-even of
 * staging it in shared memory against updating its buckets in HBM -- is updated in place with
 * global atomics. 0 = always staged, 1 = the default. Same role as gz_batch_set_route. */
GZ_API int gz_set_direct_factor(gz_alg_t *alg, double factor);
/* How queries run. mode = 2: the whole Boruvka emulation in one cooperative kernel launch, every
 * round on the device with grid barriers between its phases. mode = 1: one CUDA graph of
 * per-phase kernels whose conditional while node loops over the rounds. mode = 0: the same
 * per-phase kernels with the round loop on the host (a synchronize per round; ticket submits then
 * wait for their query), for profilers that do not see kernels inside conditional graphs.
 * mode = -1 (the default): 2 up to 2^18 vertices, 1 above (the faster of the two at each size).
 * Answers, rounds and sample traces are the same in every mode. GZ_ERR_INVALID for another mode. */
GZ_API int gz_set_query_graph(gz_alg_t *alg, int mode);
/* Sketch-update kernel of a handle: mode 1 = the tile pipeline (a producer warp loads the next
 * tiles' sketches and writes finished ones back while the other warps hash; one tile per gutter
 * bin; CameoSketch only, ignored otherwise), 2..4 = the pipeline with that many tile buffers,
 * 0 = one staged tile per CTA at a time, -1 = chosen by the handle (the default: coded entries
 * and bucket planes where they apply). Modes 0..4 select plain entries. Re-picks the default
 * tiling. */
GZ_API int gz_set_pipeline(gz_alg_t *alg, int mode);

/* ---- many graphs on one GPU ------------------------------------------------------------------
 * A gz_batch_t holds num_graphs independent CCSketchAlg instances (each its own V, seed and
 * sketch geometry, include/cc_sketch_alg.h:69) in one device allocation. One ingest call runs one
 * gutter pass and ONE persistent sketch-update launch over the tiles of every graph; one query
 * runs Boruvka for all graphs at once, each round a replayed CUDA graph, each graph stopping on
 * its own. Per graph the sketches, partition, last_query_rounds and out-of-samples outcome equal
 * those of a gz_alg_t with the same V and seed fed the same records. */
typedef struct gz_batch gz_batch_t;

/* num_vertices[g], seeds[g]: as gz_create for graph g. vertices_per_tile may be NULL (default
 * tiling per graph) or hold a power of two in [4, 64] (0 = default) per graph. */
GZ_API int gz_batch_create(uint32_t num_graphs, const uint32_t *num_vertices, const uint64_t *seeds,
                           double sketches_factor, const uint32_t *vertices_per_tile,
                           gz_batch_t **out);
GZ_API int gz_batch_destroy(gz_batch_t *batch);
/* gz_get_params of graph g (batch_factor 1). */
GZ_API int gz_batch_get_params(gz_batch_t *batch, uint32_t graph, gz_params_t *out);
/* Applies records of every graph: graph g's packed 9-byte records {u8 type, u32 src, u32 dst}
 * (reference README "Binary Stream Format") are d_records[offsets[g] .. offsets[g+1]) in device memory
 * (offsets has num_graphs + 1 entries, in records). Synchronous: the records are folded into
 * the sketches when the call returns. A vertex id >= its graph's V gives GZ_ERR_BAD_VERTEX. */
GZ_API int gz_batch_ingest_device(gz_batch_t *batch, const void *d_records, const uint64_t *offsets);
/* Same, records in host memory (copied to the device inside the call). */
GZ_API int gz_batch_ingest(gz_batch_t *batch, const void *records, const uint64_t *offsets);
/* Zeroes every graph's sketches. */
GZ_API int gz_batch_clear(gz_batch_t *batch);
/* connected_components (src/cc_sketch_alg.cpp:515-557) of every graph. labels_out (NULL or
 * sum of V entries, graph-major) gets each vertex's graph-local root; num_cc, rounds and status
 * (NULL or num_graphs entries) get each graph's component count, last_query_rounds, and
 * GZ_OK or GZ_ERR_OUT_OF_SAMPLES. The call itself fails only on device or argument errors. */
GZ_API int gz_batch_connected_components(gz_batch_t *batch, uint32_t *labels_out, uint32_t *num_cc,
                                         uint32_t *rounds, int *status);
/* Graph g's sketches, V * sketch_bytes bytes in gz_dump_sketches' layout. */
GZ_API int gz_batch_dump_sketches(gz_batch_t *batch, uint32_t graph, void *host_buf, size_t bytes);
/* Replaces graph g's sketches with V * sketch_bytes bytes in that layout (the sketch part of a
 * write_binary file, as construct_from_serialized_data reads it, src/cc_sketch_alg.cpp:30-64). */
GZ_API int gz_batch_load_sketches(gz_batch_t *batch, uint32_t graph, const void *host_buf, size_t bytes);
/* Shape of the batched sketch-update launch: threads per CTA (multiple of 32 in [64, 1024]),
 * CTAs sharing one SM (1..4, threads * CTAs <= 2048; each CTA stages its tiles in 1/ctas of the
 * SM's shared memory, so one CTA's bulk copies overlap another's XORs), and vertices per tile per
 * graph (NULL or 0 = the largest power of two <= 64 that fits). 0 picks the default (1024, 1).
 * Sketch contents are kept; only the tiling changes. */
GZ_API int gz_batch_set_tuning(gz_batch_t *batch, uint32_t threads_per_block, uint32_t ctas_per_sm,
                               const uint32_t *vertices_per_tile);
/* Routing of each ingest call, per graph: a graph whose call brings few records for its size
 * (the in-place cost estimate, 2 (C + 1) bucket sectors per record, below sparse_factor times
 * the staged cost, its sketches read and written once plus the gutter's bytes) skips the
 * gutter: each record is hashed once and XORed into both endpoints' sketches in HBM. The rest
 * are guttered and applied tile by tile in shared memory. 0 = always staged, 1 = the default,
 * a huge value = always in place. */
GZ_API int gz_batch_set_route(gz_batch_t *batch, double sparse_factor);
/* Autotuner: times trial ingests (records_per_vertex random edge records per vertex, 0 = 64) on
 * a scratch batch with one representative graph per sketch-size class (same columns and buckets
 * per column) and applies the fastest CTA shape and per-class vertices per tile to this batch.
 * vertices_per_tile_out (NULL or num_graphs entries) gets the choice. The sketches are kept. */
GZ_API int gz_batch_autotune(gz_batch_t *batch, uint32_t records_per_vertex,
                             uint32_t *vertices_per_tile_out);
GZ_API int gz_batch_set_profiling(gz_batch_t *batch, int enable);

/* ---- serving: many tenants resident in one HBM budget ------------------------------------------
 * A gz_server_t keeps the sketches of many tenants (each one CCSketchAlg with its own V and
 * seed) in one device arena of budget_bytes, admitting a tenant only while its sketch bytes
 * (V x columns x buckets x 12 B, rounded) fit. gz_server_ingest applies update batches of any set
 * of tenants with one batched gutter pass and one persistent sketch-update launch.
 * gz_server_query_submit snapshots the queried tenants' sketches (after every earlier ingest
 * call, before every later one) into a pool of snapshot_bytes and runs their batched Boruvka on
 * a second stream from a worker thread, so ingest calls made meanwhile proceed; the answer is
 * the connected_components (src/cc_sketch_alg.cpp:515-557) of each tenant at submission. */
typedef struct gz_server gz_server_t;

/* Device bytes one tenant of num_vertices takes from the budget. */
GZ_API int gz_server_tenant_bytes(uint32_t num_vertices, double sketches_factor, uint64_t *bytes);
GZ_API int gz_server_create(uint64_t budget_bytes, uint64_t snapshot_bytes, double sketches_factor,
                            gz_server_t **out);
GZ_API int gz_server_destroy(gz_server_t *server);
/* Admits a tenant with zeroed sketches; GZ_ERR_BUDGET when the budget has no room for it. */
GZ_API int gz_server_admit(gz_server_t *server, uint32_t num_vertices, uint64_t seed,
                           uint32_t *tenant_out);
/* Frees a tenant's sketches (queries already submitted for it still complete). */
GZ_API int gz_server_evict(gz_server_t *server, uint32_t tenant);
GZ_API int gz_server_usage(gz_server_t *server, uint64_t *used_bytes, uint64_t *budget_bytes,
                           uint32_t *tenants);
/* gz_batch_set_route for the server's ingest calls. */
GZ_API int gz_server_set_route(gz_server_t *server, double sparse_factor);
/* How later gz_server_query_submit calls read the tenants' sketches. snapshot = 1 (the default):
 * copied into the snapshot pool first, so ingest of those tenants may continue at once. snapshot
 * = 0: read in place, no copy; an ingest call or eviction naming a tenant of an unfinished query
 * waits until that query is done (the answer is still the state at submission). For callers that
 * hold a tenant's updates while its query runs, as a per-tenant request queue does. Queries
 * queued behind a running one are answered together by one batched Boruvka. */
GZ_API int gz_server_set_query_snapshot(gz_server_t *server, int snapshot);
GZ_API int gz_server_get_params(gz_server_t *server, uint32_t tenant, gz_params_t *out);
/* Tenant tenants[i]'s packed 9-byte records are records[offsets[i] .. offsets[i+1]) in host
 * memory (offsets: n + 1 entries; each tenant at most once per call). Synchronous. */
GZ_API int gz_server_ingest(gz_server_t *server, uint32_t n, const uint32_t *tenants,
                            const void *records, const uint64_t *offsets);
/* Same as gz_server_ingest with the records given as segments: segment k is counts[k] records
 * at host address ptrs[k] for tenant tenants[k] (a tenant's segments consecutive). Each segment
 * is copied once, straight to the device (no host-side gathering). */
GZ_API int gz_server_ingest_segments(gz_server_t *server, uint32_t num_segments,
                                     const uint32_t *tenants, const void *const *ptrs,
                                     const uint64_t *counts);
/* Page-locks (gz_host_register) or releases (gz_host_unregister) a host buffer the caller keeps
 * its incoming records in, so that gz_ingest_records and gz_server_ingest* copy from it at full
 * host-link speed; pageable buffers go through the driver's staging at a fraction of that.
 * No counterpart in the reference: its update buffers never leave host memory. */
GZ_API int gz_host_register(void *ptr, uint64_t bytes);
GZ_API int gz_host_unregister(void *ptr);
GZ_API int gz_server_query_submit(gz_server_t *server, uint32_t n, const uint32_t *tenants,
                                  uint64_t *ticket);
/* Whether a submitted query's answer is ready (gz_server_query_wait would not block). */
GZ_API int gz_server_query_ready(gz_server_t *server, uint64_t ticket, int *ready);
/* Waits for a submitted query: labels_out (NULL or the sum of the tenants' V, in submission
 * order) gets each vertex's tenant-local root; num_cc, rounds, status (NULL or n entries) as
 * gz_batch_connected_components. */
GZ_API int gz_server_query_wait(gz_server_t *server, uint64_t ticket, uint32_t *labels_out,
                                uint32_t *num_cc, uint32_t *rounds, int *status);
GZ_API int gz_server_dump_sketches(gz_server_t *server, uint32_t tenant, void *host_buf,
                                   size_t bytes);
/* Checkpoint of one tenant in CCSketchAlg::write_binary's format (src/cc_sketch_alg.cpp:614-623),
 * and admission of a tenant from such a file (construct_from_serialized_data,
 * src/cc_sketch_alg.cpp:30-64; the file's sketches_factor must be the server's): eviction and
 * re-admission without replaying the stream. */
GZ_API int gz_server_write_binary(gz_server_t *server, uint32_t tenant, const char *path);
GZ_API int gz_server_admit_serialized(gz_server_t *server, const char *path, uint32_t *tenant_out);
GZ_API int gz_batch_get_profile(gz_batch_t *batch, gz_profile_t *out);

#ifdef __cplusplus
}
#endif
#endif /* GZ_B200_H */
