// gz_capi.cu -- the C ABI (include/gz_b200.h): one handle = one CCSketchAlg whose sketches live in
// HBM, fed by a device-resident gutter and queried by device Boruvka.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <condition_variable>
#include <map>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/gz_b200.h"
#include "gz_device.cuh"
#include "gz_kernels.cuh"
#include "gz_ingest_plan.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define GZ_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? GZ_ERR_NOMEM : GZ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define GZ_TRY(expr)          \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != GZ_OK) return rc_; \
  } while (0)

template <class T>
int dev_alloc(T **p, size_t count) {
  if (*p) return GZ_OK;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess)
    return fail(GZ_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) +
                                  " bytes): " + cudaGetErrorString(e));
  *p = static_cast<T *>(q);
  return GZ_OK;
}
template <class T>
void dev_free(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <class T>
int host_alloc(T **p, size_t count) {
  if (*p) return GZ_OK;
  void *q = nullptr;
  cudaError_t e = cudaMallocHost(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(GZ_ERR_NOMEM, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
  *p = static_cast<T *>(q);
  return GZ_OK;
}
template <class T>
void host_free(T *&p) {
  if (p) cudaFreeHost(p);
  p = nullptr;
}

using gz::kStageBuffers;
using gz::kStageRecords;
constexpr uint64_t kEntStage = 1ull << 20;      // staged apply_update_batch entries per flush
constexpr uint64_t kMaxChunkEntries = 1ull << 31;

}  // namespace

namespace gz {
// Columns and buckets per column of one vertex sketch, CCSketchAlg's sizing
// (src/cc_sketch_alg.cpp:16-17; include/sketch.h:62-76, :181, :188-190) evaluated with the same
// double expressions so the results agree bit for bit: B = ceil(log2(V(V-1)/2)) + 1 buckets per
// column, C = max(18, ceil(f * log2(V) / (1 - log2(1.2)))) columns.
// CubeSketch (the reference built with -DL0_SAMPLING, include/sketch.h:183-190) takes 7 columns per
// sample and num_samples_div = log2(3) - 1; CameoSketch 1 column.
void sketch_sizing_alg(uint32_t V, double f, bool cube, uint32_t &samples, uint32_t &cps, uint32_t &B) {
  if (!cube) {
    sketch_sizing(V, f, samples, B);
    cps = 1;
    return;
  }
  const uint64_t vec_len = (uint64_t)std::ceil(double(V) * (uint32_t)(V - 1) / 2);
  B = (uint32_t)(std::ceil(std::log2((double)vec_len)) + 1);
  const double num_samples_div = std::log2(3) - 1;
  const size_t s = (size_t)std::ceil(f * std::log2((double)V) / num_samples_div);
  samples = (uint32_t)std::max<size_t>(18, s);
  cps = 7;
}

void sketch_sizing(uint32_t V, double f, uint32_t &C, uint32_t &B) {
  const uint64_t vec_len = (uint64_t)std::ceil(double(V) * (uint32_t)(V - 1) / 2);
  B = (uint32_t)(std::ceil(std::log2((double)vec_len)) + 1);
  const double num_samples_div = 1 - std::log2(2 - 0.8);
  const size_t s = (size_t)std::ceil(f * std::log2((double)V) / num_samples_div);
  C = (uint32_t)std::max<size_t>(18, s);
}
}  // namespace gz

// Error text for entry points defined in other files of this library.
void gz_internal_set_error(const std::string &msg) { g_last_error = msg; }

struct gz_alg {
  std::mutex mtx;
  int device = 0;
  // configuration
  uint32_t V = 0, C = 0, B = 0, nb = 0;
  // CubeSketch (L0_SAMPLING) or CameoSketch: samples of cps columns each (C = samples * cps)
  bool cube = false;
  uint32_t samples = 0, cps = 1;
  bool in_place = false;  // sketches too large to stage 4 in shared memory: updated in HBM
  uint64_t seed = 0;
  double sketches_factor = 1, batch_factor = 1;
  uint64_t sketch_bytes = 0, desired_batch = 0;
  uint32_t tile_shift = 2, ntiles = 0, threads = 1024;
  uint32_t bin_shift = 2, nbins = 0;
  size_t smem_optin = 227 * 1024;
  size_t num_workers = 1;
  // sketches + per-column hash constants
  uint8_t *d_sk = nullptr;
  uint64_t *d_flip = nullptr;
  uint32_t *d_status = nullptr;  // [0] status bits, [1] work counter
  uint32_t *h_status = nullptr;  // pinned mirror
  // device gutter
  uint8_t *d_gutter = nullptr;  // chunks of plain (8 B) or coded (16 B) endpoint entries
  uint64_t entry_cap = 0;       // capacity in endpoint updates
  uint64_t gutter_bytes = 0, gutter_used = 0, entries_pending = 0;
  double direct_factor = 1.0;   // scales the in-place threshold of sparse tiles (0 = never)
  int pipe_mode = -1;           // pipelined sketch update: 1 on, 2..4 on with that many buffers,
                                // 0 off, -1 automatic
  bool pipe = false;            // the pipelined kernel is the one in use
  uint32_t nbuf = 2;            // its tile buffers
  // every update so far reached both endpoints' sketches (records, gz_update): the XOR of all
  // vertex sketches is zero, which lets a query merge its largest component from the rest
  bool symmetric = true;
  // records become coded entries (each record hashed once) applied through bucket planes
  bool planes = false;
  bool codes3 = false;          // the coded entries carry 3-bit codes (kEntryCoded3)
  int planes_mode = -1;         // entry form asked for: -1 automatic, 0 plain, 1 coded (4-bit
                                // codes where they fit, else 3-bit), 2 coded with 3-bit codes
  gz::PlaneHash ph{};
  gz::ChunkTable chunks{};
  int nchunks = 0;
  uint32_t *d_bin_off = nullptr;
  uint64_t *d_hist = nullptr, *d_scan_tmp = nullptr, *d_total = nullptr, *d_cursor = nullptr;
  uint32_t *d_fill = nullptr;
  size_t hist_words = 0;
  // host-record pipeline
  uint8_t *d_stage[kStageBuffers] = {};
  uint64_t stage_cap = 0;  // records each staging buffer holds
  cudaEvent_t ev_copied[kStageBuffers] = {}, ev_free[kStageBuffers] = {};
  // apply_update_batch staging
  uint2 *h_ent[2] = {nullptr, nullptr};
  uint2 *d_ent[2] = {nullptr, nullptr};
  cudaEvent_t ev_ent_done[2] = {nullptr, nullptr};
  uint64_t h_ent_n = 0;
  int h_ent_cur = 0;
  uint32_t *d_raw = nullptr;
  // query state
  gz::BoruvkaBufs bv{};
  bool bv_alloc = false;
  uint32_t *d_final = nullptr, *d_ncc = nullptr;
  bool dsu_valid = true, update_locked = false, labels_on_host = false;
  // eager DSU (the reference's default build, src/cc_sketch_alg.cpp:87-102): a host union-find
  // and the spanning-forest edge set, kept while dsu_valid; host_answer = it holds merges the
  // device answer (d_final) lacks
  bool eager = false, host_answer = false, boruvka_ran = false;
  std::vector<uint32_t> hdsu;
  std::unordered_set<uint64_t> hforest;
  // how a query runs: 2 = one cooperative kernel (every round on the device), 1 = a CUDA graph of
  // the per-phase kernels with a conditional while node over the rounds (qgraph), 0 = the same
  // kernels with the round loop on the host, -1 = by size (query_mode_of)
  gz::BoruvkaGraph qgraph;
  int query_mode = -1;
  uint32_t *h_qpin = nullptr;  // pinned: rounds, out-of-samples flag, components
  // queries by ticket (gz_query_submit / gz_query_wait): the query graph enqueued on the
  // handle's stream behind every update submitted before it, with its own buffers, so the
  // answer is the state at submission while later updates queue up behind it
  struct Ticket {
    cudaEvent_t done = nullptr;
    uint32_t *labels = nullptr;  // pinned, V entries
    uint32_t *pin = nullptr;     // pinned: rounds, out-of-samples flag, components, status
    bool graph = true;           // ran as the query graph (its kernels are counted at the end)
  };
  struct Tickets {
    gz::BoruvkaBufs bv{};
    gz::BoruvkaGraph graph;
    uint32_t *d_final = nullptr, *d_ncc = nullptr;
    std::map<uint64_t, Ticket> live;
    std::vector<Ticket> pool;
    uint64_t next = 1;
  } tq;
  uint32_t deferred_status = 0;  // device status bits seen by a ticket, reported at the next flush
  std::atomic<bool> query_running{false};
  size_t last_rounds = 0;
  uint32_t last_ncc = 0;
  std::vector<uint32_t> h_labels;
  bool trace = false;
  // streams
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  // profiling
  bool prof = false;
  struct Ev {
    cudaEvent_t a, b;
    int phase;
  };
  std::vector<Ev> prof_pending;
  std::vector<cudaEvent_t> ev_pool;
  gz_profile_t prof_acc{};
  uint64_t launch_base = 0;

  gz::SketchGeom sgeom() const {
    gz::SketchGeom g;
    g.V = V;
    g.C = C;
    g.B = B;
    g.sketch_words = nb * 3;
    g.tile_shift = tile_shift;
    g.ntiles = ntiles;
    g.bin_shift = bin_shift;
    g.nbins = nbins;
    g.cube = cube ? 1 : 0;
    g.nbuf = nbuf;
    // Staging a tile moves its sketches twice (bulk load + write-back); updating it in place
    // costs about C + 1 bucket sectors read and written per entry. Below the break-even entry
    // count a tile goes in place (one tile per bin and plain CameoSketch entries only).
    if (bin_shift == tile_shift && !cube && !planes) {
      const double even = (double)((uint64_t)nb * 12 << tile_shift) / (32.0 * (C + 1));
      g.direct_max = (uint32_t)std::min(even * direct_factor, 4.0e9);
    }
    return g;
  }
  gz::GutterGeom ggeom() const { return gz::GutterGeom{V, bin_shift, nbins}; }
  gz::PlaneGeom pgeom() const {
    gz::PlaneGeom g;
    g.V = V;
    g.C = C;
    g.B = B;
    g.sketch_words = nb * 3;
    g.tile_shift = tile_shift;
    g.ntiles = ntiles;
    g.bin_shift = bin_shift;
    g.nbins = nbins;
    // A tile through the planes costs its write-back, about 2 x 12 x (C min(B, rows) + 1) bytes
    // per vertex read and written; in place an entry costs its C + 1 buckets' sectors, each read
    // and written by an L2 atomic. Below the break-even entry count a tile goes in place.
    const double wb = 24.0 * ((double)C * std::min<uint32_t>(B, gz::kPlaneRows - 1) + 1) *
                      (double)(1u << tile_shift);
    const double even = wb / (64.0 * (C + 1));
    g.direct_max = (uint32_t)std::min(even * direct_factor, 4.0e9);
    return g;
  }
  gz::BoruvkaGeom bgeom() const {
    gz::BoruvkaGeom g;
    g.V = V;
    g.C = C;
    g.B = B;
    g.sketch_words = nb * 3;
    g.flip_chk = gz::xxh3_flip(seed);
    g.span = gz::kBoruvkaSpan;
    g.cps = cps;
    g.complement = symmetric ? 1 : 0;
    return g;
  }

  cudaEvent_t get_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  int prof_begin() {
    if (!prof) return -1;
    Ev e{get_event(), get_event(), 0};
    cudaEventRecord(e.a, stream);
    prof_pending.push_back(e);
    return (int)prof_pending.size() - 1;
  }
  void prof_end(int i, int phase) {
    if (i < 0) return;
    prof_pending[i].phase = phase;
    cudaEventRecord(prof_pending[i].b, stream);
  }
  void prof_collect() {
    if (prof_pending.empty()) return;
    cudaStreamSynchronize(stream);
    for (auto &e : prof_pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, e.a, e.b);
      if (e.phase == 0) {
        prof_acc.gutter_ms += ms;
        prof_acc.gutter_launches++;
      } else if (e.phase == 1) {
        prof_acc.sketch_update_ms += ms;
        prof_acc.sketch_update_launches++;
      } else {
        prof_acc.query_ms += ms;
      }
      ev_pool.push_back(e.a);
      ev_pool.push_back(e.b);
    }
    prof_pending.clear();
  }
};

namespace {

// Default gutter bins: the fewest tiles per bin that brings the bin count within the
// shared-memory sort-scatter's range (each extra tile per bin costs the sketch-update kernel a
// pass over the other tiles' entries).
constexpr uint32_t kBinTarget = 4096;  // measured best on B200 at 2^17 vertices (2 tiles per bin)
constexpr uint32_t kMaxTilesPerBin = 16;

// Whether a handle uses the two-buffer sketch update when not told: past 2^18 vertices, where
// one-tile-at-a-time staging would need over 4 tiles per gutter bin and is switched to one tile
// per bin anyway, so overlapping a tile's load and write-back with the hashing pays (measured at
// 2^20 vertices: 6.1 -> 5.5 ms per 1.3e7 records). Below, the one-tile kernel keeps its larger
// tiles and coarser bins (2^17 vertices: 17.6 ms ingest against 25.8 ms pipelined).
constexpr uint32_t kPipeBuffers = 2;  // default tile buffers of the pipelined kernel

bool want_pipe(const gz_alg *h) {
  if (h->pipe_mode >= 0) return h->pipe_mode >= 1;
  return h->V > (1u << 18);
}

// Coded entries and bucket planes by default: CameoSketch of at most 31 columns up to 2^18
// vertices (asked for explicitly: while the gutter bins fit the shared-memory hash sort). By
// default a gutter bin is one tile of 32 vertices. Coarser bins (set_tuning tiles_per_bin 2..8)
// lengthen the sort's runs but make every tile filter its bin's entries; measured on B200 over
// 1.4e8 records at 2^17 vertices, gutter + sketch update took 5.2 + 6.4 ms at 1 tile per bin,
// 5.0 + 7.1 ms at 2 and 4.8 + 8.0 ms at 4.
constexpr uint32_t kPlaneBinTarget = 1024;
constexpr uint32_t kPlaneTilesPerBin = 1;
constexpr uint32_t kPlaneDefaultMaxV = 1u << 18;

int choose_planes(gz_alg *h, uint32_t vpt_req, uint32_t threads_req, uint32_t tpb_req, bool &done) {
  done = false;
  const bool asked = h->planes_mode >= 1;
  if (h->planes_mode == 0) return GZ_OK;
  if (h->cube || h->C > gz::kPlaneMaxColumns) {
    if (asked) return fail(GZ_ERR_INVALID, "coded entries need CameoSketch with at most 31 columns");
    return GZ_OK;
  }
  if ((tpb_req && ((tpb_req & (tpb_req - 1)) || tpb_req > 8)) ||
      (vpt_req && (vpt_req < 4 || (vpt_req & (vpt_req - 1)) || vpt_req > gz::kPlaneMaxTile))) {
    if (asked) return fail(GZ_ERR_INVALID, "coded entries take tiles of 4 to 32 vertices, 1 to 8 per bin");
    return GZ_OK;
  }
  // By default past 2^18 vertices the pipelined staged kernel stays in use (large sparse graphs,
  // where a wave brings few entries per tile)
  if (!asked && h->V > kPlaneDefaultMaxV) return GZ_OK;
  const uint32_t shift = vpt_req ? (uint32_t)__builtin_ctz(vpt_req) : 5;
  uint32_t bshift = shift;
  if (tpb_req) {
    bshift = shift + (uint32_t)__builtin_ctz(tpb_req);
  } else {
    while (((h->V + (1u << bshift) - 1) >> bshift) > kPlaneBinTarget &&
           (1u << (bshift - shift)) < kPlaneTilesPerBin)
      ++bshift;
    // large graphs: bins of several tiles, as many as the hash sort's shared memory holds
    while (((h->V + (1u << bshift) - 1) >> bshift) > gz::kSortBinsMax && bshift < shift + 3) ++bshift;
  }
  const uint32_t nbins = (uint32_t)((h->V + (1u << bshift) - 1) >> bshift);
  if (nbins > gz::kSortBinsMax) {
    if (asked) return fail(GZ_ERR_INVALID, "too many gutter bins for coded entries at this tile size");
    return GZ_OK;
  }
  // 4-bit codes where they fit (unless 3-bit ones are asked for), else 3-bit codes
  const bool fits4 = h->planes_mode != 2 && gz::coded_entry_fits(h->V, h->C, bshift, 4);
  if (!fits4 && !gz::coded_entry_fits(h->V, h->C, bshift, 3)) {
    if (asked) return fail(GZ_ERR_INVALID, "the codes of this sketch do not fit a 16-byte coded entry");
    return GZ_OK;
  }
  uint32_t threads = threads_req ? threads_req : 1024;
  if (threads_req && (threads_req < 64 || threads_req > 1024 || threads_req % 32))
    return fail(GZ_ERR_INVALID, "threads_per_block must be a multiple of 32 in [64, 1024]");
  if (gz::plane_update_smem(shift, (int)threads) > h->smem_optin)
    return fail(GZ_ERR_INVALID, "this tile does not fit in shared memory");
  h->planes = true;
  h->codes3 = !fits4;
  h->in_place = false;
  h->pipe = false;
  h->threads = threads;
  h->tile_shift = shift;
  h->ntiles = (uint32_t)((h->V + (1u << shift) - 1) >> shift);
  h->bin_shift = bshift;
  h->nbins = nbins;
  done = true;
  return GZ_OK;
}

int choose_tiling(gz_alg *h, uint32_t vpt_req, uint32_t threads_req, uint32_t tpb_req) {
  int dev = h->device;
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem_optin <= 0) smem_optin = 227 * 1024;
  h->smem_optin = (size_t)smem_optin;
  h->planes = false;
  h->codes3 = false;
  h->threads = 1024;
  {
    bool done = false;
    GZ_TRY(choose_planes(h, vpt_req, threads_req, tpb_req, done));
    if (done) return GZ_OK;
  }
  const size_t budget = (size_t)smem_optin - 64 - gz::kQueueBytes;
  const size_t flip_bytes = (size_t)(h->C + 1) * 8;
  uint32_t shift;
  if (vpt_req) {
    if (vpt_req < 4 || (vpt_req & (vpt_req - 1)) || vpt_req > 64)
      return fail(GZ_ERR_INVALID, "vertices_per_tile must be a power of two in [4, 64]");
    shift = (uint32_t)__builtin_ctz(vpt_req);
    if ((h->sketch_bytes << shift) + flip_bytes > budget)
      return fail(GZ_ERR_INVALID, "vertices_per_tile does not fit in shared memory");
  } else {
    shift = 2;
    const uint64_t want = std::max<uint64_t>(4, h->V / (2ull * gz::num_sms()));
    while (shift < 6 && (1ull << (shift + 1)) <= want &&
           (h->sketch_bytes << (shift + 1)) + flip_bytes <= budget)
      ++shift;
    if ((h->sketch_bytes << shift) + flip_bytes > budget) {
      // not even 4 vertex sketches fit a tile (CubeSketch at large V): updates go straight to
      // HBM, hashed once per record (apply_in_place)
      h->in_place = true;
      shift = 2;
    }
  }
  // two-buffer pipeline: two tiles (one bin each) and the hash constants in shared memory
  h->pipe = false;
  if (!h->in_place && !h->cube && !tpb_req && want_pipe(h)) {
    const size_t room = (size_t)smem_optin - 1024 - (((size_t)h->C + 2) & ~(size_t)1) * 8;
    // the most buffers asked for (or kPipeBuffers) that hold tiles of at least 4 vertices
    for (uint32_t nb = h->pipe_mode >= 2 ? (uint32_t)h->pipe_mode : kPipeBuffers; nb >= 2 && !h->pipe; --nb) {
      uint32_t ps = vpt_req ? shift : 6;
      while (ps > 2 && nb * (h->sketch_bytes << ps) > room) --ps;
      if (nb * (h->sketch_bytes << ps) <= room) {
        h->pipe = true;
        h->nbuf = nb;
        shift = ps;
      }
    }
  }
  h->tile_shift = shift;
  h->ntiles = (uint32_t)((h->V + (1u << shift) - 1) >> shift);
  uint32_t bshift = shift;
  if (h->pipe) {
    // one tile per bin
  } else if (tpb_req) {
    if (tpb_req & (tpb_req - 1) || tpb_req > 64)
      return fail(GZ_ERR_INVALID, "tiles_per_bin must be a power of two <= 64");
    bshift = shift + (uint32_t)__builtin_ctz(tpb_req);
  } else {
    while (((h->V + (1u << bshift) - 1) >> bshift) > kBinTarget &&
           (1u << (bshift - shift)) < kMaxTilesPerBin)
      ++bshift;
    // Past 4 tiles per bin every sketch-update CTA would filter most of its bin's entries away
    // (measured at 2^20 vertices: 16 tiles per bin cost 9.1 ms per 1.3e7 records against 6.3 ms
    // for one tile per bin, whose scatter uses global cursors and costs 0.25 ms more).
    if (bshift - shift > 2) bshift = shift;
  }
  h->bin_shift = bshift;
  h->nbins = (uint32_t)((h->V + (1u << bshift) - 1) >> bshift);
  if (threads_req) {
    if (threads_req < 64 || threads_req > 1024 || threads_req % 32)
      return fail(GZ_ERR_INVALID, "threads_per_block must be a multiple of 32 in [64, 1024]");
    h->threads = threads_req;
  }
  if (h->in_place || h->pipe) return GZ_OK;
  cudaError_t e = gz::sketch_update_prepare(h->sgeom(), h->threads);
  if (e != cudaSuccess) return fail(GZ_ERR_CUDA, cudaGetErrorString(e));
  return GZ_OK;
}

int init_alg(gz_alg *h, uint32_t V, uint64_t seed, double sf, double bf, bool cube) {
  if (V < 2 || V > (1u << 31)) return fail(GZ_ERR_INVALID, "num_vertices must be in [2, 2^31]");
  GZ_CUDA(cudaGetDevice(&h->device));
  h->V = V;
  h->seed = seed;
  h->sketches_factor = sf > 0 ? sf : 1;  // CCAlgConfiguration::sketches_factor
  h->batch_factor = bf > 0 ? bf : 1;     // CCAlgConfiguration::batch_factor
  h->cube = cube;
  gz::sketch_sizing_alg(V, h->sketches_factor, cube, h->samples, h->cps, h->B);
  h->C = h->samples * h->cps;
  if (h->B > 63) return fail(GZ_ERR_INVALID, "bkt_per_col above 63 is not supported");
  h->nb = h->C * h->B + 1;
  h->ph = gz::plane_hash(seed, h->C, h->B);
  h->sketch_bytes = (uint64_t)h->nb * gz::kBucketBytes;
  {
    size_t num = h->sketch_bytes / sizeof(uint32_t);
    num *= h->batch_factor;  // same size_t *= double truncation as the reference
    h->desired_batch = num;
  }
  GZ_TRY(choose_tiling(h, 0, 0, 0));
  GZ_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  GZ_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  // V rounded up to 64 so any tile size stays inside the allocation
  const uint64_t v_pad = ((uint64_t)V + 63) & ~63ull;
  // + kSketchTail: the query's bulk copies read 16-byte-aligned supersets of a vertex's buckets
  GZ_TRY(dev_alloc(&h->d_sk, v_pad * h->sketch_bytes + gz::kSketchTail));
  GZ_CUDA(cudaMemsetAsync(h->d_sk, 0, v_pad * h->sketch_bytes + gz::kSketchTail, h->stream));
  std::vector<uint64_t> flip(h->C + 1);
  for (uint32_t c = 0; c < h->C; ++c) flip[c] = gz::xxh3_flip(seed + 5ull * c);  // column_seed
  flip[h->C] = gz::xxh3_flip(seed);                                                  // checksum_seed
  GZ_TRY(dev_alloc(&h->d_flip, flip.size()));
  GZ_CUDA(cudaMemcpyAsync(h->d_flip, flip.data(), flip.size() * 8, cudaMemcpyHostToDevice, h->stream));
  GZ_TRY(dev_alloc(&h->d_status, 4));
  GZ_CUDA(cudaMemsetAsync(h->d_status, 0, 16, h->stream));
  GZ_TRY(host_alloc(&h->h_status, 4));
  h->entry_cap = std::min<uint64_t>((uint64_t)V * h->desired_batch, 1ull << 29);
  h->entry_cap = std::max<uint64_t>(h->entry_cap, 1ull << 16);
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

void tickets_shutdown(gz_alg *h);
void free_bv(gz::BoruvkaBufs &b);

void destroy_alg(gz_alg *h) {
  tickets_shutdown(h);
  gz::boruvka_graph_free(h->qgraph);
  host_free(h->h_qpin);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  dev_free(h->d_sk);
  dev_free(h->d_flip);
  dev_free(h->d_status);
  host_free(h->h_status);
  dev_free(h->d_gutter);
  dev_free(h->d_bin_off);
  dev_free(h->d_hist);
  dev_free(h->d_scan_tmp);
  dev_free(h->d_total);
  dev_free(h->d_cursor);
  dev_free(h->d_fill);
  for (int i = 0; i < kStageBuffers; ++i) {
    dev_free(h->d_stage[i]);
    if (h->ev_copied[i]) cudaEventDestroy(h->ev_copied[i]);
    if (h->ev_free[i]) cudaEventDestroy(h->ev_free[i]);
  }
  for (int i = 0; i < 2; ++i) {
    dev_free(h->d_ent[i]);
    host_free(h->h_ent[i]);
    if (h->ev_ent_done[i]) cudaEventDestroy(h->ev_ent_done[i]);
  }
  dev_free(h->d_raw);
  auto &b = h->bv;
  dev_free(b.parent);
  dev_free(b.label);
  dev_free(b.cnt);
  dev_free(b.fill);
  dev_free(b.minv);
  dev_free(b.packed);
  dev_free(b.scan_total);
  dev_free(b.scan_tmp);
  dev_free(b.order);
  dev_free(b.order_comp);
  dev_free(b.comp_start);
  dev_free(b.comp_key);
  dev_free(b.ncomp);
  dev_free(b.acc);
  dev_free(b.part);
  dev_free(b.part_comp);
  dev_free(b.big);
  dev_free(b.round);
  b.ctl = nullptr;
  dev_free(b.flags);
  dev_free(b.cross);
  dev_free(b.ncross);
  dev_free(b.qbar);
  dev_free(b.btot);
  dev_free(b.forest);
  dev_free(b.forest_n);
  if (b.trace) cudaFree(b.trace);
  dev_free(b.trace_n);
  dev_free(h->d_final);
  dev_free(h->d_ncc);
  for (auto &e : h->prof_pending) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
}

// ---- device gutter -------------------------------------------------------------------------------

// Gutter bytes per endpoint entry: 8 B {vertex, neighbour}, or 16 B with the depth codes of the
// first columns (records on the bucket-plane path).
uint64_t entry_bytes(const gz_alg *h, int input) {
  return input == gz::kInputRecords && h->planes ? 16 : 8;
}
constexpr uint64_t kGutterSlack = 64;  // 16-byte alignment of each chunk

int ensure_gutter(gz_alg *h) {
  if (!h->d_gutter) {
    h->gutter_bytes = h->entry_cap * (h->planes ? 16 : 8) + kGutterSlack;
    GZ_TRY(dev_alloc(&h->d_gutter, h->gutter_bytes));
  }
  GZ_TRY(dev_alloc(&h->d_bin_off, (size_t)gz::kMaxChunks * (h->nbins + 1)));
  const size_t words = h->nbins;
  if (h->hist_words < words) {
    dev_free(h->d_hist);
    dev_free(h->d_scan_tmp);
    dev_free(h->d_cursor);
    dev_free(h->d_fill);
    GZ_TRY(dev_alloc(&h->d_hist, words));
    GZ_TRY(dev_alloc(&h->d_cursor, words));
    GZ_TRY(dev_alloc(&h->d_fill, words));
    GZ_TRY(dev_alloc(&h->d_scan_tmp, gz::scan_tmp_words(words)));
    h->hist_words = words;
  }
  GZ_TRY(dev_alloc(&h->d_total, 1));
  return GZ_OK;
}

// Apply every buffered gutter chunk to the sketches (one sketch-update launch).
int apply_pending(gz_alg *h) {
  if (h->nchunks == 0) return GZ_OK;
  const gz::SketchGeom g = h->sgeom();
  GZ_CUDA(cudaMemsetAsync(h->d_status + 1, 0, sizeof(uint32_t), h->stream));
  const int pi = h->prof_begin();
  if (h->planes) {
    const int per_sm = gz::plane_update_ctas_per_sm(h->tile_shift, (int)h->threads);
    const int grid = (int)std::min<uint64_t>(h->ntiles, (uint64_t)gz::num_sms() * per_sm);
    GZ_CUDA(gz::plane_update(h->pgeom(), h->ph, h->d_sk, h->d_gutter, h->chunks, h->d_bin_off,
                             h->nchunks, h->d_status + 1, h->d_status, grid, (int)h->threads, h->stream));
  } else if (h->pipe) {
    const int grid = (int)std::min<uint64_t>(h->ntiles, (uint64_t)gz::num_sms());
    GZ_CUDA(gz::sketch_update_pipe(g, h->d_sk, h->d_gutter, h->chunks, h->d_bin_off, h->nchunks, h->d_flip,
                                   h->d_status + 1, h->d_status, grid, h->stream));
  } else {
    const int per_sm = gz::sketch_update_ctas_per_sm(g, (int)h->threads);
    const int grid = (int)std::min<uint64_t>(h->ntiles, (uint64_t)gz::num_sms() * per_sm);
    GZ_CUDA(gz::sketch_update(g, h->d_sk, h->d_gutter, h->chunks, h->d_bin_off, h->nchunks, h->d_flip,
                              h->d_status + 1, h->d_status, grid, h->threads, h->stream));
  }
  h->prof_end(pi, 1);
  h->prof_acc.entries_applied += h->entries_pending;
  h->nchunks = 0;
  h->gutter_used = 0;
  h->entries_pending = 0;
  return GZ_OK;
}

// Counting-sort n inputs (records or entries, device memory) into a new gutter chunk.
int gutter_chunk(gz_alg *h, int input, const void *d_in, uint64_t n) {
  if (n == 0) return GZ_OK;
  if (h->in_place) {
    const int pi = h->prof_begin();
    GZ_CUDA(gz::apply_in_place(input, d_in, n, h->sgeom(), h->d_sk, h->d_flip, h->d_status, h->stream));
    h->prof_end(pi, 1);
    return GZ_OK;
  }
  const uint64_t per = input == gz::kInputRecords ? 2 : 1;
  const uint64_t esz = entry_bytes(h, input);
  const bool coded = esz == 16;
  GZ_TRY(ensure_gutter(h));
  const uint64_t max_n = std::min((h->gutter_bytes - kGutterSlack) / esz, kMaxChunkEntries) / per;
  if (max_n == 0) return fail(GZ_ERR_INVALID, "gutter capacity is below one update");
  if (n > max_n) {
    const size_t isz = input == gz::kInputRecords ? 9 : sizeof(uint2);
    for (uint64_t off = 0; off < n; off += max_n)
      GZ_TRY(gutter_chunk(h, input, (const uint8_t *)d_in + off * isz, std::min(max_n, n - off)));
    return GZ_OK;
  }
  // a chunk's entries, 16-byte aligned
  const uint64_t n_ent = n * per;
  const uint64_t need = (n_ent * esz + 15) & ~15ull;
  if (h->gutter_used + need > h->gutter_bytes || h->nchunks == gz::kMaxChunks)
    GZ_TRY(apply_pending(h));
  const gz::GutterGeom gg = h->ggeom();
  const uint64_t unit = input == gz::kInputRecords ? gz::kRecTile : 4096;
  const int G = (int)std::max<uint64_t>(1, std::min<uint64_t>(2ull * gz::num_sms(), (n + unit - 1) / unit));
  uint8_t *out = h->d_gutter + h->gutter_used;
  uint32_t *bin_off = h->d_bin_off + (size_t)h->nchunks * (h->nbins + 1);
  const int pi = h->prof_begin();
  uint2 *out2 = reinterpret_cast<uint2 *>(out);
  GZ_CUDA(cudaMemsetAsync(h->d_hist, 0, sizeof(uint64_t) * h->nbins, h->stream));
  GZ_CUDA(gz::gutter_count(input, d_in, n, gg, G, h->d_hist, h->d_status, h->stream));
  GZ_CUDA(gz::scan_exclusive_u64(h->d_hist, h->nbins, h->d_total, h->d_scan_tmp, h->stream));
  GZ_CUDA(gz::gutter_bin_offsets(h->d_hist, 1, h->nbins, h->d_total, bin_off, h->stream));
  if (coded) {
    // records -> coded entries, each record hashed once
    const uint32_t tile = gz::hash_sort_tile(h->nbins, h->smem_optin - 1024);
    if (tile == 0) return fail(GZ_ERR_INVALID, "gutter bins do not fit the hash sort");
    GZ_CUDA(cudaMemsetAsync(h->d_fill, 0, sizeof(uint32_t) * h->nbins, h->stream));
    GZ_CUDA(gz::gutter_hash_sort(d_in, n, gg, h->ph, tile, h->d_hist, h->d_fill,
                                 reinterpret_cast<uint4 *>(out),
                                 h->codes3 ? gz::kEntryCoded3 : gz::kEntryCoded, h->stream));
  } else {
    const uint32_t tile = gz::sort_scatter_tile(input, gg, h->smem_optin - 1024);
    if (tile >= 1024) {
      GZ_CUDA(cudaMemsetAsync(h->d_fill, 0, sizeof(uint32_t) * h->nbins, h->stream));
      GZ_CUDA(gz::gutter_sort_scatter(input, d_in, n, gg, tile, h->d_hist, h->d_fill, out2, h->stream));
    } else {
      GZ_CUDA(gz::copy_u64(h->d_hist, h->d_cursor, h->nbins, h->stream));
      GZ_CUDA(gz::gutter_scatter_global(input, d_in, n, gg, G, h->d_cursor, out2, h->stream));
    }
  }
  h->prof_end(pi, 0);
  h->chunks.base[h->nchunks] = h->gutter_used;
  h->chunks.kind[h->nchunks] = !coded ? gz::kEntryPlain : h->codes3 ? gz::kEntryCoded3 : gz::kEntryCoded;
  h->nchunks++;
  h->gutter_used += need;
  h->entries_pending += n_ent;
  return GZ_OK;
}

int push_staged_entries(gz_alg *h) {
  if (h->h_ent_n == 0) return GZ_OK;
  const int i = h->h_ent_cur;
  GZ_TRY(dev_alloc(&h->d_ent[i], kEntStage));
  GZ_CUDA(cudaMemcpyAsync(h->d_ent[i], h->h_ent[i], h->h_ent_n * sizeof(uint2),
                          cudaMemcpyHostToDevice, h->stream));
  GZ_TRY(gutter_chunk(h, gz::kInputEntries, h->d_ent[i], h->h_ent_n));
  GZ_CUDA(cudaEventRecord(h->ev_ent_done[i], h->stream));
  h->h_ent_n = 0;
  h->h_ent_cur ^= 1;
  // the next buffer may still be in flight from two pushes ago
  GZ_CUDA(cudaEventSynchronize(h->ev_ent_done[h->h_ent_cur]));
  return GZ_OK;
}

int stage_entry(gz_alg *h, uint32_t v, uint32_t w) {
  if (!h->h_ent[0]) {
    for (int i = 0; i < 2; ++i) {
      GZ_TRY(host_alloc(&h->h_ent[i], kEntStage));
      GZ_CUDA(cudaEventCreateWithFlags(&h->ev_ent_done[i], cudaEventDisableTiming));
      GZ_CUDA(cudaEventRecord(h->ev_ent_done[i], h->stream));
    }
  }
  h->h_ent[h->h_ent_cur][h->h_ent_n++] = make_uint2(v, w);
  if (h->h_ent_n == kEntStage) GZ_TRY(push_staged_entries(h));
  return GZ_OK;
}

int check_status(gz_alg *h) {
  GZ_CUDA(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  const uint32_t st = h->h_status[0] | h->deferred_status;
  h->deferred_status = 0;
  if (st) {
    GZ_CUDA(cudaMemsetAsync(h->d_status, 0, sizeof(uint32_t), h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->stream));
    if (st & gz::kStatusTimeout) return fail(GZ_ERR_TIMEOUT, "a bounded device wait timed out");
    if (st & gz::kStatusBadVertex) return fail(GZ_ERR_BAD_VERTEX, "an update named a vertex id >= V; it was dropped");
    if (st & gz::kStatusBadSample) return fail(GZ_ERR_BAD_SAMPLE, "a sampled edge decoded to a vertex id >= V");
  }
  return GZ_OK;
}

int flush_all(gz_alg *h) {
  GZ_TRY(push_staged_entries(h));
  GZ_TRY(apply_pending(h));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int check_unlocked(gz_alg *h) {
  if (h->update_locked || h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  return GZ_OK;
}

// The cached answer is lost: the NO_EAGER_DSU form of pre_insert, and every update path whose
// updates the eager DSU cannot see.
void invalidate_answer(gz_alg *h) {
  h->dsu_valid = false;
  h->host_answer = false;
  h->labels_on_host = false;
}

int mark_updated(gz_alg *h) {
  GZ_TRY(check_unlocked(h));
  invalidate_answer(h);
  return GZ_OK;
}

uint32_t host_find(std::vector<uint32_t> &p, uint32_t x) {
  while (p[x] != x) {
    p[x] = p[p[x]];
    x = p[x];
  }
  return x;
}

// CCSketchAlg::pre_insert (src/cc_sketch_alg.cpp:79-104) for one update (u, v).
void pre_insert_one(gz_alg *h, uint32_t u, uint32_t v) {
  if (!h->dsu_valid) return;
  if (!h->eager || u >= h->V || v >= h->V) {
    invalidate_answer(h);
    return;
  }
  const uint32_t a = std::min(u, v), b = std::max(u, v);
  const uint64_t key = ((uint64_t)a << 32) | b;
  const uint32_t ra = host_find(h->hdsu, a), rb = host_find(h->hdsu, b);
  if (ra != rb) {  // new connectivity: merge, and the edge joins the spanning forest
    h->hdsu[std::max(ra, rb)] = std::min(ra, rb);
    h->hforest.insert(key);
    h->host_answer = true;
    h->labels_on_host = false;
  } else if (h->hforest.count(key)) {  // one of the forest's edges changed
    invalidate_answer(h);
  }
}

// Seed the eager DSU from the device answer (labels and Boruvka's spanning forest).
int eager_from_device(gz_alg *h, bool have_forest) {
  h->hdsu.resize(h->V);
  GZ_CUDA(cudaMemcpyAsync(h->hdsu.data(), h->d_final, sizeof(uint32_t) * h->V, cudaMemcpyDeviceToHost, h->stream));
  uint32_t n = 0;
  std::vector<uint64_t> idx;
  if (have_forest) {
    GZ_CUDA(cudaMemcpyAsync(h->h_status + 3, h->bv.forest_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->stream));
    n = std::min<uint32_t>(h->h_status[3], h->V);
    idx.resize(n);
    if (n) GZ_CUDA(cudaMemcpyAsync(idx.data(), h->bv.forest, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  }
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  h->hforest.clear();
  h->hforest.insert(idx.begin(), idx.end());
  h->host_answer = false;
  return GZ_OK;
}

// ---- Boruvka ---------------------------------------------------------------------------------------

// Boruvka buffers for V vertices; acc_words per component spanning warps (and per merge warp)
int alloc_bv(gz::BoruvkaBufs &b, size_t V, size_t acc_words, uint32_t *status) {
  GZ_TRY(dev_alloc(&b.parent, V));
  GZ_TRY(dev_alloc(&b.label, V));
  GZ_TRY(dev_alloc(&b.cnt, V));
  GZ_TRY(dev_alloc(&b.fill, V));
  GZ_TRY(dev_alloc(&b.minv, V));
  GZ_TRY(dev_alloc(&b.packed, V));
  GZ_TRY(dev_alloc(&b.scan_total, 1));
  GZ_TRY(dev_alloc(&b.scan_tmp, gz::scan_tmp_words(V)));
  GZ_TRY(dev_alloc(&b.order, V));
  GZ_TRY(dev_alloc(&b.order_comp, V));
  GZ_TRY(dev_alloc(&b.comp_start, V + 1));
  GZ_TRY(dev_alloc(&b.comp_key, V));
  GZ_TRY(dev_alloc(&b.ncomp, 1));
  const size_t warps = (V + gz::kBoruvkaSpan - 1) / gz::kBoruvkaSpan;
  GZ_TRY(dev_alloc(&b.acc, (warps + 1) * acc_words));
  GZ_TRY(dev_alloc(&b.part, warps * acc_words));
  GZ_TRY(dev_alloc(&b.part_comp, warps));
  GZ_TRY(dev_alloc(&b.big, 1));
  GZ_TRY(dev_alloc(&b.round, 4));
  b.ctl = b.round + 1;
  GZ_TRY(dev_alloc(&b.flags, 4));
  GZ_TRY(dev_alloc(&b.cross, warps + 1));
  GZ_TRY(dev_alloc(&b.ncross, 1));
  GZ_TRY(dev_alloc(&b.qbar, 1));
  GZ_TRY(dev_alloc(&b.btot, gz::kBvQueryMaxBlocks));
  GZ_TRY(dev_alloc(&b.forest, V));
  GZ_TRY(dev_alloc(&b.forest_n, 1));
  GZ_TRY(dev_alloc(&b.trace_n, 1));
  b.status = status;
  return GZ_OK;
}

void free_bv(gz::BoruvkaBufs &b) {
  dev_free(b.parent);
  dev_free(b.label);
  dev_free(b.cnt);
  dev_free(b.fill);
  dev_free(b.minv);
  dev_free(b.packed);
  dev_free(b.scan_total);
  dev_free(b.scan_tmp);
  dev_free(b.order);
  dev_free(b.order_comp);
  dev_free(b.comp_start);
  dev_free(b.comp_key);
  dev_free(b.ncomp);
  dev_free(b.acc);
  dev_free(b.part);
  dev_free(b.part_comp);
  dev_free(b.big);
  dev_free(b.round);
  b.ctl = nullptr;
  dev_free(b.flags);
  dev_free(b.cross);
  dev_free(b.ncross);
  dev_free(b.qbar);
  dev_free(b.btot);
  dev_free(b.forest);
  dev_free(b.forest_n);
  dev_free(b.trace_n);
}

// boruvka_emulation (src/cc_sketch_alg.cpp:464-513) on the sketches at sk with buffers b: the
// query graph (every round on the device, no host round trip) enqueued on stream s, then the
// rounds, the out-of-samples flag and the component count copied to pin[0..2] (pinned).
// The query mode in effect. By size: the one-launch query up to 2^18 vertices (a round's phases
// are short there, and launches and gaps between them dominated: 0.59 against 0.64 ms at 2^17);
// the graph of per-phase kernels above (each phase then has work for more resident warps than the
// cooperative kernel's registers allow: 1.8-2.0 against 2.1-2.2 ms per query at 2^20).
constexpr uint32_t kOneLaunchQueryMaxV = 1u << 18;
int query_mode_of(const gz_alg *h) {
  if (h->query_mode >= 0) return h->query_mode;
  return h->V <= kOneLaunchQueryMaxV ? 2 : 1;
}

int boruvka_enqueue(gz_alg *h, gz::BoruvkaGraph &q, const gz::BoruvkaGeom &g, const uint8_t *sk,
                    gz::BoruvkaBufs &b, uint32_t *d_final, uint32_t *d_ncc, uint32_t *pin,
                    cudaStream_t s) {
  const int mode = query_mode_of(h);
  if (mode == 2) GZ_CUDA(gz::boruvka_query_launch(g, h->samples, sk, b, d_final, d_ncc, s));
  else if (mode == 1) GZ_CUDA(gz::boruvka_graph_launch(q, g, h->samples, sk, b, d_final, d_ncc, s));
  else GZ_CUDA(gz::boruvka_host_loop(g, h->samples, sk, b, d_final, d_ncc, pin, s));
  GZ_CUDA(cudaMemcpyAsync(pin, b.ctl, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GZ_CUDA(cudaMemcpyAsync(pin + 2, d_ncc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  return GZ_OK;
}

// Kernel launches of a finished query graph (its loop body ran once per round >= 1).
void boruvka_account(const gz::BoruvkaGraph &q, const uint32_t *pin, bool graph) {
  if (!graph) return;  // the host loop counted its launches as it went
  const uint32_t body_runs = pin[1] ? pin[0] - 1 : pin[0];
  gz::add_launches(q.fixed_kernels + (uint64_t)body_runs * q.round_kernels);
}

std::string out_of_samples_msg(const gz_alg *h, uint32_t round) {
  return "This sketch (seed=" + std::to_string(h->seed) + ", max samples=" + std::to_string(h->samples) +
         ") cannot be sampled more times (cur idx=" + std::to_string(round) + ")!";
}

// ---- queries by ticket ----------------------------------------------------------------------------
int tickets_ensure(gz_alg *h) {
  auto &T = h->tq;
  if (T.d_final) return GZ_OK;
  GZ_TRY(alloc_bv(T.bv, h->V, (size_t)(h->cps * h->B + 1) * 3, h->d_status));
  GZ_TRY(dev_alloc(&T.d_ncc, 1));
  GZ_TRY(dev_alloc(&T.d_final, h->V));
  return GZ_OK;
}

void ticket_free(gz_alg::Ticket &t) {
  if (t.done) cudaEventDestroy(t.done);
  host_free(t.labels);
  host_free(t.pin);
  t = gz_alg::Ticket{};
}

void tickets_shutdown(gz_alg *h) {
  auto &T = h->tq;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto &kv : T.live) ticket_free(kv.second);
  for (auto &t : T.pool) ticket_free(t);
  T.live.clear();
  T.pool.clear();
  gz::boruvka_graph_free(T.graph);
  free_bv(T.bv);
  dev_free(T.d_final);
  dev_free(T.d_ncc);
}

int ensure_query(gz_alg *h) {
  auto &b = h->bv;
  const size_t V = h->V;
  GZ_TRY(alloc_bv(b, V, (size_t)(h->cps * h->B + 1) * 3, h->d_status));
  GZ_TRY(dev_alloc(&h->d_final, V));
  GZ_TRY(dev_alloc(&h->d_ncc, 1));
  if (h->trace && !b.trace) {
    const size_t cap = V * (size_t)(h->C + 1);
    void *p = nullptr;
    GZ_CUDA(cudaMalloc(&p, cap * sizeof(gz_trace_rec_t)));
    b.trace = p;
    b.trace_cap = (uint32_t)std::min<size_t>(cap, 0xffffffffu);
  }
  if (!h->trace) {
    if (b.trace) cudaFree(b.trace);
    b.trace = nullptr;
    b.trace_cap = 0;
  }
  return GZ_OK;
}

// boruvka_emulation (src/cc_sketch_alg.cpp:464-513) driven from the host, one device round per
// iteration until a round neither FAILs nor merges.
int run_boruvka(gz_alg *h) {
  GZ_TRY(ensure_query(h));
  if (!h->h_qpin) GZ_TRY(host_alloc(&h->h_qpin, 4));
  h->update_locked = true;  // stays set if the query fails, as in the reference
  const int pi = h->prof_begin();
  GZ_TRY(boruvka_enqueue(h, h->qgraph, h->bgeom(), h->d_sk, h->bv, h->d_final, h->d_ncc, h->h_qpin,
                         h->stream));
  h->prof_end(pi, 2);
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  boruvka_account(h->qgraph, h->h_qpin, query_mode_of(h) == 1);
  const uint32_t round = h->h_qpin[0];
  if (h->h_qpin[1]) {
    h->last_rounds = round;
    return fail(GZ_ERR_OUT_OF_SAMPLES, out_of_samples_msg(h, round));
  }
  h->prof_acc.query_rounds += round + 1;
  GZ_TRY(check_status(h));
  h->last_ncc = h->h_qpin[2];
  h->last_rounds = round;
  h->dsu_valid = true;
  h->labels_on_host = false;
  h->update_locked = false;
  h->boruvka_ran = true;
  if (h->eager) GZ_TRY(eager_from_device(h, true));
  return GZ_OK;
}

// The partition: either the cached one or a fresh Boruvka. Identity when nothing was ever
// inserted (a fresh CCSketchAlg starts with a valid, empty DSU).
int ensure_answer(gz_alg *h) {
  GZ_TRY(flush_all(h));
  if (h->dsu_valid && h->host_answer) {
    // the eager DSU's partition: labels computed here, copied to the device answer
    GZ_TRY(ensure_query(h));
    h->h_labels.resize(h->V);
    uint32_t ncc = 0;
    for (uint32_t v = 0; v < h->V; ++v) {
      h->h_labels[v] = host_find(h->hdsu, v);
      ncc += h->h_labels[v] == v;
    }
    GZ_CUDA(cudaMemcpyAsync(h->d_final, h->h_labels.data(), sizeof(uint32_t) * h->V, cudaMemcpyHostToDevice, h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->stream));
    h->last_ncc = ncc;
    h->labels_on_host = true;
    h->host_answer = false;
    return GZ_OK;
  }
  if (h->dsu_valid && h->d_final) return GZ_OK;
  if (h->dsu_valid) {
    GZ_TRY(ensure_query(h));
    GZ_CUDA(gz::boruvka_reset(h->bgeom(), h->bv, h->stream));
    GZ_CUDA(gz::boruvka_final(h->bgeom(), h->bv, h->d_final, h->d_ncc, h->stream));
    GZ_CUDA(cudaMemcpyAsync(h->h_status + 2, h->d_ncc, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->stream));
    h->last_ncc = h->h_status[2];
    return GZ_OK;
  }
  h->query_running = true;
  const int rc = run_boruvka(h);
  h->query_running = false;
  return rc;
}

int labels_to_host(gz_alg *h) {
  if (h->labels_on_host) return GZ_OK;
  h->h_labels.resize(h->V);
  GZ_CUDA(cudaMemcpyAsync(h->h_labels.data(), h->d_final, sizeof(uint32_t) * h->V, cudaMemcpyDeviceToHost, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  h->labels_on_host = true;
  return GZ_OK;
}

// Best of `repeats` timed launches of a probe kernel (after one warm-up) on a private stream:
// units / second, units = the work count of one launch.
template <class F>
int time_probe(int repeats, double units, F launch, double *rate) {
  cudaStream_t s = nullptr;
  GZ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0;
  cudaError_t e = launch(s, 0);
  for (int r = 0; r < repeats && e == cudaSuccess; ++r) {
    cudaEventRecord(a, s);
    e = launch(s, 1);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms > 0) best = std::max(best, units / (ms * 1e-3));
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return fail(GZ_ERR_CUDA, cudaGetErrorString(e));
  *rate = best;
  return GZ_OK;
}

struct Guard {
  gz_alg *h;
  std::lock_guard<std::mutex> lk;
  explicit Guard(gz_alg *a) : h(a), lk(a->mtx) { cudaSetDevice(a->device); }
};

}  // namespace

// =================================================================================================
// C ABI
// =================================================================================================
extern "C" {

const char *gz_version(void) { return "graphzeppelin_b200 0.1.0 (sm_100a)"; }

const char *gz_status_string(int s) {
  switch (s) {
    case GZ_OK: return "ok";
    case GZ_ERR_INVALID: return "invalid argument";
    case GZ_ERR_CUDA: return "CUDA error";
    case GZ_ERR_OUT_OF_SAMPLES: return "out of samples";
    case GZ_ERR_LOCKED: return "updates locked";
    case GZ_ERR_BAD_VERTEX: return "vertex id out of range";
    case GZ_ERR_NOMEM: return "out of memory";
    case GZ_ERR_IO: return "I/O error";
    case GZ_ERR_TIMEOUT: return "device wait timed out";
    case GZ_ERR_BAD_SAMPLE: return "sampled edge out of range";
    case GZ_ERR_NO_DEVICE: return "no CUDA device";
    case GZ_ERR_BUDGET: return "sketch-byte budget exhausted";
    default: return "unknown status";
  }
}

const char *gz_last_error(void) { return g_last_error.c_str(); }

int gz_create(uint32_t num_vertices, uint64_t seed, double sketches_factor, double batch_factor,
              gz_alg_t **out) {
  return gz_create_ex(num_vertices, seed, sketches_factor, batch_factor, GZ_CAMEO_SKETCH, out);
}

int gz_create_ex(uint32_t num_vertices, uint64_t seed, double sketches_factor, double batch_factor,
                 int sketch_algorithm, gz_alg_t **out) {
  if (!out) return fail(GZ_ERR_INVALID, "out is null");
  if (sketch_algorithm != GZ_CAMEO_SKETCH && sketch_algorithm != GZ_CUBE_SKETCH)
    return fail(GZ_ERR_INVALID, "sketch_algorithm must be GZ_CAMEO_SKETCH or GZ_CUBE_SKETCH");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(GZ_ERR_NO_DEVICE, "no CUDA device is available (this library has no CPU path)");
  gz_alg *h = new gz_alg();
  const int rc = init_alg(h, num_vertices, seed, sketches_factor, batch_factor,
                          sketch_algorithm == GZ_CUBE_SKETCH);
  if (rc != GZ_OK) {
    destroy_alg(h);
    delete h;
    return rc;
  }
  *out = h;
  return GZ_OK;
}

int gz_create_from_serialized(const char *path, double batch_factor, gz_alg_t **out) {
  return gz_create_from_serialized_ex(path, batch_factor, GZ_CAMEO_SKETCH, out);
}

int gz_create_from_serialized_ex(const char *path, double batch_factor, int sketch_algorithm,
                                 gz_alg_t **out) {
  if (!path || !out) return fail(GZ_ERR_INVALID, "null argument");
  *out = nullptr;
  FILE *f = fopen(path, "rb");
  if (!f) return fail(GZ_ERR_IO, std::string("cannot open ") + path);
  uint64_t seed = 0;
  uint32_t V = 0;
  double sf = 0;
  if (fread(&seed, 8, 1, f) != 1 || fread(&V, 4, 1, f) != 1 || fread(&sf, 8, 1, f) != 1) {
    fclose(f);
    return fail(GZ_ERR_IO, "truncated header");
  }
  gz_alg_t *h = nullptr;
  int rc = gz_create_ex(V, seed, sf, batch_factor, sketch_algorithm, &h);
  if (rc != GZ_OK) {
    fclose(f);
    return rc;
  }
  std::vector<uint8_t> buf((size_t)h->sketch_bytes * V);
  const size_t got = fread(buf.data(), 1, buf.size(), f);
  fclose(f);
  if (got != buf.size()) {
    gz_destroy(h);
    return fail(GZ_ERR_IO, "truncated sketch data");
  }
  cudaError_t e = cudaMemcpy(h->d_sk, buf.data(), buf.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    gz_destroy(h);
    return fail(GZ_ERR_CUDA, cudaGetErrorString(e));
  }
  h->dsu_valid = false;  // src/cc_sketch_alg.cpp:62-63
  // loaded sketches keep the complement merge only if their XOR over all vertices is zero
  {
    uint32_t *d_tot = nullptr;
    const uint32_t words = h->nb * 3;
    std::vector<uint32_t> tot(words, 1);
    e = cudaMalloc(&d_tot, words * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_tot, 0, words * sizeof(uint32_t), h->stream);
    if (e == cudaSuccess) e = gz::sketch_total_xor(h->d_sk, V, words, d_tot, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tot.data(), d_tot, words * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (d_tot) cudaFree(d_tot);
    if (e != cudaSuccess) {
      gz_destroy(h);
      return fail(GZ_ERR_CUDA, cudaGetErrorString(e));
    }
    h->symmetric = std::all_of(tot.begin(), tot.end(), [](uint32_t x) { return x == 0; });
  }
  *out = h;
  return GZ_OK;
}

int gz_destroy(gz_alg_t *h) {
  if (!h) return GZ_OK;
  cudaSetDevice(h->device);
  destroy_alg(h);
  delete h;
  return GZ_OK;
}

int gz_get_params(const gz_alg_t *h, gz_params_t *o) {
  if (!h || !o) return fail(GZ_ERR_INVALID, "null argument");
  o->num_vertices = h->V;
  o->num_columns = h->C;
  o->bkt_per_col = h->B;
  o->num_buckets = h->nb;
  o->seed = h->seed;
  o->sketch_bytes = h->sketch_bytes;
  o->desired_updates_per_batch = h->desired_batch;
  o->max_rounds = h->samples;
  o->sketches_factor = h->sketches_factor;
  o->batch_factor = h->batch_factor;
  o->vertices_per_tile = 1u << h->tile_shift;
  o->num_tiles = h->ntiles;
  o->vertices_per_bin = 1u << h->bin_shift;
  o->num_bins = h->nbins;
  o->cols_per_sample = h->cps;
  o->sketch_algorithm = h->cube ? GZ_CUBE_SKETCH : GZ_CAMEO_SKETCH;
  o->in_place = h->in_place ? 1 : 0;
  o->entry_form = h->planes ? (h->codes3 ? 3 : 2) : 1;
  return GZ_OK;
}

int gz_set_gutter_capacity(gz_alg_t *h, uint64_t n) {
  if (!h || n < 2) return fail(GZ_ERR_INVALID, "capacity must be >= 2");
  Guard g(h);
  GZ_TRY(push_staged_entries(h));
  GZ_TRY(apply_pending(h));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  dev_free(h->d_gutter);
  h->entry_cap = n;
  return GZ_OK;
}

int gz_allocate_worker_memory(gz_alg_t *h, size_t num_workers) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  h->num_workers = std::max<size_t>(1, num_workers);
  return GZ_OK;
}

int gz_pre_insert(gz_alg_t *h, uint32_t src, uint32_t dst, int, int) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  pre_insert_one(h, src, dst);
  return GZ_OK;
}

int gz_set_eager_dsu(gz_alg_t *h, int enable) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  if ((enable != 0) == h->eager) return GZ_OK;
  h->eager = enable != 0;
  h->host_answer = false;
  h->hforest.clear();
  if (!h->eager || !h->dsu_valid) {
    h->hdsu.clear();
    return GZ_OK;
  }
  // a valid answer exists: start the eager DSU from it
  GZ_TRY(ensure_answer(h));
  return eager_from_device(h, h->boruvka_ran);
}

int gz_apply_update_batch(gz_alg_t *h, int, uint32_t src, const uint32_t *dsts, size_t n) {
  if (!h || (n && !dsts)) return fail(GZ_ERR_INVALID, "null argument");
  if (h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  Guard g(h);
  // the reference leaves the DSU to pre_insert, which the driver calls for every update; without
  // the eager DSU the cached answer is dropped here as well
  GZ_TRY(check_unlocked(h));
  if (!h->eager) invalidate_answer(h);
  if (src >= h->V) return fail(GZ_ERR_BAD_VERTEX, "src vertex id >= V");
  for (size_t i = 0; i < n; ++i) {
    if (dsts[i] >= h->V) return fail(GZ_ERR_BAD_VERTEX, "dst vertex id >= V");
  }
  h->symmetric = false;  // one endpoint's sketch only
  for (size_t i = 0; i < n; ++i) GZ_TRY(stage_entry(h, src, dsts[i]));
  return GZ_OK;
}

int gz_apply_raw_buckets_update(gz_alg_t *h, uint32_t src, const void *raw) {
  if (!h || !raw) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  if (src >= h->V) return fail(GZ_ERR_BAD_VERTEX, "src vertex id >= V");
  invalidate_answer(h);
  h->symmetric = false;
  GZ_TRY(dev_alloc(&h->d_raw, (size_t)h->nb * 3));
  GZ_CUDA(cudaMemcpyAsync(h->d_raw, raw, h->sketch_bytes, cudaMemcpyHostToDevice, h->stream));
  GZ_CUDA(gz::sketch_xor_raw(h->d_sk, h->nb * 3, src, h->d_raw, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int gz_update(gz_alg_t *h, uint32_t src, uint32_t dst, int) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  if (h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  Guard g(h);
  GZ_TRY(check_unlocked(h));
  pre_insert_one(h, src, dst);  // CCSketchAlg::update calls pre_insert first
  if (src >= h->V || dst >= h->V) return fail(GZ_ERR_BAD_VERTEX, "vertex id >= V");
  GZ_TRY(stage_entry(h, src, dst));
  GZ_TRY(stage_entry(h, dst, src));
  return GZ_OK;
}

int gz_ingest_records_device(gz_alg_t *h, const void *d_rec, size_t n) {
  if (!h || (n && !d_rec)) return fail(GZ_ERR_INVALID, "null argument");
  if (h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  Guard g(h);
  GZ_TRY(mark_updated(h));
  return gutter_chunk(h, gz::kInputRecords, d_rec, n);
}

int gz_ingest_records(gz_alg_t *h, const void *rec, size_t n) {
  if (!h || (n && !rec)) return fail(GZ_ERR_INVALID, "null argument");
  if (h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  Guard g(h);
  GZ_TRY(check_unlocked(h));
  if (h->eager) {
    // the driver's per-update pre_insert, in stream order, until the DSU is invalidated
    const uint8_t *r = static_cast<const uint8_t *>(rec);
    for (size_t i = 0; i < n && h->dsu_valid; ++i) {
      uint32_t u, v;
      std::memcpy(&u, r + 9 * i + 1, 4);
      std::memcpy(&v, r + 9 * i + 5, 4);
      pre_insert_one(h, u, v);
    }
  } else {
    invalidate_answer(h);
  }
  if (n == 0) return GZ_OK;
  gz::IngestPlan plan(n, h->in_place, (uint64_t)h->V * h->sketch_bytes);
  const uint64_t chunk = plan.chunk;
  const int nbuf = (int)std::min<uint64_t>(kStageBuffers, (n + chunk - 1) / chunk);
  if (chunk > h->stage_cap) {
    // staging buffers are sized for the largest chunk seen (small update batches stay small)
    GZ_CUDA(cudaStreamSynchronize(h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->copy_stream));
    for (int i = 0; i < kStageBuffers; ++i) {
      dev_free(h->d_stage[i]);
      if (h->ev_copied[i]) cudaEventDestroy(h->ev_copied[i]);
      if (h->ev_free[i]) cudaEventDestroy(h->ev_free[i]);
      h->ev_copied[i] = h->ev_free[i] = nullptr;
    }
    h->stage_cap = std::min<uint64_t>(kStageRecords, std::max<uint64_t>(chunk, 1ull << 16));
  }
  for (int i = 0; i < nbuf; ++i) {
    if (!h->d_stage[i]) {
      GZ_TRY(dev_alloc(&h->d_stage[i], h->stage_cap * 9 + 16));
      GZ_CUDA(cudaEventCreateWithFlags(&h->ev_copied[i], cudaEventDisableTiming));
      GZ_CUDA(cudaEventCreateWithFlags(&h->ev_free[i], cudaEventDisableTiming));
      GZ_CUDA(cudaEventRecord(h->ev_free[i], h->stream));
    }
  }
  const uint8_t *src = static_cast<const uint8_t *>(rec);
  int buf = 0;
  for (uint64_t off = 0, m = 0; off < n; off += m, buf = (buf + 1) % nbuf) {
    m = plan.next(off);
    GZ_CUDA(cudaStreamWaitEvent(h->copy_stream, h->ev_free[buf], 0));
    GZ_CUDA(cudaMemcpyAsync(h->d_stage[buf], src + off * 9, m * 9, cudaMemcpyHostToDevice, h->copy_stream));
    GZ_CUDA(cudaEventRecord(h->ev_copied[buf], h->copy_stream));
    GZ_CUDA(cudaStreamWaitEvent(h->stream, h->ev_copied[buf], 0));
    GZ_TRY(gutter_chunk(h, gz::kInputRecords, h->d_stage[buf], m));
    GZ_CUDA(cudaEventRecord(h->ev_free[buf], h->stream));
    // fold a wave into the sketches while the copy engine keeps streaming records
    if (plan.wave_after(off + m, h->entries_pending)) GZ_TRY(apply_pending(h));
  }
  // the caller's buffer may be reused once every copy has landed
  GZ_CUDA(cudaStreamSynchronize(h->copy_stream));
  return GZ_OK;
}

int gz_flush(gz_alg_t *h) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  return flush_all(h);
}

int gz_query_submit(gz_alg_t *h, uint64_t *ticket) {
  if (!h || !ticket) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  // every update so far goes to the stream ahead of the query; nothing waits here
  GZ_TRY(push_staged_entries(h));
  GZ_TRY(apply_pending(h));
  GZ_TRY(tickets_ensure(h));
  auto &T = h->tq;
  gz_alg::Ticket t;
  if (!T.pool.empty()) {
    t = T.pool.back();
    T.pool.pop_back();
  } else {
    GZ_CUDA(cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming));
    const int rc1 = host_alloc(&t.labels, h->V);
    const int rc2 = rc1 == GZ_OK ? host_alloc(&t.pin, 4) : rc1;
    if (rc2 != GZ_OK) {
      ticket_free(t);
      return rc2;
    }
  }
  const int pi = h->prof_begin();
  t.graph = query_mode_of(h) == 1;
  int rc = boruvka_enqueue(h, T.graph, h->bgeom(), h->d_sk, T.bv, T.d_final, T.d_ncc, t.pin, h->stream);
  h->prof_end(pi, 2);
  cudaError_t e = cudaSuccess;
  if (rc == GZ_OK) e = cudaMemcpyAsync(t.labels, T.d_final, sizeof(uint32_t) * h->V, cudaMemcpyDeviceToHost, h->stream);
  // the device status as the query left it (bits of earlier updates too), then cleared
  if (rc == GZ_OK && e == cudaSuccess)
    e = cudaMemcpyAsync(t.pin + 3, h->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
  if (rc == GZ_OK && e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, sizeof(uint32_t), h->stream);
  if (rc == GZ_OK && e == cudaSuccess) e = cudaEventRecord(t.done, h->stream);
  if (rc == GZ_OK && e != cudaSuccess) rc = fail(GZ_ERR_CUDA, cudaGetErrorString(e));
  if (rc != GZ_OK) {
    T.pool.push_back(t);
    return rc;
  }
  *ticket = T.next++;
  T.live[*ticket] = t;
  return GZ_OK;
}

int gz_query_wait(gz_alg_t *h, uint64_t ticket, uint32_t *parent_out, uint32_t *num_cc, size_t *rounds) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  gz_alg::Ticket t;
  {
    std::lock_guard<std::mutex> lk(h->mtx);
    auto it = h->tq.live.find(ticket);
    if (it == h->tq.live.end()) return fail(GZ_ERR_INVALID, "unknown or already collected ticket");
    t = it->second;
    h->tq.live.erase(it);
  }
  cudaSetDevice(h->device);
  const cudaError_t e = cudaEventSynchronize(t.done);  // no handle lock held: ingest goes on
  std::lock_guard<std::mutex> lk(h->mtx);
  if (e != cudaSuccess) {
    h->tq.pool.push_back(t);
    return fail(GZ_ERR_CUDA, cudaGetErrorString(e));
  }
  boruvka_account(h->tq.graph, t.pin, t.graph);
  const uint32_t round = t.pin[0], oos = t.pin[1], ncc = t.pin[2], st = t.pin[3];
  // bits of updates submitted before the query are reported by the next flush, as usual
  h->deferred_status |= st & (gz::kStatusBadVertex | gz::kStatusTimeout);
  if (rounds) *rounds = round;
  int rc = GZ_OK;
  if (oos) {
    rc = fail(GZ_ERR_OUT_OF_SAMPLES, out_of_samples_msg(h, round));
  } else if (st & gz::kStatusBadSample) {
    rc = fail(GZ_ERR_BAD_SAMPLE, "a sampled edge decoded to a vertex id >= V");
  } else {
    h->prof_acc.query_rounds += round + 1;
    if (num_cc) *num_cc = ncc;
    if (parent_out) std::copy(t.labels, t.labels + h->V, parent_out);
  }
  h->tq.pool.push_back(t);
  return rc;
}

int gz_has_cached_query(const gz_alg_t *h, int code, int *out) {
  if (!h || !out) return fail(GZ_ERR_INVALID, "null argument");
  *out = code == GZ_CONNECTIVITY ? (h->dsu_valid ? 1 : 0) : 0;
  return GZ_OK;
}

int gz_connected_components(gz_alg_t *h, uint32_t *parent_out, uint32_t *num_cc) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  GZ_TRY(ensure_answer(h));
  if (num_cc) *num_cc = h->last_ncc;
  if (parent_out) {
    GZ_CUDA(cudaMemcpyAsync(parent_out, h->d_final, sizeof(uint32_t) * h->V, cudaMemcpyDeviceToHost, h->stream));
    GZ_CUDA(cudaStreamSynchronize(h->stream));
  }
  return GZ_OK;
}

int gz_point_query(gz_alg_t *h, uint32_t a, uint32_t b, int *out) {
  if (!h || !out) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  if (a >= h->V || b >= h->V) return fail(GZ_ERR_BAD_VERTEX, "vertex id >= V");
  GZ_TRY(ensure_answer(h));
  GZ_TRY(labels_to_host(h));
  *out = h->h_labels[a] == h->h_labels[b] ? 1 : 0;
  return GZ_OK;
}

int gz_last_query_rounds(const gz_alg_t *h, size_t *out) {
  if (!h || !out) return fail(GZ_ERR_INVALID, "null argument");
  *out = h->last_rounds;
  return GZ_OK;
}

int gz_spanning_forest(gz_alg_t *h, uint32_t *edges_out, size_t cap, size_t *n_edges) {
  if (!h || !n_edges) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  GZ_TRY(ensure_answer(h));
  if (h->eager) {  // Boruvka's forest plus the edges the eager DSU merged since
    std::vector<uint64_t> idx(h->hforest.begin(), h->hforest.end());
    std::sort(idx.begin(), idx.end());
    *n_edges = idx.size();
    for (size_t i = 0; edges_out && i < std::min(cap, idx.size()); ++i) {
      edges_out[2 * i] = (uint32_t)(idx[i] >> 32);
      edges_out[2 * i + 1] = (uint32_t)idx[i];
    }
    return GZ_OK;
  }
  uint32_t n = 0;
  GZ_CUDA(cudaMemcpyAsync(h->h_status + 3, h->bv.forest_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  n = std::min<uint32_t>(h->h_status[3], h->V);
  *n_edges = n;
  if (edges_out && cap) {
    std::vector<uint64_t> idx(n);
    if (n) GZ_CUDA(cudaMemcpy(idx.data(), h->bv.forest, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < std::min<size_t>(cap, n); ++i) {
      edges_out[2 * i] = (uint32_t)(idx[i] >> 32);
      edges_out[2 * i + 1] = (uint32_t)idx[i];
    }
  }
  return GZ_OK;
}

int gz_dump_sketches(gz_alg_t *h, void *buf, size_t bytes) {
  if (!h || !buf) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  if (bytes != h->sketch_bytes * h->V) return fail(GZ_ERR_INVALID, "buffer must hold V * sketch_bytes bytes");
  GZ_TRY(flush_all(h));
  GZ_CUDA(cudaMemcpyAsync(buf, h->d_sk, bytes, cudaMemcpyDeviceToHost, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int gz_write_binary(gz_alg_t *h, const char *path) {
  if (!h || !path) return fail(GZ_ERR_INVALID, "null argument");
  std::vector<uint8_t> buf((size_t)h->sketch_bytes * h->V);
  GZ_TRY(gz_dump_sketches(h, buf.data(), buf.size()));
  FILE *f = fopen(path, "wb");
  if (!f) return fail(GZ_ERR_IO, std::string("cannot open ") + path);
  const uint64_t seed = h->seed;
  const uint32_t V = h->V;
  const double sf = h->sketches_factor;
  bool ok = fwrite(&seed, 8, 1, f) == 1 && fwrite(&V, 4, 1, f) == 1 && fwrite(&sf, 8, 1, f) == 1 &&
            fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? GZ_OK : fail(GZ_ERR_IO, "short write");
}

int gz_set_trace(gz_alg_t *h, int enable) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  h->trace = enable != 0;
  return GZ_OK;
}

int gz_get_trace(gz_alg_t *h, gz_trace_rec_t *out, size_t cap, size_t *len) {
  if (!h || !len) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  *len = 0;
  if (!h->bv.trace) return GZ_OK;
  GZ_CUDA(cudaMemcpyAsync(h->h_status + 3, h->bv.trace_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  const size_t n = std::min<size_t>(h->h_status[3], h->bv.trace_cap);
  *len = n;
  if (out && cap) GZ_CUDA(cudaMemcpy(out, h->bv.trace, std::min(cap, n) * sizeof(gz_trace_rec_t), cudaMemcpyDeviceToHost));
  return GZ_OK;
}

int gz_set_pipeline(gz_alg_t *h, int mode) {
  if (!h || mode < -1 || mode > 4) return fail(GZ_ERR_INVALID, "mode must be -1 .. 4");
  {
    Guard g(h);
    h->pipe_mode = mode;
  }
  // re-pick the default tiling for the chosen kernel; the staged-tile kernels take plain entries
  return gz_set_tuning(h, 0, 0, 0, mode >= 0 ? 1 : 0);
}

int gz_set_query_graph(gz_alg_t *h, int enable) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  if (enable < -1 || enable > 2) return fail(GZ_ERR_INVALID, "query mode is -1, 0, 1 or 2");
  h->query_mode = enable;
  return GZ_OK;
}

int gz_set_direct_factor(gz_alg_t *h, double factor) {
  if (!h || !(factor >= 0)) return fail(GZ_ERR_INVALID, "bad argument");
  Guard g(h);
  GZ_TRY(push_staged_entries(h));
  GZ_TRY(apply_pending(h));
  h->direct_factor = factor;
  return GZ_OK;
}

int gz_set_profiling(gz_alg_t *h, int enable) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  Guard g(h);
  h->prof_collect();
  h->prof = enable != 0;
  h->prof_acc = gz_profile_t{};
  h->launch_base = gz::launch_count();
  return GZ_OK;
}

int gz_get_profile(gz_alg_t *h, gz_profile_t *out) {
  if (!h || !out) return fail(GZ_ERR_INVALID, "null argument");
  Guard g(h);
  h->prof_collect();
  *out = h->prof_acc;
  out->kernel_launches = gz::launch_count() - h->launch_base;
  return GZ_OK;
}

int gz_clear(gz_alg_t *h) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  if (h->query_running.load()) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  Guard g(h);
  if (h->update_locked) return fail(GZ_ERR_LOCKED, "Cannot update the algorithm: Connected components currently running");
  h->nchunks = 0;
  h->gutter_used = 0;
  h->entries_pending = 0;
  h->h_ent_n = 0;
  const uint64_t v_pad = ((uint64_t)h->V + 63) & ~63ull;
  GZ_CUDA(cudaMemsetAsync(h->d_sk, 0, v_pad * h->sketch_bytes, h->stream));
  invalidate_answer(h);
  h->symmetric = true;
  if (h->eager) {  // empty sketches: the eager DSU restarts from singletons, as at construction
    h->hdsu.resize(h->V);
    for (uint32_t v = 0; v < h->V; ++v) h->hdsu[v] = v;
    h->hforest.clear();
    h->dsu_valid = true;
    h->host_answer = true;
  }
  return GZ_OK;
}

// Page-locks a caller's host buffer for this process (portable across contexts), so copies of
// records from it run at full host-link speed instead of through the driver's pageable staging;
// gz_host_unregister releases it. Used by callers that keep incoming update batches in one long
// lived buffer (a serving loop's receive buffers).
int gz_host_register(void *ptr, uint64_t bytes) {
  if (!ptr || bytes == 0) return fail(GZ_ERR_INVALID, "null or empty host buffer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(GZ_ERR_NO_DEVICE, "no CUDA device");
  GZ_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterPortable));
  return GZ_OK;
}

int gz_host_unregister(void *ptr) {
  if (!ptr) return fail(GZ_ERR_INVALID, "null host buffer");
  GZ_CUDA(cudaHostUnregister(ptr));
  return GZ_OK;
}

int gz_measure_update_rate(int repeats, double *updates_per_s) {
  if (!updates_per_s || repeats < 1) return fail(GZ_ERR_INVALID, "bad argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(GZ_ERR_NO_DEVICE, "no CUDA device");
  const int blocks = gz::num_sms();
  const uint32_t iters = 512;  // entries per thread; 32 bucket slots each
  uint32_t *out = nullptr;
  GZ_CUDA(cudaMalloc(&out, sizeof(uint32_t) * 1024 * blocks));
  const int rc = time_probe(repeats, (double)blocks * 1024 * iters * gz::kPlaneSlots,
                            [&](cudaStream_t s, int timed) {
                              return gz::plane_update_peak(timed ? iters : 8, blocks, out, s);
                            },
                            updates_per_s);
  cudaFree(out);
  return rc;
}

int gz_measure_hash_rate(int repeats, double *hashes_per_s) {
  if (!hashes_per_s || repeats < 1) return fail(GZ_ERR_INVALID, "bad argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(GZ_ERR_NO_DEVICE, "no CUDA device");
  const int threads = 256, blocks = gz::num_sms() * 8;
  const uint32_t iters = 4096;
  uint64_t *out = nullptr;
  GZ_CUDA(cudaMalloc(&out, sizeof(uint64_t) * threads * blocks));
  const int rc = time_probe(repeats, (double)threads * blocks * iters * 8,
                            [&](cudaStream_t s, int timed) {
                              return gz::plane_hash_peak(timed ? iters : 16, blocks, threads, out, s);
                            },
                            hashes_per_s);
  cudaFree(out);
  return rc;
}

int gz_get_stream(gz_alg_t *h, void **s) {
  if (!h || !s) return fail(GZ_ERR_INVALID, "null argument");
  *s = (void *)h->stream;
  return GZ_OK;
}

int gz_set_tuning(gz_alg_t *h, uint32_t vpt, uint32_t threads, uint32_t tiles_per_bin,
                  uint32_t entry_form) {
  if (!h) return fail(GZ_ERR_INVALID, "null handle");
  if (entry_form > 3) return fail(GZ_ERR_INVALID, "entry_form must be 0, 1, 2 or 3");
  if (entry_form >= 2 && (h->C > gz::kPlaneMaxColumns || h->cube))
    return fail(GZ_ERR_INVALID, "coded entries need CameoSketch with at most 31 columns");
  if (h->in_place && (vpt || threads || tiles_per_bin || entry_form >= 2))
    return fail(GZ_ERR_INVALID, "this handle updates its sketches in place: there are no tiles to tune");
  Guard g(h);
  GZ_TRY(push_staged_entries(h));
  GZ_TRY(apply_pending(h));
  GZ_CUDA(cudaStreamSynchronize(h->stream));
  const int keep_mode = h->planes_mode;
  const bool keep_planes = h->planes, keep_pipe = h->pipe, keep_codes3 = h->codes3;
  const uint32_t keep[5] = {h->tile_shift, h->ntiles, h->bin_shift, h->nbins, h->threads};
  h->planes_mode = entry_form == 0 ? -1 : (int)entry_form - 1;
  const uint32_t old_nb = h->nbins;
  const int rc = choose_tiling(h, vpt, threads, tiles_per_bin);
  if (rc != GZ_OK) {
    h->planes_mode = keep_mode;
    h->planes = keep_planes;
    h->codes3 = keep_codes3;
    h->pipe = keep_pipe;
    h->tile_shift = keep[0];
    h->ntiles = keep[1];
    h->bin_shift = keep[2];
    h->nbins = keep[3];
    h->threads = keep[4];
    return rc;
  }
  if (h->planes != keep_planes) dev_free(h->d_gutter);  // entry size changes: reallocated on the next ingest
  if (h->nbins != old_nb) {
    dev_free(h->d_bin_off);
    dev_free(h->d_hist);
    dev_free(h->d_scan_tmp);
    h->hist_words = 0;
  }
  return GZ_OK;
}

}  // extern "C"
