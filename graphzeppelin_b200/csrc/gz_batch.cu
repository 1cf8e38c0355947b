// gz_batch.cu -- many independent graph streams on one GPU: one gutter pass and one persistent
// sketch-update launch for all graphs, and a batched Boruvka whose round is a captured CUDA graph.
//
// Every graph keeps its own sketch geometry (vertex count, seed, columns, buckets per column) and
// its own shared-memory tile size; a device table describes them. Vertices of all graphs share one
// global id space (graph g owns [vbase_g, vbase_g + V_g)), so a single CAS union-find serves all
// graphs (unions never cross graphs). Per graph the result equals the single-graph path exactly:
// same sketch bytes, same partition, same last_query_rounds, same out-of-samples behaviour.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gz_b200.h"
#include "gz_common.cuh"
#include "gz_device.cuh"
#include "gz_kernels.cuh"

void gz_internal_set_error(const std::string &msg);

namespace gz {
namespace {

using namespace gz::dev;

struct GraphDesc {
  uint64_t sk_off;    // byte offset of the graph's sketches in the batch buffer
  uint32_t V, C, B, sketch_words;
  uint32_t tile_shift, bin_shift;
  uint32_t vbase;     // first global vertex id
  uint32_t bin_base;  // first global gutter bin
  uint32_t tile_base; // first global tile
  uint32_t flip_off;  // first of the graph's C + 1 hash constants
  uint32_t nbins, ntiles;
  uint32_t pad;
};

// index of the last base <= x in a sorted array of n bases (base[0] == 0)
__device__ __forceinline__ uint32_t find_base(const uint32_t *base, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ---- gutter ----------------------------------------------------------------------------------
// record tile: {graph, first record (lo, hi), count}
template <bool COUNT>
__global__ void __launch_bounds__(512)
k_mb_gutter(const uint8_t *__restrict__ rec, const uint4 *__restrict__ rtiles,
            const GraphDesc *__restrict__ graphs, uint64_t *__restrict__ bins,
            uint2 *__restrict__ entries, uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) uint8_t bsm[];
  const uint4 rt = rtiles[blockIdx.x];
  const GraphDesc gd = graphs[rt.x];
  const uint64_t start = ((uint64_t)rt.z << 32) | rt.y;
  const uint32_t shift = stage_records(rec, start, rt.w, bsm);
  __syncthreads();
  bool bad = false;
  for (uint32_t i = threadIdx.x; i < rt.w; i += blockDim.x) {
    uint32_t u, v;
    parse_record(bsm, shift, i, u, v);
    if (u >= gd.V || v >= gd.V) {
      bad = true;
      continue;
    }
    unsigned long long *bu = reinterpret_cast<unsigned long long *>(bins + gd.bin_base + (u >> gd.bin_shift));
    unsigned long long *bv = reinterpret_cast<unsigned long long *>(bins + gd.bin_base + (v >> gd.bin_shift));
    if (COUNT) {
      atomicAdd(bu, 1ull);
      atomicAdd(bv, 1ull);
    } else {
      entries[atomicAdd(bu, 1ull)] = make_uint2(u, v);
      entries[atomicAdd(bv, 1ull)] = make_uint2(v, u);
    }
  }
  if (COUNT && bad) atomicOr(status, kStatusBadVertex);
}

__global__ void k_mb_bin_off(const uint64_t *scanned, uint64_t nbins, const uint64_t *total,
                             uint32_t *bin_off) {
  const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b < nbins) bin_off[b] = (uint32_t)scanned[b];
  if (b == nbins) bin_off[b] = (uint32_t)*total;
}

// ---- sketch update -------------------------------------------------------------------------------
// One persistent launch over the (graph, tile) items of every graph: stage the tile with bulk
// async copies, XOR in the entries of the tile's gutter bin that belong to it, write it back.
__global__ void __launch_bounds__(1024, 1)
k_mb_sketch_update(const GraphDesc *__restrict__ graphs, const uint32_t *__restrict__ tile_base,
                   uint32_t G, uint32_t total_tiles, uint8_t *__restrict__ sketches,
                   const uint2 *__restrict__ entries, const uint32_t *__restrict__ bin_off,
                   const uint64_t *__restrict__ flip, uint32_t max_tile_bytes,
                   uint32_t *work_counter, uint32_t *status) {
  extern __shared__ __align__(128) uint8_t dsm[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_item, s_graph, s_b, s_e;
  uint32_t *s_sk = reinterpret_cast<uint32_t *>(dsm);
  uint32_t *s_queue = reinterpret_cast<uint32_t *>(dsm + max_tile_bytes);
  uint64_t *s_flip = reinterpret_cast<uint64_t *>(dsm + max_tile_bytes + kQueueBytes);
  const uint32_t bar = smem_u32(&s_bar);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t *q = s_queue + warp * 64;
  uint32_t parity = 0, cur_graph = 0xffffffffu;
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(work_counter, 1u);
      s_item = t;
      if (t < total_tiles) {
        const uint32_t g = find_base(tile_base, G, t);
        const GraphDesc gd = graphs[g];
        const uint32_t lt = t - gd.tile_base;
        const uint32_t bin = gd.bin_base + (lt >> (gd.bin_shift - gd.tile_shift));
        s_graph = g;
        s_b = bin_off[bin];
        s_e = bin_off[bin + 1];
        if (s_e > s_b) {
          const uint32_t bytes = (gd.sketch_words * 4) << gd.tile_shift;
          const uint8_t *src = sketches + gd.sk_off + (uint64_t)lt * bytes;
          mbar_expect_tx(bar, bytes);
          for (uint32_t off = 0; off < bytes; off += kBulkPiece)
            bulk_g2s(smem_u32(dsm) + off, src + off, min(kBulkPiece, bytes - off), bar);
        }
      }
    }
    __syncthreads();
    const uint32_t t = s_item;
    if (t >= total_tiles) break;
    if (s_e > s_b) {
      const uint32_t g = s_graph;
      const GraphDesc gd = graphs[g];
      if (g != cur_graph) {  // this CTA's flips belong to another graph: reload
        for (uint32_t i = threadIdx.x; i <= gd.C; i += blockDim.x) s_flip[i] = flip[gd.flip_off + i];
        cur_graph = g;
      }
      const bool ok = mbar_wait_bounded(bar, parity, kWaitLimitNs);
      parity ^= 1u;
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
          atomicOr(status, kStatusTimeout);
          mbar_wait_bounded(bar, parity ^ 1u, kWaitLimitNs);
        }
        return;
      }
      const uint32_t lt = t - gd.tile_base;
      const uint32_t vmask = (1u << gd.tile_shift) - 1;
      const uint64_t flip_chk = s_flip[gd.C];
      const uint32_t b = s_b, e = s_e;
      if (gd.bin_shift == gd.tile_shift) {
        for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x)
          apply_entry(entries[i], s_sk, vmask, gd.sketch_words, s_flip, flip_chk, gd.C, gd.B);
      } else {
        uint32_t qn = 0;
        for (uint32_t i0 = b + warp * 32; i0 < e; i0 += nwarps * 32) {
          const uint32_t i = i0 + lane;
          const bool mine = i < e && (entries[i].x >> gd.tile_shift) == lt;
          const uint32_t m = __ballot_sync(0xffffffffu, mine);
          if (mine) q[qn + __popc(m & ((1u << lane) - 1u))] = i;
          qn += __popc(m);
          __syncwarp();
          if (qn >= 32) {
            apply_entry(entries[q[lane]], s_sk, vmask, gd.sketch_words, s_flip, flip_chk, gd.C, gd.B);
            __syncwarp();
            qn -= 32;
            if (lane < qn) q[lane] = q[32 + lane];
            __syncwarp();
          }
        }
        if (lane < qn)
          apply_entry(entries[q[lane]], s_sk, vmask, gd.sketch_words, s_flip, flip_chk, gd.C, gd.B);
      }
      fence_proxy_async_smem();
      __syncthreads();
      if (threadIdx.x == 0) {
        const uint32_t bytes = (gd.sketch_words * 4) << gd.tile_shift;
        uint8_t *dst = sketches + gd.sk_off + (uint64_t)lt * bytes;
        for (uint32_t off = 0; off < bytes; off += kBulkPiece)
          bulk_s2g(dst + off, smem_u32(dsm) + off, min(kBulkPiece, bytes - off));
        bulk_commit();
        bulk_wait_read_all();
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// ---- batched Boruvka -------------------------------------------------------------------------------
struct MBBufs {
  const GraphDesc *graphs;
  const uint32_t *gov;  // graph of each global vertex
  const uint8_t *sketches;
  const uint64_t *flip;
  uint32_t *parent, *label, *cnt, *fill;
  uint64_t *packed, *scan_total;
  uint32_t *order, *comp_start, *ncomp, *acc;
  uint32_t *active, *modified;  // per graph
  const uint32_t *round;        // current round (device)
  uint32_t *status;
  uint32_t total_V, acc_words;  // acc words per component = (max B + 1) * 3
  uint32_t span;
};

// dsu_unite with the link order taken on graph-local ids, so every graph's roots (the highest
// ranked member of each component) are the ones its single-graph query finds.
__device__ bool mb_unite(uint32_t *parent, uint32_t a, uint32_t b, uint32_t vbase) {
  for (;;) {
    a = dsu_find(parent, a);
    b = dsu_find(parent, b);
    if (a == b) return false;
    if (rank_of(a - vbase) < rank_of(b - vbase)) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(parent + b, b, a) == b) return true;
  }
}

__device__ void mb_handle(int res, uint64_t idx, uint32_t g, const GraphDesc &gd, const MBBufs &b) {
  if (res == 2) {
    atomicOr(b.modified + g, 1u);
  } else if (res == 0) {
    const uint32_t x = (uint32_t)(idx >> 32), y = (uint32_t)idx;
    if (x >= gd.V || y >= gd.V) {
      atomicOr(b.status, kStatusBadSample);
      return;
    }
    if (mb_unite(b.parent, gd.vbase + x, gd.vbase + y, gd.vbase)) atomicOr(b.modified + g, 1u);
  }
}

__device__ __forceinline__ const uint32_t *mb_sketch(const MBBufs &b, const GraphDesc &gd,
                                                     uint32_t v) {
  return reinterpret_cast<const uint32_t *>(b.sketches + gd.sk_off) +
         (uint64_t)(v - gd.vbase) * gd.sketch_words;
}

__global__ void k_mb_round0(MBBufs b) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < b.total_V; v += nwarps) {
    const uint32_t g = b.gov[v];
    if (!b.active[g]) continue;
    const GraphDesc gd = b.graphs[g];
    const uint32_t *sk = mb_sketch(b, gd, v);
    uint32_t d[3], a[2][3] = {{0, 0, 0}, {0, 0, 0}};
    load_bucket(sk + 3 * gd.C * gd.B, d);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const uint32_t j = s * 32 + lane;
      if (j < gd.B) load_bucket(sk + 3 * j, a[s]);
    }
    uint64_t idx;
    const int res = warp_sample(d, a, gd.B, b.flip[gd.flip_off + gd.C], &idx);
    if (lane == 0) mb_handle(res, idx, g, gd, b);
  }
}

__global__ void k_mb_label(MBBufs b) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= b.total_V || !b.active[b.gov[v]]) return;
  const uint32_t r = dsu_find(b.parent, v);
  b.label[v] = r;
  atomicAdd(&b.cnt[r], 1u);
}

__global__ void k_mb_pack(MBBufs b) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= b.total_V) return;
  const uint32_t c = b.cnt[v];
  b.packed[v] = (uint64_t)c | (c ? (1ull << 32) : 0ull);
}

__global__ void k_mb_group(MBBufs b) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v == 0) {
    const uint32_t nc = (uint32_t)(*b.scan_total >> 32), members = (uint32_t)*b.scan_total;
    b.comp_start[nc] = members;
    *b.ncomp = nc;
  }
  if (v >= b.total_V || !b.active[b.gov[v]]) return;
  const uint32_t r = b.label[v];
  const uint64_t s = b.packed[r];
  const uint32_t start = (uint32_t)s, c = (uint32_t)(s >> 32);
  b.order[start + atomicAdd(&b.fill[r], 1u)] = v;
  if (v == r) {
    b.comp_start[c] = start;
    const uint32_t end = start + b.cnt[r];
    if (start / b.span != (end - 1) / b.span) {
      uint32_t *ac = b.acc + (uint64_t)c * b.acc_words;
      for (uint32_t i = 0; i < b.acc_words; ++i) ac[i] = 0;
    }
  }
}

// component index of grouped position p (comp_start is sorted)
__device__ __forceinline__ uint32_t comp_of(const MBBufs &b, uint32_t nc, uint32_t p) {
  uint32_t lo = 0, hi = nc;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (b.comp_start[mid] <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_mb_merge(MBBufs b) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nc = *b.ncomp;
  const uint32_t members = b.comp_start[nc];
  const uint64_t p0 = (uint64_t)w * b.span;
  if (p0 >= members) return;
  const uint32_t p1 = (p0 + b.span < members) ? (uint32_t)(p0 + b.span) : members;
  const uint32_t round = *b.round;
  uint32_t a[2][3] = {{0, 0, 0}, {0, 0, 0}}, d[3] = {0, 0, 0};
  uint32_t cur = comp_of(b, nc, (uint32_t)p0);
  uint32_t next_start = b.comp_start[cur + 1];
  uint32_t g = b.gov[b.order[p0]];
  GraphDesc gd = b.graphs[g];
  auto flush = [&]() {
    const uint32_t s = b.comp_start[cur], e = b.comp_start[cur + 1];
    if (s >= p0 && e <= p1) {
      uint64_t idx;
      const int res = warp_sample(d, a, gd.B, b.flip[gd.flip_off + gd.C], &idx);
      if (lane == 0) mb_handle(res, idx, g, gd, b);
    } else {
      uint32_t *ac = b.acc + (uint64_t)cur * b.acc_words;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const uint32_t j = q * 32 + lane;
        if (j < gd.B) {
          atomicXor(ac + 3 * j, a[q][0]);
          atomicXor(ac + 3 * j + 1, a[q][1]);
          atomicXor(ac + 3 * j + 2, a[q][2]);
        }
      }
      if (lane == 0) {
        atomicXor(ac + 3 * gd.B, d[0]);
        atomicXor(ac + 3 * gd.B + 1, d[1]);
        atomicXor(ac + 3 * gd.B + 2, d[2]);
      }
    }
  };
  for (uint32_t p = (uint32_t)p0; p < p1; ++p) {
    if (p == next_start) {
      flush();
      ++cur;
      next_start = b.comp_start[cur + 1];
      g = b.gov[b.order[p]];
      gd = b.graphs[g];
#pragma unroll
      for (int q = 0; q < 2; ++q) a[q][0] = a[q][1] = a[q][2] = 0;
      d[0] = d[1] = d[2] = 0;
    }
    const uint32_t *sk = mb_sketch(b, gd, b.order[p]);
    const uint32_t col = 3 * round * gd.B, detw = 3 * gd.C * gd.B;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t j = q * 32 + lane;
      if (j < gd.B) {
        const uint32_t *bk = sk + col + 3 * j;
        a[q][0] ^= bk[0];
        a[q][1] ^= bk[1];
        a[q][2] ^= bk[2];
      }
    }
    d[0] ^= sk[detw];
    d[1] ^= sk[detw + 1];
    d[2] ^= sk[detw + 2];
  }
  flush();
}

__global__ void k_mb_sample_spanning(MBBufs b) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nc = *b.ncomp;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc; c += nwarps) {
    const uint32_t s = b.comp_start[c], e = b.comp_start[c + 1];
    if (s / b.span == (e - 1) / b.span) continue;
    const uint32_t g = b.gov[b.order[s]];
    const GraphDesc gd = b.graphs[g];
    const uint32_t *ac = b.acc + (uint64_t)c * b.acc_words;
    uint32_t a[2][3] = {{0, 0, 0}, {0, 0, 0}}, d[3];
    d[0] = __ldcg(ac + 3 * gd.B);
    d[1] = __ldcg(ac + 3 * gd.B + 1);
    d[2] = __ldcg(ac + 3 * gd.B + 2);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t j = q * 32 + lane;
      if (j < gd.B) {
        a[q][0] = __ldcg(ac + 3 * j);
        a[q][1] = __ldcg(ac + 3 * j + 1);
        a[q][2] = __ldcg(ac + 3 * j + 2);
      }
    }
    uint64_t idx;
    const int res = warp_sample(d, a, gd.B, b.flip[gd.flip_off + gd.C], &idx);
    if (lane == 0) mb_handle(res, idx, g, gd, b);
  }
}

__global__ void k_mb_reset(uint32_t n, uint32_t *parent) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) parent[v] = v;
}

// labels_out[v] = graph-local representative; ncc[g] += roots of graph g
__global__ void k_mb_final(MBBufs b, uint32_t *labels_out, uint32_t *ncc) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= b.total_V) return;
  const uint32_t g = b.gov[v];
  const uint32_t r = dsu_find(b.parent, v);
  labels_out[v] = r - b.graphs[g].vbase;
  if (r == v) atomicAdd(ncc + g, 1u);
}

inline unsigned cdiv(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

#define MB_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      gz_internal_set_error(std::string(#call) + ": " + cudaGetErrorString(e_));            \
      return e_ == cudaErrorMemoryAllocation ? GZ_ERR_NOMEM : GZ_ERR_CUDA;                  \
    }                                                                                       \
  } while (0)
#define MB_TRY(expr)          \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != GZ_OK) return rc_; \
  } while (0)

int mb_fail(int code, const std::string &msg) {
  gz_internal_set_error(msg);
  return code;
}

template <class T>
int mb_alloc(T **p, size_t count) {
  if (*p) return GZ_OK;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return mb_fail(GZ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  *p = static_cast<T *>(q);
  return GZ_OK;
}
template <class T>
void mb_free(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}


}  // namespace
}  // namespace gz

using gz::GraphDesc;

struct gz_batch {
  std::mutex mtx;
  int device = 0;
  uint32_t G = 0;
  double factor = 1;
  std::vector<GraphDesc> graphs;
  std::vector<uint64_t> seeds;
  uint64_t total_V = 0, total_bins = 0, total_tiles = 0, sk_bytes = 0;
  uint32_t max_B = 0, max_C = 0, max_tile_bytes = 0, threads = 1024;
  GraphDesc *d_graphs = nullptr;
  uint32_t *d_tile_base = nullptr, *d_gov = nullptr;
  uint8_t *d_sk = nullptr;
  uint64_t *d_flip = nullptr;
  uint32_t *d_status = nullptr, *h_small = nullptr;
  // gutter
  uint2 *d_entries = nullptr;
  uint64_t entry_cap = 0;
  uint64_t *d_bins = nullptr, *d_scan_tmp = nullptr, *d_total = nullptr;
  uint32_t *d_bin_off = nullptr;
  uint4 *d_rtiles = nullptr;
  size_t rtiles_cap = 0;
  uint8_t *d_rec = nullptr;  // device copy of host records (gz_batch_ingest)
  uint64_t rec_cap = 0;
  // Boruvka
  uint32_t *d_parent = nullptr, *d_label = nullptr, *d_cnt = nullptr, *d_fill = nullptr;
  uint64_t *d_packed = nullptr, *d_vscan_total = nullptr, *d_vscan_tmp = nullptr;
  uint32_t *d_order = nullptr, *d_comp_start = nullptr, *d_ncomp = nullptr, *d_acc = nullptr;
  uint32_t *d_active = nullptr, *d_modified = nullptr, *d_round = nullptr, *d_ncc = nullptr;
  cudaGraphExec_t round_exec = nullptr;
  cudaGraph_t round_graph = nullptr;
  std::vector<uint32_t> rounds, status, ncc;
  cudaStream_t stream = nullptr;
  bool prof = false;
  uint64_t launches = 0;       // kernels this handle launched (graph replays count their kernels)
  uint32_t round_kernels = 0;  // kernel nodes of the captured round
  double prof_gutter_ms = 0, prof_sketch_ms = 0, prof_query_ms = 0;
  uint64_t prof_rounds = 0;

  gz::MBBufs bufs() const {
    gz::MBBufs b;
    b.graphs = d_graphs;
    b.gov = d_gov;
    b.sketches = d_sk;
    b.flip = d_flip;
    b.parent = d_parent;
    b.label = d_label;
    b.cnt = d_cnt;
    b.fill = d_fill;
    b.packed = d_packed;
    b.scan_total = d_vscan_total;
    b.order = d_order;
    b.comp_start = d_comp_start;
    b.ncomp = d_ncomp;
    b.acc = d_acc;
    b.active = d_active;
    b.modified = d_modified;
    b.round = d_round;
    b.status = d_status;
    b.total_V = (uint32_t)total_V;
    b.acc_words = (max_B + 1) * 3;
    b.span = 64;
    return b;
  }
};

namespace {

using namespace gz;

void batch_destroy(gz_batch *h) {
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->round_exec) cudaGraphExecDestroy(h->round_exec);
  if (h->round_graph) cudaGraphDestroy(h->round_graph);
  mb_free(h->d_graphs);
  mb_free(h->d_tile_base);
  mb_free(h->d_gov);
  mb_free(h->d_sk);
  mb_free(h->d_flip);
  mb_free(h->d_status);
  if (h->h_small) cudaFreeHost(h->h_small);
  mb_free(h->d_entries);
  mb_free(h->d_bins);
  mb_free(h->d_scan_tmp);
  mb_free(h->d_total);
  mb_free(h->d_bin_off);
  mb_free(h->d_rtiles);
  mb_free(h->d_rec);
  mb_free(h->d_parent);
  mb_free(h->d_label);
  mb_free(h->d_cnt);
  mb_free(h->d_fill);
  mb_free(h->d_packed);
  mb_free(h->d_vscan_total);
  mb_free(h->d_vscan_tmp);
  mb_free(h->d_order);
  mb_free(h->d_comp_start);
  mb_free(h->d_ncomp);
  mb_free(h->d_acc);
  mb_free(h->d_active);
  mb_free(h->d_modified);
  mb_free(h->d_round);
  mb_free(h->d_ncc);
  if (h->stream) cudaStreamDestroy(h->stream);
}

// Per-graph tile/bin geometry: the single-graph default rule (tile of at most 64 vertices that
// fits in shared memory, bins of up to 16 tiles), or an explicit vertices-per-tile.
int layout(gz_batch *h, const std::vector<uint32_t> &vpt_req) {
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  if (smem_optin <= 0) smem_optin = 227 * 1024;
  uint64_t sk_off = 0, vbase = 0, bin_base = 0, tile_base = 0, flip_off = 0;
  h->max_tile_bytes = 0;
  h->max_B = h->max_C = 0;
  for (const GraphDesc &gd : h->graphs) {
    h->max_B = std::max(h->max_B, gd.B);
    h->max_C = std::max(h->max_C, gd.C);
  }
  // one launch serves every graph: its shared memory holds the largest tile and the most flips
  const size_t budget = (size_t)smem_optin - 64 - kQueueBytes - (size_t)(h->max_C + 1) * 8;
  for (uint32_t g = 0; g < h->G; ++g) {
    GraphDesc &gd = h->graphs[g];
    const uint64_t sketch_bytes = (uint64_t)gd.sketch_words * 4;
    uint32_t shift = 2;
    if (!vpt_req.empty() && vpt_req[g]) {
      shift = (uint32_t)__builtin_ctz(vpt_req[g]);
    } else {
      const uint64_t want = std::max<uint64_t>(4, gd.V / (2ull * num_sms()));
      while (shift < 6 && (1ull << (shift + 1)) <= want && (sketch_bytes << (shift + 1)) <= budget)
        ++shift;
    }
    if ((sketch_bytes << shift) > budget) return mb_fail(GZ_ERR_INVALID, "sketch too large for a tile");
    uint32_t bshift = shift;
    while (((gd.V + (1u << bshift) - 1) >> bshift) > 4096 && (1u << (bshift - shift)) < 16) ++bshift;
    gd.tile_shift = shift;
    gd.bin_shift = bshift;
    gd.ntiles = (gd.V + (1u << shift) - 1) >> shift;
    gd.nbins = (gd.V + (1u << bshift) - 1) >> bshift;
    gd.sk_off = sk_off;
    gd.vbase = (uint32_t)vbase;
    gd.bin_base = (uint32_t)bin_base;
    gd.tile_base = (uint32_t)tile_base;
    gd.flip_off = (uint32_t)flip_off;
    const uint64_t v_pad = ((uint64_t)gd.V + 63) & ~63ull;
    sk_off += (v_pad * sketch_bytes + 255) & ~255ull;
    vbase += gd.V;
    bin_base += gd.nbins;
    tile_base += gd.ntiles;
    flip_off += gd.C + 1;
    h->max_tile_bytes = std::max<uint32_t>(h->max_tile_bytes, (uint32_t)(sketch_bytes << shift));
  }
  if (vbase > 0xFFFFFFF0ull || bin_base > 0xFFFFFFF0ull || tile_base > 0xFFFFFFF0ull)
    return mb_fail(GZ_ERR_INVALID, "batch too large for 32-bit global vertex ids");
  h->sk_bytes = sk_off;
  h->total_V = vbase;
  h->total_bins = bin_base;
  h->total_tiles = tile_base;
  return GZ_OK;
}

int upload_tables(gz_batch *h) {
  std::vector<uint32_t> tb(h->G);
  for (uint32_t g = 0; g < h->G; ++g) tb[g] = h->graphs[g].tile_base;
  MB_CUDA(cudaMemcpyAsync(h->d_graphs, h->graphs.data(), sizeof(GraphDesc) * h->G, cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaMemcpyAsync(h->d_tile_base, tb.data(), sizeof(uint32_t) * h->G, cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int batch_flush_status(gz_batch *h) {
  MB_CUDA(cudaMemcpyAsync(h->h_small, h->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  MB_CUDA(cudaStreamSynchronize(h->stream));
  const uint32_t st = h->h_small[0];
  if (st) {
    MB_CUDA(cudaMemsetAsync(h->d_status, 0, sizeof(uint32_t), h->stream));
    MB_CUDA(cudaStreamSynchronize(h->stream));
    if (st & kStatusTimeout) return mb_fail(GZ_ERR_TIMEOUT, "a bounded device wait timed out");
    if (st & kStatusBadVertex) return mb_fail(GZ_ERR_BAD_VERTEX, "a record named a vertex id >= its graph's V");
    if (st & kStatusBadSample) return mb_fail(GZ_ERR_BAD_SAMPLE, "a sampled edge decoded to a vertex id >= V");
  }
  return GZ_OK;
}

// records of graph g are d_rec[off[g] .. off[g+1]) (9-byte records)
int batch_ingest(gz_batch *h, const void *d_rec, const uint64_t *off) {
  std::vector<uint4> rt;
  uint64_t n_total = 0;
  for (uint32_t g = 0; g < h->G; ++g) {
    if (off[g + 1] < off[g]) return mb_fail(GZ_ERR_INVALID, "record offsets must be non-decreasing");
    for (uint64_t s = off[g]; s < off[g + 1]; s += kRecTile) {
      const uint32_t cnt = (uint32_t)std::min<uint64_t>(kRecTile, off[g + 1] - s);
      rt.push_back(make_uint4(g, (uint32_t)s, (uint32_t)(s >> 32), cnt));
    }
    n_total += off[g + 1] - off[g];
  }
  if (rt.empty()) return GZ_OK;
  if (2 * n_total >= 0xFFFFFFF0ull) return mb_fail(GZ_ERR_INVALID, "more than 2^31 records in one batch ingest");
  if (h->entry_cap < 2 * n_total) {
    mb_free(h->d_entries);
    h->entry_cap = 0;
    MB_TRY(mb_alloc(&h->d_entries, 2 * n_total));
    h->entry_cap = 2 * n_total;
  }
  if (h->rtiles_cap < rt.size()) {
    mb_free(h->d_rtiles);
    h->rtiles_cap = 0;
    MB_TRY(mb_alloc(&h->d_rtiles, rt.size()));
    h->rtiles_cap = rt.size();
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
  if (h->prof) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, h->stream);
  }
  MB_CUDA(cudaMemcpyAsync(h->d_rtiles, rt.data(), sizeof(uint4) * rt.size(), cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaMemsetAsync(h->d_bins, 0, sizeof(uint64_t) * h->total_bins, h->stream));
  const size_t smem = kRecTile * 9 + 48;
  const uint8_t *rec = static_cast<const uint8_t *>(d_rec);
  k_mb_gutter<true><<<(unsigned)rt.size(), 512, smem, h->stream>>>(rec, h->d_rtiles, h->d_graphs, h->d_bins,
                                                                    nullptr, h->d_status);
  h->launches++;
  MB_CUDA(cudaGetLastError());
  const uint64_t l0 = launch_count();
  MB_CUDA(scan_exclusive_u64(h->d_bins, h->total_bins, h->d_total, h->d_scan_tmp, h->stream));
  h->launches += launch_count() - l0;
  k_mb_bin_off<<<cdiv(h->total_bins + 1, 256), 256, 0, h->stream>>>(h->d_bins, h->total_bins, h->d_total,
                                                                     h->d_bin_off);
  k_mb_gutter<false><<<(unsigned)rt.size(), 512, smem, h->stream>>>(rec, h->d_rtiles, h->d_graphs, h->d_bins,
                                                                     h->d_entries, h->d_status);
  h->launches += 2;
  MB_CUDA(cudaGetLastError());
  if (h->prof) cudaEventRecord(e1, h->stream);
  // one persistent launch for every (graph, tile)
  MB_CUDA(cudaMemsetAsync(h->d_status + 1, 0, sizeof(uint32_t), h->stream));
  const size_t ksmem = h->max_tile_bytes + kQueueBytes + (size_t)(h->max_C + 1) * 8;
  MB_CUDA(cudaFuncSetAttribute(k_mb_sketch_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ksmem));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mb_sketch_update, (int)h->threads, ksmem);
  const int grid = (int)std::min<uint64_t>(h->total_tiles, (uint64_t)num_sms() * std::max(per_sm, 1));
  k_mb_sketch_update<<<grid, h->threads, ksmem, h->stream>>>(
      h->d_graphs, h->d_tile_base, h->G, (uint32_t)h->total_tiles, h->d_sk, h->d_entries, h->d_bin_off,
      h->d_flip, h->max_tile_bytes, h->d_status + 1, h->d_status);
  h->launches++;
  MB_CUDA(cudaGetLastError());
  if (h->prof) {
    cudaEventRecord(e2, h->stream);
    cudaEventSynchronize(e2);
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    h->prof_gutter_ms += a;
    h->prof_sketch_ms += b;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
  }
  return batch_flush_status(h);
}

int ensure_boruvka(gz_batch *h) {
  const size_t V = h->total_V;
  MB_TRY(mb_alloc(&h->d_parent, V));
  MB_TRY(mb_alloc(&h->d_label, V));
  MB_TRY(mb_alloc(&h->d_cnt, V));
  MB_TRY(mb_alloc(&h->d_fill, V));
  MB_TRY(mb_alloc(&h->d_packed, V));
  MB_TRY(mb_alloc(&h->d_vscan_total, 1));
  MB_TRY(mb_alloc(&h->d_vscan_tmp, scan_tmp_words(V)));
  MB_TRY(mb_alloc(&h->d_order, V));
  MB_TRY(mb_alloc(&h->d_comp_start, V + 1));
  MB_TRY(mb_alloc(&h->d_ncomp, 1));
  MB_TRY(mb_alloc(&h->d_acc, V * (size_t)(h->max_B + 1) * 3));
  MB_TRY(mb_alloc(&h->d_active, h->G));
  MB_TRY(mb_alloc(&h->d_modified, h->G));
  MB_TRY(mb_alloc(&h->d_round, 1));
  MB_TRY(mb_alloc(&h->d_ncc, h->G));
  return GZ_OK;
}

// Kernels of one round >= 1, enqueued on s (captured once into a CUDA graph).
int enqueue_round(gz_batch *h, cudaStream_t s) {
  const MBBufs b = h->bufs();
  const size_t V = h->total_V;
  MB_CUDA(cudaMemsetAsync(h->d_cnt, 0, sizeof(uint32_t) * V, s));
  MB_CUDA(cudaMemsetAsync(h->d_fill, 0, sizeof(uint32_t) * V, s));
  MB_CUDA(cudaMemsetAsync(h->d_modified, 0, sizeof(uint32_t) * h->G, s));
  k_mb_label<<<cdiv(V, 256), 256, 0, s>>>(b);
  k_mb_pack<<<cdiv(V, 256), 256, 0, s>>>(b);
  MB_CUDA(scan_exclusive_u64(h->d_packed, V, h->d_vscan_total, h->d_vscan_tmp, s));
  k_mb_group<<<cdiv(V, 256), 256, 0, s>>>(b);
  const uint64_t warps = (V + b.span - 1) / b.span;
  k_mb_merge<<<cdiv(warps * 32, 256), 256, 0, s>>>(b);
  k_mb_sample_spanning<<<std::min<unsigned>(cdiv(V * 32, 256), num_sms() * 16), 256, 0, s>>>(b);
  MB_CUDA(cudaGetLastError());
  return GZ_OK;
}

// boruvka_emulation for every graph at once; per graph the rounds stop independently.
int batch_query(gz_batch *h, uint32_t *labels_out) {
  MB_TRY(ensure_boruvka(h));
  const MBBufs b = h->bufs();
  const size_t V = h->total_V;
  const uint32_t G = h->G;
  cudaEvent_t q0 = nullptr, q1 = nullptr;
  if (h->prof) {
    cudaEventCreate(&q0);
    cudaEventCreate(&q1);
    cudaEventRecord(q0, h->stream);
  }
  std::vector<uint32_t> active(G, 1), modified(G, 0);
  h->rounds.assign(G, 0);
  h->status.assign(G, GZ_OK);
  h->ncc.assign(G, 0);
  k_mb_reset<<<cdiv(V, 256), 256, 0, h->stream>>>((uint32_t)V, h->d_parent);
  MB_CUDA(cudaMemcpyAsync(h->d_active, active.data(), sizeof(uint32_t) * G, cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaMemsetAsync(h->d_modified, 0, sizeof(uint32_t) * G, h->stream));
  k_mb_round0<<<std::min<unsigned>(cdiv(V * 32, 256), num_sms() * 16), 256, 0, h->stream>>>(b);
  h->launches += 2;
  MB_CUDA(cudaGetLastError());
  if (!h->round_exec) {
    // capture the round once: it reads the round number and the active flags from device memory
    cudaStream_t cs = nullptr;
    MB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    MB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_round(h, cs);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (rc != GZ_OK) return rc;
    MB_CUDA(ec);
    h->round_graph = graph;
    MB_CUDA(cudaGraphInstantiate(&h->round_exec, graph, 0));
    size_t n = 0;
    MB_CUDA(cudaGraphGetNodes(graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    MB_CUDA(cudaGraphGetNodes(graph, nodes.data(), &n));
    h->round_kernels = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) h->round_kernels++;
    }
  }
  uint32_t round = 0;
  for (;;) {
    MB_CUDA(cudaMemcpyAsync(modified.data(), h->d_modified, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, h->stream));
    MB_CUDA(cudaStreamSynchronize(h->stream));
    bool any = false;
    for (uint32_t g = 0; g < G; ++g) {
      if (!active[g]) continue;
      if (!modified[g]) {  // this graph's round changed nothing: its Boruvka is done
        active[g] = 0;
        h->rounds[g] = round;
      } else if (round + 1 >= h->graphs[g].C) {  // Sketch::sample would throw next round
        active[g] = 0;
        h->rounds[g] = round + 1;
        h->status[g] = GZ_ERR_OUT_OF_SAMPLES;
      } else {
        any = true;
      }
    }
    if (!any) break;
    ++round;
    MB_CUDA(cudaMemcpyAsync(h->d_active, active.data(), sizeof(uint32_t) * G, cudaMemcpyHostToDevice, h->stream));
    MB_CUDA(cudaMemcpyAsync(h->d_round, &round, sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    MB_CUDA(cudaGraphLaunch(h->round_exec, h->stream));
    h->launches += h->round_kernels;
    h->prof_rounds++;
  }
  MB_CUDA(cudaMemsetAsync(h->d_ncc, 0, sizeof(uint32_t) * G, h->stream));
  k_mb_final<<<cdiv(V, 256), 256, 0, h->stream>>>(b, h->d_label, h->d_ncc);
  h->launches++;
  MB_CUDA(cudaGetLastError());
  if (labels_out)
    MB_CUDA(cudaMemcpyAsync(labels_out, h->d_label, sizeof(uint32_t) * V, cudaMemcpyDeviceToHost, h->stream));
  MB_CUDA(cudaMemcpyAsync(h->ncc.data(), h->d_ncc, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, h->stream));
  if (h->prof) cudaEventRecord(q1, h->stream);
  MB_CUDA(cudaStreamSynchronize(h->stream));
  if (h->prof) {
    float ms = 0;
    cudaEventElapsedTime(&ms, q0, q1);
    h->prof_query_ms += ms;
    cudaEventDestroy(q0);
    cudaEventDestroy(q1);
  }
  return batch_flush_status(h);
}

}  // namespace

extern "C" {

int gz_batch_create(uint32_t num_graphs, const uint32_t *num_vertices, const uint64_t *seeds,
                    double sketches_factor, const uint32_t *vertices_per_tile, gz_batch_t **out) {
  if (!out || !num_vertices || !seeds || num_graphs == 0) return mb_fail(GZ_ERR_INVALID, "bad argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return mb_fail(GZ_ERR_NO_DEVICE, "no CUDA device");
  gz_batch *h = new gz_batch();
  auto bail = [&](int rc) {
    batch_destroy(h);
    delete h;
    return rc;
  };
  cudaGetDevice(&h->device);
  h->G = num_graphs;
  h->factor = sketches_factor > 0 ? sketches_factor : 1;
  h->graphs.resize(num_graphs);
  h->seeds.assign(seeds, seeds + num_graphs);
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const uint32_t V = num_vertices[g];
    if (V < 2 || V > (1u << 31)) return bail(mb_fail(GZ_ERR_INVALID, "every graph needs 2 <= V <= 2^31"));
    if (vertices_per_tile && vertices_per_tile[g] &&
        (vertices_per_tile[g] < 4 || vertices_per_tile[g] > 64 || (vertices_per_tile[g] & (vertices_per_tile[g] - 1))))
      return bail(mb_fail(GZ_ERR_INVALID, "vertices_per_tile must be 0 or a power of two in [4, 64]"));
    GraphDesc &gd = h->graphs[g];
    std::memset(&gd, 0, sizeof(gd));
    gd.V = V;
    sketch_sizing(V, h->factor, gd.C, gd.B);
    if (gd.B > 63) return bail(mb_fail(GZ_ERR_INVALID, "bkt_per_col above 63 is not supported"));
    gd.sketch_words = (gd.C * gd.B + 1) * 3;
  }
  std::vector<uint32_t> vpt;
  if (vertices_per_tile) vpt.assign(vertices_per_tile, vertices_per_tile + num_graphs);
  int rc = layout(h, vpt);
  if (rc != GZ_OK) return bail(rc);
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(mb_fail(GZ_ERR_CUDA, cudaGetErrorString(e)));
  if ((rc = mb_alloc(&h->d_graphs, num_graphs)) || (rc = mb_alloc(&h->d_tile_base, num_graphs)) ||
      (rc = mb_alloc(&h->d_gov, h->total_V)) || (rc = mb_alloc(&h->d_sk, h->sk_bytes)) ||
      (rc = mb_alloc(&h->d_status, 4)) || (rc = mb_alloc(&h->d_bins, h->total_bins)) ||
      (rc = mb_alloc(&h->d_scan_tmp, scan_tmp_words(h->total_bins))) || (rc = mb_alloc(&h->d_total, 1)) ||
      (rc = mb_alloc(&h->d_bin_off, h->total_bins + 1)))
    return bail(rc);
  uint64_t nflip = 0;
  for (auto &gd : h->graphs) nflip += gd.C + 1;
  if ((rc = mb_alloc(&h->d_flip, nflip))) return bail(rc);
  std::vector<uint64_t> flip(nflip);
  std::vector<uint32_t> gov(h->total_V);
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const GraphDesc &gd = h->graphs[g];
    for (uint32_t c = 0; c < gd.C; ++c) flip[gd.flip_off + c] = xxh3_flip(seeds[g] + 5ull * c);
    flip[gd.flip_off + gd.C] = xxh3_flip(seeds[g]);
    std::fill(gov.begin() + gd.vbase, gov.begin() + gd.vbase + gd.V, g);
  }
  if (cudaMallocHost(&h->h_small, 64) != cudaSuccess) return bail(mb_fail(GZ_ERR_NOMEM, "cudaMallocHost"));
  e = cudaMemcpyAsync(h->d_flip, flip.data(), nflip * 8, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_gov, gov.data(), gov.size() * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_sk, 0, h->sk_bytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, 16, h->stream);
  if (e != cudaSuccess) return bail(mb_fail(GZ_ERR_CUDA, cudaGetErrorString(e)));
  if ((rc = upload_tables(h))) return bail(rc);
  *out = h;
  return GZ_OK;
}

int gz_batch_destroy(gz_batch_t *h) {
  if (!h) return GZ_OK;
  cudaSetDevice(h->device);
  batch_destroy(h);
  delete h;
  return GZ_OK;
}

int gz_batch_get_params(gz_batch_t *h, uint32_t graph, gz_params_t *o) {
  if (!h || !o || graph >= h->G) return mb_fail(GZ_ERR_INVALID, "bad argument");
  const GraphDesc &gd = h->graphs[graph];
  std::memset(o, 0, sizeof(*o));
  o->num_vertices = gd.V;
  o->num_columns = gd.C;
  o->bkt_per_col = gd.B;
  o->num_buckets = gd.C * gd.B + 1;
  o->seed = h->seeds[graph];
  o->sketch_bytes = (uint64_t)gd.sketch_words * 4;
  o->max_rounds = gd.C;
  o->sketches_factor = h->factor;
  o->batch_factor = 1;
  o->vertices_per_tile = 1u << gd.tile_shift;
  o->num_tiles = gd.ntiles;
  o->vertices_per_bin = 1u << gd.bin_shift;
  o->num_bins = gd.nbins;
  return GZ_OK;
}

int gz_batch_ingest_device(gz_batch_t *h, const void *d_records, const uint64_t *offsets) {
  if (!h || !offsets) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  return batch_ingest(h, d_records, offsets);
}

int gz_batch_ingest(gz_batch_t *h, const void *records, const uint64_t *offsets) {
  if (!h || !offsets || (!records && offsets[h->G] > offsets[0]))
    return mb_fail(GZ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  const uint64_t n = offsets[h->G];
  if (n == 0) return GZ_OK;
  if (h->rec_cap < n * 9) {
    mb_free(h->d_rec);
    h->rec_cap = 0;
    MB_TRY(mb_alloc(&h->d_rec, n * 9));
    h->rec_cap = n * 9;
  }
  MB_CUDA(cudaMemcpyAsync(h->d_rec, records, n * 9, cudaMemcpyHostToDevice, h->stream));
  return batch_ingest(h, h->d_rec, offsets);
}

int gz_batch_clear(gz_batch_t *h) {
  if (!h) return mb_fail(GZ_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  MB_CUDA(cudaMemsetAsync(h->d_sk, 0, h->sk_bytes, h->stream));
  MB_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int gz_batch_connected_components(gz_batch_t *h, uint32_t *labels_out, uint32_t *num_cc,
                                  uint32_t *rounds, int *status) {
  if (!h) return mb_fail(GZ_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  MB_TRY(batch_query(h, labels_out));
  for (uint32_t g = 0; g < h->G; ++g) {
    if (num_cc) num_cc[g] = h->ncc[g];
    if (rounds) rounds[g] = h->rounds[g];
    if (status) status[g] = (int)h->status[g];
  }
  return GZ_OK;
}

int gz_batch_dump_sketches(gz_batch_t *h, uint32_t graph, void *host_buf, size_t bytes) {
  if (!h || !host_buf || graph >= h->G) return mb_fail(GZ_ERR_INVALID, "bad argument");
  const GraphDesc &gd = h->graphs[graph];
  if (bytes != (uint64_t)gd.V * gd.sketch_words * 4) return mb_fail(GZ_ERR_INVALID, "buffer must hold V * sketch_bytes");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  MB_CUDA(cudaMemcpyAsync(host_buf, h->d_sk + gd.sk_off, bytes, cudaMemcpyDeviceToHost, h->stream));
  MB_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int gz_batch_load_sketches(gz_batch_t *h, uint32_t graph, const void *host_buf, size_t bytes) {
  if (!h || !host_buf || graph >= h->G) return mb_fail(GZ_ERR_INVALID, "bad argument");
  const GraphDesc &gd = h->graphs[graph];
  if (bytes != (uint64_t)gd.V * gd.sketch_words * 4) return mb_fail(GZ_ERR_INVALID, "buffer must hold V * sketch_bytes");
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  MB_CUDA(cudaMemcpyAsync(h->d_sk + gd.sk_off, host_buf, bytes, cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaStreamSynchronize(h->stream));
  return GZ_OK;
}

int gz_batch_set_profiling(gz_batch_t *h, int enable) {
  if (!h) return mb_fail(GZ_ERR_INVALID, "null handle");
  h->prof = enable != 0;
  h->prof_gutter_ms = h->prof_sketch_ms = h->prof_query_ms = 0;
  h->prof_rounds = 0;
  return GZ_OK;
}

int gz_batch_get_profile(gz_batch_t *h, gz_profile_t *out) {
  if (!h || !out) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::memset(out, 0, sizeof(*out));
  out->gutter_ms = h->prof_gutter_ms;
  out->sketch_update_ms = h->prof_sketch_ms;
  out->query_ms = h->prof_query_ms;
  out->query_rounds = h->prof_rounds;
  out->kernel_launches = h->launches;
  return GZ_OK;
}

}  // extern "C"
