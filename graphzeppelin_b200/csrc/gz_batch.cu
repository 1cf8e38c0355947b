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
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
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
  uint32_t direct_max;  // tiles with fewer entries are updated in place in HBM, unstaged
};

// ---- gutter ----------------------------------------------------------------------------------
// The records of each graph are cut into record tiles of at most kMbRecTile records; a record
// tile {graph, first record (lo, hi), count} belongs to one graph, so its endpoint entries land in
// that graph's gutter bins only (at most kMbBinsMax of them).
constexpr uint32_t kMbRecTile = 4096;
constexpr uint32_t kMbSpan = 32;  // grouped members merged per Boruvka merge warp
constexpr uint32_t kMbBinsMax = 4096;
constexpr uint32_t kMbTilesPerBinMax = 64;
constexpr uint32_t kMbBinTarget = 4096;  // bins per graph aimed for with at most 16 tiles per bin

// Counting pass: per record tile, a shared-memory histogram over the graph's bins, added to the
// global bin counts once per non-empty bin.
__global__ void __launch_bounds__(1024)
k_mb_count(const uint8_t *__restrict__ rec, const uint4 *__restrict__ rtiles, uint32_t n_rt,
           const GraphDesc *__restrict__ graphs, uint64_t *__restrict__ bins,
           uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) uint8_t bsm[];
  uint32_t *s_bin = reinterpret_cast<uint32_t *>(bsm);
  uint8_t *s_rec = bsm + kMbBinsMax * 4;
  bool bad = false;
  for (uint32_t t = blockIdx.x; t < n_rt; t += gridDim.x) {
    const uint4 rt = rtiles[t];
    const GraphDesc gd = graphs[rt.x];
    for (uint32_t b = threadIdx.x; b < gd.nbins; b += blockDim.x) s_bin[b] = 0u;
    const uint32_t shift = stage_records(rec, ((uint64_t)rt.z << 32) | rt.y, rt.w, s_rec);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < rt.w; i += blockDim.x) {
      uint32_t u, v;
      parse_record(s_rec, shift, i, u, v);
      if (u >= gd.V || v >= gd.V) {
        bad = true;
        continue;
      }
      atomicAdd(&s_bin[u >> gd.bin_shift], 1u);
      atomicAdd(&s_bin[v >> gd.bin_shift], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < gd.nbins; b += blockDim.x)
      if (s_bin[b])
        atomicAdd(reinterpret_cast<unsigned long long *>(bins + gd.bin_base + b),
                  (unsigned long long)s_bin[b]);
    __syncthreads();
  }
  if (bad) atomicOr(status, kStatusBadVertex);
}

// Sort-scatter pass: per record tile, counting-sort its endpoint entries by bin in shared memory,
// reserve one run per non-empty bin in the bin's gutter region (one global atomic per tile and
// bin), and write the runs out with consecutive threads on consecutive addresses.
// base[b] = first slot of global bin b (scanned counts), fill[b] = slots taken so far.
__global__ void __launch_bounds__(1024, 1)
k_mb_sort_scatter(const uint8_t *__restrict__ rec, const uint4 *__restrict__ rtiles, uint32_t n_rt,
                  const GraphDesc *__restrict__ graphs, const uint64_t *__restrict__ base,
                  uint32_t *__restrict__ fill, uint2 *__restrict__ entries) {
  extern __shared__ __align__(16) uint8_t bsm[];
  __shared__ uint32_t ws[32];
  uint32_t *s_cur = reinterpret_cast<uint32_t *>(bsm);  // counts, then placement cursors
  uint32_t *s_off = s_cur + kMbBinsMax;                  // run start inside the tile
  uint32_t *s_dst = s_off + kMbBinsMax;                  // run start inside the gutter
  uint2 *s_sorted = reinterpret_cast<uint2 *>(s_dst + kMbBinsMax);
  uint8_t *s_rec = reinterpret_cast<uint8_t *>(s_sorted + 2 * kMbRecTile);
  for (uint32_t t = blockIdx.x; t < n_rt; t += gridDim.x) {
    const uint4 rt = rtiles[t];
    const GraphDesc gd = graphs[rt.x];
    const uint32_t nb = gd.nbins, cnt = rt.w;
    const uint32_t per_thread = (nb + blockDim.x - 1) / blockDim.x;  // <= 4
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s_cur[b] = 0u;
    const uint32_t shift = stage_records(rec, ((uint64_t)rt.z << 32) | rt.y, cnt, s_rec);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
      uint32_t u, v;
      parse_record(s_rec, shift, i, u, v);
      if (u >= gd.V || v >= gd.V) continue;
      atomicAdd(&s_cur[u >> gd.bin_shift], 1u);
      atomicAdd(&s_cur[v >> gd.bin_shift], 1u);
    }
    __syncthreads();
    uint32_t local[4] = {0, 0, 0, 0}, sum = 0;
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      local[k] = b < nb ? s_cur[b] : 0u;
      sum += local[k];
    }
    uint32_t run = block_scan_1024(sum, ws);
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      if (b < nb) {
        const uint32_t gb = gd.bin_base + b;
        s_off[b] = run;
        s_dst[b] = local[k] ? (uint32_t)base[gb] + atomicAdd(&fill[gb], local[k]) : 0u;
        s_cur[b] = run;
      }
      run += local[k];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
      uint32_t u, v;
      parse_record(s_rec, shift, i, u, v);
      if (u >= gd.V || v >= gd.V) continue;
      s_sorted[atomicAdd(&s_cur[u >> gd.bin_shift], 1u)] = make_uint2(u, v);
      s_sorted[atomicAdd(&s_cur[v >> gd.bin_shift], 1u)] = make_uint2(v, u);
    }
    __syncthreads();
    const uint32_t total = s_cur[nb - 1];
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
      const uint2 x = s_sorted[j];
      const uint32_t b = x.x >> gd.bin_shift;
      entries[s_dst[b] + (j - s_off[b])] = x;
    }
    __syncthreads();
  }
}

constexpr size_t kMbCountSmem = kMbBinsMax * 4 + kMbRecTile * 9 + 48;
constexpr size_t kMbSortSmem = 3 * kMbBinsMax * 4 + 2 * kMbRecTile * 8 + kMbRecTile * 9 + 48;

__global__ void k_mb_bin_off(const uint64_t *scanned, uint64_t nbins, const uint64_t *total,
                             uint32_t *bin_off) {
  const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b < nbins) bin_off[b] = (uint32_t)scanned[b];
  if (b == nbins) bin_off[b] = (uint32_t)*total;
}

// ---- sparse route: records applied in place ---------------------------------------------------
// For a graph whose call brings too few records to pay for the gutter and tile staging, each
// record is hashed once (checksum and C depths, shared by both endpoints) and XORed into both
// endpoints' sketches in HBM with global atomics. A self-loop XORs one sketch twice: no change,
// as in the gutter path.
constexpr uint32_t kMbFlipMax = 64;

__global__ void __launch_bounds__(512)
k_mb_direct(const uint8_t *__restrict__ rec, const uint4 *__restrict__ rtiles, uint32_t n_rt,
            const GraphDesc *__restrict__ graphs, uint8_t *__restrict__ sketches,
            const uint64_t *__restrict__ flip, uint32_t *__restrict__ status) {
  extern __shared__ __align__(128) uint8_t dsm[];
  uint64_t *s_flip = reinterpret_cast<uint64_t *>(dsm);
  uint8_t *s_rec = dsm + kMbFlipMax * 8;
  bool bad = false;
  for (uint32_t t = blockIdx.x; t < n_rt; t += gridDim.x) {
    const uint4 rt = rtiles[t];
    const GraphDesc gd = graphs[rt.x];
    for (uint32_t i = threadIdx.x; i <= gd.C; i += blockDim.x) s_flip[i] = flip[gd.flip_off + i];
    const uint32_t shift = stage_records(rec, ((uint64_t)rt.z << 32) | rt.y, rt.w, s_rec);
    __syncthreads();
    uint32_t *gsk = reinterpret_cast<uint32_t *>(sketches + gd.sk_off);
    const uint64_t flip_chk = s_flip[gd.C];
    for (uint32_t i = threadIdx.x; i < rt.w; i += blockDim.x) {
      uint32_t u, v;
      parse_record(s_rec, shift, i, u, v);
      if (u >= gd.V || v >= gd.V) {
        bad = true;
        continue;
      }
      if (u == v) continue;
      const uint32_t lo = max(u, v), hi = min(u, v);
      const uint64_t in64 = ((uint64_t)lo << 32) | hi;
      const uint32_t chk = hash_lo32(in64 ^ flip_chk);
      uint32_t *su = gsk + (uint64_t)u * gd.sketch_words;
      uint32_t *sv = gsk + (uint64_t)v * gd.sketch_words;
      const uint32_t det = 3 * gd.C * gd.B;
      xor_bucket(su + det, lo, hi, chk);
      xor_bucket(sv + det, lo, hi, chk);
      for (uint32_t c = 0; c < gd.C; ++c) {
        const uint32_t d = hash_depth(in64 ^ s_flip[c], gd.B);
        if (d < gd.B) {
          const uint32_t o = 3 * (c * gd.B + d);
          xor_bucket(su + o, lo, hi, chk);
          xor_bucket(sv + o, lo, hi, chk);
        }
      }
    }
    __syncthreads();
  }
  if (bad) atomicOr(status, kStatusBadVertex);
}

constexpr size_t kMbDirectSmem = kMbFlipMax * 8 + kMbRecTile * 9 + 48;

// Work list of the tile kernel: the global tiles whose gutter bin holds entries.
__global__ void k_mb_worklist(const GraphDesc *__restrict__ graphs, const uint32_t *__restrict__ tile_graph,
                              uint32_t total_tiles, const uint32_t *__restrict__ bin_off,
                              uint32_t *__restrict__ list, uint32_t *__restrict__ count) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  bool take = false;
  if (t < total_tiles) {
    const GraphDesc gd = graphs[tile_graph[t]];
    const uint32_t bin = gd.bin_base + ((t - gd.tile_base) >> (gd.bin_shift - gd.tile_shift));
    take = bin_off[bin + 1] > bin_off[bin];
  }
  const uint32_t m = __ballot_sync(kFull, take);
  uint32_t base = 0;
  if ((threadIdx.x & 31) == 0 && m) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(kFull, base, 0);
  if (take) list[base + __popc(m & ((1u << (threadIdx.x & 31)) - 1u))] = t;
}

// ---- sketch update -------------------------------------------------------------------------------
// One persistent launch over the (graph, tile) items of every graph, warp-specialised: lane 0 of
// the last warp is the producer -- it claims items from a device work counter, bulk-loads each
// tile and its graph's hash constants into one of two buffers, and writes finished tiles back;
// the other warps consume, XORing the tile's gutter entries into the staged buckets. Buffers
// are handed over with mbarriers (full: tile landed; empty: every consumer thread is done), so
// claiming, loading and writing back overlap the hashing of the other buffer and no CTA-wide
// barrier ever waits on the producer.
struct MbSlot {
  uint32_t item, b, e, lt;                 // work item, entry range of its bin, tile in graph
  uint32_t C, B, words, tile_shift, bin_shift;
  uint32_t direct;                         // apply in place in HBM (no staged tile)
  uint64_t sk_off;                         // the graph's sketches
};

__global__ void __launch_bounds__(1024, 1)
k_mb_sketch_update(const GraphDesc *__restrict__ graphs, const uint32_t *__restrict__ tile_graph,
                   const uint32_t *__restrict__ worklist, const uint32_t *__restrict__ worklist_len,
                   uint8_t *__restrict__ sketches,
                   const uint2 *__restrict__ entries, const uint32_t *__restrict__ bin_off,
                   const uint64_t *__restrict__ flip, uint32_t tile_stride, uint32_t flip_stride,
                   uint32_t *work_counter, uint32_t *status) {
  extern __shared__ __align__(128) uint8_t dsm[];
  __shared__ __align__(8) uint64_t s_full[2], s_empty[2];
  __shared__ MbSlot s_slot[2];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ncw = (blockDim.x >> 5) - 1;  // consumer warps
  const uint32_t total_tiles = *worklist_len;  // items; item k is global tile worklist[k]
  const uint32_t nct = ncw * 32;               // consumer threads
  uint8_t *s_flipb = dsm + 2 * tile_stride;    // 2 x flip_stride bytes
  uint32_t *s_queue = reinterpret_cast<uint32_t *>(s_flipb + 2 * flip_stride);
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&s_full[0]), 1);
    mbar_init(smem_u32(&s_full[1]), 1);
    mbar_init(smem_u32(&s_empty[0]), nct);
    mbar_init(smem_u32(&s_empty[1]), nct);
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == ncw) {  // ---------------- producer ----------------
    if (lane != 0) return;
    // claim the next item: its slot, and where its tile and hash constants live
    struct Claim {
      MbSlot m;
      const uint8_t *src;
      const uint64_t *fsrc;
      uint32_t bytes, fbytes;
    };
    auto claim = [&]() {
      Claim c;
      c.m.item = atomicAdd(work_counter, 1u);
      c.m.b = c.m.e = 0;
      c.bytes = c.fbytes = 0;
      c.src = nullptr;
      c.fsrc = nullptr;
      if (c.m.item < total_tiles) {
        const uint32_t tile = worklist[c.m.item];
        const GraphDesc gd = graphs[tile_graph[tile]];
        c.m.lt = tile - gd.tile_base;
        c.m.C = gd.C;
        c.m.B = gd.B;
        c.m.words = gd.sketch_words;
        c.m.tile_shift = gd.tile_shift;
        c.m.bin_shift = gd.bin_shift;
        const uint32_t bin = gd.bin_base + (c.m.lt >> (gd.bin_shift - gd.tile_shift));
        c.m.b = bin_off[bin];
        c.m.e = bin_off[bin + 1];
        c.m.sk_off = gd.sk_off;
        // a bin shared by several tiles is staged (its entries are filtered per tile)
        c.m.direct = gd.bin_shift == gd.tile_shift && c.m.e - c.m.b < gd.direct_max;
        if (c.m.e > c.m.b) {
          c.fbytes = ((gd.C + 2) & ~1u) * 8;
          c.fsrc = flip + gd.flip_off;
          if (!c.m.direct) {
            c.bytes = (gd.sketch_words * 4) << gd.tile_shift;
            c.src = sketches + gd.sk_off + (uint64_t)c.m.lt * c.bytes;
          }
        }
      }
      return c;
    };
    uint8_t *pdst[2] = {nullptr, nullptr};
    uint32_t pbytes[2] = {0, 0};
    uint32_t issued = 0;         // bit s: a load into buffer s was issued
    uint32_t lastk[2] = {0, 0};  // item index k of the last load into buffer s
    uint32_t k = 0;
    bool ok = true;
    Claim c = claim();
    for (;; ++k) {
      const uint32_t s = k & 1;
      if (k >= 2) {  // consumers must be done with tile k - 2 (same buffer) before reuse
        if (!mbar_wait_bounded(smem_u32(&s_empty[s]), ((k - 2) >> 1) & 1, kWaitLimitNs)) {
          ok = false;
          break;
        }
        if (pbytes[s]) {
          for (uint32_t off = 0; off < pbytes[s]; off += kBulkPiece)
            bulk_s2g(pdst[s] + off, smem_u32(dsm + s * tile_stride) + off, min(kBulkPiece, pbytes[s] - off));
          bulk_commit();
          bulk_wait_read_all();
        }
      }
      const uint32_t full = smem_u32(&s_full[s]);
      s_slot[s] = c.m;
      pbytes[s] = c.bytes;
      pdst[s] = const_cast<uint8_t *>(c.src);
      if (c.fbytes) {  // entries to apply: the hash constants, and the tile unless in place
        const uint32_t dst = smem_u32(dsm + s * tile_stride);
        mbar_expect_tx(full, c.bytes + c.fbytes);
        for (uint32_t off = 0; off < c.bytes; off += kBulkPiece)
          bulk_g2s(dst + off, c.src + off, min(kBulkPiece, c.bytes - off), full);
        bulk_g2s(smem_u32(s_flipb + s * flip_stride), c.fsrc, c.fbytes, full);
        issued |= 1u << s;
        lastk[s] = k;
      } else {
        mbar_arrive(full);  // nothing to apply, or end of work: hand the slot over at once
      }
      if (c.m.item >= total_tiles) break;
      c = claim();  // the next item's lookups overlap this tile's load
    }
    if (ok && k >= 1) {  // write back the last tile
      const uint32_t s = (k - 1) & 1;
      ok = mbar_wait_bounded(smem_u32(&s_empty[s]), ((k - 1) >> 1) & 1, kWaitLimitNs);
      if (ok && pbytes[s]) {
        for (uint32_t off = 0; off < pbytes[s]; off += kBulkPiece)
          bulk_s2g(pdst[s] + off, smem_u32(dsm + s * tile_stride) + off, min(kBulkPiece, pbytes[s] - off));
        bulk_commit();
      }
    }
    if (!ok) {
      atomicOr(status, kStatusTimeout);
      // every load issued must land before the CTA's shared memory goes away
      for (uint32_t s = 0; s < 2; ++s)
        if (issued & (1u << s)) mbar_wait_bounded(smem_u32(&s_full[s]), (lastk[s] >> 1) & 1, kWaitLimitNs);
    }
    bulk_wait_all();
    return;
  }

  // ---------------- consumers ----------------
  const uint32_t ct = threadIdx.x;  // consumer thread index (warps 0 .. ncw - 1)
  uint32_t *q = s_queue + warp * 64;
  for (uint32_t k = 0;; ++k) {
    const uint32_t s = k & 1;
    if (!mbar_wait_bounded(smem_u32(&s_full[s]), (k >> 1) & 1, kWaitLimitNs)) {
      if (lane == 0) atomicOr(status, kStatusTimeout);
      return;
    }
    const MbSlot m = s_slot[s];
    if (m.item >= total_tiles) return;
    if (m.e > m.b) {
      uint32_t *s_sk = reinterpret_cast<uint32_t *>(dsm + s * tile_stride);
      const uint64_t *s_flip = reinterpret_cast<const uint64_t *>(s_flipb + s * flip_stride);
      const uint32_t vmask = (1u << m.tile_shift) - 1;
      const uint64_t flip_chk = s_flip[m.C];
      if (m.direct) {
        uint32_t *gsk = reinterpret_cast<uint32_t *>(sketches + m.sk_off);
        for (uint32_t i = m.b + ct; i < m.e; i += nct)
          apply_entry_global(entries[i], gsk, m.words, s_flip, flip_chk, m.C, m.B);
      } else if (m.bin_shift == m.tile_shift) {
        // every entry of the bin is this tile's; the next entry's load is in flight while the
        // current one is hashed
        uint32_t i = m.b + ct;
        uint2 cur = i < m.e ? entries[i] : make_uint2(0, 0);
        for (; i < m.e; i += nct) {
          const uint2 e = cur;
          if (i + nct < m.e) cur = entries[i + nct];
          apply_entry(e, s_sk, vmask, m.words, s_flip, flip_chk, m.C, m.B);
        }
      } else {
        uint32_t qn = 0;
        for (uint32_t i0 = m.b + warp * 32; i0 < m.e; i0 += nct) {
          const uint32_t i = i0 + lane;
          const bool mine = i < m.e && (entries[i].x >> m.tile_shift) == m.lt;
          const uint32_t bal = __ballot_sync(0xffffffffu, mine);
          if (mine) q[qn + __popc(bal & ((1u << lane) - 1u))] = i;
          qn += __popc(bal);
          __syncwarp();
          if (qn >= 32) {
            apply_entry(entries[q[lane]], s_sk, vmask, m.words, s_flip, flip_chk, m.C, m.B);
            __syncwarp();
            qn -= 32;
            if (lane < qn) q[lane] = q[32 + lane];
            __syncwarp();
          }
        }
        if (lane < qn) apply_entry(entries[q[lane]], s_sk, vmask, m.words, s_flip, flip_chk, m.C, m.B);
        __syncwarp();
      }
      fence_proxy_async_smem();  // this thread's bucket writes, before the bulk write-back
    }
    mbar_arrive(smem_u32(&s_empty[s]));
  }
}

// ---- batched Boruvka -------------------------------------------------------------------------------
struct MBBufs {
  const GraphDesc *graphs;
  const uint32_t *gov;  // graph of each global vertex
  const uint8_t *sketches;
  const uint64_t *flip;
  uint32_t *parent, *label, *cnt, *fill;
  uint64_t *packed, *scan_total;
  uint32_t *order, *order_comp, *comp_start, *ncomp, *acc;
  uint32_t *part, *part_comp;  // per merge warp: its XOR when one component covers its span
  // sample results of the round, per vertex (round 0) or per component (rounds >= 1): the
  // sampled edge, or kResZero / kResFail; res_g = the component's graph
  uint64_t *res;
  uint32_t *res_g;
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

constexpr uint64_t kResZero = ~0ull, kResFail = ~0ull - 1;  // never an edge index (min < max)
__device__ __forceinline__ uint64_t res_code(int res, uint64_t idx) {
  return res == 0 ? idx : res == 2 ? kResFail : kResZero;
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

// Per-lane view of one vertex's graph for the query kernels: where its sketch lives and the
// sizes of its sample regions. Each lane loads the descriptor of its own vertex; a warp then
// hands them round with shuffles, one vertex at a time.
struct MbVert {
  const uint32_t *sk;  // the vertex's sketch (words)
  uint32_t g, B, det;  // graph, buckets per column, word offset of the deterministic bucket
  uint64_t chk;        // the graph's checksum flip
};
__device__ __forceinline__ MbVert mb_vert(const MBBufs &b, uint32_t v) {
  MbVert m;
  m.g = b.gov[v];
  const GraphDesc gd = b.graphs[m.g];
  m.sk = mb_sketch(b, gd, v);
  m.B = gd.B;
  m.det = 3 * gd.C * gd.B;
  m.chk = b.flip[gd.flip_off + gd.C];
  return m;
}
__device__ __forceinline__ MbVert mb_vert_shfl(const MbVert &m, uint32_t src) {
  MbVert o;
  o.sk = reinterpret_cast<const uint32_t *>(__shfl_sync(kFull, reinterpret_cast<unsigned long long>(m.sk), src));
  o.g = __shfl_sync(kFull, m.g, src);
  o.B = __shfl_sync(kFull, m.B, src);
  o.det = __shfl_sync(kFull, m.det, src);
  o.chk = __shfl_sync(kFull, (unsigned long long)m.chk, src);
  return o;
}

constexpr int kMbKB = 8;  // members per cp.async batch
// dynamic shared memory of a 256-thread query block: per warp two batches of kMbKB member slots
// and one stage, each slot acc_words (the largest graph's sample region + its deterministic
// bucket)
inline size_t mb_query_smem(uint32_t acc_words) { return 8 * (size_t)bv_warp_bytes(acc_words - 3, kMbKB); }

// Round 0 for every active graph (run_round_zero, src/cc_sketch_alg.cpp:223-244): a warp takes
// 32 consecutive global vertices, copies their sample-0 regions to shared memory with cp.async
// in batches of kMbKB (one batch ahead), samples each there, and the 32 lanes then apply their
// vertex's result together.
__global__ void __launch_bounds__(256) k_mb_round0(MBBufs b) {
  extern __shared__ __align__(16) uint8_t mb_smem[];
  const uint32_t lane = threadIdx.x & 31;
  BvRing ring;
  ring.init(mb_smem + (threadIdx.x >> 5) * bv_warp_bytes(b.acc_words - 3, kMbKB), b.acc_words - 3, kMbKB);
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t tb = 0;  // batches this warp ran before the current group (the ring's phases go on)
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < b.total_V;
       base += nwarps * 32) {
    const uint32_t n = b.total_V - base < 32 ? b.total_V - base : 32;
    MbVert me{};
    bool my_act = false;
    if (lane < n) {
      me = mb_vert(b, base + lane);
      my_act = b.active[me.g] != 0;
    }
    const uint32_t act = __ballot_sync(kFull, my_act);
    // batch t of this group: lane k < kMbKB copies vertex t * kMbKB + k
    auto issue = [&](uint32_t t) {
      const uint32_t m = t * kMbKB + lane;
      const MbVert mk = mb_vert_shfl(me, m & 31);
      const bool mine = lane < (uint32_t)kMbKB && m < n && (act >> m & 1);
      ring.issue(tb + t, mine, mk.sk, 3 * mk.B, mk.sk + mk.det, kMbKB);
    };
    int my_res = 1;
    uint64_t my_idx = 0;
    const uint32_t nb = (n + kMbKB - 1) / kMbKB;
    issue(0);
    bool ok = true;
    for (uint32_t t = 0; t < nb && ok; ++t) {
      if (t + 1 < nb) issue(t + 1);
      if (!ring.wait(tb + t)) {
        if (lane == 0) atomicOr(b.status, kStatusTimeout);
        if (t + 1 < nb) ring.wait(tb + t + 1);  // its copies must land before shared memory goes away
        ok = false;
        break;
      }
#pragma unroll 1
      for (int k = 0; k < kMbKB; ++k) {
        const uint32_t m = t * kMbKB + k;
        if (m >= n) break;
        if (!(act >> m & 1)) continue;
        const MbVert mk = mb_vert_shfl(me, m);
        const uint8_t *sl = ring.slot(tb + t, k, kMbKB);
        uint64_t idx;
        const int res = warp_sample_smem_split<1>(bulk_run_at(sl, mk.sk), bulk_run_at(sl + ring.run_cap, mk.sk + mk.det),
                                                  mk.B, mk.chk, &idx);
        if (lane == m) {
          my_res = res;
          my_idx = idx;
        }
      }
      __syncwarp();
    }
    if (!ok) return;
    tb += nb;
    if (lane < n) b.res[base + lane] = my_act ? res_code(my_res, my_idx) : kResZero;
    __syncwarp();
  }
}

// Roots and members per root of the active graphs' vertices (one atomic per root per warp).
__global__ void __launch_bounds__(256) k_mb_label(MBBufs b) {
  __shared__ uint32_t s_r0;
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = v < b.total_V;
  const bool ok = in && b.active[b.gov[v]];
  uint32_t r = 0xffffffffu;
  if (ok) {
    r = dsu_find(b.parent, v);
    b.label[v] = r;
    // full path compression (no union runs during the labelling)
    if (__ldcg(b.parent + v) != r) __stcg(b.parent + v, r);
  }
  if (threadIdx.x == 0) s_r0 = r;
  __syncthreads();
  // every in-range vertex of the block active and under one root: one counter add for all
  if (__syncthreads_and(!in || (ok && r == s_r0))) {
    if (threadIdx.x == 0 && ok) {
      const uint32_t nin = b.total_V - blockIdx.x * blockDim.x < blockDim.x ? b.total_V - blockIdx.x * blockDim.x : blockDim.x;
      atomicAdd(&b.cnt[r], nin);
    }
    return;
  }
  const uint32_t act = __ballot_sync(kFull, ok);
  if (!ok) return;
  const uint32_t peers = __match_any_sync(act, r);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&b.cnt[r], (uint32_t)__popc(peers));
}

__global__ void k_mb_pack(MBBufs b) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= b.total_V) return;
  const uint32_t c = b.cnt[v];
  b.packed[v] = (uint64_t)c | (c ? (1ull << 32) : 0ull);
}

__global__ void __launch_bounds__(256) k_mb_group(MBBufs b) {
  __shared__ uint32_t stage[8][32];
  __shared__ uint32_t s_r0, s_base;
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v == 0) {
    const uint32_t nc = (uint32_t)(*b.scan_total >> 32), members = (uint32_t)*b.scan_total;
    b.comp_start[nc] = members;
    *b.ncomp = nc;
  }
  const bool in = v < b.total_V;
  const bool ok = in && b.active[b.gov[v]];
  const uint32_t r = ok ? b.label[v] : 0xffffffffu;
  if (threadIdx.x == 0) s_r0 = r;
  __syncthreads();
  uint32_t slot;
  if (__syncthreads_and(!in || (ok && r == s_r0))) {
    // every in-range vertex of the block active and under one root: one cursor claim
    if (threadIdx.x == 0 && ok) {
      const uint32_t nin = b.total_V - blockIdx.x * blockDim.x < blockDim.x ? b.total_V - blockIdx.x * blockDim.x : blockDim.x;
      s_base = atomicAdd(&b.fill[r], nin);
    }
    __syncthreads();
    if (!ok) return;
    slot = s_base + threadIdx.x;
  } else {
    const uint32_t act = __ballot_sync(kFull, ok);
    if (!ok) return;
    slot = warp_agg_inc(b.fill, r, act, stage[threadIdx.x >> 5]);
  }
  const uint64_t s = b.packed[r];
  const uint32_t start = (uint32_t)s, c = (uint32_t)(s >> 32);
  const uint32_t pos = start + slot;
  b.order[pos] = v;
  b.order_comp[pos] = c;
  if (v == r) {
    b.comp_start[c] = start;
    const uint32_t end = start + b.cnt[r];
    if (start / b.span != (end - 1) / b.span) {
      uint32_t *ac = b.acc + (uint64_t)(start / b.span) * b.acc_words;
      for (uint32_t i = 0; i < b.acc_words; ++i) ac[i] = 0;
    }
  }
}

// Round >= 1 merge (perform_boruvka_round, src/cc_sketch_alg.cpp:246-380) over the grouped
// members of every active graph: a warp takes kMbSpan consecutive members, copies column
// `round` of each (its graph's B buckets) and the deterministic bucket to shared memory with
// cp.async, one batch ahead, and XORs them in registers. A component wholly inside the span is
// sampled here (the results applied 32 at a time by the lanes); a component covering the whole
// span leaves the warp's XOR in its partial slot (folded by k_mb_reduce_parts); the parts of
// components crossing a span edge go to acc with one atomicXor per word.
__global__ void __launch_bounds__(256) k_mb_merge(MBBufs b) {
  constexpr int NW = Region<1>::kNW;
  extern __shared__ __align__(16) uint8_t mb_smem[];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t SW = b.acc_words;
  BvRing ring;
  ring.init(mb_smem + (threadIdx.x >> 5) * bv_warp_bytes(SW - 3, kMbKB), SW - 3, kMbKB);
  uint32_t *st = ring.stage;
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nc = *b.ncomp;
  const uint32_t members = b.comp_start[nc];
  const uint64_t p0 = (uint64_t)w * kMbSpan;
  if (p0 >= members) {  // past the active graphs' members: this slot holds nothing this round
    if (lane == 0) b.part_comp[w] = 0xffffffffu;
    return;
  }
  const uint32_t n = members - p0 < kMbSpan ? members - (uint32_t)p0 : kMbSpan;
  const uint32_t p1 = (uint32_t)p0 + n;
  const uint32_t round = *b.round;
  MbVert me{};
  uint32_t my_c = 0;
  if (lane < n) {
    me = mb_vert(b, b.order[p0 + lane]);
    my_c = b.order_comp[p0 + lane];
  }
  // components of the positions just outside the span (members of a component are contiguous)
  uint32_t edge_c = 0xffffffffu;
  if (lane == 0 && p0 > 0) edge_c = b.order_comp[p0 - 1];
  if (lane == 1 && p1 < members) edge_c = b.order_comp[p1];
  const uint32_t prev_c = __shfl_sync(kFull, edge_c, 0), next_c = __shfl_sync(kFull, edge_c, 1);
  // batch t: lane k < kMbKB copies member t * kMbKB + k
  auto issue = [&](uint32_t t) {
    const uint32_t m = t * kMbKB + lane;
    const MbVert mk = mb_vert_shfl(me, m & 31);
    const bool mine = lane < (uint32_t)kMbKB && m < n;
    ring.issue(t, mine, mk.sk + 3 * round * mk.B, 3 * mk.B, mk.sk + mk.det, kMbKB);
  };
  issue(0);
  uint32_t acc[NW], dacc = 0;
#pragma unroll
  for (int k = 0; k < NW; ++k) acc[k] = 0;
  uint32_t cur = 0xffffffffu;
  MbVert cm{};  // a member of the current component (its graph's geometry)
  bool whole = false;
  auto flush = [&]() {
    const bool before = cur == prev_c, after = cur == next_c;
    const uint32_t W = 3 * cm.B;
    if (!before && !after) {
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W) st[wi] = acc[k];
      }
      if (lane < 3) st[W + lane] = dacc;
      __syncwarp();
      uint64_t idx;
      const int res = warp_sample_smem<1>(st, W, cm.B, cm.chk, &idx);
      __syncwarp();
      if (lane == 0) {
        b.res[cur] = res_code(res, idx);
        b.res_g[cur] = cm.g;
      }
    } else if (before && after) {
      uint32_t *pt = b.part + (uint64_t)w * SW;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W) pt[wi] = acc[k];
      }
      if (lane < 3) pt[W + lane] = dacc;
      if (lane == 0) b.part_comp[w] = cur;
      whole = true;
    } else {
      // a component crossing a span edge owns acc slot (its first position / span)
      const uint32_t slot = before ? b.comp_start[cur] / kMbSpan : w;
      uint32_t *ac = b.acc + (uint64_t)slot * SW;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W && acc[k]) atomicXor(ac + wi, acc[k]);
      }
      if (lane < 3 && dacc) atomicXor(ac + W + lane, dacc);
    }
  };
  const uint32_t nb = (n + kMbKB - 1) / kMbKB;
  for (uint32_t t = 0; t < nb; ++t) {
    if (t + 1 < nb) issue(t + 1);
    if (!ring.wait(t)) {
      if (lane == 0) atomicOr(b.status, kStatusTimeout);
      if (t + 1 < nb) ring.wait(t + 1);  // its copies must land before shared memory goes away
      return;
    }
    // not unrolled: one copy of the flush keeps the kernel small for the instruction cache
#pragma unroll 1
    for (int k = 0; k < kMbKB; ++k) {
      const uint32_t m = t * kMbKB + k;
      if (m >= n) break;
      const uint32_t c = __shfl_sync(kFull, my_c, m);
      const MbVert mk = mb_vert_shfl(me, m);
      if (c != cur) {
        if (cur != 0xffffffffu) flush();
        cur = c;
        cm = mk;
#pragma unroll
        for (int q = 0; q < NW; ++q) acc[q] = 0;
        dacc = 0;
      }
      const uint32_t W = 3 * cm.B;
      const uint8_t *slt = ring.slot(t, k, kMbKB);
      const uint32_t *sl = bulk_run_at(slt, mk.sk + 3 * round * mk.B);
      const uint32_t *sd = bulk_run_at(slt + ring.run_cap, mk.sk + mk.det);
#pragma unroll
      for (int q = 0; q < NW; ++q) {
        const uint32_t wi = q * 32 + lane;
        if (wi < W) acc[q] ^= sl[wi];
      }
      if (lane < 3) dacc ^= sd[lane];
    }
    __syncwarp();
  }
  flush();
  if (!whole && lane == 0) b.part_comp[w] = 0xffffffffu;
}

// Folds the partial slots of merge warps covered by one component into its acc: one warp per
// 32 consecutive slots, one atomicXor per word per component per warp. Slots are folded whole
// (acc_words): a smaller graph's slot tail lands in its acc's unused tail.
__global__ void __launch_bounds__(256) k_mb_reduce_parts(MBBufs b, uint32_t nslots) {
  constexpr int NW = Region<1>::kNW;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
  if (s0 >= nslots) return;
  const uint32_t n = nslots - s0 < 32 ? nslots - s0 : 32;
  const uint32_t SW = b.acc_words, W = SW - 3;
  const uint32_t my_c = lane < n ? b.part_comp[s0 + lane] : 0xffffffffu;
  uint32_t live = __ballot_sync(kFull, my_c != 0xffffffffu);
  if (!live) return;
  uint32_t acc[NW], dacc = 0, cur = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < NW; ++k) acc[k] = 0;
  auto flush = [&]() {
    uint32_t *ac = b.acc + (uint64_t)(b.comp_start[cur] / kMbSpan) * SW;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const uint32_t wi = k * 32 + lane;
      if (wi < W && acc[k]) atomicXor(ac + wi, acc[k]);
    }
    if (lane < 3 && dacc) atomicXor(ac + W + lane, dacc);
  };
  while (live) {
    constexpr int KB = 4;
    uint32_t x[KB][NW], dw[KB], sl[KB];
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      sl[k] = live ? __ffs(live) - 1 : 32u;
      if (live) live &= live - 1;
      if (sl[k] < 32) {
        const uint32_t *pt = b.part + (uint64_t)(s0 + sl[k]) * SW;
        region_load(pt, pt + W, W, lane, x[k], dw[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      if (sl[k] >= 32) break;
      const uint32_t c = __shfl_sync(kFull, my_c, sl[k]);
      if (c != cur) {
        if (cur != 0xffffffffu) flush();
        cur = c;
#pragma unroll
        for (int q = 0; q < NW; ++q) acc[q] = 0;
        dacc = 0;
      }
#pragma unroll
      for (int q = 0; q < NW; ++q) acc[q] ^= x[k][q];
      dacc ^= dw[k];
    }
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
    const uint32_t *ac = b.acc + (uint64_t)(s / b.span) * b.acc_words;
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
    if (lane == 0) {
      b.res[c] = res_code(res, idx);
      b.res_g[c] = g;
    }
  }
}

// sample_supernode (src/cc_sketch_alg.cpp:137-166) for every result of the round: n results
// (all vertices in round 0, else the components), visited transposed -- lane l of a warp takes
// result l * ceil(n / 32) + warp -- so that the lanes of one warp work on distant components
// (other graphs, mostly) rather than on neighbours that would race for one root's CAS.
__global__ void k_mb_unite(MBBufs b, int round0) {
  const uint32_t n = round0 ? b.total_V : *b.ncomp;
  const uint32_t q = (n + 31) / 32;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 32ull * q) return;
  const uint64_t i64 = (t & 31) * (uint64_t)q + (t >> 5);
  if (i64 >= n) return;
  const uint32_t i = (uint32_t)i64;
  const uint64_t r = b.res[i];
  if (r == kResZero) return;
  const uint32_t g = round0 ? b.gov[i] : b.res_g[i];
  mb_handle(r == kResFail ? 2 : 0, r, g, b.graphs[g], b);
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

// Stream-ordered reallocation of scratch that grows while the engine runs: cudaFree would wait
// for the whole device (every request in flight, on every stream); cudaFreeAsync/cudaMallocAsync
// only order against the engine's own stream. The device's default pool keeps freed memory
// (release threshold raised once per process), so regrowth does not go back to the driver.
template <class T>
int mb_realloc_async(T **p, size_t count, cudaStream_t s) {
  static std::once_flag keep;
  std::call_once(keep, [] {
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep_all = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    }
  });
  if (*p) cudaFreeAsync(*p, s);
  *p = nullptr;
  void *q = nullptr;
  cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(count, 1) * sizeof(T), s);
  if (e != cudaSuccess) return mb_fail(GZ_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  *p = static_cast<T *>(q);
  return GZ_OK;
}

// graph g owns global tiles [tile_base, +ntiles) and global vertices [vbase, +V)
__global__ void k_mb_fill_tables(const GraphDesc *graphs, uint32_t G, uint32_t *tile_graph, uint32_t *gov) {
  for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
    const GraphDesc gd = graphs[g];
    for (uint32_t i = threadIdx.x; i < gd.ntiles; i += blockDim.x) tile_graph[gd.tile_base + i] = g;
    for (uint32_t i = threadIdx.x; i < gd.V; i += blockDim.x) gov[gd.vbase + i] = g;
  }
}

// ---- autotuning trials -----------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Trial records: record r of graph g (records off[g] .. off[g+1]) joins two distinct vertices
// drawn uniformly from [0, nv[g]) by a counter-based hash.
__global__ void k_trial_records(uint8_t *out, const uint64_t *off, const uint32_t *nv, uint32_t G,
                                uint64_t seed) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= off[G]) return;
  uint32_t lo = 0, hi = G;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= r) lo = mid;
    else hi = mid;
  }
  const uint32_t n = nv[lo];
  const uint64_t h = splitmix64(seed ^ (r * 0xD1B54A32D192ED03ull));
  const uint32_t u = (uint32_t)(((h & 0xffffffffull) * n) >> 32);
  uint32_t v = (uint32_t)(((h >> 32) * (n - 1)) >> 32);
  if (v >= u) ++v;
  uint8_t *p = out + 9 * r;
  p[0] = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p[1 + k] = (uint8_t)(u >> (8 * k));
    p[5 + k] = (uint8_t)(v >> (8 * k));
  }
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
  uint32_t max_B = 0, max_C = 0, max_tile_bytes = 0;
  uint32_t threads = 1024, ctas_per_sm = 1;  // sketch-update CTA shape
  std::vector<uint32_t> vpt_req;             // requested vertices per tile (0 = default)
  bool own_storage = true;                   // d_sk / d_flip allocated (and freed) by this handle
  double sparse_factor = 1.0;                // scales the sparse-route threshold (0 = never)
  uint32_t *d_worklist = nullptr, *d_wl_len = nullptr;
  uint64_t cap_worklist = 0;
  // capacities of the device tables (grown, never shrunk)
  uint64_t cap_graphs = 0, cap_tiles = 0, cap_V = 0, cap_bins = 0;
  uint64_t cap_bv_V = 0, cap_bv_G = 0, cap_acc = 0;
  gz::MBBufs captured{};    // buffers the captured Boruvka round was recorded with
  gz::MBBufs last_query{};  // buffers of the previous query
  GraphDesc *d_graphs = nullptr;
  uint32_t *d_tile_graph = nullptr, *d_gov = nullptr;  // graph of each global tile / vertex
  uint8_t *d_sk = nullptr;
  uint64_t *d_flip = nullptr;
  uint32_t *d_status = nullptr, *h_small = nullptr;
  // gutter
  uint2 *d_entries = nullptr;
  uint64_t entry_cap = 0;
  uint64_t *d_bins = nullptr, *d_scan_tmp = nullptr, *d_total = nullptr;
  uint32_t *d_bin_fill = nullptr;  // per-bin slots taken by the sort-scatter pass
  uint32_t *d_bin_off = nullptr;
  uint4 *d_rtiles = nullptr;
  size_t rtiles_cap = 0;
  uint8_t *d_rec = nullptr;  // device copy of host records (gz_batch_ingest)
  uint64_t rec_cap = 0;
  // Boruvka
  uint32_t *d_parent = nullptr, *d_label = nullptr, *d_cnt = nullptr, *d_fill = nullptr;
  uint64_t *d_packed = nullptr, *d_vscan_total = nullptr, *d_vscan_tmp = nullptr;
  uint32_t *d_part = nullptr, *d_part_comp = nullptr;
  uint64_t cap_part = 0, cap_part_comp = 0;
  uint64_t *d_res = nullptr;
  uint32_t *d_res_g = nullptr;
  uint64_t cap_res = 0, cap_res_g = 0;
  uint32_t *d_order = nullptr, *d_order_comp = nullptr, *d_comp_start = nullptr, *d_ncomp = nullptr, *d_acc = nullptr;
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
    b.order_comp = d_order_comp;
    b.part = d_part;
    b.part_comp = d_part_comp;
    b.res = d_res;
    b.res_g = d_res_g;
    b.comp_start = d_comp_start;
    b.ncomp = d_ncomp;
    b.acc = d_acc;
    b.active = d_active;
    b.modified = d_modified;
    b.round = d_round;
    b.status = d_status;
    b.total_V = (uint32_t)total_V;
    b.acc_words = (max_B + 1) * 3;
    b.span = gz::kMbSpan;
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
  mb_free(h->d_tile_graph);
  mb_free(h->d_gov);
  if (h->own_storage) {
    mb_free(h->d_sk);
    mb_free(h->d_flip);
  }
  mb_free(h->d_status);
  if (h->h_small) cudaFreeHost(h->h_small);
  mb_free(h->d_entries);
  mb_free(h->d_bins);
  mb_free(h->d_bin_fill);
  mb_free(h->d_scan_tmp);
  mb_free(h->d_total);
  mb_free(h->d_bin_off);
  mb_free(h->d_rtiles);
  mb_free(h->d_rec);
  mb_free(h->d_worklist);
  mb_free(h->d_wl_len);
  mb_free(h->d_parent);
  mb_free(h->d_label);
  mb_free(h->d_cnt);
  mb_free(h->d_fill);
  mb_free(h->d_packed);
  mb_free(h->d_vscan_total);
  mb_free(h->d_vscan_tmp);
  mb_free(h->d_order);
  mb_free(h->d_order_comp);
  mb_free(h->d_part);
  mb_free(h->d_part_comp);
  mb_free(h->d_res);
  mb_free(h->d_res_g);
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
// Shared memory one sketch-update CTA may use when ctas_per_sm of them share an SM.
size_t cta_smem_budget(const gz_batch *h) {
  int optin = 0, per_sm = 0, reserved = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->device);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, h->device);
  if (optin <= 0) optin = 227 * 1024;
  if (per_sm <= 0) per_sm = 228 * 1024;
  const size_t share = (size_t)per_sm / h->ctas_per_sm - (size_t)std::max(reserved, 0);
  return std::min<size_t>((size_t)optin, share);
}

// Bytes of one tile buffer when the launch's graphs have at most max_C columns: two buffers, two
// padded hash-constant arrays, the consumer warps' queues and static shared memory share the CTA.
size_t tile_budget(const gz_batch *h, uint32_t max_C) {
  const size_t cta_smem = cta_smem_budget(h);
  const size_t fixed = 256 + (size_t)(h->threads / 32) * 256 + 2 * (size_t)((max_C + 2) & ~1u) * 8;
  if (cta_smem <= fixed) return 0;
  return ((cta_smem - fixed) / 2) & ~(size_t)127;
}

// Tile and bin geometry of one graph. A requested vertices-per-tile (vpt != 0) is used as given;
// otherwise the largest power of two <= 64 whose tile fits `budget` bytes (a batch has enough
// tiles to fill the GPU, and bigger tiles spread the shared-memory atomics over more buckets).
int choose_tiles(GraphDesc &gd, uint32_t vpt, size_t budget) {
  const uint64_t sketch_bytes = (uint64_t)gd.sketch_words * 4;
  uint32_t shift = 2;
  if (vpt) {
    shift = (uint32_t)__builtin_ctz(vpt);
  } else {
    while (shift < 6 && (sketch_bytes << (shift + 1)) <= budget) ++shift;
  }
  if ((sketch_bytes << shift) > budget) return mb_fail(GZ_ERR_INVALID, "sketch too large for a tile");
  uint32_t bshift = shift;
  while (((gd.V + (1u << bshift) - 1) >> bshift) > kMbBinTarget && (1u << (bshift - shift)) < 16) ++bshift;
  while (((gd.V + (1u << bshift) - 1) >> bshift) > kMbBinsMax && (1u << (bshift - shift)) < kMbTilesPerBinMax)
    ++bshift;
  if (((gd.V + (1u << bshift) - 1) >> bshift) > kMbBinsMax)
    return mb_fail(GZ_ERR_INVALID, "a graph with V=" + std::to_string(gd.V) +
                                       " is too large for a batch: use a single-graph handle");
  gd.tile_shift = shift;
  gd.bin_shift = bshift;
  gd.ntiles = (gd.V + (1u << shift) - 1) >> shift;
  gd.nbins = (gd.V + (1u << bshift) - 1) >> bshift;
  // Staging a tile moves 2 x tile bytes over HBM; updating in place moves about one 32-byte
  // sector read and written per bucket, C + 1 buckets per entry: in place wins below this.
  gd.direct_max = (uint32_t)((sketch_bytes << shift) / (32ull * (gd.C + 1)));
  return GZ_OK;
}

// Device bytes of one graph's sketches: V rounded up to 64 (any tile stays inside), 256-aligned.
uint64_t graph_sketch_bytes(const GraphDesc &gd) {
  const uint64_t v_pad = ((uint64_t)gd.V + 63) & ~63ull;
  return (v_pad * gd.sketch_words * 4 + 255) & ~255ull;
}

// Scratch grows by at least half its size each time it is outgrown: a server whose calls vary in
// size reallocates (a device-wide synchronisation, and a latency spike for every request in
// flight) a few times while warming up instead of on every larger call.
inline uint64_t headroom(uint64_t cap, uint64_t need) {
  return need <= cap ? cap : std::max<uint64_t>(need, cap + cap / 2);
}

template <class T>
int grow(T **p, uint64_t &cap, uint64_t need, cudaStream_t s) {
  if (*p && cap >= need) return GZ_OK;
  const uint64_t n = headroom(cap, need);
  cap = 0;
  MB_TRY(mb_realloc_async(p, std::max<uint64_t>(n, 1), s));
  cap = n;
  return GZ_OK;
}

// h->graphs hold tiling, sketch and hash-constant offsets: number their tiles, bins and vertices
// globally, size the device tables for them and upload them.
int finalize_graphs(gz_batch *h) {
  uint64_t vbase = 0, bin_base = 0, tile_base = 0;
  h->G = (uint32_t)h->graphs.size();
  h->max_tile_bytes = 0;
  h->max_B = h->max_C = 0;
  for (GraphDesc &gd : h->graphs) {
    gd.vbase = (uint32_t)vbase;
    gd.bin_base = (uint32_t)bin_base;
    gd.tile_base = (uint32_t)tile_base;
    vbase += gd.V;
    bin_base += gd.nbins;
    tile_base += gd.ntiles;
    h->max_B = std::max(h->max_B, gd.B);
    h->max_C = std::max(h->max_C, gd.C);
    h->max_tile_bytes = std::max<uint32_t>(h->max_tile_bytes, (gd.sketch_words * 4) << gd.tile_shift);
  }
  if (vbase > 0xFFFFFFF0ull || bin_base > 0xFFFFFFF0ull || tile_base > 0xFFFFFFF0ull)
    return mb_fail(GZ_ERR_INVALID, "batch too large for 32-bit global vertex ids");
  h->total_V = vbase;
  h->total_bins = bin_base;
  h->total_tiles = tile_base;
  if (h->G == 0) return GZ_OK;
  MB_TRY(grow(&h->d_graphs, h->cap_graphs, h->G, h->stream));
  MB_TRY(grow(&h->d_tile_graph, h->cap_tiles, h->total_tiles, h->stream));
  MB_TRY(grow(&h->d_gov, h->cap_V, h->total_V, h->stream));
  if (!h->d_bins || h->cap_bins < h->total_bins) {
    const uint64_t nb = headroom(h->cap_bins, h->total_bins);
    h->cap_bins = 0;
    MB_TRY(mb_realloc_async(&h->d_bins, nb, h->stream));
    MB_TRY(mb_realloc_async(&h->d_bin_fill, nb, h->stream));
    MB_TRY(mb_realloc_async(&h->d_scan_tmp, scan_tmp_words(nb), h->stream));
    MB_TRY(mb_realloc_async(&h->d_bin_off, nb + 1, h->stream));
    h->cap_bins = nb;
  }
  MB_CUDA(cudaMemcpyAsync(h->d_graphs, h->graphs.data(), sizeof(GraphDesc) * h->G, cudaMemcpyHostToDevice, h->stream));
  k_mb_fill_tables<<<std::min<uint32_t>(h->G, 4096), 256, 0, h->stream>>>(h->d_graphs, h->G, h->d_tile_graph, h->d_gov);
  h->launches++;
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(h->stream));  // the host descriptor vector may change next call
  return GZ_OK;
}

// Layout of a batch that owns its storage: every graph's tiling, then its sketches and hash
// constants back to back.
int layout(gz_batch *h, const std::vector<uint32_t> &vpt_req) {
  uint32_t max_C = 0;
  for (const GraphDesc &gd : h->graphs) max_C = std::max(max_C, gd.C);
  const size_t budget = tile_budget(h, max_C);
  if (!budget) return mb_fail(GZ_ERR_INVALID, "no shared memory left for a tile");
  uint64_t sk_off = 0, flip_off = 0;
  for (uint32_t g = 0; g < h->graphs.size(); ++g) {
    GraphDesc &gd = h->graphs[g];
    MB_TRY(choose_tiles(gd, vpt_req.empty() ? 0 : vpt_req[g], budget));
    gd.sk_off = sk_off;
    gd.flip_off = (uint32_t)flip_off;
    sk_off += graph_sketch_bytes(gd);
    flip_off += (gd.C + 2) & ~1u;  // even: every graph's constants start 16-byte aligned
  }
  h->sk_bytes = sk_off;
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

// Whether graph gd takes n records of one call in place (sparse route): staging its touched
// tiles moves about 2 x V x sketch bytes over HBM plus the gutter's bytes, updating in place
// about 2 (C + 1) bucket sectors of 64 B read + written per record.
bool route_sparse(const gz_batch *h, const GraphDesc &gd, uint64_t n) {
  const double staged = 2.0 * gd.V * (gd.sketch_words * 4.0) + 50.0 * n;
  const double in_place = 128.0 * (gd.C + 1) * (double)n;
  return in_place < staged * h->sparse_factor;
}

// records of graph g are d_rec[off[g] .. off[g+1]) (9-byte records)
int batch_ingest(gz_batch *h, const void *d_rec, const uint64_t *off) {
  std::vector<uint4> rt_dense, rt_sparse;
  uint64_t n_dense = 0;
  for (uint32_t g = 0; g < h->G; ++g) {
    if (off[g + 1] < off[g]) return mb_fail(GZ_ERR_INVALID, "record offsets must be non-decreasing");
    const uint64_t n = off[g + 1] - off[g];
    if (!n) continue;
    const bool sparse = route_sparse(h, h->graphs[g], n);
    auto &rt = sparse ? rt_sparse : rt_dense;
    for (uint64_t s = off[g]; s < off[g + 1]; s += kMbRecTile) {
      const uint32_t cnt = (uint32_t)std::min<uint64_t>(kMbRecTile, off[g + 1] - s);
      rt.push_back(make_uint4(g, (uint32_t)s, (uint32_t)(s >> 32), cnt));
    }
    if (!sparse) n_dense += n;
  }
  if (rt_dense.empty() && rt_sparse.empty()) return GZ_OK;
  if (2 * n_dense >= 0xFFFFFFF0ull) return mb_fail(GZ_ERR_INVALID, "more than 2^31 records in one batch ingest");
  const size_t n_rt = rt_dense.size() + rt_sparse.size();
  MB_TRY(grow(&h->d_rtiles, h->rtiles_cap, n_rt, h->stream));
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
  if (h->prof) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, h->stream);
  }
  rt_dense.insert(rt_dense.end(), rt_sparse.begin(), rt_sparse.end());
  MB_CUDA(cudaMemcpyAsync(h->d_rtiles, rt_dense.data(), sizeof(uint4) * n_rt, cudaMemcpyHostToDevice, h->stream));
  const uint32_t n_rt_dense = (uint32_t)(n_rt - rt_sparse.size());
  const uint8_t *rec = static_cast<const uint8_t *>(d_rec);
  if (n_rt_dense) {
    MB_TRY(grow(&h->d_entries, h->entry_cap, 2 * n_dense, h->stream));
    MB_TRY(grow(&h->d_worklist, h->cap_worklist, h->total_tiles, h->stream));
    MB_TRY(mb_alloc(&h->d_wl_len, 1));
    MB_CUDA(cudaMemsetAsync(h->d_bins, 0, sizeof(uint64_t) * h->total_bins, h->stream));
    MB_CUDA(cudaMemsetAsync(h->d_bin_fill, 0, sizeof(uint32_t) * h->total_bins, h->stream));
    MB_CUDA(cudaMemsetAsync(h->d_wl_len, 0, sizeof(uint32_t), h->stream));
    {
      MB_CUDA(smem_optin(k_mb_count));
      int per_sm = 1;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mb_count, 1024, kMbCountSmem);
      const unsigned grid = (unsigned)std::min<uint64_t>(n_rt_dense, (uint64_t)num_sms() * std::max(per_sm, 1));
      k_mb_count<<<grid, 1024, kMbCountSmem, h->stream>>>(rec, h->d_rtiles, n_rt_dense, h->d_graphs, h->d_bins,
                                                         h->d_status);
      h->launches++;
      MB_CUDA(cudaGetLastError());
    }
    const uint64_t l0 = launch_count();
    MB_CUDA(scan_exclusive_u64(h->d_bins, h->total_bins, h->d_total, h->d_scan_tmp, h->stream));
    h->launches += launch_count() - l0;
    k_mb_bin_off<<<cdiv(h->total_bins + 1, 256), 256, 0, h->stream>>>(h->d_bins, h->total_bins, h->d_total,
                                                                       h->d_bin_off);
    h->launches++;
    {
      MB_CUDA(smem_optin(k_mb_sort_scatter));
      const unsigned grid = (unsigned)std::min<uint64_t>(n_rt_dense, (uint64_t)num_sms());
      k_mb_sort_scatter<<<grid, 1024, kMbSortSmem, h->stream>>>(rec, h->d_rtiles, n_rt_dense, h->d_graphs,
                                                                h->d_bins, h->d_bin_fill, h->d_entries);
      h->launches++;
      MB_CUDA(cudaGetLastError());
    }
    k_mb_worklist<<<cdiv(h->total_tiles, 256), 256, 0, h->stream>>>(
        h->d_graphs, h->d_tile_graph, (uint32_t)h->total_tiles, h->d_bin_off, h->d_worklist, h->d_wl_len);
    h->launches++;
    MB_CUDA(cudaGetLastError());
  }
  if (h->prof) cudaEventRecord(e1, h->stream);
  if (n_rt_dense) {
    // one persistent launch over every non-empty tile
    MB_CUDA(cudaMemsetAsync(h->d_status + 1, 0, sizeof(uint32_t), h->stream));
    const uint32_t tile_stride = (h->max_tile_bytes + 127) & ~127u;
    const uint32_t flip_stride = ((h->max_C + 2) & ~1u) * 8;
    const size_t ksmem = 2 * (size_t)tile_stride + 2 * (size_t)flip_stride + (size_t)(h->threads / 32) * 256;
    MB_CUDA(smem_optin(k_mb_sketch_update));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mb_sketch_update, (int)h->threads, ksmem);
    const int grid = (int)std::min<uint64_t>(h->total_tiles, (uint64_t)num_sms() * std::max(per_sm, 1));
    k_mb_sketch_update<<<grid, h->threads, ksmem, h->stream>>>(
        h->d_graphs, h->d_tile_graph, h->d_worklist, h->d_wl_len, h->d_sk, h->d_entries, h->d_bin_off,
        h->d_flip, tile_stride, flip_stride, h->d_status + 1, h->d_status);
    h->launches++;
    MB_CUDA(cudaGetLastError());
  }
  if (!rt_sparse.empty()) {
    MB_CUDA(smem_optin(k_mb_direct));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mb_direct, 512, kMbDirectSmem);
    const unsigned grid = (unsigned)std::min<uint64_t>(rt_sparse.size(), (uint64_t)num_sms() * std::max(per_sm, 1));
    k_mb_direct<<<grid, 512, kMbDirectSmem, h->stream>>>(rec, h->d_rtiles + n_rt_dense, (uint32_t)rt_sparse.size(),
                                                         h->d_graphs, h->d_sk, h->d_flip, h->d_status);
    h->launches++;
    MB_CUDA(cudaGetLastError());
  }
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
  const uint64_t V = h->total_V, G = h->G;
  if (!h->d_parent || h->cap_bv_V < V) {
    const uint64_t Vn = headroom(h->cap_bv_V, V);
    h->cap_bv_V = 0;
    MB_TRY(mb_realloc_async(&h->d_parent, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_label, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_cnt, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_fill, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_packed, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_vscan_tmp, scan_tmp_words(Vn), h->stream));
    MB_TRY(mb_realloc_async(&h->d_order, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_order_comp, Vn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_comp_start, Vn + 1, h->stream));
    h->cap_bv_V = Vn;
  }
  const uint64_t slots = (V + kMbSpan - 1) / kMbSpan;
  MB_TRY(grow(&h->d_acc, h->cap_acc, (slots + 1) * (uint64_t)(h->max_B + 1) * 3, h->stream));
  MB_TRY(grow(&h->d_part, h->cap_part, slots * (uint64_t)(h->max_B + 1) * 3, h->stream));
  MB_TRY(grow(&h->d_part_comp, h->cap_part_comp, slots, h->stream));
  MB_TRY(grow(&h->d_res, h->cap_res, V, h->stream));
  MB_TRY(grow(&h->d_res_g, h->cap_res_g, V, h->stream));
  if (!h->d_active || h->cap_bv_G < G) {
    const uint64_t Gn = headroom(h->cap_bv_G, G);
    h->cap_bv_G = 0;
    MB_TRY(mb_realloc_async(&h->d_active, Gn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_modified, Gn, h->stream));
    MB_TRY(mb_realloc_async(&h->d_ncc, Gn, h->stream));
    h->cap_bv_G = Gn;
  }
  MB_TRY(mb_alloc(&h->d_vscan_total, 1));
  MB_TRY(mb_alloc(&h->d_ncomp, 1));
  MB_TRY(mb_alloc(&h->d_round, 1));
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
  const uint64_t warps = (V + kMbSpan - 1) / kMbSpan;
  const size_t smem = mb_query_smem(b.acc_words);
  MB_CUDA(smem_optin(k_mb_merge));
  k_mb_merge<<<cdiv(warps * 32, 256), 256, smem, s>>>(b);
  k_mb_reduce_parts<<<cdiv(warps, 256), 256, 0, s>>>(b, (uint32_t)warps);
  k_mb_sample_spanning<<<std::min<unsigned>(cdiv(V * 32, 256), num_sms() * 16), 256, 0, s>>>(b);
  k_mb_unite<<<cdiv(32 * ((V + 31) / 32), 256), 256, 0, s>>>(b, 0);
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
  {
    const size_t smem = mb_query_smem(b.acc_words);
    MB_CUDA(smem_optin(k_mb_round0));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mb_round0, 256, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    k_mb_round0<<<std::min<unsigned>(cdiv(V, 256), num_sms() * per_sm), 256, smem, h->stream>>>(b);
    k_mb_unite<<<cdiv(32 * ((V + 31) / 32), 256), 256, 0, h->stream>>>(b, 1);
    h->launches++;
  }
  h->launches += 2;
  MB_CUDA(cudaGetLastError());
  // The round runs as a captured CUDA graph once the same graphs and buffers come back (a batch
  // queried repeatedly); a one-off set of graphs (a server query job) launches it directly
  // rather than paying for a capture it would use once.
  const MBBufs cur = h->bufs();
  const bool same_as_capture = h->round_exec && std::memcmp(&cur, &h->captured, sizeof(MBBufs)) == 0;
  const bool seen_before = std::memcmp(&cur, &h->last_query, sizeof(MBBufs)) == 0;
  h->last_query = cur;
  if (h->round_exec && !same_as_capture) {
    cudaGraphExecDestroy(h->round_exec);  // the graphs or buffers changed since the capture
    cudaGraphDestroy(h->round_graph);
    h->round_exec = nullptr;
    h->round_graph = nullptr;
  }
  const bool use_graph = same_as_capture || seen_before;
  if (use_graph && !h->round_exec) {
    // capture the round: it reads the round number and the active flags from device memory
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
    h->captured = cur;
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
    if (use_graph) {
      MB_CUDA(cudaGraphLaunch(h->round_exec, h->stream));
      h->launches += h->round_kernels;
    } else {
      const uint64_t l0 = launch_count();
      MB_TRY(enqueue_round(h, h->stream));
      h->launches += 7 + (launch_count() - l0);  // label, pack, group, merge, reduce, sample, unite
    }
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
  if (vertices_per_tile) h->vpt_req.assign(vertices_per_tile, vertices_per_tile + num_graphs);
  int rc = layout(h, h->vpt_req);
  if (rc != GZ_OK) return bail(rc);
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(mb_fail(GZ_ERR_CUDA, cudaGetErrorString(e)));
  if ((rc = mb_alloc(&h->d_sk, h->sk_bytes + kSketchTail)) || (rc = mb_alloc(&h->d_status, 4)) ||
      (rc = mb_alloc(&h->d_total, 1)))
    return bail(rc);
  uint64_t nflip = 0;
  for (auto &gd : h->graphs) nflip += (gd.C + 2) & ~1u;
  if ((rc = mb_alloc(&h->d_flip, nflip))) return bail(rc);
  std::vector<uint64_t> flip(nflip);
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const GraphDesc &gd = h->graphs[g];
    for (uint32_t c = 0; c < gd.C; ++c) flip[gd.flip_off + c] = xxh3_flip(seeds[g] + 5ull * c);
    flip[gd.flip_off + gd.C] = xxh3_flip(seeds[g]);
  }
  if (cudaMallocHost(&h->h_small, 64) != cudaSuccess) return bail(mb_fail(GZ_ERR_NOMEM, "cudaMallocHost"));
  e = cudaMemcpyAsync(h->d_flip, flip.data(), nflip * 8, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_sk, 0, h->sk_bytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, 16, h->stream);
  if (e != cudaSuccess) return bail(mb_fail(GZ_ERR_CUDA, cudaGetErrorString(e)));
  if ((rc = finalize_graphs(h))) return bail(rc);
  *out = h;
  return GZ_OK;
}

int gz_batch_set_tuning(gz_batch_t *h, uint32_t threads_per_block, uint32_t ctas_per_sm,
                        const uint32_t *vertices_per_tile) {
  if (!h) return mb_fail(GZ_ERR_INVALID, "null handle");
  const uint32_t threads = threads_per_block ? threads_per_block : 1024;
  const uint32_t ctas = ctas_per_sm ? ctas_per_sm : 1;
  if (threads < 64 || threads > 1024 || threads % 32)
    return mb_fail(GZ_ERR_INVALID, "threads_per_block must be a multiple of 32 in [64, 1024]");
  if (ctas > 4 || threads * ctas > 2048)
    return mb_fail(GZ_ERR_INVALID, "ctas_per_sm must be in [1, 4] with threads * ctas <= 2048");
  if (vertices_per_tile)
    for (uint32_t g = 0; g < h->G; ++g) {
      const uint32_t v = vertices_per_tile[g];
      if (v && (v < 4 || v > 64 || (v & (v - 1))))
        return mb_fail(GZ_ERR_INVALID, "vertices_per_tile must be 0 or a power of two in [4, 64]");
    }
  std::lock_guard<std::mutex> lk(h->mtx);
  cudaSetDevice(h->device);
  MB_CUDA(cudaStreamSynchronize(h->stream));
  const uint32_t old_threads = h->threads, old_ctas = h->ctas_per_sm;
  const std::vector<uint32_t> old_vpt = h->vpt_req;
  h->threads = threads;
  h->ctas_per_sm = ctas;
  if (vertices_per_tile) h->vpt_req.assign(vertices_per_tile, vertices_per_tile + h->G);
  else h->vpt_req.clear();
  int rc = layout(h, h->vpt_req);
  if (rc != GZ_OK) {  // keep the previous tuning
    const std::string msg = gz_last_error();
    h->threads = old_threads;
    h->ctas_per_sm = old_ctas;
    h->vpt_req = old_vpt;
    layout(h, h->vpt_req);
    gz_internal_set_error(msg);
    return rc;
  }
  return finalize_graphs(h);
}

int gz_batch_set_route(gz_batch_t *h, double sparse_factor) {
  if (!h || !(sparse_factor >= 0)) return mb_fail(GZ_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(h->mtx);
  h->sparse_factor = sparse_factor;
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
  o->cols_per_sample = 1;
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
    const uint64_t nr = headroom(h->rec_cap, n * 9);
    h->rec_cap = 0;
    MB_TRY(mb_realloc_async(&h->d_rec, nr, h->stream));
    h->rec_cap = nr;
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

// Picks, per sketch-size class (graphs with the same columns and buckets per column), the
// vertices per tile of the batched sketch update -- i.e. the buckets each CTA stages and the warps
// per vertex -- and the CTA shape, by timing trial ingests on a scratch batch holding one
// representative graph per class. The caller's sketches are not touched.
int gz_batch_autotune(gz_batch_t *h, uint32_t records_per_vertex, uint32_t *vpt_out) {
  if (!h) return mb_fail(GZ_ERR_INVALID, "null handle");
  const uint32_t rpv = records_per_vertex ? records_per_vertex : 64;
  cudaSetDevice(h->device);
  std::vector<std::pair<uint32_t, uint32_t>> keys;  // (C, B) per class
  std::vector<uint32_t> rep_v, cls_of(h->G);
  for (uint32_t g = 0; g < h->G; ++g) {
    const auto key = std::make_pair(h->graphs[g].C, h->graphs[g].B);
    uint32_t k = 0;
    while (k < keys.size() && keys[k] != key) ++k;
    if (k == keys.size()) {
      keys.push_back(key);
      rep_v.push_back(0);
    }
    rep_v[k] = std::max(rep_v[k], h->graphs[g].V);
    cls_of[g] = k;
  }
  const uint32_t K = (uint32_t)keys.size();
  // scratch graphs: copies of each class's largest graph, enough (>= 16384 vertices, i.e. >= 4
  // tiles per SM at 16 vertices per tile) that a class's trial fills the GPU like the real batch
  std::vector<uint32_t> sv, first(K + 1, 0);
  std::vector<uint64_t> seeds;
  for (uint32_t k = 0; k < K; ++k) {
    const uint32_t copies = std::max<uint32_t>(1, std::min<uint32_t>(64, (16384 + rep_v[k] - 1) / rep_v[k]));
    first[k] = (uint32_t)sv.size();
    for (uint32_t c = 0; c < copies; ++c) {
      sv.push_back(rep_v[k]);
      seeds.push_back(0x5EEDull + sv.size());
    }
  }
  first[K] = (uint32_t)sv.size();
  const uint32_t S = (uint32_t)sv.size();
  std::vector<uint64_t> off(S + 1, 0);
  for (uint32_t g = 0; g < S; ++g)
    off[g + 1] = off[g] + std::min<uint64_t>(std::max<uint64_t>(1, (uint64_t)rpv * sv[g] / 2), 1ull << 22);
  gz_batch_t *sc = nullptr;
  MB_TRY(gz_batch_create(S, sv.data(), seeds.data(), h->factor, nullptr, &sc));
  struct Guard {
    gz_batch_t *b;
    uint8_t *rec = nullptr;
    uint64_t *off = nullptr;
    uint32_t *nv = nullptr;
    ~Guard() {
      if (rec) cudaFree(rec);
      if (off) cudaFree(off);
      if (nv) cudaFree(nv);
      gz_batch_destroy(b);
    }
  } guard{sc};
  MB_TRY(mb_alloc(&guard.rec, off[S] * 9));
  MB_TRY(mb_alloc(&guard.off, S + 1));
  MB_TRY(mb_alloc(&guard.nv, S));
  MB_CUDA(cudaMemcpyAsync(guard.off, off.data(), 8 * (S + 1), cudaMemcpyHostToDevice, sc->stream));
  MB_CUDA(cudaMemcpyAsync(guard.nv, sv.data(), 4 * S, cudaMemcpyHostToDevice, sc->stream));
  k_trial_records<<<cdiv(off[S], 256), 256, 0, sc->stream>>>(guard.rec, guard.off, guard.nv, S, 0xA070ull);
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(sc->stream));

  struct Shape {
    uint32_t threads, ctas;
  };
  const Shape shapes[] = {{1024, 1}, {768, 1}, {512, 2}};
  double best_total = 1e300;
  Shape best_shape = shapes[0];
  std::vector<uint32_t> best_vpt(K, 0);
  for (const Shape &sh : shapes) {
    double total = 0;
    std::vector<uint32_t> pick(K, 0);
    bool feasible = true;
    for (uint32_t k = 0; k < K && feasible; ++k) {
      std::vector<uint64_t> o(S + 1);  // only class k's records
      for (uint32_t g = 0; g <= S; ++g) o[g] = std::min(std::max(off[g], off[first[k]]), off[first[k + 1]]);
      double best = 1e300;
      for (uint32_t vpt = 4; vpt <= 64; vpt <<= 1) {
        std::vector<uint32_t> vv(S, 0);
        for (uint32_t g = first[k]; g < first[k + 1]; ++g) vv[g] = vpt;
        if (gz_batch_set_tuning(sc, sh.threads, sh.ctas, vv.data()) != GZ_OK) continue;
        double t = 1e300;
        for (int rep = 0; rep < 3; ++rep) {
          gz_batch_set_profiling(sc, 1);
          MB_TRY(gz_batch_ingest_device(sc, guard.rec, o.data()));
          if (rep) t = std::min(t, sc->prof_sketch_ms);
        }
        if (t < best) {
          best = t;
          pick[k] = vpt;
        }
      }
      if (!pick[k]) feasible = false;
      total += best;
    }
    if (feasible && total < best_total) {
      best_total = total;
      best_shape = sh;
      best_vpt = pick;
    }
  }
  gz_batch_set_profiling(sc, 0);
  std::vector<uint32_t> vpt(h->G);
  for (uint32_t g = 0; g < h->G; ++g) vpt[g] = best_vpt[cls_of[g]];
  MB_TRY(gz_batch_set_tuning(h, best_shape.threads, best_shape.ctas, vpt.data()));
  if (vpt_out) std::copy(vpt.begin(), vpt.end(), vpt_out);
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

// =================================================================================================
// Serving: many tenants' sketches resident in one HBM arena
// =================================================================================================
// A tenant is one CCSketchAlg (its own V and seed) admitted against a sketch-byte budget. Each
// ingest call applies update batches of any set of tenants with one batched gutter pass and one
// persistent sketch-update launch (the kernels above, with the tenants' arena offsets in the
// descriptor table). A connectivity query copies the queried tenants' sketches into a snapshot
// pool on the query stream and runs the batched Boruvka there from a worker thread, so later
// ingest calls proceed while it runs; the answer is that of the state at submission.
namespace {

constexpr uint32_t kServeFlipWords = 64;  // hash-constant slot per tenant (C <= 62)
constexpr uint32_t kServeTileC = 62;      // column count the tiling budget is reserved for
constexpr uint64_t kServeQueryMaxV = 1ull << 24;  // vertices of queued jobs merged into one run

// First-fit allocator over [0, size) in 256-byte units.
struct RangeAlloc {
  std::map<uint64_t, uint64_t> free_;  // offset -> length
  uint64_t size = 0;
  void init(uint64_t n) {
    size = n;
    free_.clear();
    if (n) free_[0] = n;
  }
  bool alloc(uint64_t n, uint64_t &off) {
    n = (n + 255) & ~255ull;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      off = it->first;
      const uint64_t rest = it->second - n;
      free_.erase(it);
      if (rest) free_[off + n] = rest;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t n) {
    n = (n + 255) & ~255ull;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct ServeTenant {
  bool alive = false;
  GraphDesc desc{};  // tiling, sketch geometry, arena offset, flip slot offset
  uint64_t seed = 0, bytes = 0;
  std::vector<uint64_t> flips;  // C + 1 hash constants, padded to even
};

struct QueryJob {
  uint64_t ticket = 0;
  std::vector<uint32_t> tenants;
  std::vector<GraphDesc> descs;  // sk_off into the snapshot pool (or the arena), flip_off into `flips`
  std::vector<uint64_t> flips;
  std::vector<std::pair<uint64_t, uint64_t>> snaps;  // snapshot regions to release
  bool live = false;  // reads the tenants' sketches in the arena (sk_off into the arena), no snapshot
  bool done = false;
  int rc = GZ_OK;
  std::string err;
  std::vector<uint32_t> labels, ncc, rounds;
  std::vector<int> status;
};

}  // namespace

struct gz_server {
  std::mutex mtx;  // tenant registry and ingest
  int device = 0;
  double factor = 1;
  uint64_t budget = 0, used = 0;
  uint8_t *arena = nullptr;
  RangeAlloc arena_alloc;
  uint64_t *d_flip = nullptr;  // kServeFlipWords per slot
  uint32_t slot_cap = 0;
  std::vector<uint32_t> free_slots;
  std::vector<ServeTenant> tenants;
  uint32_t alive = 0;
  gz_batch ingest;  // engine over the arena
  gz_batch query;   // engine over the snapshot pool
  uint64_t *d_qflip = nullptr;
  uint64_t qflip_cap = 0;
  uint8_t *d_rec = nullptr;
  uint64_t rec_cap = 0;
  // snapshots and the query worker
  uint8_t *snap = nullptr;
  RangeAlloc snap_alloc;
  std::mutex qmtx;
  std::condition_variable qcv, done_cv;
  std::deque<QueryJob *> queue;
  std::map<uint64_t, QueryJob *> jobs;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread worker;
  cudaEvent_t snap_done = nullptr;
  bool live = false;  // queries submitted now read the arena in place (gz_server_set_query_snapshot)
};

namespace {

// Blocks until no unfinished in-place query reads any of the n tenants, whose sketches may then be
// written or freed. The worker never takes s->mtx, so callers may hold it.
void serve_wait_live(gz_server *s, const uint32_t *ids, uint32_t n) {
  std::unique_lock<std::mutex> ql(s->qmtx);
  s->done_cv.wait(ql, [&] {
    for (const auto &kv : s->jobs) {
      const QueryJob *j = kv.second;
      if (!j->live || j->done) continue;
      for (uint32_t t : j->tenants)
        for (uint32_t k = 0; k < n; ++k)
          if (ids[k] == t) return false;
    }
    return true;
  });
}

// One batched Boruvka over every tenant of the given jobs (all live, or all on snapshots); each
// job gets its own tenants' slice of the answer.
int serve_run_jobs(gz_server *s, const std::vector<QueryJob *> &js) {
  gz_batch *q = &s->query;
  std::vector<uint64_t> flips;
  std::vector<GraphDesc> descs;
  for (QueryJob *j : js) {
    const uint32_t base = (uint32_t)flips.size();  // even: every job's constants stay 16-byte aligned
    flips.insert(flips.end(), j->flips.begin(), j->flips.end());
    for (GraphDesc gd : j->descs) {
      gd.flip_off += base;
      descs.push_back(gd);
    }
  }
  MB_TRY(grow(&s->d_qflip, s->qflip_cap, flips.size(), s->query.stream));
  q->d_flip = s->d_qflip;
  q->d_sk = js[0]->live ? s->arena : s->snap;
  MB_CUDA(cudaMemcpyAsync(s->d_qflip, flips.data(), 8 * flips.size(), cudaMemcpyHostToDevice, q->stream));
  q->graphs = descs;
  MB_TRY(finalize_graphs(q));
  std::vector<uint32_t> labels(q->total_V);
  MB_TRY(batch_query(q, labels.data()));
  size_t v0 = 0, g0 = 0;
  for (QueryJob *j : js) {
    size_t nv = 0;
    for (const GraphDesc &gd : j->descs) nv += gd.V;
    const size_t ng = j->descs.size();
    j->labels.assign(labels.begin() + v0, labels.begin() + v0 + nv);
    j->ncc.assign(q->ncc.begin() + g0, q->ncc.begin() + g0 + ng);
    j->rounds.assign(q->rounds.begin() + g0, q->rounds.begin() + g0 + ng);
    j->status.assign(q->status.begin() + g0, q->status.begin() + g0 + ng);
    v0 += nv;
    g0 += ng;
  }
  return GZ_OK;
}

void serve_worker(gz_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<QueryJob *> js;
    {
      std::unique_lock<std::mutex> lk(s->qmtx);
      s->qcv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->queue.empty()) return;
      // every queued job of the same kind as the first runs in one batched query: jobs that
      // arrive while one runs wait for it anyway, and one run over all their tenants costs
      // about as many rounds as the longest of them
      uint64_t nv = 0;
      while (!s->queue.empty() && s->queue.front()->live == (js.empty() ? s->queue.front()->live : js[0]->live)) {
        uint64_t v = 0;
        for (const GraphDesc &gd : s->queue.front()->descs) v += gd.V;
        if (!js.empty() && nv + v > kServeQueryMaxV) break;
        nv += v;
        js.push_back(s->queue.front());
        s->queue.pop_front();
      }
    }
    const int rc = serve_run_jobs(s, js);
    const std::string err = rc != GZ_OK ? std::string(gz_last_error()) : std::string();
    {
      std::lock_guard<std::mutex> lk(s->qmtx);
      for (QueryJob *j : js) {
        j->rc = rc;
        j->err = err;
        for (auto &r : j->snaps) s->snap_alloc.release(r.first, r.second);
        j->done = true;
      }
    }
    s->done_cv.notify_all();
  }
}

void serve_destroy(gz_server *s) {
  {
    std::lock_guard<std::mutex> lk(s->qmtx);
    s->stop = true;
  }
  s->qcv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto &kv : s->jobs) delete kv.second;
  s->jobs.clear();
  s->ingest.d_sk = nullptr;
  s->query.d_sk = nullptr;
  batch_destroy(&s->ingest);
  batch_destroy(&s->query);
  if (s->snap_done) cudaEventDestroy(s->snap_done);
  mb_free(s->arena);
  mb_free(s->snap);
  mb_free(s->d_flip);
  mb_free(s->d_qflip);
  mb_free(s->d_rec);
}

int serve_engine_init(gz_server *s, gz_batch *e, uint8_t *storage, bool urgent) {
  e->device = s->device;
  e->factor = s->factor;
  e->own_storage = false;
  e->d_sk = storage;
  int least = 0, greatest = 0;
  MB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  MB_CUDA(cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, urgent ? greatest : least));
  MB_TRY(mb_alloc(&e->d_status, 4));
  MB_TRY(mb_alloc(&e->d_total, 1));
  MB_CUDA(cudaMemsetAsync(e->d_status, 0, 16, e->stream));
  if (cudaMallocHost(&e->h_small, 64) != cudaSuccess) return mb_fail(GZ_ERR_NOMEM, "cudaMallocHost");
  return GZ_OK;
}

int serve_check_tenants(gz_server *s, uint32_t n, const uint32_t *ids) {
  std::vector<uint32_t> seen(ids, ids + n);
  std::sort(seen.begin(), seen.end());
  for (uint32_t i = 0; i < n; ++i) {
    if (ids[i] >= s->tenants.size() || !s->tenants[ids[i]].alive)
      return mb_fail(GZ_ERR_INVALID, "tenant " + std::to_string(ids[i]) + " is not admitted");
    if (i && seen[i] == seen[i - 1]) return mb_fail(GZ_ERR_INVALID, "a tenant is listed twice");
  }
  return GZ_OK;
}

}  // namespace

extern "C" {

int gz_server_tenant_bytes(uint32_t num_vertices, double sketches_factor, uint64_t *bytes) {
  if (!bytes || num_vertices < 2) return mb_fail(GZ_ERR_INVALID, "bad argument");
  GraphDesc gd{};
  gd.V = num_vertices;
  sketch_sizing(num_vertices, sketches_factor > 0 ? sketches_factor : 1, gd.C, gd.B);
  gd.sketch_words = (gd.C * gd.B + 1) * 3;
  *bytes = graph_sketch_bytes(gd);
  return GZ_OK;
}

int gz_server_create(uint64_t budget_bytes, uint64_t snapshot_bytes, double sketches_factor,
                     gz_server_t **out) {
  if (!out || budget_bytes < 256 || snapshot_bytes < 256) return mb_fail(GZ_ERR_INVALID, "bad argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return mb_fail(GZ_ERR_NO_DEVICE, "no CUDA device");
  gz_server *s = new gz_server();
  auto bail = [&](int rc) {
    serve_destroy(s);
    delete s;
    return rc;
  };
  cudaGetDevice(&s->device);
  s->factor = sketches_factor > 0 ? sketches_factor : 1;
  s->budget = (budget_bytes + 255) & ~255ull;
  int rc;
  if ((rc = mb_alloc(&s->arena, s->budget + kSketchTail)) ||
      (rc = mb_alloc(&s->snap, ((snapshot_bytes + 255) & ~255ull) + kSketchTail)))
    return bail(rc);
  s->arena_alloc.init(s->budget);
  s->snap_alloc.init((snapshot_bytes + 255) & ~255ull);
  // the query stream has the greatest priority: its kernels take SMs ahead of queued ingest blocks
  if ((rc = serve_engine_init(s, &s->ingest, s->arena, false)) || (rc = serve_engine_init(s, &s->query, s->snap, true)))
    return bail(rc);
  if (cudaEventCreateWithFlags(&s->snap_done, cudaEventDisableTiming) != cudaSuccess)
    return bail(mb_fail(GZ_ERR_CUDA, "cudaEventCreate"));
  s->worker = std::thread(serve_worker, s);
  *out = s;
  return GZ_OK;
}

int gz_server_destroy(gz_server_t *s) {
  if (!s) return GZ_OK;
  cudaSetDevice(s->device);
  serve_destroy(s);
  delete s;
  return GZ_OK;
}

int gz_server_admit(gz_server_t *s, uint32_t num_vertices, uint64_t seed, uint32_t *tenant_out) {
  if (!s || !tenant_out) return mb_fail(GZ_ERR_INVALID, "null argument");
  if (num_vertices < 2 || num_vertices > (1u << 31)) return mb_fail(GZ_ERR_INVALID, "a tenant needs 2 <= V <= 2^31");
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  ServeTenant t;
  GraphDesc &gd = t.desc;
  gd.V = num_vertices;
  sketch_sizing(num_vertices, s->factor, gd.C, gd.B);
  if (gd.B > 63 || gd.C > kServeTileC) return mb_fail(GZ_ERR_INVALID, "sketch geometry not supported by the server");
  gd.sketch_words = (gd.C * gd.B + 1) * 3;
  const size_t budget = tile_budget(&s->ingest, kServeTileC);
  MB_TRY(choose_tiles(gd, 0, budget));
  t.bytes = graph_sketch_bytes(gd);
  uint64_t off = 0;
  if (s->used + t.bytes > s->budget || !s->arena_alloc.alloc(t.bytes, off))
    return mb_fail(GZ_ERR_BUDGET, "sketch-byte budget exhausted: " + std::to_string(t.bytes) + " more bytes needed, " +
                                      std::to_string(s->budget - s->used) + " free");
  gd.sk_off = off;
  uint32_t slot;
  if (!s->free_slots.empty()) {
    slot = s->free_slots.back();
    s->free_slots.pop_back();
  } else {
    slot = s->slot_cap;
    if (slot >= (1u << 20)) {
      s->arena_alloc.release(off, t.bytes);
      return mb_fail(GZ_ERR_INVALID, "too many tenants");
    }
    const uint32_t cap = std::max<uint32_t>(64, s->slot_cap * 2);
    uint64_t *nf = nullptr;
    if (cudaMalloc(&nf, (size_t)cap * kServeFlipWords * 8) != cudaSuccess) {
      s->arena_alloc.release(off, t.bytes);
      return mb_fail(GZ_ERR_NOMEM, "cudaMalloc of hash constants");
    }
    if (s->d_flip) {
      cudaMemcpyAsync(nf, s->d_flip, (size_t)s->slot_cap * kServeFlipWords * 8, cudaMemcpyDeviceToDevice, s->ingest.stream);
      cudaStreamSynchronize(s->ingest.stream);
      cudaFree(s->d_flip);
    }
    s->d_flip = nf;
    for (uint32_t k = cap; k-- > s->slot_cap + 1;) s->free_slots.push_back(k);
    s->slot_cap = cap;
  }
  gd.flip_off = slot * kServeFlipWords;
  t.seed = seed;
  t.flips.assign((gd.C + 2) & ~1u, 0);
  for (uint32_t c = 0; c < gd.C; ++c) t.flips[c] = xxh3_flip(seed + 5ull * c);
  t.flips[gd.C] = xxh3_flip(seed);
  t.alive = true;
  // pageable source: the call returns once the bytes are staged, so t may move afterwards
  MB_CUDA(cudaMemcpyAsync(s->d_flip + gd.flip_off, t.flips.data(), 8 * t.flips.size(), cudaMemcpyHostToDevice,
                          s->ingest.stream));
  // zeroed on the ingest stream: ordered before every later ingest of this tenant, and after
  // every snapshot copy of the range's previous owner (the ingest stream waits for those)
  MB_CUDA(cudaMemsetAsync(s->arena + off, 0, t.bytes, s->ingest.stream));
  s->used += t.bytes;
  uint32_t id = (uint32_t)s->tenants.size();
  s->tenants.push_back(std::move(t));
  s->alive++;
  *tenant_out = id;
  return GZ_OK;
}

int gz_server_evict(gz_server_t *s, uint32_t tenant) {
  if (!s) return mb_fail(GZ_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  MB_TRY(serve_check_tenants(s, 1, &tenant));
  serve_wait_live(s, &tenant, 1);
  ServeTenant &t = s->tenants[tenant];
  // queries already submitted read their snapshots, whose copies the ingest stream waits for
  // before any later work on the range (a new tenant's zeroing included)
  s->arena_alloc.release(t.desc.sk_off, t.bytes);
  s->free_slots.push_back(t.desc.flip_off / kServeFlipWords);
  s->used -= t.bytes;
  t.alive = false;
  t.flips.clear();
  t.flips.shrink_to_fit();
  s->alive--;
  return GZ_OK;
}

int gz_server_set_route(gz_server_t *s, double sparse_factor) {
  if (!s || !(sparse_factor >= 0)) return mb_fail(GZ_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(s->mtx);
  s->ingest.sparse_factor = sparse_factor;
  return GZ_OK;
}

int gz_server_set_query_snapshot(gz_server_t *s, int snapshot) {
  if (!s) return mb_fail(GZ_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(s->mtx);
  s->live = snapshot == 0;
  return GZ_OK;
}

int gz_server_usage(gz_server_t *s, uint64_t *used, uint64_t *budget, uint32_t *tenants) {
  if (!s) return mb_fail(GZ_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(s->mtx);
  if (used) *used = s->used;
  if (budget) *budget = s->budget;
  if (tenants) *tenants = s->alive;
  return GZ_OK;
}

int gz_server_get_params(gz_server_t *s, uint32_t tenant, gz_params_t *o) {
  if (!s || !o) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mtx);
  MB_TRY(serve_check_tenants(s, 1, &tenant));
  const GraphDesc &gd = s->tenants[tenant].desc;
  std::memset(o, 0, sizeof(*o));
  o->num_vertices = gd.V;
  o->num_columns = gd.C;
  o->bkt_per_col = gd.B;
  o->num_buckets = gd.C * gd.B + 1;
  o->seed = s->tenants[tenant].seed;
  o->sketch_bytes = (uint64_t)gd.sketch_words * 4;
  o->max_rounds = gd.C;
  o->sketches_factor = s->factor;
  o->batch_factor = 1;
  o->vertices_per_tile = 1u << gd.tile_shift;
  o->num_tiles = gd.ntiles;
  o->vertices_per_bin = 1u << gd.bin_shift;
  o->num_bins = gd.nbins;
  o->cols_per_sample = 1;
  return GZ_OK;
}

// Applies update batches: tenant ids[i]'s packed 9-byte records are records[offsets[i] ..
// offsets[i+1]) in host memory. Synchronous.
int gz_server_ingest(gz_server_t *s, uint32_t n, const uint32_t *ids, const void *records,
                     const uint64_t *offsets) {
  if (!s || (n && (!ids || !offsets))) return mb_fail(GZ_ERR_INVALID, "null argument");
  if (n == 0) return GZ_OK;
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  MB_TRY(serve_check_tenants(s, n, ids));
  serve_wait_live(s, ids, n);
  const uint64_t nrec = offsets[n] - offsets[0];
  if (nrec == 0) return GZ_OK;
  if (!records) return mb_fail(GZ_ERR_INVALID, "null records");
  gz_batch *e = &s->ingest;
  e->graphs.resize(n);
  for (uint32_t i = 0; i < n; ++i) e->graphs[i] = s->tenants[ids[i]].desc;
  e->d_flip = s->d_flip;
  MB_TRY(finalize_graphs(e));
  MB_TRY(grow(&s->d_rec, s->rec_cap, nrec * 9, s->ingest.stream));
  MB_CUDA(cudaMemcpyAsync(s->d_rec, static_cast<const uint8_t *>(records) + offsets[0] * 9, nrec * 9,
                          cudaMemcpyHostToDevice, e->stream));
  std::vector<uint64_t> rel(n + 1);
  for (uint32_t i = 0; i <= n; ++i) rel[i] = offsets[i] - offsets[0];
  return batch_ingest(e, s->d_rec, rel.data());
}

// Applies update batches given as segments: segment k holds counts[k] packed records at host
// address ptrs[k] for tenant tenants[k]; the segments of one tenant must be consecutive. Each
// segment is one copy into the device staging buffer (pinned sources copy at full link speed).
int gz_server_ingest_segments(gz_server_t *s, uint32_t nseg, const uint32_t *tenants,
                              const void *const *ptrs, const uint64_t *counts) {
  if (!s || (nseg && (!tenants || !ptrs || !counts))) return mb_fail(GZ_ERR_INVALID, "null argument");
  if (nseg == 0) return GZ_OK;
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  std::vector<uint32_t> ids;
  std::vector<uint64_t> off(1, 0);
  for (uint32_t k = 0; k < nseg; ++k) {
    if (ids.empty() || ids.back() != tenants[k]) {
      ids.push_back(tenants[k]);
      off.push_back(off.back());
    }
    off.back() += counts[k];
  }
  MB_TRY(serve_check_tenants(s, (uint32_t)ids.size(), ids.data()));
  serve_wait_live(s, ids.data(), (uint32_t)ids.size());
  const uint64_t nrec = off.back();
  if (nrec == 0) return GZ_OK;
  gz_batch *e = &s->ingest;
  e->graphs.resize(ids.size());
  for (size_t i = 0; i < ids.size(); ++i) e->graphs[i] = s->tenants[ids[i]].desc;
  e->d_flip = s->d_flip;
  MB_TRY(finalize_graphs(e));
  MB_TRY(grow(&s->d_rec, s->rec_cap, nrec * 9, s->ingest.stream));
  uint64_t pos = 0;
  for (uint32_t k = 0; k < nseg; ++k) {
    if (!counts[k]) continue;
    if (!ptrs[k]) return mb_fail(GZ_ERR_INVALID, "null segment");
    MB_CUDA(cudaMemcpyAsync(s->d_rec + pos * 9, ptrs[k], counts[k] * 9, cudaMemcpyHostToDevice, e->stream));
    pos += counts[k];
  }
  return batch_ingest(e, s->d_rec, off.data());
}

// Snapshots the listed tenants' sketches (ordered after every earlier ingest call, before every
// later one) and queues their connected-components query; *ticket identifies it.
int gz_server_query_submit(gz_server_t *s, uint32_t n, const uint32_t *ids, uint64_t *ticket) {
  if (!s || !ids || !ticket || n == 0) return mb_fail(GZ_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  MB_TRY(serve_check_tenants(s, n, ids));
  QueryJob *j = new QueryJob();
  j->tenants.assign(ids, ids + n);
  if (s->live) {
    // read in place: ordered after every earlier ingest call; the tenants' later ingest calls and
    // evictions wait for the query (serve_wait_live)
    j->live = true;
    cudaEvent_t ev;
    MB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    MB_CUDA(cudaEventRecord(ev, s->ingest.stream));
    MB_CUDA(cudaStreamWaitEvent(s->query.stream, ev, 0));
    cudaEventDestroy(ev);
    uint64_t flip_off = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const ServeTenant &t = s->tenants[ids[i]];
      GraphDesc gd = t.desc;
      gd.flip_off = (uint32_t)flip_off;
      j->flips.insert(j->flips.end(), t.flips.begin(), t.flips.end());
      flip_off += t.flips.size();
      j->descs.push_back(gd);
    }
    {
      std::lock_guard<std::mutex> ql(s->qmtx);
      j->ticket = s->next_ticket++;
      s->jobs[j->ticket] = j;
      s->queue.push_back(j);
      *ticket = j->ticket;
    }
    s->qcv.notify_all();
    return GZ_OK;
  }
  uint64_t need = 0;
  for (uint32_t i = 0; i < n; ++i) need += (s->tenants[ids[i]].bytes + 255) & ~255ull;
  if (need > s->snap_alloc.size) {
    delete j;
    return mb_fail(GZ_ERR_INVALID, "the snapshot pool is smaller than this query's tenants");
  }
  {
    // wait for snapshot space (the worker releases it as queries finish)
    std::unique_lock<std::mutex> ql(s->qmtx);
    for (;;) {
      std::vector<std::pair<uint64_t, uint64_t>> got;
      bool ok = true;
      for (uint32_t i = 0; i < n && ok; ++i) {
        uint64_t off;
        if (s->snap_alloc.alloc(s->tenants[ids[i]].bytes, off)) got.emplace_back(off, s->tenants[ids[i]].bytes);
        else ok = false;
      }
      if (ok) {
        j->snaps = std::move(got);
        break;
      }
      for (auto &r : got) s->snap_alloc.release(r.first, r.second);
      if (s->queue.empty() && std::all_of(s->jobs.begin(), s->jobs.end(), [](auto &kv) { return kv.second->done; })) {
        delete j;
        return mb_fail(GZ_ERR_NOMEM, "snapshot pool fragmented");
      }
      s->done_cv.wait(ql);
    }
  }
  // copies on the query stream after all ingest work so far; later ingest work waits for them
  cudaEvent_t ev;
  MB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  MB_CUDA(cudaEventRecord(ev, s->ingest.stream));
  MB_CUDA(cudaStreamWaitEvent(s->query.stream, ev, 0));
  cudaEventDestroy(ev);
  uint64_t flip_off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const ServeTenant &t = s->tenants[ids[i]];
    GraphDesc gd = t.desc;
    MB_CUDA(cudaMemcpyAsync(s->snap + j->snaps[i].first, s->arena + t.desc.sk_off, t.bytes, cudaMemcpyDeviceToDevice,
                            s->query.stream));
    gd.sk_off = j->snaps[i].first;
    gd.flip_off = (uint32_t)flip_off;
    j->flips.insert(j->flips.end(), t.flips.begin(), t.flips.end());
    flip_off += t.flips.size();
    j->descs.push_back(gd);
  }
  MB_CUDA(cudaEventRecord(s->snap_done, s->query.stream));
  MB_CUDA(cudaStreamWaitEvent(s->ingest.stream, s->snap_done, 0));
  {
    std::lock_guard<std::mutex> ql(s->qmtx);
    j->ticket = s->next_ticket++;
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    *ticket = j->ticket;
  }
  s->qcv.notify_all();
  return GZ_OK;
}

// Waits for a submitted query. labels_out (NULL or the sum of the tenants' V, in submission
// order) gets each vertex's tenant-local root; num_cc, rounds and status (NULL or one per tenant)
// as gz_batch_connected_components.
int gz_server_query_ready(gz_server_t *s, uint64_t ticket, int *ready) {
  if (!s || !ready) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> ql(s->qmtx);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return mb_fail(GZ_ERR_INVALID, "unknown ticket");
  *ready = it->second->done ? 1 : 0;
  return GZ_OK;
}

int gz_server_query_wait(gz_server_t *s, uint64_t ticket, uint32_t *labels_out, uint32_t *num_cc,
                         uint32_t *rounds, int *status) {
  if (!s) return mb_fail(GZ_ERR_INVALID, "null handle");
  QueryJob *j = nullptr;
  {
    std::unique_lock<std::mutex> ql(s->qmtx);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return mb_fail(GZ_ERR_INVALID, "unknown ticket");
    j = it->second;
    s->done_cv.wait(ql, [&] { return j->done; });
    s->jobs.erase(it);
  }
  std::unique_ptr<QueryJob> owned(j);
  if (j->rc != GZ_OK) return mb_fail(j->rc, j->err);
  if (labels_out) std::copy(j->labels.begin(), j->labels.end(), labels_out);
  for (size_t i = 0; i < j->tenants.size(); ++i) {
    if (num_cc) num_cc[i] = j->ncc[i];
    if (rounds) rounds[i] = j->rounds[i];
    if (status) status[i] = j->status[i];
  }
  return GZ_OK;
}

// CCSketchAlg::write_binary (src/cc_sketch_alg.cpp:614-623) of one tenant: u64 seed, u32 V,
// f64 sketches_factor, then the V sketches.
int gz_server_write_binary(gz_server_t *s, uint32_t tenant, const char *path) {
  if (!s || !path) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::vector<uint8_t> buf;
  uint64_t seed;
  uint32_t V;
  {
    std::lock_guard<std::mutex> lk(s->mtx);
    MB_TRY(serve_check_tenants(s, 1, &tenant));
    const ServeTenant &t = s->tenants[tenant];
    seed = t.seed;
    V = t.desc.V;
    buf.resize((size_t)V * t.desc.sketch_words * 4);
  }
  MB_TRY(gz_server_dump_sketches(s, tenant, buf.data(), buf.size()));
  FILE *f = fopen(path, "wb");
  if (!f) return mb_fail(GZ_ERR_IO, std::string("cannot open ") + path);
  const double sf = s->factor;
  const bool ok = fwrite(&seed, 8, 1, f) == 1 && fwrite(&V, 4, 1, f) == 1 && fwrite(&sf, 8, 1, f) == 1 &&
                  fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (fclose(f) != 0 || !ok) return mb_fail(GZ_ERR_IO, std::string("cannot write ") + path);
  return GZ_OK;
}

// Re-admission from a write_binary file (construct_from_serialized_data,
// src/cc_sketch_alg.cpp:30-64): the tenant gets the file's V, seed and sketches; the file's
// sketches_factor must be the server's.
int gz_server_admit_serialized(gz_server_t *s, const char *path, uint32_t *tenant_out) {
  if (!s || !path || !tenant_out) return mb_fail(GZ_ERR_INVALID, "null argument");
  FILE *f = fopen(path, "rb");
  if (!f) return mb_fail(GZ_ERR_IO, std::string("cannot open ") + path);
  uint64_t seed = 0;
  uint32_t V = 0;
  double sf = 0;
  if (fread(&seed, 8, 1, f) != 1 || fread(&V, 4, 1, f) != 1 || fread(&sf, 8, 1, f) != 1) {
    fclose(f);
    return mb_fail(GZ_ERR_IO, "truncated header");
  }
  if ((sf > 0 ? sf : 1.0) != s->factor) {
    fclose(f);
    return mb_fail(GZ_ERR_INVALID, "the file's sketches_factor differs from the server's");
  }
  uint32_t C, B;
  sketch_sizing(V, s->factor, C, B);
  std::vector<uint8_t> buf((size_t)V * (C * B + 1) * 12);
  const size_t got = fread(buf.data(), 1, buf.size(), f);
  fclose(f);
  if (got != buf.size()) return mb_fail(GZ_ERR_IO, "truncated sketch data");
  uint32_t id;
  MB_TRY(gz_server_admit(s, V, seed, &id));
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  MB_CUDA(cudaMemcpyAsync(s->arena + s->tenants[id].desc.sk_off, buf.data(), buf.size(), cudaMemcpyHostToDevice,
                          s->ingest.stream));
  MB_CUDA(cudaStreamSynchronize(s->ingest.stream));
  *tenant_out = id;
  return GZ_OK;
}

int gz_server_dump_sketches(gz_server_t *s, uint32_t tenant, void *host_buf, size_t bytes) {
  if (!s || !host_buf) return mb_fail(GZ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mtx);
  cudaSetDevice(s->device);
  MB_TRY(serve_check_tenants(s, 1, &tenant));
  const GraphDesc &gd = s->tenants[tenant].desc;
  if (bytes != (uint64_t)gd.V * gd.sketch_words * 4) return mb_fail(GZ_ERR_INVALID, "buffer must hold V * sketch_bytes");
  MB_CUDA(cudaMemcpyAsync(host_buf, s->arena + gd.sk_off, bytes, cudaMemcpyDeviceToHost, s->ingest.stream));
  MB_CUDA(cudaStreamSynchronize(s->ingest.stream));
  return GZ_OK;
}

}  // extern "C"
