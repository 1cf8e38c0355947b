// gz_kernels.cu -- sm_100a kernels of the sketch-ingest and Boruvka-query path.
//
//   device gutter   : 9-byte records -> per-tile endpoint entries (counting sort by vertex tile)
//                     (replaces the GutteringSystem + driver reader threads,
//                      include/graph_sketch_driver.h:148-179)
//   sketch update   : per tile, sketches staged in shared memory by bulk async copies, every
//                     entry hashed per column and XORed in with shared-memory atomics
//                     (Sketch::update src/sketch.cpp:69-83 + apply_update_batch
//                      src/cc_sketch_alg.cpp:106-118)
//   Boruvka         : per-component sample, lock-free CAS union-find with path halving,
//                     segmented XOR merge of column r (boruvka_emulation and friends,
//                     src/cc_sketch_alg.cpp:137-513; DisjointSetUnion_MT include/dsu.h:101-174)
//
// All work is integer / XOR; results are bit-identical to the reference CPU build.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

#include "gz_common.cuh"
#include "gz_device.cuh"
#include "gz_kernels.cuh"

namespace gz {

namespace {

using namespace gz::dev;
std::atomic<uint64_t> g_launches{0};  // kernel launches issued from this file

// ------------------------------------------------------------------------------------------------
// device gutter
// ------------------------------------------------------------------------------------------------
// Counting pass (COUNT) or global-cursor scatter (!COUNT, used only when there are too many
// bins for the shared-memory sort). With SMEM the per-bin counts of a CTA are gathered in shared
// memory and added to the global counts once per bin.
template <int INPUT, bool COUNT, bool SMEM>
__global__ void __launch_bounds__(512)
k_gutter(const void *__restrict__ in, uint64_t n, GutterGeom g, uint64_t *__restrict__ hist,
         uint2 *__restrict__ entries, uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) uint8_t gsm[];
  uint32_t *s_bin = reinterpret_cast<uint32_t *>(gsm);
  const uint32_t nt_pad = (g.nbins + 3) & ~3u;
  uint8_t *s_rec = gsm + (SMEM ? nt_pad * 4 : 0);
  const uint32_t G = gridDim.x, cta = blockIdx.x;
  if (SMEM) {
    for (uint32_t b = threadIdx.x; b < g.nbins; b += blockDim.x) s_bin[b] = 0u;
    __syncthreads();
  }
  const uint64_t r0 = n * cta / G, r1 = n * (cta + 1) / G;
  bool bad = false;
  auto emit = [&](uint32_t v, uint32_t w) {
    const uint32_t t = v >> g.bin_shift;
    if (COUNT) {
      if (SMEM) atomicAdd(&s_bin[t], 1u);
      else atomicAdd(reinterpret_cast<unsigned long long *>(&hist[t]), 1ull);
    } else {
      const uint64_t p = atomicAdd(reinterpret_cast<unsigned long long *>(&hist[t]), 1ull);
      entries[p] = make_uint2(v, w);
    }
  };
  if (INPUT == kInputRecords) {
    const uint8_t *rec = reinterpret_cast<const uint8_t *>(in);
    for (uint64_t t = r0; t < r1; t += kRecTile) {
      const uint32_t cnt = (uint32_t)(r1 - t < (uint64_t)kRecTile ? r1 - t : (uint64_t)kRecTile);
      const uint32_t shift = stage_records(rec, t, cnt, s_rec);
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
        uint32_t u, v;
        parse_record(s_rec, shift, i, u, v);
        if (u >= g.V || v >= g.V) {
          bad = true;
          continue;
        }
        emit(u, v);
        emit(v, u);
      }
      __syncthreads();
    }
  } else {
    const uint2 *e = reinterpret_cast<const uint2 *>(in);
    for (uint64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const uint2 x = e[i];
      if (x.x >= g.V || x.y >= g.V) {
        bad = true;
        continue;
      }
      emit(x.x, x.y);
    }
  }
  if (COUNT && SMEM) {
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < g.nbins; b += blockDim.x)
      if (s_bin[b]) atomicAdd(reinterpret_cast<unsigned long long *>(&hist[b]), (unsigned long long)s_bin[b]);
  }
  if (COUNT && bad) atomicOr(status, kStatusBadVertex);
}

// Counting pass over records, unstaged: each thread takes RPI records per iteration (all their
// loads in flight together, straight from global memory), the block counts bins in shared
// memory, and adds its counts to the global ones once per bin.
template <int RPI>
__global__ void __launch_bounds__(512)
k_count_records(const uint8_t *__restrict__ rec, uint64_t n, GutterGeom g, uint64_t *__restrict__ hist,
                uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) uint32_t s_cnt[];
  for (uint32_t b = threadIdx.x; b < g.nbins; b += blockDim.x) s_cnt[b] = 0u;
  __syncthreads();
  const uint8_t *rec_end = rec + 9 * n;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x * RPI;
  bool bad = false;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x * RPI + threadIdx.x; i0 < n; i0 += step) {
    uint32_t u[RPI], v[RPI];
#pragma unroll
    for (int k = 0; k < RPI; ++k) {
      const uint64_t i = i0 + (uint64_t)k * blockDim.x;
      u[k] = v[k] = 0xffffffffu;
      if (i < n) load_record(rec, rec_end, i, u[k], v[k]);
    }
#pragma unroll
    for (int k = 0; k < RPI; ++k) {
      if (i0 + (uint64_t)k * blockDim.x >= n) continue;
      if (u[k] >= g.V || v[k] >= g.V) {
        bad = true;
        continue;
      }
      atomicAdd(&s_cnt[u[k] >> g.bin_shift], 1u);
      atomicAdd(&s_cnt[v[k] >> g.bin_shift], 1u);
    }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < g.nbins; b += blockDim.x)
    if (s_cnt[b]) atomicAdd(reinterpret_cast<unsigned long long *>(&hist[b]), (unsigned long long)s_cnt[b]);
  if (bad) atomicOr(status, kStatusBadVertex);
}

size_t gutter_smem(int input, GutterGeom g, bool smem) {
  size_t s = smem ? ((g.nbins + 3) & ~3u) * 4 : 0;
  if (input == kInputRecords) s += kRecStageBytes;
  return s;
}

template <int INPUT, bool COUNT, bool SMEM>
cudaError_t launch_gutter(const void *in, uint64_t n, GutterGeom g, int G, uint64_t *hist,
                          uint2 *entries, uint32_t *status, cudaStream_t s) {
  const size_t smem = gutter_smem(INPUT, g, SMEM);
  auto kern = k_gutter<INPUT, COUNT, SMEM>;
  if (smem > 48 * 1024) {
    cudaError_t e = smem_optin(kern);
    if (e != cudaSuccess) return e;
  }
  kern<<<G, 512, smem, s>>>(in, n, g, hist, entries, status);
  g_launches++;
  return cudaGetLastError();
}

// Sort-scatter pass: each CTA takes `rec_tile` inputs at a time, counting-sorts their endpoint
// entries by bin in shared memory, reserves one contiguous run per bin in the bin's region of the
// gutter (one global atomic per bin and tile), and writes the runs out, so consecutive threads
// store to consecutive addresses. base[b] = first slot of bin b, fill[b] = slots taken so far.
template <int INPUT>
__global__ void __launch_bounds__(1024, 1)
k_gutter_sort_scatter(const void *__restrict__ in, uint64_t n, GutterGeom g, uint32_t rec_tile,
                      const uint64_t *__restrict__ base, uint32_t *__restrict__ fill,
                      uint2 *__restrict__ entries) {
  extern __shared__ __align__(16) uint8_t gsm[];
  __shared__ uint32_t ws[32];
  const uint32_t nb = g.nbins, nb4 = (nb + 3) & ~3u;
  uint32_t *s_cur = reinterpret_cast<uint32_t *>(gsm);  // counts, then placement cursors
  uint32_t *s_off = s_cur + nb4;                         // run start inside the tile
  uint32_t *s_dst = s_off + nb4;                         // run start inside the gutter
  uint2 *s_sorted = reinterpret_cast<uint2 *>(s_dst + nb4);
  // the staged records share the sorted-entry area: they are parsed into registers before the
  // first entry is placed, and the next tile is staged only after the write-out
  uint8_t *s_rec = reinterpret_cast<uint8_t *>(s_sorted);
  const uint8_t *rec = reinterpret_cast<const uint8_t *>(in);
  const uint2 *ein = reinterpret_cast<const uint2 *>(in);
  const uint32_t per_thread = (nb + blockDim.x - 1) / blockDim.x;  // bins per thread (<= 8)
  for (uint64_t t0 = blockIdx.x * (uint64_t)rec_tile; t0 < n; t0 += (uint64_t)gridDim.x * rec_tile) {
    const uint32_t cnt = (uint32_t)(n - t0 < rec_tile ? n - t0 : rec_tile);
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s_cur[b] = 0u;
    uint32_t shift = 0;
    if (INPUT == kInputRecords) shift = stage_records(rec, t0, cnt, s_rec);
    __syncthreads();
    // 1. this thread's inputs (at most RPT; blockDim = 1024 and rec_tile <= RPT * 1024) into
    //    registers, then their per-bin counts
    constexpr int RPT = INPUT == kInputRecords ? 8 : 16;
    uint32_t ru[RPT], rv[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const uint32_t i = threadIdx.x + k * blockDim.x;
      ru[k] = rv[k] = 0xffffffffu;
      if (i < cnt) {
        if (INPUT == kInputRecords) {
          parse_record(s_rec, shift, i, ru[k], rv[k]);
        } else {
          const uint2 x = ein[t0 + i];
          ru[k] = x.x;
          rv[k] = x.y;
        }
        if (ru[k] >= g.V || rv[k] >= g.V) ru[k] = 0xffffffffu;  // dropped (status set by the count pass)
      }
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        atomicAdd(&s_cur[ru[k] >> g.bin_shift], 1u);
        if (INPUT == kInputRecords) atomicAdd(&s_cur[rv[k] >> g.bin_shift], 1u);
      }
    __syncthreads();
    // 2. run offsets inside the tile (bins [tid*per_thread, +per_thread) per thread)
    uint32_t local[8] = {0, 0, 0, 0, 0, 0, 0, 0}, sum = 0;
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      local[k] = b < nb ? s_cur[b] : 0u;
      sum += local[k];
    }
    uint32_t run = block_scan_1024(sum, ws);
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      if (b < nb) {
        s_off[b] = run;
        s_dst[b] = local[k] ? (uint32_t)base[b] + atomicAdd(&fill[b], local[k]) : 0u;
        s_cur[b] = run;
      }
      run += local[k];
    }
    __syncthreads();
    // 3. place entries in bin order: every slot claimed first (independent atomics in flight
    //    together), then the stores
    uint32_t pu[RPT], pv[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        pu[k] = atomicAdd(&s_cur[ru[k] >> g.bin_shift], 1u);
        if (INPUT == kInputRecords) pv[k] = atomicAdd(&s_cur[rv[k] >> g.bin_shift], 1u);
      }
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        s_sorted[pu[k]] = make_uint2(ru[k], rv[k]);
        if (INPUT == kInputRecords) s_sorted[pv[k]] = make_uint2(rv[k], ru[k]);
      }
    __syncthreads();
    // 4. coalesced write-out of the runs
    const uint32_t total = s_cur[nb - 1];
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
      const uint2 x = s_sorted[j];
      const uint32_t b = x.x >> g.bin_shift;
      entries[s_dst[b] + (j - s_off[b])] = x;
    }
    __syncthreads();
  }
}

__global__ void k_bin_offsets(const uint64_t *scanned, uint32_t stride, uint32_t nbins,
                              const uint64_t *total, uint32_t *bin_off) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins) bin_off[b] = (uint32_t)scanned[(uint64_t)b * stride];
  if (b == nbins) bin_off[b] = (uint32_t)*total;
}

__global__ void k_copy_u64(const uint64_t *src, uint64_t *dst, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// ------------------------------------------------------------------------------------------------
// scan (exclusive, u64, in place)
// ------------------------------------------------------------------------------------------------
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr uint64_t kScanBlock = (uint64_t)kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t block_exclusive(uint64_t x, uint64_t *block_total) {
  __shared__ uint64_t ws[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane < kScanThreads / 32 ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) ws[lane] = w;
  }
  __syncthreads();
  const uint64_t before = warp ? ws[warp - 1] : 0;
  *block_total = ws[kScanThreads / 32 - 1];
  __syncthreads();
  return before + inc - x;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const uint64_t *__restrict__ d, uint64_t n, uint64_t *__restrict__ sums) {
  const uint64_t base = blockIdx.x * kScanBlock + (uint64_t)threadIdx.x * kScanItems;
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += d[base + k];
  uint64_t tot;
  block_exclusive(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_down(uint64_t *__restrict__ d, uint64_t n, const uint64_t *__restrict__ prefix,
            uint64_t *__restrict__ total) {
  const uint64_t base = blockIdx.x * kScanBlock + (uint64_t)threadIdx.x * kScanItems;
  uint64_t v[kScanItems];
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? d[base + k] : 0;
    s += v[k];
  }
  uint64_t tot;
  uint64_t run = block_exclusive(s, &tot) + (prefix ? prefix[blockIdx.x] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) d[base + k] = run;
    run += v[k];
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total = run;
}

// ------------------------------------------------------------------------------------------------
// sketch update
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void apply_any(const uint8_t *cb, uint64_t i, uint32_t *s_sk,
                                          uint32_t vmask, const SketchGeom &g,
                                          const uint64_t *s_flip, uint64_t flip_chk) {
  const uint2 e = reinterpret_cast<const uint2 *>(cb)[i];
  if (g.cube)
    apply_entry_cube(e, s_sk, vmask, g.sketch_words, s_flip, flip_chk, g.C, g.B);
  else
    apply_entry(e, s_sk, vmask, g.sketch_words, s_flip, flip_chk, g.C, g.B);
}

__global__ void __launch_bounds__(1024, 1)
k_sketch_update(SketchGeom g, uint8_t *__restrict__ sketches, const uint8_t *__restrict__ gutter,
                ChunkTable chunks, const uint32_t *__restrict__ bin_off, int nchunks,
                const uint64_t *__restrict__ flip, uint32_t *work_counter, uint32_t *status) {
  extern __shared__ __align__(128) uint8_t dsm[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_tile, s_total, s_direct;
  const uint32_t vpt = 1u << g.tile_shift;
  const uint32_t tile_bytes = vpt * g.sketch_words * 4;
  const uint32_t per_bin = g.bin_shift - g.tile_shift;  // log2(tiles per bin)
  uint32_t *s_sk = reinterpret_cast<uint32_t *>(dsm);
  uint32_t *s_queue = reinterpret_cast<uint32_t *>(dsm + tile_bytes);
  uint64_t *s_flip = reinterpret_cast<uint64_t *>(dsm + tile_bytes + kQueueBytes);
  for (uint32_t i = threadIdx.x; i <= g.C; i += blockDim.x) s_flip[i] = flip[i];
  const uint32_t bar = smem_u32(&s_bar);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  const uint64_t flip_chk = s_flip[g.C];
  const uint32_t stride = g.nbins + 1;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t *q = s_queue + warp * 64;
  uint32_t parity = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(work_counter, 1u);
      uint32_t total = 0;
      if (t < g.ntiles) {
        const uint32_t bin = t >> per_bin;
        for (int k = 0; k < nchunks; ++k)
          total += bin_off[(uint64_t)k * stride + bin + 1] - bin_off[(uint64_t)k * stride + bin];
      }
      // a tile with too few entries to pay for staging its sketches is updated in place in HBM
      const bool direct = per_bin == 0 && total < g.direct_max;
      s_tile = t;
      s_total = total;
      s_direct = direct;
      if (t < g.ntiles && total && !direct) {
        const uint8_t *src = sketches + (uint64_t)t * tile_bytes;
        mbar_expect_tx(bar, tile_bytes);
        for (uint32_t off = 0; off < tile_bytes; off += kBulkPiece)
          bulk_g2s(smem_u32(dsm) + off, src + off, min(kBulkPiece, tile_bytes - off), bar);
      }
    }
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= g.ntiles) break;
    if (s_total && s_direct) {
      uint32_t *gsk = reinterpret_cast<uint32_t *>(sketches);
      for (int k = 0; k < nchunks; ++k) {
        const uint2 *E = reinterpret_cast<const uint2 *>(gutter + chunks.base[k]);
        const uint64_t b = bin_off[(uint64_t)k * stride + t];
        const uint64_t e = bin_off[(uint64_t)k * stride + t + 1];
        for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x)
          apply_entry_global(E[i], gsk, g.sketch_words, s_flip, flip_chk, g.C, g.B);
      }
    } else if (s_total) {
      const bool ok = mbar_wait_bounded(bar, parity, kWaitLimitNs);
      parity ^= 1u;
      if (__syncthreads_or(!ok)) {
        // the staged copy never completed: report it and leave without touching the tile
        if (threadIdx.x == 0) {
          atomicOr(status, kStatusTimeout);
          mbar_wait_bounded(bar, parity ^ 1u, kWaitLimitNs);
        }
        return;
      }
      const uint32_t bin = t >> per_bin;
      for (int k = 0; k < nchunks; ++k) {
        const uint8_t *cb = gutter + chunks.base[k];
        const uint64_t b = bin_off[(uint64_t)k * stride + bin];
        const uint64_t e = bin_off[(uint64_t)k * stride + bin + 1];
        if (per_bin == 0) {
          // the bin is this tile: every entry applies
          for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x)
            apply_any(cb, i, s_sk, vpt - 1, g, s_flip, flip_chk);
        } else {
          // the bin holds several tiles: each warp ballots 32 entries, queues the indices of
          // this tile's, and applies only full warps of queued entries
          uint32_t qn = 0;
          for (uint64_t i0 = b + (uint64_t)warp * 32; i0 < e; i0 += (uint64_t)nwarps * 32) {
            const uint64_t i = i0 + lane;
            const bool mine = i < e && (reinterpret_cast<const uint2 *>(cb)[i].x >> g.tile_shift) == t;
            const uint32_t m = __ballot_sync(kFull, mine);
            if (mine) q[qn + __popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
            qn += __popc(m);
            __syncwarp();
            if (qn >= 32) {
              apply_any(cb, q[lane], s_sk, vpt - 1, g, s_flip, flip_chk);
              __syncwarp();
              qn -= 32;
              if (lane < qn) q[lane] = q[32 + lane];
              __syncwarp();
            }
          }
          if (lane < qn) apply_any(cb, q[lane], s_sk, vpt - 1, g, s_flip, flip_chk);
          __syncwarp();
        }
      }
      fence_proxy_async_smem();
      __syncthreads();
      if (threadIdx.x == 0) {
        uint8_t *dst = sketches + (uint64_t)t * tile_bytes;
        for (uint32_t off = 0; off < tile_bytes; off += kBulkPiece)
          bulk_s2g(dst + off, smem_u32(dsm) + off, min(kBulkPiece, tile_bytes - off));
        bulk_commit();
        bulk_wait_read_all();
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// Pipelined variant of k_sketch_update for tiles of one bin each and plain CameoSketch entries
// (large graphs, where a tile's sketches dwarf its entries and staging dominates): a ring of
// g.nbuf tile buffers. The last warp's lane 0 claims tiles, bulk-loads them up to nbuf - 1 ahead
// and writes finished ones back, while the other 31 warps XOR each tile's entries into its
// buffer. Buffers change hands through full/empty mbarriers (bounded waits), so loads and
// write-backs of several tiles overlap the hashing. A tile with fewer entries than g.direct_max
// is updated in place in HBM without staging.
struct PipeSlot {
  uint32_t t, total, direct;
};
constexpr uint32_t kPipeMaxBuf = 4;

__global__ void __launch_bounds__(1024, 1)
k_sketch_update_pipe(SketchGeom g, uint8_t *__restrict__ sketches, const uint8_t *__restrict__ gutter,
                     ChunkTable chunks, const uint32_t *__restrict__ bin_off, int nchunks,
                     const uint64_t *__restrict__ flip, uint32_t *work_counter, uint32_t *status) {
  extern __shared__ __align__(128) uint8_t dsm[];
  __shared__ __align__(8) uint64_t s_full[kPipeMaxBuf], s_empty[kPipeMaxBuf];
  __shared__ PipeSlot s_slot[kPipeMaxBuf];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ncw = (blockDim.x >> 5) - 1, nct = ncw * 32;
  const uint32_t nbuf = g.nbuf;
  const uint32_t vpt = 1u << g.tile_shift;
  const uint32_t tile_bytes = vpt * g.sketch_words * 4;
  uint64_t *s_flip = reinterpret_cast<uint64_t *>(dsm + (size_t)nbuf * tile_bytes);
  for (uint32_t i = threadIdx.x; i <= g.C; i += blockDim.x) s_flip[i] = flip[i];
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < nbuf; ++i) {
      mbar_init(smem_u32(&s_full[i]), 1);
      mbar_init(smem_u32(&s_empty[i]), nct);
    }
    mbar_fence_init();
  }
  __syncthreads();
  const uint32_t stride = g.nbins + 1;

  if (warp == ncw) {  // ---------------- producer ----------------
    if (lane != 0) return;
    auto claim = [&]() {
      PipeSlot c;
      c.t = atomicAdd(work_counter, 1u);
      c.total = 0;
      c.direct = 0;
      if (c.t < g.ntiles) {
        for (int k = 0; k < nchunks; ++k)
          c.total += bin_off[(uint64_t)k * stride + c.t + 1] - bin_off[(uint64_t)k * stride + c.t];
        c.direct = c.total < g.direct_max;
      }
      return c;
    };
    uint8_t *pdst[kPipeMaxBuf] = {nullptr, nullptr, nullptr, nullptr};  // where a staged buffer goes back
    uint32_t issued = 0, lastk[kPipeMaxBuf] = {0, 0, 0, 0};
    uint32_t k = 0;
    bool ok = true;
    PipeSlot c = claim();
    for (;; ++k) {
      const uint32_t s = k % nbuf;
      if (k >= nbuf) {  // consumers must be done with tile k - nbuf (same buffer) before reuse
        if (!mbar_wait_bounded(smem_u32(&s_empty[s]), ((k - nbuf) / nbuf) & 1, kWaitLimitNs)) {
          ok = false;
          break;
        }
        if (pdst[s]) {
          for (uint32_t off = 0; off < tile_bytes; off += kBulkPiece)
            bulk_s2g(pdst[s] + off, smem_u32(dsm + (size_t)s * tile_bytes) + off, min(kBulkPiece, tile_bytes - off));
          bulk_commit();
          bulk_wait_read_all();
        }
      }
      s_slot[s] = c;
      const uint32_t full = smem_u32(&s_full[s]);
      const bool stage = c.t < g.ntiles && c.total && !c.direct;
      pdst[s] = stage ? sketches + (uint64_t)c.t * tile_bytes : nullptr;
      if (stage) {
        mbar_expect_tx(full, tile_bytes);
        for (uint32_t off = 0; off < tile_bytes; off += kBulkPiece)
          bulk_g2s(smem_u32(dsm + (size_t)s * tile_bytes) + off, pdst[s] + off, min(kBulkPiece, tile_bytes - off), full);
        issued |= 1u << s;
        lastk[s] = k;
      } else {
        mbar_arrive(full);  // in place, empty, or the end of the work: hand over at once
      }
      if (c.t >= g.ntiles) break;
      c = claim();  // the next tile's counts are read while this tile loads
    }
    if (ok) {  // write back the tiles still in the ring, oldest first
      const uint32_t first = k + 1 > nbuf ? k + 1 - nbuf : 0;
      for (uint32_t j = first; j < k && ok; ++j) {
        const uint32_t s = j % nbuf;
        ok = mbar_wait_bounded(smem_u32(&s_empty[s]), (j / nbuf) & 1, kWaitLimitNs);
        if (ok && pdst[s]) {
          for (uint32_t off = 0; off < tile_bytes; off += kBulkPiece)
            bulk_s2g(pdst[s] + off, smem_u32(dsm + (size_t)s * tile_bytes) + off, min(kBulkPiece, tile_bytes - off));
          bulk_commit();
        }
      }
    }
    if (!ok) {
      atomicOr(status, kStatusTimeout);
      // every load issued must land before the CTA's shared memory goes away
      for (uint32_t s = 0; s < nbuf; ++s)
        if (issued & (1u << s)) mbar_wait_bounded(smem_u32(&s_full[s]), (lastk[s] / nbuf) & 1, kWaitLimitNs);
    }
    bulk_wait_all();
    return;
  }

  // ---------------- consumers ----------------
  const uint64_t flip_chk = s_flip[g.C];
  const uint32_t ct = threadIdx.x;
  for (uint32_t k = 0;; ++k) {
    const uint32_t s = k % nbuf;
    if (!mbar_wait_bounded(smem_u32(&s_full[s]), (k / nbuf) & 1, kWaitLimitNs)) {
      if (lane == 0) atomicOr(status, kStatusTimeout);
      return;
    }
    const PipeSlot m = s_slot[s];
    if (m.t >= g.ntiles) return;
    if (m.total) {
      uint32_t *s_sk = reinterpret_cast<uint32_t *>(dsm + (size_t)s * tile_bytes);
      uint32_t *gsk = reinterpret_cast<uint32_t *>(sketches);
      for (int c = 0; c < nchunks; ++c) {
        const uint2 *E = reinterpret_cast<const uint2 *>(gutter + chunks.base[c]);
        const uint32_t b = bin_off[(uint64_t)c * stride + m.t], e = bin_off[(uint64_t)c * stride + m.t + 1];
        // the next entry's load is in flight while the current one is hashed
        uint32_t i = b + ct;
        uint2 cur = i < e ? E[i] : make_uint2(0, 0);
        for (; i < e; i += nct) {
          const uint2 x = cur;
          if (i + nct < e) cur = E[i + nct];
          if (m.direct) apply_entry_global(x, gsk, g.sketch_words, s_flip, flip_chk, g.C, g.B);
          else apply_entry(x, s_sk, vpt - 1, g.sketch_words, s_flip, flip_chk, g.C, g.B);
        }
      }
      fence_proxy_async_smem();  // this thread's bucket writes, before the bulk write-back
    }
    mbar_arrive(smem_u32(&s_empty[s]));
  }
}

template <int INPUT, bool CUBE>
__global__ void __launch_bounds__(512)
k_in_place(const void *__restrict__ in, uint64_t n, SketchGeom g, uint32_t *__restrict__ sk_words,
           const uint64_t *__restrict__ flip, uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) uint8_t ism[];
  uint64_t *s_flip = reinterpret_cast<uint64_t *>(ism);
  for (uint32_t i = threadIdx.x; i <= g.C; i += blockDim.x) s_flip[i] = flip[i];
  __syncthreads();
  const uint64_t flip_chk = s_flip[g.C];
  bool bad = false;
  if (INPUT == kInputRecords) {
    uint8_t *s_rec = ism + (((size_t)g.C + 2) & ~(size_t)1) * 8;
    const uint8_t *rec = reinterpret_cast<const uint8_t *>(in);
    for (uint64_t t = (uint64_t)blockIdx.x * kRecTile; t < n; t += (uint64_t)gridDim.x * kRecTile) {
      const uint32_t cnt = (uint32_t)(n - t < (uint64_t)kRecTile ? n - t : (uint64_t)kRecTile);
      const uint32_t shift = stage_records(rec, t, cnt, s_rec);
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
        uint32_t u, v;
        parse_record(s_rec, shift, i, u, v);
        if (u >= g.V || v >= g.V) {
          bad = true;
          continue;
        }
        if (u == v) continue;  // both endpoint updates land in one sketch and cancel
        xor_update_in_place<CUBE>(sk_words + (uint64_t)u * g.sketch_words,
                                  sk_words + (uint64_t)v * g.sketch_words, u, v, s_flip, flip_chk,
                                  g.C, g.B);
      }
      __syncthreads();
    }
  } else {
    const uint2 *e = reinterpret_cast<const uint2 *>(in);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
      const uint2 x = e[i];
      if (x.x >= g.V || x.y >= g.V) {
        bad = true;
        continue;
      }
      xor_update_in_place<CUBE>(sk_words + (uint64_t)x.x * g.sketch_words, nullptr, x.x, x.y, s_flip,
                                flip_chk, g.C, g.B);
    }
  }
  if (bad) atomicOr(status, kStatusBadVertex);
}

__global__ void k_sketch_xor_raw(uint32_t *sketches, uint32_t words, uint32_t v,
                                 const uint32_t *raw) {
  uint32_t *sk = sketches + (uint64_t)v * words;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
    sk[i] ^= raw[i];
}

// ------------------------------------------------------------------------------------------------
// Boruvka
// ------------------------------------------------------------------------------------------------
// sample_supernode (src/cc_sketch_alg.cpp:137-166): FAIL marks the round modified, GOOD unions
// the sampled edge and marks modified if the partition changed. flags = the round's modified word.
__device__ void handle_result(int res, uint64_t idx, uint32_t round, uint32_t key,
                              const BoruvkaGeom &g, const BoruvkaBufs &b, uint32_t *flags) {
  if (b.trace) {
    const uint32_t ti = atomicAdd(b.trace_n, 1u);
    if (ti < b.trace_cap) {
      TraceRec r;
      r.round = round;
      r.key = key;
      r.result = (uint32_t)res;
      r.pad = 0;
      r.idx = idx;
      reinterpret_cast<TraceRec *>(b.trace)[ti] = r;
    }
  }
  if (res == 2) {
    atomicOr(flags, 1u);
  } else if (res == 0) {
    const uint32_t x = (uint32_t)(idx >> 32), y = (uint32_t)idx;
    if (x >= g.V || y >= g.V) {
      atomicOr(b.status, kStatusBadSample);
      return;
    }
    if (dsu_unite(b.parent, x, y)) {
      atomicOr(flags, 1u);
      const uint32_t fi = atomicAdd(b.forest_n, 1u);
      if (fi < g.V) b.forest[fi] = idx;
    }
  }
}

__global__ void k_bv_reset(uint32_t V, uint32_t *parent) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) parent[v] = v;
}

// The Boruvka phases below are device functions shared by the per-phase kernels (one launch
// each, the CUDA-graph and host-loop queries) and by k_bv_query (every phase of every round in
// one cooperative launch). Data written earlier in the same query is read through L2 (__ldcg):
// in k_bv_query another SM wrote it in an earlier phase of the same kernel. A warp's copy ring
// counts its batches in T across calls, so its two mbarriers' phases stay in step.

// Round 0 (run_round_zero, src/cc_sketch_alg.cpp:223-244) for warp gw of nwarps: every vertex
// sketch samples its sample 0 -- columns 0..CPS-1 and the deterministic bucket. The warp takes
// 32 consecutive vertices at a time, in batches of KB whose runs are bulk-copied to shared memory
// one batch ahead (also across its 32-vertex groups), and samples each vertex from there; lane i
// keeps vertex i's result, and the 32 results are applied by the 32 lanes at once. False when a
// copy did not land in time (status set).
template <int CPS, int KB, int NS>
__device__ bool bv_round0_warp(const BoruvkaGeom &g, const uint32_t *__restrict__ sk_words,
                               const BoruvkaBufs &b, uint32_t *flags, BvRingN<NS> &ring, uint32_t &T,
                               uint32_t gw, uint32_t nwarps) {
  constexpr uint32_t BPG = 32 / KB;  // batches per 32-vertex group
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t W = 3 * CPS * g.B, detw = 3 * g.C * g.B;
  const uint32_t ngroups = (g.V + 31) / 32;
  if (gw >= ngroups) return true;
  auto first_vertex = [&](uint32_t t) {  // first vertex of batch t, or ~0 past the work
    const uint32_t grp = gw + (t / BPG) * nwarps;
    return grp < ngroups ? grp * 32 + (t % BPG) * KB : 0xffffffffu;
  };
  auto issue = [&](uint32_t t) {
    const uint32_t v0 = first_vertex(t);
    const bool mine = v0 != 0xffffffffu && lane < (uint32_t)KB && v0 + lane < g.V;
    const uint32_t *sk = sk_words + (uint64_t)(mine ? v0 + lane : 0) * g.sketch_words;
    ring.issue(T + t, mine, sk, W, sk + detw, KB);
  };
  int my_res = 1;
  uint64_t my_idx = 0;
  for (uint32_t a = 0; a + 1 < (uint32_t)NS; ++a) issue(a);
  uint32_t t = 0;
  for (;; ++t) {
    const uint32_t v0 = first_vertex(t);
    if (v0 == 0xffffffffu) break;
    issue(t + NS - 1);
    if (!ring.wait(T + t)) {
      if (lane == 0) atomicOr(b.status, kStatusTimeout);
      // their copies must land before the shared memory is reused or freed
      for (uint32_t a = 1; a < (uint32_t)NS; ++a) ring.wait(T + t + a);
      return false;
    }
#pragma unroll 1
    for (int k = 0; k < KB; ++k)
      if (v0 + k < g.V) {
        const uint32_t *sk = sk_words + (uint64_t)(v0 + k) * g.sketch_words;
        const uint8_t *sl = ring.slot(T + t, k, KB);
        const uint32_t *run = bulk_run_at(sl, sk), *det = bulk_run_at(sl + ring.run_cap, sk + detw);
        uint64_t idx;
        const int res = warp_sample_smem_split<CPS>(run, det, g.B, g.flip_chk, &idx);
        if (lane == (t % BPG) * KB + k) {
          my_res = res;
          my_idx = idx;
        }
      }
    __syncwarp();
    if (t % BPG == BPG - 1) {  // end of a 32-vertex group: its results, one lane each
      const uint32_t base = v0 - (t % BPG) * KB;
      if (base + lane < g.V) handle_result(my_res, my_idx, 0, base + lane, g, b, flags);
      __syncwarp();
      my_res = 1;
      my_idx = 0;
    }
  }
  // batches 0 .. t + NS - 2 were issued; those from t on covered no vertex (nothing in flight)
  T += t + NS - 1;
  return true;
}

template <int CPS, int KB>
__global__ void __launch_bounds__(256) k_bv_round0(BoruvkaGeom g, const uint32_t *__restrict__ sk_words,
                                                   BoruvkaBufs b) {
  extern __shared__ __align__(16) uint8_t bv_smem[];
  const uint32_t W = 3 * CPS * g.B;
  BvRing ring;
  ring.init(bv_smem + (threadIdx.x >> 5) * bv_warp_bytes(W, KB), W, KB);
  uint32_t T = 0;
  bv_round0_warp<CPS, KB, 2>(g, sk_words, b, b.flags, ring, T,
                          (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                          (gridDim.x * blockDim.x) >> 5);
}

// Per-block table of the distinct roots among a block's vertices (at most 512 of them in 1024
// slots, open addressing): the block's members per root are counted in shared memory, so a root
// shared by many vertices (late rounds: a few large components) gets one global atomic per block
// instead of one per warp.
constexpr uint32_t kRootSlots = 1024;
struct RootTable {
  uint32_t key[kRootSlots], cnt[kRootSlots], aux[kRootSlots];
};
__device__ __forceinline__ void root_table_clear(RootTable &t, uint32_t aux0) {
  for (uint32_t e = threadIdx.x; e < kRootSlots; e += blockDim.x) {
    t.key[e] = 0xffffffffu;
    t.cnt[e] = 0;
    t.aux[e] = aux0;
  }
}
// Slot of root r (inserted if new); the table has room for every distinct root of a block.
__device__ __forceinline__ uint32_t root_slot(RootTable &t, uint32_t r) {
  uint32_t h = (r * 0x9E3779B1u) >> 22;
  for (uint32_t i = 0; i < kRootSlots; ++i, h = (h + 1) & (kRootSlots - 1)) {
    const uint32_t k = atomicCAS(&t.key[h], 0xffffffffu, r);
    if (k == 0xffffffffu || k == r) break;
  }
  return h;
}

// Root of every vertex of [v0, v0 + VPT * blockDim.x) (thread t: vertices v0 + k * blockDim.x + t)
// and members per root (cnt) and smallest member per root (minv, for trace keys). The VPT parent
// chains of a thread are followed together, one hop per pass with all VPT loads in flight (no
// union runs during the labelling), then each vertex's parent is set to its root: later rounds
// find it in a hop or two. VPT * blockDim.x <= 512. Every thread of the block calls it.
template <int VPT>
__device__ __forceinline__ void bv_label_block(uint32_t V, uint32_t v0, uint32_t *parent,
                                               uint32_t *label, uint32_t *cnt, uint32_t *minv,
                                               RootTable &tab) {
  uint32_t r[VPT], p1[VPT];
  bool in[VPT];
  root_table_clear(tab, 0xffffffffu);
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint32_t v = v0 + k * blockDim.x + threadIdx.x;
    in[k] = v < V;
    r[k] = in[k] ? v : 0u;
    p1[k] = in[k] ? __ldcg(parent + v) : 0u;
  }
  // x[k] = parent of r[k]; r[k] is the root once they are equal
  uint32_t x[VPT];
#pragma unroll
  for (int k = 0; k < VPT; ++k) x[k] = in[k] ? p1[k] : r[k];
  for (;;) {
    bool more = false;
#pragma unroll
    for (int k = 0; k < VPT; ++k) more = more || x[k] != r[k];
    if (!more) break;
#pragma unroll
    for (int k = 0; k < VPT; ++k)
      if (x[k] != r[k]) {
        r[k] = x[k];
        x[k] = __ldcg(parent + x[k]);
      }
  }
  __syncthreads();  // the table is clear
#pragma unroll
  for (int k = 0; k < VPT; ++k)
    if (in[k]) {
      const uint32_t v = v0 + k * blockDim.x + threadIdx.x;
      label[v] = r[k];
      if (p1[k] != r[k]) __stcg(parent + v, r[k]);
      const uint32_t h = root_slot(tab, r[k]);
      atomicAdd(&tab.cnt[h], 1u);
      if (minv) atomicMin(&tab.aux[h], v);
    }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < kRootSlots; e += blockDim.x) {
    const uint32_t key = tab.key[e];
    if (key != 0xffffffffu) {
      atomicAdd(&cnt[key], tab.cnt[e]);
      if (minv) atomicMin(&minv[key], tab.aux[e]);
    }
  }
  __syncthreads();  // the table's next user clears it
}

__global__ void __launch_bounds__(256) k_bv_label(uint32_t V, uint32_t *parent, uint32_t *label,
                                                  uint32_t *cnt, uint32_t *minv) {
  __shared__ RootTable tab;
  bv_label_block<1>(V, blockIdx.x * blockDim.x, parent, label, cnt, minv, tab);
}

// Per-round counters: members and scatter cursors per root, smallest member (traces), and no
// component marked as merged from its complement yet.
__global__ void k_bv_prep(uint32_t V, BoruvkaBufs b) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  b.cnt[v] = 0;
  b.fill[v] = 0;
  if (b.trace) b.minv[v] = 0xffffffffu;
  if (v == 0) {
    *b.big = 0xffffffffu;
    *b.ncross = 0;
  }
}

__global__ void k_bv_pack(uint32_t V, const uint32_t *cnt, uint64_t *packed) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const uint32_t c = cnt[v];
  packed[v] = (uint64_t)c | (c ? (1ull << 32) : 0ull);
}

// create_merge_instructions (src/cc_sketch_alg.cpp:382-462) for the vertices [v0, v0 + VPT *
// blockDim.x) (thread t: vertices v0 + k * blockDim.x + t): group vertices by root so each
// component's members are contiguous in `order` (slots taken with warp-aggregated atomics, or one
// claim when the block's vertices share one root). packed_at(r) = the exclusive scan over the
// roots below r of (members | 1 << 32): root r's first grouped position and its component index;
// nc = the number of components. Components crossing a span edge get their acc slot cleared and
// are listed in cross. Every thread of the block (8 warps) calls it.
template <int VPT, class PackedAt>
__device__ __forceinline__ void bv_group_block(uint32_t V, uint32_t v0, uint32_t acc_words,
                                               uint32_t span, const uint32_t *label,
                                               PackedAt packed_at, uint32_t nc, const uint32_t *cnt,
                                               uint32_t *fill, const uint32_t *minv, uint32_t *order,
                                               uint32_t *order_comp, uint32_t *comp_start,
                                               uint32_t *comp_key, uint32_t *ncomp, uint32_t *acc,
                                               uint32_t *big, uint32_t *cross, uint32_t *ncross,
                                               RootTable &tab) {
  uint32_t r[VPT], slot[VPT], h[VPT];
  bool in[VPT];
  root_table_clear(tab, 0u);
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint32_t v = v0 + k * blockDim.x + threadIdx.x;
    in[k] = v < V;
    r[k] = in[k] ? __ldcg(label + v) : 0u;
  }
  __syncthreads();  // the table is clear
  // rank of each vertex among the block's members of its root, then one cursor claim per root
#pragma unroll
  for (int k = 0; k < VPT; ++k)
    if (in[k]) {
      h[k] = root_slot(tab, r[k]);
      slot[k] = atomicAdd(&tab.cnt[h[k]], 1u);
    }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < kRootSlots; e += blockDim.x) {
    const uint32_t key = tab.key[e];
    if (key != 0xffffffffu) tab.aux[e] = atomicAdd(&fill[key], tab.cnt[e]);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < VPT; ++k)
    if (in[k]) slot[k] += tab.aux[h[k]];
  __syncthreads();  // the table's next user clears it
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    if (!in[k]) continue;
    const uint32_t v = v0 + k * blockDim.x + threadIdx.x;
    const uint64_t s = packed_at(r[k]);
    const uint32_t start = (uint32_t)s, c = (uint32_t)(s >> 32);
    const uint32_t pos = start + slot[k];
    order[pos] = v;
    order_comp[pos] = c;
    if (v == r[k]) {
      const uint32_t members = __ldcg(cnt + v);
      comp_start[c] = start;
      comp_key[c] = minv ? __ldcg(minv + v) : v;
      const uint32_t end = start + members;
      if (start / span != (end - 1) / span) {
        uint32_t *ac = acc + (uint64_t)(start / span) * acc_words;
        for (uint32_t i = 0; i < acc_words; ++i) ac[i] = 0;
        if (2ull * members > V) *big = c;  // at most one component holds over half the vertices
        // listed for the sampling from acc (one component at most per span edge)
        cross[atomicAdd(ncross, 1u)] = c;
      }
    }
    if (v == 0) {
      comp_start[nc] = V;
      *ncomp = nc;
    }
  }
}

__global__ void __launch_bounds__(256) k_bv_group(uint32_t V, uint32_t acc_words, uint32_t span,
                                                  const uint32_t *label, const uint64_t *packed,
                                                  const uint64_t *total, const uint32_t *cnt,
                                                  uint32_t *fill, const uint32_t *minv,
                                                  uint32_t *order, uint32_t *order_comp,
                                                  uint32_t *comp_start, uint32_t *comp_key,
                                                  uint32_t *ncomp, uint32_t *acc, uint32_t *big,
                                                  uint32_t *cross, uint32_t *ncross) {
  const uint32_t nc = (uint32_t)(*total >> 32);
  __shared__ RootTable tab;
  bv_group_block<1>(V, blockIdx.x * blockDim.x, acc_words, span, label,
                    [&](uint32_t r) { return packed[r]; }, nc, cnt, fill, minv, order, order_comp,
                    comp_start, comp_key, ncomp, acc, big, cross, ncross, tab);
}

// perform_boruvka_round (src/cc_sketch_alg.cpp:246-380) for round >= 1, grouped positions
// [w * span, w * span + span) (span <= 32): the warp XOR-merges sample `round` (columns
// round*CPS .. +CPS, one contiguous word run) + the deterministic bucket of those members, copied
// to shared memory with bulk copies in batches of KB, one batch ahead. A component wholly inside
// the span is sampled right here (results applied 32 at a time by the lanes); a component
// covering the whole span leaves this warp's XOR in its partial slot w (bv_reduce_parts_warp folds
// those); the parts of components crossing a span edge go to acc (per component: CPS*B column
// buckets, then the deterministic one) with one coalesced atomicXor per word. False when a copy did
// not land in time (status set).
template <int CPS, int NW, int KB, int NS>
__device__ bool bv_merge_span(const BoruvkaGeom &g, const uint32_t *__restrict__ sk_words,
                              const BoruvkaBufs &b, uint32_t round, uint32_t *flags,
                              BvRingN<NS> &ring, uint32_t &T, uint32_t w) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t W = 3 * CPS * g.B, SW = W + 3;
  uint32_t *st = ring.stage;
  const uint64_t p0 = (uint64_t)w * g.span;
  if (p0 >= g.V) return true;
  const uint32_t n = (uint32_t)(g.V - p0 < g.span ? g.V - p0 : g.span);  // span <= 32
  const uint32_t p1 = (uint32_t)p0 + n;
  const uint32_t col = 3 * round * CPS * g.B, detw = 3 * g.C * g.B;
  // the component merged from its complement: its members are skipped, and every other
  // member's words are also XORed into its acc
  const uint32_t big = g.complement ? __ldcg(b.big) : 0xffffffffu;
  if (big != 0xffffffffu && __ldcg(b.comp_start + big) <= p0 && __ldcg(b.comp_start + big + 1) >= p1) {
    if (lane == 0) b.part_comp[w] = 0xffffffffu;
    return true;
  }
  const uint32_t my_v = lane < n ? __ldcg(b.order + p0 + lane) : 0u;
  const uint32_t my_c = lane < n ? __ldcg(b.order_comp + p0 + lane) : 0u;
  // the components of the positions just before and after the span: a component that also
  // holds one of them crosses a span edge (members of a component are contiguous)
  uint32_t edge_c = 0xffffffffu;
  if (lane == 0 && p0 > 0) edge_c = __ldcg(b.order_comp + p0 - 1);
  if (lane == 1 && p1 < g.V) edge_c = __ldcg(b.order_comp + p1);
  const uint32_t prev_c = __shfl_sync(kFull, edge_c, 0), next_c = __shfl_sync(kFull, edge_c, 1);
  // lane k < KB copies member t * KB + k of batch t (its vertex and component come by shuffle)
  auto member_sketch = [&](uint32_t m) {
    const uint32_t v = __shfl_sync(kFull, my_v, m & 31);
    return sk_words + (uint64_t)v * g.sketch_words;
  };
  auto issue = [&](uint32_t t) {
    const uint32_t m = t * KB + lane;
    const uint32_t *sk = member_sketch(m);
    const uint32_t c = __shfl_sync(kFull, my_c, m & 31);
    const bool mine = lane < (uint32_t)KB && m < n && c != big;
    ring.issue(T + t, mine, sk + col, W, sk + detw, KB);
  };
  const uint32_t nb = (n + KB - 1) / KB;
  for (uint32_t a = 0; a + 1 < (uint32_t)NS && a < nb; ++a) issue(a);
  uint32_t acc[NW], dacc = 0, cpl[NW], dcpl = 0;
#pragma unroll
  for (int k = 0; k < NW; ++k) acc[k] = cpl[k] = 0;
  uint32_t cur = 0xffffffffu;
  bool whole = false;  // one component covers [p0, p1)
  // results of components sampled here: lane j holds the j-th, applied 32 at a time
  int my_res = 1;
  uint64_t my_idx = 0;
  uint32_t my_key = 0, nres = 0;
  auto apply = [&]() {
    if (lane < nres) handle_result(my_res, my_idx, round, my_key, g, b, flags);
    __syncwarp();
    nres = 0;
  };
  auto flush = [&](uint32_t comp) {
    const bool before = comp == prev_c, after = comp == next_c;
    if (!before && !after) {
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W) st[wi] = acc[k];
      }
      if (lane < 3) st[W + lane] = dacc;
      __syncwarp();
      uint64_t idx;
      const int res = warp_sample_smem<CPS>(st, W, g.B, g.flip_chk, &idx);
      __syncwarp();
      if (lane == nres) {
        my_res = res;
        my_idx = idx;
        my_key = __ldcg(b.comp_key + comp);
      }
      if (++nres == 32) apply();
    } else if (before && after) {
      uint32_t *pt = b.part + (uint64_t)w * SW;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W) pt[wi] = acc[k];
      }
      if (lane < 3) pt[W + lane] = dacc;
      if (lane == 0) b.part_comp[w] = comp;
      whole = true;
    } else {
      // a component crossing a span edge owns acc slot (its first position / span)
      const uint32_t slot = before ? __ldcg(b.comp_start + comp) / g.span : w;
      uint32_t *ac = b.acc + (uint64_t)slot * SW;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t wi = k * 32 + lane;
        if (wi < W && acc[k]) atomicXor(ac + wi, acc[k]);
      }
      if (lane < 3 && dacc) atomicXor(ac + W + lane, dacc);
    }
  };
  for (uint32_t t = 0; t < nb; ++t) {
    if (t + NS - 1 < nb) issue(t + NS - 1);
    if (!ring.wait(T + t)) {
      if (lane == 0) atomicOr(b.status, kStatusTimeout);
      // their copies must land before the shared memory is reused or freed
      for (uint32_t a = 1; a < (uint32_t)NS && t + a < nb; ++a) ring.wait(T + t + a);
      return false;
    }
    // not unrolled: one copy of the flush (and the sampling it inlines) keeps the kernel small
    // enough for the instruction cache
#pragma unroll 1
    for (int k = 0; k < KB; ++k) {
      const uint32_t m = t * KB + k;
      const uint32_t c = __shfl_sync(kFull, my_c, m < n ? m : 0);
      const uint32_t *sk = member_sketch(m < n ? m : 0);
      if (m < n && c != big) {
        if (c != cur) {
          if (cur != 0xffffffffu) flush(cur);
          cur = c;
#pragma unroll
          for (int q = 0; q < NW; ++q) acc[q] = 0;
          dacc = 0;
        }
        const uint8_t *slt = ring.slot(T + t, k, KB);
        const uint32_t *sl = bulk_run_at(slt, sk + col);
        const uint32_t *sd = bulk_run_at(slt + ring.run_cap, sk + detw);
#pragma unroll
        for (int q = 0; q < NW; ++q) {
          const uint32_t wi = q * 32 + lane;
          if (wi < W) acc[q] ^= sl[wi];
        }
        if (lane < 3) dacc ^= sd[lane];
        if (big != 0xffffffffu) {
#pragma unroll
          for (int q = 0; q < NW; ++q) {
            const uint32_t wi = q * 32 + lane;
            if (wi < W) cpl[q] ^= sl[wi];
          }
          if (lane < 3) dcpl ^= sd[lane];
        }
      }
    }
    __syncwarp();
  }
  T += nb;
  if (cur != 0xffffffffu) flush(cur);
  apply();
  if (big != 0xffffffffu) {
    uint32_t *ac = b.acc + (uint64_t)(__ldcg(b.comp_start + big) / g.span) * SW;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const uint32_t wi = k * 32 + lane;
      if (wi < W && cpl[k]) atomicXor(ac + wi, cpl[k]);
    }
    if (lane < 3 && dcpl) atomicXor(ac + W + lane, dcpl);
  }
  if (!whole && lane == 0) b.part_comp[w] = 0xffffffffu;
  return true;
}

template <int CPS, int NW, int KB>
__global__ void __launch_bounds__(256) k_bv_merge(BoruvkaGeom g, const uint32_t *__restrict__ sk_words,
                                                  BoruvkaBufs b) {
  extern __shared__ __align__(16) uint8_t bv_smem[];
  const uint32_t W = 3 * CPS * g.B;
  BvRing ring;
  ring.init(bv_smem + (threadIdx.x >> 5) * bv_warp_bytes(W, KB), W, KB);
  uint32_t T = 0;
  bv_merge_span<CPS, NW, KB, 2>(g, sk_words, b, *b.round, b.flags, ring, T,
                             (blockIdx.x * blockDim.x + threadIdx.x) >> 5);
}

// Folds the partial slots [s0, s0 + per) (per <= 32) of merge warps covered by one component into
// that component's acc (KB slots' loads in flight), one atomicXor per word per component.
template <int CPS, int NW, int KB>
__device__ void bv_reduce_parts_warp(const BoruvkaGeom &g, uint32_t nslots, const BoruvkaBufs &b,
                                     uint32_t s0, uint32_t per) {
  const uint32_t lane = threadIdx.x & 31;
  if (s0 >= nslots) return;
  const uint32_t n = nslots - s0 < per ? nslots - s0 : per;
  const uint32_t W = 3 * CPS * g.B;
  const uint32_t my_c = lane < n ? __ldcg(b.part_comp + s0 + lane) : 0xffffffffu;
  uint32_t live = __ballot_sync(kFull, my_c != 0xffffffffu);
  if (!live) return;
  uint32_t acc[NW], dacc = 0, cur = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < NW; ++k) acc[k] = 0;
  auto flush = [&]() {
    uint32_t *ac = b.acc + (uint64_t)(__ldcg(b.comp_start + cur) / g.span) * (W + 3);
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const uint32_t wi = k * 32 + lane;
      if (wi < W && acc[k]) atomicXor(ac + wi, acc[k]);
    }
    if (lane < 3 && dacc) atomicXor(ac + W + lane, dacc);
  };
  while (live) {
    uint32_t x[KB][NW], dw[KB], sl[KB];
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      sl[k] = live ? __ffs(live) - 1 : 32u;
      if (live) live &= live - 1;
      if (sl[k] < 32) {
        const uint32_t *pt = b.part + (uint64_t)(s0 + sl[k]) * (W + 3);
        region_load<NW, true>(pt, pt + W, W, lane, x[k], dw[k]);
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

// Partial slots folded per warp.
constexpr uint32_t kPartsPerWarp = 8;

template <int CPS, int NW, int KB>
__global__ void __launch_bounds__(256) k_bv_reduce_parts(BoruvkaGeom g, uint32_t nslots, BoruvkaBufs b) {
  bv_reduce_parts_warp<CPS, NW, KB>(g, nslots, b,
                                    ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kPartsPerWarp,
                                    kPartsPerWarp);
}

// Sampling of component comp when it crosses a span edge (its merged sample is in acc).
template <int CPS>
__device__ void bv_sample_spanning_comp(const BoruvkaGeom &g, const BoruvkaBufs &b, uint32_t round,
                                        uint32_t *flags, uint32_t comp) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t acc_words = (CPS * g.B + 1) * 3;
  const uint32_t s = __ldcg(b.comp_start + comp), e = __ldcg(b.comp_start + comp + 1);
  if (s / g.span == (e - 1) / g.span) return;
  const uint32_t *ac = b.acc + (uint64_t)(s / g.span) * acc_words;
  uint32_t a[CPS][2][3], d[3];
  d[0] = __ldcg(ac + 3 * CPS * g.B);
  d[1] = __ldcg(ac + 3 * CPS * g.B + 1);
  d[2] = __ldcg(ac + 3 * CPS * g.B + 2);
#pragma unroll
  for (int c = 0; c < CPS; ++c)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t j = q * 32 + lane;
      a[c][q][0] = a[c][q][1] = a[c][q][2] = 0;
      if (j < g.B) {
        const uint32_t *bk = ac + 3 * (c * g.B + j);
        a[c][q][0] = __ldcg(bk);
        a[c][q][1] = __ldcg(bk + 1);
        a[c][q][2] = __ldcg(bk + 2);
      }
    }
  uint64_t idx;
  const int res = warp_sample_cols<CPS>(d, a, g.B, g.flip_chk, &idx);
  if (lane == 0) handle_result(res, idx, round, __ldcg(b.comp_key + comp), g, b, flags);
}

template <int CPS>
__global__ void k_bv_sample_spanning(BoruvkaGeom g, BoruvkaBufs b) {
  const uint32_t round = *b.round;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nx = *b.ncross;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nx; i += nwarps)
    bv_sample_spanning_comp<CPS>(g, b, round, b.flags, b.cross[i]);
}

// End of a round (the loop test of boruvka_emulation, src/cc_sketch_alg.cpp:490-509): stop when
// nothing FAILed or merged, or when the next round would ask Sketch::sample for sample
// `samples` (OutOfSamplesException); otherwise start the next round.
// In a query graph (in_graph) the verdict drives its while node; b.ctl[2] carries it for a loop
// run from the host.
__global__ void k_bv_check(BoruvkaBufs b, uint32_t samples, cudaGraphConditionalHandle cond,
                           int in_graph) {
  const uint32_t r = *b.round;
  uint32_t go = 0;
  if (*b.flags == 0) {
    b.ctl[0] = r;
    b.ctl[1] = 0;
  } else if (r + 1 >= samples) {
    b.ctl[0] = r + 1;
    b.ctl[1] = 1;
  } else {
    *b.round = r + 1;
    *b.flags = 0;
    go = 1;
  }
  b.ctl[2] = go;
  if (in_graph) cudaGraphSetConditional(cond, go);
}

__device__ __forceinline__ void bv_final_vertex(uint32_t v, uint32_t *parent, uint32_t *out,
                                                uint32_t *ncc) {
  const uint32_t r = dsu_find(parent, v);
  out[v] = r;
  if (r == v) atomicAdd(ncc, 1u);
}

__global__ void k_bv_final(uint32_t V, uint32_t *parent, uint32_t *out, uint32_t *ncc) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) bv_final_vertex(v, parent, out, ncc);
}

// ---- the whole query in one cooperative launch ------------------------------------------------
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of a cooperative launch: the blocks count their arrivals in *count (zeroed
// before the launch); barrier number k completes at k * gridDim.x arrivals. Writes before it are
// seen by every block after it (fence, arrival, acquire, fence). A block with a failed warp
// (failed = true in any thread) leaves without arriving; a block that waits longer than
// kWaitLimitNs sets the timeout status. Both return false, and the caller returns from the kernel
// (the other blocks then time out at their next barrier).
__device__ bool grid_barrier(uint32_t *count, uint32_t k, bool failed, uint32_t *status) {
  __shared__ uint32_t s_ok;
  if (__syncthreads_or(failed)) return false;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1u);
    const uint32_t target = k * gridDim.x;
    uint32_t ok = 1;
    if (ld_acquire_gpu(count) < target) {
      const uint64_t t0 = global_ns();
      while (ld_acquire_gpu(count) < target) {
        if (global_ns() - t0 > kWaitLimitNs) {
          atomicOr(status, kStatusTimeout);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Batches of the one-launch query's copy rings: NS - 1 of them in flight while one is read (a
// third batch measured no faster than two).
constexpr int kBvQueryRing = 2;

// Exclusive scan of one u64 per thread over a block of 256 threads.
__device__ __forceinline__ uint64_t block_scan_u64_256(uint64_t x, uint64_t *ws /*8*/) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, inc, o);
    if (lane >= (uint32_t)o) inc += y;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  uint64_t pre = 0;
  for (uint32_t k = 0; k < warp; ++k) pre += ws[k];
  __syncthreads();
  return pre + inc - x;
}

// boruvka_emulation (src/cc_sketch_alg.cpp:464-513) in one cooperative launch of 256-thread
// blocks: a fresh DSU, round 0, then per round the phases of the per-phase kernels separated by
// grid barriers -- (1) roots and members per root; (2) each block's exclusive scan of (members |
// 1 << 32) over its range of CH vertices; (3) each block's scan of the blocks' totals, then the
// grouping; (4) the merge over spans, sampling the components inside a span, with the next round's
// counters cleared; (5) the partial slots folded; (6) the components crossing span edges sampled
// -- then the loop test of k_bv_check, taken by every block alike, and the labels. A round's
// "modified" word is b.flags[round % 3]: the word of round r + 1 is cleared during round r, long
// after every block read it as the word of round r - 2.
template <int CPS, int NW, int KB, int KBP>
__global__ void __launch_bounds__(256) k_bv_query(BoruvkaGeom g, const uint32_t *__restrict__ sk_words,
                                                  BoruvkaBufs b, uint32_t samples,
                                                  uint32_t *labels_out, uint32_t *ncc) {
  extern __shared__ __align__(16) uint8_t bv_smem[];
  __shared__ uint64_t s_pref[kBvQueryMaxBlocks + 1];
  __shared__ uint64_t s_ws[8];
  __shared__ RootTable tab;
  const uint32_t V = g.V, nblk = gridDim.x, tid = threadIdx.x;
  const uint32_t W = 3 * CPS * g.B;
  BvRingN<kBvQueryRing> ring;
  ring.init(bv_smem + (tid >> 5) * bv_warp_bytes(W, KB, kBvQueryRing), W, KB);
  uint32_t T = 0;     // batches through this warp's copy ring
  uint32_t nbar = 0;  // grid barriers passed
  bool failed = false;
  auto sync = [&]() { return grid_barrier(b.qbar, ++nbar, failed, b.status); };
  const uint32_t gw = (blockIdx.x * blockDim.x + tid) >> 5, nwarps = (nblk * blockDim.x) >> 5;
  const uint32_t gt = blockIdx.x * blockDim.x + tid, nthreads = nblk * blockDim.x;
  uint32_t *minv = b.trace ? b.minv : nullptr;
  for (uint32_t v = gt; v < V; v += nthreads) {
    b.parent[v] = v;
    b.cnt[v] = 0;
    b.fill[v] = 0;
    if (minv) minv[v] = 0xffffffffu;
  }
  if (gt == 0) {
    *b.forest_n = 0;
    if (b.trace) *b.trace_n = 0;
    b.flags[0] = b.flags[1] = b.flags[2] = 0;
    *b.big = 0xffffffffu;
    *b.ncross = 0;
    *ncc = 0;
  }
  if (!sync()) return;
  failed = !bv_round0_warp<CPS, KB, kBvQueryRing>(g, sk_words, b, b.flags, ring, T, gw, nwarps);
  if (!sync()) return;
  const uint32_t CH = (((V + nblk - 1) / nblk) + 255) & ~255u;  // scan range of a block
  const uint32_t nspans = (V + g.span - 1) / g.span;
  const uint32_t acc_words = (CPS * g.B + 1) * 3;
  uint32_t round = 0;
  for (;;) {
    const uint32_t modified = __ldcg(b.flags + round % 3);
    if (modified == 0 || round + 1 >= samples) {
      if (gt == 0) {
        b.ctl[0] = modified ? round + 1 : round;
        b.ctl[1] = modified ? 1u : 0u;
        b.ctl[2] = 0;
        *b.round = round;
      }
      break;
    }
    ++round;
    uint32_t *flags = b.flags + round % 3;
    // (1)
    if (gt == 0) {
      b.flags[(round + 1) % 3] = 0;
      if (round > 1) *b.ncross = 0;  // the previous round's list was read before the last barrier
    }
    for (uint32_t v0 = blockIdx.x * 512; v0 < V; v0 += nblk * 512)
      bv_label_block<2>(V, v0, b.parent, b.label, b.cnt, minv, tab);
    if (!sync()) return;
    // (2)
    {
      const uint32_t ipt = CH / 256, a = blockIdx.x * CH + tid * ipt;
      uint64_t sum = 0;
      for (uint32_t i = 0; i < ipt; ++i)
        if (a + i < V) {
          const uint32_t c = __ldcg(b.cnt + a + i);
          sum += (uint64_t)c | (c ? (1ull << 32) : 0ull);
        }
      uint64_t run = block_scan_u64_256(sum, s_ws);
      for (uint32_t i = 0; i < ipt; ++i)
        if (a + i < V) {
          const uint32_t c = __ldcg(b.cnt + a + i);
          b.packed[a + i] = run;
          run += (uint64_t)c | (c ? (1ull << 32) : 0ull);
        }
      if (tid == 255) b.btot[blockIdx.x] = run;
    }
    if (!sync()) return;
    // (3)
    {
      const uint32_t per = (nblk + 255) / 256;
      uint64_t sum = 0;
      for (uint32_t k = 0; k < per; ++k) {
        const uint32_t i = tid * per + k;
        if (i < nblk) sum += __ldcg(b.btot + i);
      }
      uint64_t run = block_scan_u64_256(sum, s_ws);
      for (uint32_t k = 0; k < per; ++k) {
        const uint32_t i = tid * per + k;
        if (i < nblk) {
          s_pref[i] = run;
          run += __ldcg(b.btot + i);
        }
      }
      if (tid == 255) s_pref[nblk] = run;
      __syncthreads();
      const uint32_t nc = (uint32_t)(s_pref[nblk] >> 32);
      for (uint32_t v0 = blockIdx.x * 512; v0 < V; v0 += nblk * 512)
        bv_group_block<2>(V, v0, acc_words, g.span, b.label,
                       [&](uint32_t r) { return __ldcg(b.packed + r) + s_pref[r / CH]; }, nc, b.cnt,
                       b.fill, minv, b.order, b.order_comp, b.comp_start, b.comp_key, b.ncomp,
                       b.acc, b.big, b.cross, b.ncross, tab);
    }
    if (!sync()) return;
    // (4)
    for (uint32_t w = gw; w < nspans && !failed; w += nwarps)
      failed = !bv_merge_span<CPS, NW, KB, kBvQueryRing>(g, sk_words, b, round, flags, ring, T, w);
    for (uint32_t v = gt; v < V; v += nthreads) {
      b.cnt[v] = 0;
      b.fill[v] = 0;
      if (minv) minv[v] = 0xffffffffu;
    }
    if (!sync()) return;
    // (5)
    for (uint32_t s0 = gw * kPartsPerWarp; s0 < nspans; s0 += nwarps * kPartsPerWarp)
      bv_reduce_parts_warp<CPS, NW, KBP>(g, nspans, b, s0, kPartsPerWarp);
    if (gt == 0) *b.big = 0xffffffffu;
    if (!sync()) return;
    // (6)
    const uint32_t nx = __ldcg(b.ncross);
    for (uint32_t i = gw; i < nx; i += nwarps)
      bv_sample_spanning_comp<CPS>(g, b, round, flags, __ldcg(b.cross + i));
    if (!sync()) return;
  }
  for (uint32_t v = gt; v < V; v += nthreads) bv_final_vertex(v, b.parent, labels_out, ncc);
}

// Shared-memory bucket-update probe: every thread XORs 96-bit updates into random 12-byte
// buckets of a 16-vertex staged tile with three 32-bit atomicXor each -- the sketch-update
// kernel's per-bucket operation, without hashing or global traffic.
inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ================================================================================================
// host wrappers
// ================================================================================================
uint64_t launch_count() { return g_launches.load(); }
void add_launches(uint64_t n) { g_launches += n; }

cudaError_t smem_optin_fn(const void *fn) {
  static std::mutex mtx;
  static std::set<std::pair<const void *, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mtx);
  if (done.count({fn, dev})) return cudaSuccess;
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa{};
  e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           optin - (int)fa.sharedSizeBytes);
  if (e != cudaSuccess) return e;
  done.insert({fn, dev});
  return cudaSuccess;
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

size_t scan_tmp_words(uint64_t n) {
  size_t w = 0;
  while (n > kScanBlock) {
    n = (n + kScanBlock - 1) / kScanBlock;
    w += n;
  }
  return w + 1;
}

cudaError_t scan_exclusive_u64(uint64_t *d, uint64_t n, uint64_t *total, uint64_t *tmp,
                               cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
  const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb == 1) {
    k_scan_down<<<1, kScanThreads, 0, s>>>(d, n, nullptr, total);
    g_launches++;
    return cudaGetLastError();
  }
  uint64_t *sums = tmp;
  k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(d, n, sums);
  g_launches++;
  cudaError_t e = scan_exclusive_u64(sums, nb, total, tmp + nb, s);
  if (e != cudaSuccess) return e;
  k_scan_down<<<(unsigned)nb, kScanThreads, 0, s>>>(d, n, sums, nullptr);
  g_launches++;
  return cudaGetLastError();
}

constexpr int kCountRpi = 8;  // records per thread per iteration of the counting pass

cudaError_t gutter_count(int input, const void *in, uint64_t n, GutterGeom g, int G,
                         uint64_t *counts, uint32_t *status, cudaStream_t s) {
  const bool smem = g.nbins <= kSmemBinsMax;
  if (input == kInputRecords && smem) {
    auto kern = k_count_records<kCountRpi>;
    const size_t sm = (size_t)((g.nbins + 3) & ~3u) * 4;
    if (sm > 48 * 1024) {
      cudaError_t e = smem_optin(kern);
      if (e != cudaSuccess) return e;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, sm) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    const uint64_t need = (n + 512ull * kCountRpi - 1) / (512ull * kCountRpi);
    const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)num_sms() * per_sm));
    kern<<<blocks, 512, sm, s>>>(reinterpret_cast<const uint8_t *>(in), n, g, counts, status);
    g_launches++;
    return cudaGetLastError();
  }
  if (input == kInputRecords)
    return smem ? launch_gutter<kInputRecords, true, true>(in, n, g, G, counts, nullptr, status, s)
                : launch_gutter<kInputRecords, true, false>(in, n, g, G, counts, nullptr, status, s);
  return smem ? launch_gutter<kInputEntries, true, true>(in, n, g, G, counts, nullptr, status, s)
              : launch_gutter<kInputEntries, true, false>(in, n, g, G, counts, nullptr, status, s);
}

cudaError_t gutter_scatter_global(int input, const void *in, uint64_t n, GutterGeom g, int G,
                                  uint64_t *cursor, uint2 *entries, cudaStream_t s) {
  return input == kInputRecords
             ? launch_gutter<kInputRecords, false, false>(in, n, g, G, cursor, entries, nullptr, s)
             : launch_gutter<kInputEntries, false, false>(in, n, g, G, cursor, entries, nullptr, s);
}


uint32_t sort_scatter_tile(int input, GutterGeom g, size_t smem_budget) {
  const size_t fixed = (size_t)3 * ((g.nbins + 3) & ~3u) * 4 + 64;
  if (g.nbins > kSortBinsMax || fixed >= smem_budget) return 0;
  const size_t per = input == kInputRecords ? 16 : 8;  // records are staged in the entry area
  size_t t = (smem_budget - fixed) / per;
  t = std::min<size_t>(t, input == kInputRecords ? 8192 : 16384);
  t &= ~(size_t)127;
  return (uint32_t)t;
}

cudaError_t gutter_sort_scatter(int input, const void *in, uint64_t n, GutterGeom g,
                                uint32_t rec_tile, const uint64_t *base, uint32_t *fill,
                                uint2 *entries, cudaStream_t s) {
  const size_t nb4 = (g.nbins + 3) & ~3u;
  // records: 16 B of sorted entries per record, which also hold the 9 B staged record (plus the
  // 16-byte alignment slack of the staging) as long as the tile has at least 7 records
  const size_t smem = 3 * nb4 * 4 + (size_t)rec_tile * (input == kInputRecords ? 16 : 8);
  if (input == kInputRecords && rec_tile < 7) return cudaErrorInvalidValue;
  const int G = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)num_sms(),
                                                               (n + rec_tile - 1) / rec_tile));
  if (input == kInputRecords) {
    cudaError_t e = smem_optin(k_gutter_sort_scatter<kInputRecords>);
    if (e != cudaSuccess) return e;
    k_gutter_sort_scatter<kInputRecords><<<G, 1024, smem, s>>>(in, n, g, rec_tile, base, fill, entries);
  } else {
    cudaError_t e = smem_optin(k_gutter_sort_scatter<kInputEntries>);
    if (e != cudaSuccess) return e;
    k_gutter_sort_scatter<kInputEntries><<<G, 1024, smem, s>>>(in, n, g, rec_tile, base, fill, entries);
  }
  g_launches++;
  return cudaGetLastError();
}

cudaError_t gutter_bin_offsets(const uint64_t *scanned, uint32_t stride, uint32_t nbins,
                               const uint64_t *total, uint32_t *bin_off, cudaStream_t s) {
  k_bin_offsets<<<blocks_for(nbins + 1, 256), 256, 0, s>>>(scanned, stride, nbins, total,
                                                           bin_off);
  g_launches++;
  return cudaGetLastError();
}
cudaError_t copy_u64(const uint64_t *src, uint64_t *dst, uint64_t n, cudaStream_t s) {
  k_copy_u64<<<(unsigned)std::min<uint64_t>(blocks_for(n, 256), 4096), 256, 0, s>>>(src, dst, n);
  g_launches++;
  return cudaGetLastError();
}

size_t sketch_update_smem_bytes(SketchGeom g) {
  return ((size_t)g.sketch_words * 4 << g.tile_shift) + kQueueBytes + (size_t)(g.C + 1) * 8;
}

cudaError_t sketch_update_prepare(SketchGeom g, int /*threads*/) {
  (void)g;
  return smem_optin(k_sketch_update);
}

int sketch_update_ctas_per_sm(SketchGeom g, int threads) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sketch_update, threads,
                                                    sketch_update_smem_bytes(g)) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

cudaError_t sketch_update(SketchGeom g, uint8_t *sketches, const uint8_t *gutter,
                          const ChunkTable &chunks, const uint32_t *bin_off, int nchunks,
                          const uint64_t *flip, uint32_t *work_counter, uint32_t *status, int grid,
                          int threads, cudaStream_t s) {
  const size_t smem = sketch_update_smem_bytes(g);
  cudaError_t e = smem_optin(k_sketch_update);
  if (e != cudaSuccess) return e;
  k_sketch_update<<<grid, threads, smem, s>>>(g, sketches, gutter, chunks, bin_off, nchunks, flip,
                                              work_counter, status);
  g_launches++;
  return cudaGetLastError();
}

size_t sketch_update_pipe_smem_bytes(SketchGeom g) {
  return (size_t)g.nbuf * ((size_t)g.sketch_words * 4 << g.tile_shift) + (((size_t)g.C + 2) & ~(size_t)1) * 8;
}

cudaError_t sketch_update_pipe(SketchGeom g, uint8_t *sketches, const uint8_t *gutter,
                               const ChunkTable &chunks, const uint32_t *bin_off, int nchunks,
                               const uint64_t *flip, uint32_t *work_counter, uint32_t *status,
                               int grid, cudaStream_t s) {
  const size_t smem = sketch_update_pipe_smem_bytes(g);
  cudaError_t e = smem_optin(k_sketch_update_pipe);
  if (e != cudaSuccess) return e;
  k_sketch_update_pipe<<<grid, 1024, smem, s>>>(g, sketches, gutter, chunks, bin_off, nchunks, flip,
                                                work_counter, status);
  g_launches++;
  return cudaGetLastError();
}

cudaError_t apply_in_place(int input, const void *in, uint64_t n, SketchGeom g, uint8_t *sketches,
                           const uint64_t *flip, uint32_t *status, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const size_t flip_bytes = (((size_t)g.C + 2) & ~(size_t)1) * 8;
  const size_t smem = flip_bytes + (input == kInputRecords ? kRecStageBytes : 0);
  const uint64_t units = input == kInputRecords ? (n + kRecTile - 1) / kRecTile : (n + 511) / 512;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(units, (uint64_t)num_sms() * 4));
  uint32_t *sk = reinterpret_cast<uint32_t *>(sketches);
  auto launch = [&](auto kern) -> cudaError_t {
    if (smem > 48 * 1024) {
      cudaError_t e = smem_optin(kern);
      if (e != cudaSuccess) return e;
    }
    kern<<<grid, 512, smem, s>>>(in, n, g, sk, flip, status);
    g_launches++;
    return cudaGetLastError();
  };
  if (input == kInputRecords)
    return g.cube ? launch(k_in_place<kInputRecords, true>) : launch(k_in_place<kInputRecords, false>);
  return g.cube ? launch(k_in_place<kInputEntries, true>) : launch(k_in_place<kInputEntries, false>);
}

cudaError_t sketch_xor_raw(uint8_t *sketches, uint32_t words, uint32_t v, const uint32_t *raw,
                           cudaStream_t s) {
  k_sketch_xor_raw<<<blocks_for(words, 256), 256, 0, s>>>(reinterpret_cast<uint32_t *>(sketches),
                                                          words, v, raw);
  g_launches++;
  return cudaGetLastError();
}

__global__ void k_total_xor(const uint32_t *__restrict__ sk, uint32_t V, uint32_t words,
                            uint32_t *total) {
  const uint32_t wd = blockIdx.x * blockDim.x + threadIdx.x;
  if (wd >= words) return;
  uint32_t x = 0;
  for (uint32_t v = blockIdx.y; v < V; v += gridDim.y) x ^= sk[(uint64_t)v * words + wd];
  if (x) atomicXor(total + wd, x);
}

// Launch shape of the round-0 and merge kernels: members per bulk-copy batch, and the dynamic
// shared memory of a 256-thread block (8 warps).
int bv_batch(int cps) { return cps == 1 ? 8 : 1; }
size_t bv_smem_bytes(const BoruvkaGeom &g) {
  return 8 * (size_t)bv_warp_bytes(3 * g.cps * g.B, bv_batch(g.cps));
}
template <class K>
cudaError_t bv_smem_attr(K kern, size_t smem) {
  return smem_optin(kern);
}

cudaError_t sketch_total_xor(const uint8_t *sketches, uint32_t V, uint32_t sketch_words,
                             uint32_t *total, cudaStream_t s) {
  const dim3 grid(blocks_for(sketch_words, 256), std::max<uint32_t>(1, std::min<uint32_t>(V, 512)));
  k_total_xor<<<grid, 256, 0, s>>>(reinterpret_cast<const uint32_t *>(sketches), V, sketch_words, total);
  g_launches++;
  return cudaGetLastError();
}

cudaError_t boruvka_reset(const BoruvkaGeom &g, const BoruvkaBufs &b, cudaStream_t s) {
  k_bv_reset<<<blocks_for(g.V, 256), 256, 0, s>>>(g.V, b.parent);
  g_launches++;
  cudaMemsetAsync(b.forest_n, 0, sizeof(uint32_t), s);
  if (b.trace) cudaMemsetAsync(b.trace_n, 0, sizeof(uint32_t), s);
  return cudaGetLastError();
}

cudaError_t boruvka_round0(const BoruvkaGeom &g, const uint8_t *sketches, const BoruvkaBufs &b,
                           cudaStream_t s) {
  // one warp per 32 vertices, 8 warps per block; a grid of the resident blocks strides on
  const uint32_t *sk = reinterpret_cast<const uint32_t *>(sketches);
  const size_t smem = bv_smem_bytes(g);
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t e = bv_smem_attr(kern, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    const unsigned blocks = std::min<unsigned>(blocks_for((uint64_t)g.V, 256), num_sms() * per_sm);
    kern<<<blocks, 256, smem, s>>>(g, sk, b);
    return cudaSuccess;
  };
  cudaError_t e = g.cps == 1 ? launch(k_bv_round0<1, 8>)
                  : g.cps == 7 ? launch(k_bv_round0<7, 1>) : cudaErrorInvalidValue;
  if (e != cudaSuccess) return e;
  g_launches++;
  return cudaGetLastError();
}

cudaError_t boruvka_round(const BoruvkaGeom &g, const uint8_t *sketches, const BoruvkaBufs &b,
                          cudaStream_t s) {
  const bool trace = b.trace != nullptr;
  const uint32_t V = g.V;
  k_bv_prep<<<blocks_for(V, 256), 256, 0, s>>>(V, b);
  g_launches++;
  k_bv_label<<<blocks_for(V, 256), 256, 0, s>>>(V, b.parent, b.label, b.cnt,
                                                 trace ? b.minv : nullptr);
  g_launches++;
  k_bv_pack<<<blocks_for(V, 256), 256, 0, s>>>(V, b.cnt, b.packed);
  g_launches++;
  cudaError_t e = scan_exclusive_u64(b.packed, V, b.scan_total, b.scan_tmp, s);
  if (e != cudaSuccess) return e;
  if (g.cps != 1 && g.cps != 7) return cudaErrorInvalidValue;
  k_bv_group<<<blocks_for(V, 256), 256, 0, s>>>(V, (g.cps * g.B + 1) * 3, g.span, b.label, b.packed, b.scan_total,
                                                 b.cnt, b.fill, trace ? b.minv : nullptr, b.order,
                                                 b.order_comp, b.comp_start, b.comp_key, b.ncomp,
                                                 b.acc, b.big, b.cross, b.ncross);
  g_launches++;
  const uint64_t warps = (V + g.span - 1) / g.span;
  const uint32_t *sk = reinterpret_cast<const uint32_t *>(sketches);
  const unsigned sblocks = std::min<unsigned>(blocks_for((uint64_t)V * 32, 256), num_sms() * 16);
  const unsigned mblocks = blocks_for(warps * 32, 256);
  const unsigned rblocks = blocks_for((warps + kPartsPerWarp - 1) / kPartsPerWarp * 32, 256);
  const size_t smem = bv_smem_bytes(g);
  if (g.cps == 1 && g.B <= 42) {
    if ((e = bv_smem_attr(k_bv_merge<1, 4, 8>, smem)) != cudaSuccess) return e;
    k_bv_merge<1, 4, 8><<<mblocks, 256, smem, s>>>(g, sk, b);
    k_bv_reduce_parts<1, 4, 8><<<rblocks, 256, 0, s>>>(g, (uint32_t)warps, b);
  } else if (g.cps == 1) {
    if ((e = bv_smem_attr(k_bv_merge<1, 6, 8>, smem)) != cudaSuccess) return e;
    k_bv_merge<1, 6, 8><<<mblocks, 256, smem, s>>>(g, sk, b);
    k_bv_reduce_parts<1, 6, 4><<<rblocks, 256, 0, s>>>(g, (uint32_t)warps, b);
  } else {
    if ((e = bv_smem_attr(k_bv_merge<7, dev::Region<7>::kNW, 1>, smem)) != cudaSuccess) return e;
    k_bv_merge<7, dev::Region<7>::kNW, 1><<<mblocks, 256, smem, s>>>(g, sk, b);
    k_bv_reduce_parts<7, dev::Region<7>::kNW, 1><<<rblocks, 256, 0, s>>>(g, (uint32_t)warps, b);
  }
  g_launches += 2;
  if (g.cps == 1) k_bv_sample_spanning<1><<<sblocks, 256, 0, s>>>(g, b);
  else k_bv_sample_spanning<7><<<sblocks, 256, 0, s>>>(g, b);
  g_launches++;
  return cudaGetLastError();
}

constexpr int kBvQueryBlocksPerSm = 4;

cudaError_t boruvka_query_launch(const BoruvkaGeom &g, uint32_t samples, const uint8_t *sketches,
                                 const BoruvkaBufs &b, uint32_t *labels_out, uint32_t *ncc,
                                 cudaStream_t s) {
  const size_t smem = 8 * (size_t)bv_warp_bytes(3 * g.cps * g.B, bv_batch(g.cps), kBvQueryRing);
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t e = smem_optin(kern);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    // every block resident at once (the launch fails otherwise): a grid barrier never waits for
    // a block that has not started
    const int blocks = std::min<int>(std::min(per_sm, kBvQueryBlocksPerSm) * num_sms(), (int)kBvQueryMaxBlocks);
    e = cudaMemsetAsync(b.qbar, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    BoruvkaGeom a_g = g;
    const uint32_t *a_sk = reinterpret_cast<const uint32_t *>(sketches);
    BoruvkaBufs a_b = b;
    uint32_t a_samples = samples;
    uint32_t *a_labels = labels_out, *a_ncc = ncc;
    void *args[] = {&a_g, &a_sk, &a_b, &a_samples, &a_labels, &a_ncc};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(blocks), dim3(256), args,
                                    smem, s);
    g_launches++;
    return e;
  };
  if (g.cps == 1 && g.B <= 42) return launch(k_bv_query<1, 4, 8, 4>);
  if (g.cps == 1) return launch(k_bv_query<1, 6, 8, 4>);
  if (g.cps == 7) return launch(k_bv_query<7, dev::Region<7>::kNW, 1, 1>);
  return cudaErrorInvalidValue;
}

cudaError_t boruvka_final(const BoruvkaGeom &g, const BoruvkaBufs &b, uint32_t *labels_out,
                          uint32_t *ncc, cudaStream_t s) {
  cudaMemsetAsync(ncc, 0, sizeof(uint32_t), s);
  k_bv_final<<<blocks_for(g.V, 256), 256, 0, s>>>(g.V, b.parent, labels_out, ncc);
  g_launches++;
  return cudaGetLastError();
}

namespace {
cudaError_t build_graph(BoruvkaGraph &q, const BoruvkaGeom &g, uint32_t samples,
                        const uint8_t *sketches, const BoruvkaBufs &b, uint32_t *labels_out,
                        uint32_t *ncc) {
  cudaStream_t cs = nullptr, bs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaGraphCreate(&graph, 0);
  cudaGraphConditionalHandle cond{};
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, graph, 0, cudaGraphCondAssignDefault);
  bool capturing = false;
  if (e == cudaSuccess) {
    e = cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    capturing = e == cudaSuccess;
  }
  // kernels are counted as they are captured (the launch counter is this file's)
  const uint64_t l0 = g_launches.load();
  uint64_t l_body0 = 0, l_body1 = 0;
  if (capturing) {
    // round 0
    e = boruvka_reset(g, b, cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.flags, 0, sizeof(uint32_t), cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.round, 0, sizeof(uint32_t), cs);
    if (e == cudaSuccess) e = boruvka_round0(g, sketches, b, cs);
    if (e == cudaSuccess) {
      k_bv_check<<<1, 1, 0, cs>>>(b, samples, cond, 1);
      e = cudaGetLastError();
    }
    // while (cond) { one round; check }
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &deps, &ndeps);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&wnode, graph, deps, ndeps, &cp);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &wnode, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        l_body0 = g_launches.load();
        cudaError_t eb = boruvka_round(g, sketches, b, bs);
        if (eb == cudaSuccess) {
          k_bv_check<<<1, 1, 0, bs>>>(b, samples, cond, 1);
          eb = cudaGetLastError();
        }
        l_body1 = g_launches.load() + 1;  // + the check kernel
        e = cudaStreamEndCapture(bs, &body);
        if (e == cudaSuccess) e = eb;
      }
    }
    if (e == cudaSuccess) e = boruvka_final(g, b, labels_out, ncc, cs);
    cudaGraph_t out = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &out);
    if (e == cudaSuccess) e = ec;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&q.exec, graph, 0);
  const cudaError_t d1 = bs ? cudaStreamDestroy(bs) : cudaSuccess;
  const cudaError_t d2 = cs ? cudaStreamDestroy(cs) : cudaSuccess;
  if (e == cudaSuccess) e = d1 != cudaSuccess ? d1 : d2;
  if (e == cudaSuccess) {
    // a call whose status was not returned to us must not surface in a later launch's check
    const cudaError_t stale = cudaGetLastError();
    if (stale != cudaSuccess)
      std::fprintf(stderr, "gz: Boruvka query graph built; a runtime call reported %s\n",
                   cudaGetErrorString(stale));
  }
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    q.exec = nullptr;
    return e;
  }
  q.graph = graph;
  const uint64_t captured = g_launches.load() - l0 + 2;  // + the two check kernels
  q.round_kernels = (uint32_t)(l_body1 - l_body0);
  q.fixed_kernels = (uint32_t)(captured - q.round_kernels);
  g_launches -= captured - 2;  // captured, not launched
  q.g = g;
  q.b = b;
  q.sketches = sketches;
  q.labels = labels_out;
  q.ncc = ncc;
  q.samples = samples;
  return cudaSuccess;
}
}  // namespace

cudaError_t boruvka_host_loop(const BoruvkaGeom &g, uint32_t samples, const uint8_t *sketches,
                              const BoruvkaBufs &b, uint32_t *labels_out, uint32_t *ncc,
                              uint32_t *pin, cudaStream_t s) {
  cudaError_t e = boruvka_reset(g, b, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.flags, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.round, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) e = boruvka_round0(g, sketches, b, s);
  for (bool first = true; e == cudaSuccess; first = false) {
    if (!first) e = boruvka_round(g, sketches, b, s);
    if (e != cudaSuccess) break;
    k_bv_check<<<1, 1, 0, s>>>(b, samples, cudaGraphConditionalHandle{}, 0);
    g_launches++;
    e = cudaMemcpyAsync(pin, b.ctl, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || !pin[2]) break;
  }
  if (e == cudaSuccess) e = boruvka_final(g, b, labels_out, ncc, s);
  return e;
}

void boruvka_graph_free(BoruvkaGraph &q) {
  if (q.exec) cudaGraphExecDestroy(q.exec);
  if (q.graph) cudaGraphDestroy(q.graph);
  q.exec = nullptr;
  q.graph = nullptr;
}

cudaError_t boruvka_graph_launch(BoruvkaGraph &q, const BoruvkaGeom &g, uint32_t samples,
                                 const uint8_t *sketches, const BoruvkaBufs &b, uint32_t *labels_out,
                                 uint32_t *ncc, cudaStream_t s) {
  const bool same = q.exec && std::memcmp(&q.g, &g, sizeof(g)) == 0 &&
                    std::memcmp(&q.b, &b, sizeof(b)) == 0 && q.sketches == sketches &&
                    q.labels == labels_out && q.ncc == ncc && q.samples == samples;
  if (!same) {
    boruvka_graph_free(q);
    cudaError_t e = build_graph(q, g, samples, sketches, b, labels_out, ncc);
    if (e != cudaSuccess) return e;
  }
  return cudaGraphLaunch(q.exec, s);
}

}  // namespace gz
