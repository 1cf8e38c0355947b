// gz_common.cuh -- device helpers shared by the single-graph kernels (gz_kernels.cu) and the
// multi-graph engine (gz_batch.cu): bulk async copy + mbarrier PTX, 9-byte record staging,
// the CAS union-find, the warp-cooperative Sketch::sample and the per-entry sketch update.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "gz_device.cuh"
#include "gz_kernels.cuh"

namespace gz {
namespace dev {

constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t fmix32_(uint32_t h) {  // murmur3 finaliser
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// ------------------------------------------------------------------------------------------------
// small PTX helpers (bulk async copy + mbarrier)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait that may suspend the thread for up to hint_ns until the phase completes.
__device__ __forceinline__ bool mbar_try_wait_hint(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase: gives up after limit_ns of wall time.
static __device__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 1; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 31u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr uint32_t kBulkPiece = 32768;       // bytes per bulk copy instruction
constexpr uint64_t kWaitLimitNs = 2000000000;  // 2 s bound on any device-side wait

// ------------------------------------------------------------------------------------------------
// record staging: coalesced 128-bit loads of a range of packed 9-byte records into shared memory
// ------------------------------------------------------------------------------------------------
constexpr uint32_t kRecStageBytes = kRecTile * 9 + 48;

// Loads records [r, r + cnt) into s. Shared byte k mirrors global byte align16(start) + k.
// Whole 16-byte blocks inside the range use one 128-bit load; the partial first/last block is
// read byte by byte so no byte outside the caller's range is touched. Returns the offset of
// record r inside s.
__device__ __forceinline__ uint32_t stage_records(const uint8_t *base, uint64_t r, uint32_t cnt,
                                                  uint8_t *s) {
  const uintptr_t start = (uintptr_t)(base + r * 9);
  const uintptr_t end = start + (uintptr_t)cnt * 9;
  const uintptr_t a0 = start & ~(uintptr_t)15;
  const uint32_t nvec = (uint32_t)((((end + 15) & ~(uintptr_t)15) - a0) >> 4);
  for (uint32_t i = threadIdx.x; i < nvec; i += blockDim.x) {
    const uintptr_t blk = a0 + ((uintptr_t)i << 4);
    if (blk >= start && blk + 16 <= end) {
      *reinterpret_cast<uint4 *>(s + i * 16) = __ldcs(reinterpret_cast<const uint4 *>(blk));
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uintptr_t p = blk + k;
        if (p >= start && p < end) s[i * 16 + k] = *reinterpret_cast<const uint8_t *>(p);
      }
    }
  }
  return (uint32_t)(start - a0);
}

// src / dst of record i of the stream [rec, rec_end) straight from global memory: three 4-byte
// loads (through L1, which a warp's 32 consecutive records share) from the aligned words that
// hold bytes 9i + 1 .. 9i + 8, or byte loads where those words would reach outside the stream.
__device__ __forceinline__ void load_record(const uint8_t *rec, const uint8_t *rec_end, uint64_t i,
                                            uint32_t &u, uint32_t &v) {
  const uint8_t *p = rec + 9 * i + 1;
  const uintptr_t w0 = (uintptr_t)p & ~(uintptr_t)3;
  if (w0 >= (uintptr_t)rec && w0 + 12 <= (uintptr_t)rec_end) {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(w0);
    const uint32_t a0 = __ldg(w), a1 = __ldg(w + 1), a2 = __ldg(w + 2);
    const uint32_t sh = ((uintptr_t)p & 3) * 8;
    u = __funnelshift_r(a0, a1, sh);
    v = __funnelshift_r(a1, a2, sh);
  } else {
    u = v = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      u |= (uint32_t)__ldg(p + k) << (8 * k);
      v |= (uint32_t)__ldg(p + 4 + k) << (8 * k);
    }
  }
}

// src / dst of staged record i (the type byte is not needed).
__device__ __forceinline__ void parse_record(const uint8_t *s, uint32_t shift, uint32_t i,
                                             uint32_t &u, uint32_t &v) {
  const uint32_t off = shift + 9 * i + 1;
  const uint32_t *w = reinterpret_cast<const uint32_t *>(s) + (off >> 2);
  const uint32_t sh = (off & 3) * 8;
  u = __funnelshift_r(w[0], w[1], sh);
  v = __funnelshift_r(w[1], w[2], sh);
}


// Folds one endpoint update (vertex v, neighbour w) into v's staged sketch: the deterministic
// bucket always, then in each column the bucket at depth ctz(hash_c(idx) | 1 << B) when < B.
// Columns are hashed two at a time: the two XXH3 chains are independent, which hides the
// latency of each other's dependent integer ops.
__device__ __forceinline__ void xor_bucket(uint32_t *bk, uint32_t lo, uint32_t hi, uint32_t chk) {
  atomicXor(bk, lo);
  atomicXor(bk + 1, hi);
  atomicXor(bk + 2, chk);
}
__device__ __forceinline__ void apply_entry(uint2 e, uint32_t *s_sk, uint32_t vmask,
                                            uint32_t sketch_words, const uint64_t *s_flip,
                                            uint64_t flip_chk, uint32_t C, uint32_t B) {
  const uint32_t v = e.x, w = e.y;
  const uint32_t lo = max(v, w), hi = min(v, w);  // idx = (min << 32) | max
  uint32_t *sk = s_sk + (v & vmask) * sketch_words;
  const uint64_t in64 = ((uint64_t)lo << 32) | hi;
  const uint32_t chk = hash_lo32(in64 ^ flip_chk);
  xor_bucket(sk + 3 * C * B, lo, hi, chk);
  uint32_t c = 0;
  // four independent hash chains per step keep the integer pipes fed between dependent ops
  for (; c + 3 < C; c += 4) {
    const uint32_t d0 = hash_depth(in64 ^ s_flip[c], B);
    const uint32_t d1 = hash_depth(in64 ^ s_flip[c + 1], B);
    const uint32_t d2 = hash_depth(in64 ^ s_flip[c + 2], B);
    const uint32_t d3 = hash_depth(in64 ^ s_flip[c + 3], B);
    if (d0 < B) xor_bucket(sk + 3 * (c * B + d0), lo, hi, chk);
    if (d1 < B) xor_bucket(sk + 3 * ((c + 1) * B + d1), lo, hi, chk);
    if (d2 < B) xor_bucket(sk + 3 * ((c + 2) * B + d2), lo, hi, chk);
    if (d3 < B) xor_bucket(sk + 3 * ((c + 3) * B + d3), lo, hi, chk);
  }
  for (; c < C; ++c) {
    const uint32_t d = hash_depth(in64 ^ s_flip[c], B);
    if (d < B) xor_bucket(sk + 3 * (c * B + d), lo, hi, chk);
  }
}


// Exclusive scan over the 1024 threads of a block (one value per thread).
__device__ __forceinline__ uint32_t block_scan_1024(uint32_t x, uint32_t *ws /*32*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    ws[lane] = w;
  }
  __syncthreads();
  const uint32_t r = (warp ? ws[warp - 1] : 0) + inc - x;
  __syncthreads();
  return r;
}


// apply_entry on an unstaged sketch in global memory: the bucket XORs are global atomics (used
// when a tile has too few entries to pay for staging it). gsk = the graph's first sketch.
__device__ __forceinline__ void apply_entry_global(uint2 e, uint32_t *gsk, uint32_t sketch_words,
                                                   const uint64_t *s_flip, uint64_t flip_chk,
                                                   uint32_t C, uint32_t B) {
  const uint32_t v = e.x, w = e.y;
  const uint32_t lo = max(v, w), hi = min(v, w);
  uint32_t *sk = gsk + (uint64_t)v * sketch_words;
  const uint64_t in64 = ((uint64_t)lo << 32) | hi;
  const uint32_t chk = hash_lo32(in64 ^ flip_chk);
  xor_bucket(sk + 3 * C * B, lo, hi, chk);
  uint32_t c = 0;
  for (; c + 1 < C; c += 2) {
    const uint32_t d0 = hash_depth(in64 ^ s_flip[c], B);
    const uint32_t d1 = hash_depth(in64 ^ s_flip[c + 1], B);
    if (d0 < B) xor_bucket(sk + 3 * (c * B + d0), lo, hi, chk);
    if (d1 < B) xor_bucket(sk + 3 * ((c + 1) * B + d1), lo, hi, chk);
  }
  if (c < C) {
    const uint32_t d = hash_depth(in64 ^ s_flip[c], B);
    if (d < B) xor_bucket(sk + 3 * (c * B + d), lo, hi, chk);
  }
}


// CubeSketch update (src/sketch.cpp:50-67, the reference built with -DL0_SAMPLING): the
// deterministic bucket, then in each column every bucket of depth 0..d when d < B.
__device__ __forceinline__ void apply_entry_cube(uint2 e, uint32_t *sk_base, uint32_t vmask,
                                                 uint32_t sketch_words, const uint64_t *s_flip,
                                                 uint64_t flip_chk, uint32_t C, uint32_t B) {
  const uint32_t v = e.x, w = e.y;
  const uint32_t lo = max(v, w), hi = min(v, w);
  uint32_t *sk = sk_base + (uint64_t)(v & vmask) * sketch_words;
  const uint64_t in64 = ((uint64_t)lo << 32) | hi;
  const uint32_t chk = hash_lo32(in64 ^ flip_chk);
  xor_bucket(sk + 3 * C * B, lo, hi, chk);
  for (uint32_t c = 0; c < C; ++c) {
    const uint32_t d = hash_depth(in64 ^ s_flip[c], B);
    if (d < B)
      for (uint32_t j = 0; j <= d; ++j) xor_bucket(sk + 3 * (c * B + j), lo, hi, chk);
  }
}

// One update (u, v) XORed in place (global memory) into the sketch su of u and, when sv is not
// null, into the sketch sv of v; hashed once, since the checksum and each column's depth are
// the same for both endpoints. CUBE selects the CubeSketch rule (depths 0..d) over
// CameoSketch's (depth d).
template <bool CUBE>
__device__ __forceinline__ void xor_update_in_place(uint32_t *su, uint32_t *sv, uint32_t u, uint32_t v,
                                                    const uint64_t *s_flip, uint64_t flip_chk,
                                                    uint32_t C, uint32_t B) {
  const uint32_t lo = max(u, v), hi = min(u, v);
  const uint64_t in64 = ((uint64_t)lo << 32) | hi;
  const uint32_t chk = hash_lo32(in64 ^ flip_chk);
  xor_bucket(su + 3 * C * B, lo, hi, chk);
  if (sv) xor_bucket(sv + 3 * C * B, lo, hi, chk);
  for (uint32_t c = 0; c < C; ++c) {
    const uint32_t d = hash_depth(in64 ^ s_flip[c], B);
    if (d < B) {
      for (uint32_t j = CUBE ? 0 : d; j <= d; ++j) {
        xor_bucket(su + 3 * (c * B + j), lo, hi, chk);
        if (sv) xor_bucket(sv + 3 * (c * B + j), lo, hi, chk);
      }
    }
  }
}

// warp_sample over NC columns merged in registers (lane j holds buckets j and j + 32 of each
// column): the deterministic bucket, then columns 0..NC-1 in order, depths 0..B-1 in each --
// Sketch::sample's scan over a sample's columns (src/sketch.cpp:94-116).
template <int NC>
__device__ __forceinline__ int warp_sample_cols(const uint32_t (&d)[3], const uint32_t (&a)[NC][2][3],
                                                uint32_t B, uint64_t flip_chk, uint64_t *idx) {
  const int lane = threadIdx.x & 31;
  if ((d[0] | d[1] | d[2]) == 0) {
    *idx = 0;
    return 1;  // ZERO
  }
  if (bucket_good(d[0], d[1], d[2], flip_chk)) {
    *idx = ((uint64_t)d[1] << 32) | d[0];
    return 0;  // GOOD
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      if ((uint32_t)s * 32 >= B) break;
      const uint32_t j = s * 32 + lane;
      const bool good = j < B && bucket_good(a[c][s][0], a[c][s][1], a[c][s][2], flip_chk);
      const uint32_t m = __ballot_sync(kFull, good);
      if (m) {
        const int src = __ffs(m) - 1;
        const uint32_t x0 = __shfl_sync(kFull, a[c][s][0], src);
        const uint32_t x1 = __shfl_sync(kFull, a[c][s][1], src);
        *idx = ((uint64_t)x1 << 32) | x0;
        return 0;
      }
    }
  }
  *idx = 0;
  return 2;  // FAIL
}


// ---- sample regions in word space --------------------------------------------------------------
// The columns of one sample (CPS consecutive columns, column-major) are one contiguous run of
// W = 3 * CPS * B words, and merging sketches is a plain XOR of those words. The query kernels
// therefore load, XOR and combine a region as W words spread over the warp (lane l holds words
// l, l + 32, ...; fully coalesced), plus the deterministic bucket's 3 words on lanes 0..2, and
// go to bucket order only to sample, through a per-warp shared-memory stage.
template <int CPS>
struct Region {
  static constexpr int kNW = (3 * CPS * 64 + 31) / 32;  // word slots per lane (B <= 64)
};

// Load region words [0, W) at src and the deterministic bucket at det into x / dw (CG: through
// L2 only, for words written earlier in the same kernel by another SM).
template <int NW, bool CG = false>
__device__ __forceinline__ void region_load(const uint32_t *__restrict__ src,
                                            const uint32_t *__restrict__ det, uint32_t W,
                                            uint32_t lane, uint32_t (&x)[NW], uint32_t &dw) {
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const uint32_t w = k * 32 + lane;
    x[k] = w < W ? (CG ? __ldcg(src + w) : src[w]) : 0u;
  }
  dw = lane < 3 ? (CG ? __ldcg(det + lane) : det[lane]) : 0u;
}

// Sketch::sample (src/sketch.cpp:94-116) of a region in shared memory: s[0, 3 * CPS * B) the
// columns, det[0, 3) the deterministic bucket; the deterministic bucket first, then columns
// 0..CPS-1, depths 0..B-1 in each, the first good bucket wins (ballot + lowest lane). Returns 0
// GOOD / 1 ZERO / 2 FAIL.
template <int CPS>
__device__ __forceinline__ int warp_sample_smem_split(const uint32_t *s, const uint32_t *det,
                                                      uint32_t B, uint64_t flip_chk, uint64_t *idx) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t d0 = det[0], d1 = det[1], d2 = det[2];
  if ((d0 | d1 | d2) == 0) {
    *idx = 0;
    return 1;  // ZERO
  }
  if (bucket_good(d0, d1, d2, flip_chk)) {
    *idx = ((uint64_t)d1 << 32) | d0;
    return 0;  // GOOD
  }
  int res = 2;
  *idx = 0;
#pragma unroll
  for (int c = 0; c < CPS && res == 2; ++c) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if ((uint32_t)q * 32 >= B || res != 2) break;
      const uint32_t j = q * 32 + lane;
      uint32_t a0 = 0, a1 = 0, a2 = 0;
      if (j < B) {
        const uint32_t *bk = s + 3 * (c * B + j);
        a0 = bk[0];
        a1 = bk[1];
        a2 = bk[2];
      }
      const bool good = j < B && bucket_good(a0, a1, a2, flip_chk);
      const uint32_t m = __ballot_sync(kFull, good);
      if (m) {
        const int src = __ffs(m) - 1;
        const uint32_t x0 = __shfl_sync(kFull, a0, src);
        const uint32_t x1 = __shfl_sync(kFull, a1, src);
        *idx = ((uint64_t)x1 << 32) | x0;
        res = 0;
      }
    }
  }
  return res;
}

// The same with the deterministic bucket right after the columns: s[W, W + 3).
template <int CPS>
__device__ __forceinline__ int warp_sample_smem(const uint32_t *s, uint32_t W, uint32_t B,
                                                uint64_t flip_chk, uint64_t *idx) {
  return warp_sample_smem_split<CPS>(s, s + W, B, flip_chk, idx);
}

// ---- bulk-copied bucket runs (cp.async.bulk) -----------------------------------------------------
// One lane moves a member's whole bucket run with one bulk copy instead of every lane issuing
// 4-byte copies. A bulk copy needs 16-byte-aligned addresses and sizes, so the 16-byte-aligned
// superset of the run is copied (up to 15 bytes either side, inside the sketch buffer's tail
// padding at the end) and the run starts (p & 15) bytes into its slot.
__host__ __device__ constexpr uint32_t bulk_run_cap(uint32_t words) {  // slot bytes for a run
  return (words * 4 + 12 + 15) & ~15u;
}
__device__ __forceinline__ uint32_t bulk_run_bytes(const uint32_t *p, uint32_t words) {
  const uintptr_t a = (uintptr_t)p & ~(uintptr_t)15, e = ((uintptr_t)(p + words) + 15) & ~(uintptr_t)15;
  return (uint32_t)(e - a);
}
__device__ __forceinline__ void bulk_run_copy(uint8_t *slot, const uint32_t *p, uint32_t words, uint32_t bar) {
  const uintptr_t a = (uintptr_t)p & ~(uintptr_t)15;
  bulk_g2s(smem_u32(slot), reinterpret_cast<const void *>(a), bulk_run_bytes(p, words), bar);
}
__device__ __forceinline__ const uint32_t *bulk_run_at(const uint8_t *slot, const uint32_t *p) {
  return reinterpret_cast<const uint32_t *>(slot + ((uintptr_t)p & 15));
}

// Shared memory of the query kernels' bulk-copy rings, per warp: NS batches of KB member slots
// (a slot holds the 16-byte-aligned supersets of a member's column run, up to Wmax words, and of
// its deterministic bucket), one stage of Wmax + 3 words, and one mbarrier per batch.
__host__ __device__ constexpr uint32_t bv_slot_bytes(uint32_t Wmax) { return bulk_run_cap(Wmax) + bulk_run_cap(3); }
__host__ __device__ constexpr uint32_t bv_warp_bytes(uint32_t Wmax, int KB, int NS = 2) {
  return NS * KB * bv_slot_bytes(Wmax) + (((Wmax + 3) * 4 + 15) & ~15u) + ((8 * NS + 15) & ~15u);
}

// A warp's NS batch buffers: init of their mbarriers (one arrival: lane 0's expect_tx), issue of
// a batch's bulk copies, and the bounded wait for a batch. Batch t uses buffer t % NS; its
// barrier completes its (t / NS)-th phase.
template <int NS>
struct BvRingN {
  uint8_t *slots;   // NS * KB slots
  uint32_t *stage;  // Wmax + 3 words
  uint64_t *bars;   // NS
  uint32_t slot_bytes, run_cap;
  __device__ void init(uint8_t *warp_smem, uint32_t Wmax, int KB) {
    run_cap = bulk_run_cap(Wmax);
    slot_bytes = bv_slot_bytes(Wmax);
    slots = warp_smem;
    stage = reinterpret_cast<uint32_t *>(warp_smem + NS * KB * slot_bytes);
    bars = reinterpret_cast<uint64_t *>(warp_smem + NS * KB * slot_bytes + (((Wmax + 3) * 4 + 15) & ~15u));
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
      for (int i = 0; i < NS; ++i) mbar_init(smem_u32(&bars[i]), 1);
      mbar_fence_init();
    }
    __syncwarp();
  }
  __device__ uint8_t *slot(uint32_t t, uint32_t k, int KB) const { return slots + ((t % NS) * KB + k) * slot_bytes; }
  // Lane k < KB with `mine` copies its run [run, run + words) (words <= Wmax) and its
  // deterministic bucket det into slot k of batch t; lane 0 arms the batch's barrier with the
  // bytes of the whole batch first. Every lane of the warp calls it.
  __device__ void issue(uint32_t t, bool mine, const uint32_t *run, uint32_t words, const uint32_t *det, int KB) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t bar = smem_u32(&bars[t % NS]);
    const uint32_t bytes = mine ? bulk_run_bytes(run, words) + bulk_run_bytes(det, 3) : 0;
    const uint32_t total = __reduce_add_sync(kFull, bytes);
    // this lane's reads of the slots about to be overwritten, before the async proxy writes
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      if (total) mbar_expect_tx(bar, total);
      else mbar_arrive(bar);
    }
    __syncwarp();
    if (mine) {
      uint8_t *sl = slot(t, lane, KB);
      bulk_run_copy(sl, run, words, bar);
      bulk_run_copy(sl + run_cap, det, 3, bar);
    }
  }
  // The thread sleeps in the barrier (20 us per try) instead of spinning; limit_ns bounds the wait.
  __device__ bool wait(uint32_t t) const {
    const uint32_t bar = smem_u32(&bars[t % NS]), parity = (t / NS) & 1;
    bool ok = mbar_try_wait_hint(bar, parity, 20000);
    if (!ok) {
      const uint64_t t0 = global_ns();
      while (!(ok = mbar_try_wait_hint(bar, parity, 20000)) && global_ns() - t0 < kWaitLimitNs) {
      }
    }
    return __all_sync(kFull, ok);
  }
};
using BvRing = BvRingN<2>;

// Warp-aggregated counter add: lanes in `active` holding the same key add one each to ctr[key]
// with one atomic per distinct key; returns this lane's slot (old value + rank among its key's
// lanes). stage is a 32-word per-warp shared array used to hand the base to the key's lanes.
__device__ __forceinline__ uint32_t warp_agg_inc(uint32_t *ctr, uint32_t key, uint32_t active,
                                                 uint32_t *stage) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t peers = __match_any_sync(active, key);
  const uint32_t leader = __ffs(peers) - 1;
  if (lane == leader) stage[lane] = atomicAdd(ctr + key, (uint32_t)__popc(peers));
  __syncwarp(active);
  const uint32_t base = stage[leader];
  __syncwarp(active);
  return base + __popc(peers & ((1u << lane) - 1u));
}

struct TraceRec {
  uint32_t round, key, result, pad;
  uint64_t idx;
};


// Total order used to link roots (lower rank goes under higher): no cycles can form, the same
// role as the random priorities of DisjointSetUnion_MT::order_edge (include/dsu.h:113-117).
__device__ __forceinline__ uint64_t rank_of(uint32_t x) {
  return ((uint64_t)fmix32_(x) << 32) | x;
}

// find_root with path halving (include/dsu.h:145-152); loads/stores go to L2 so updates by other
// SMs are seen.
static __device__ uint32_t dsu_find(uint32_t *parent, uint32_t x) {
  for (;;) {
    const uint32_t p = __ldcg(parent + x);
    if (p == x) return x;
    const uint32_t gp = __ldcg(parent + p);
    if (gp == p) return p;
    __stcg(parent + x, gp);
    x = gp;
  }
}

// merge with CAS (include/dsu.h:155-167). Returns true when this call linked two roots.
static __device__ bool dsu_unite(uint32_t *parent, uint32_t a, uint32_t b) {
  for (;;) {
    a = dsu_find(parent, a);
    b = dsu_find(parent, b);
    if (a == b) return false;
    if (rank_of(a) < rank_of(b)) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(parent + b, b, a) == b) return true;
  }
}

// Sketch::sample (src/sketch.cpp:94-116) on one merged column held one or two buckets per lane
// (lane j holds bucket j and j + 32) plus the deterministic bucket (same on every lane).
__device__ __forceinline__ int warp_sample(const uint32_t (&d)[3], const uint32_t (&a)[2][3],
                                           uint32_t B, uint64_t flip_chk, uint64_t *idx) {
  const int lane = threadIdx.x & 31;
  if ((d[0] | d[1] | d[2]) == 0) {
    *idx = 0;
    return 1;  // ZERO
  }
  if (bucket_good(d[0], d[1], d[2], flip_chk)) {
    *idx = ((uint64_t)d[1] << 32) | d[0];
    return 0;  // GOOD
  }
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    if ((uint32_t)s * 32 >= B) break;
    const uint32_t j = s * 32 + lane;
    const bool good = j < B && bucket_good(a[s][0], a[s][1], a[s][2], flip_chk);
    const uint32_t m = __ballot_sync(kFull, good);
    if (m) {
      const int src = __ffs(m) - 1;
      const uint32_t x0 = __shfl_sync(kFull, a[s][0], src);
      const uint32_t x1 = __shfl_sync(kFull, a[s][1], src);
      *idx = ((uint64_t)x1 << 32) | x0;
      return 0;
    }
  }
  *idx = 0;
  return 2;  // FAIL
}


}  // namespace dev
}  // namespace gz
