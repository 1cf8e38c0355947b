// gz_planes.cu -- coded-entry record ingest for CameoSketch sketches of at most 31 columns.
//
// Sketch::update (src/sketch.cpp:69-83) XORs an edge index and its checksum into the
// deterministic bucket and into bucket (c, depth_c(idx)) of every column c, and
// CCSketchAlg::update / apply_update_batch (src/cc_sketch_alg.cpp:106-133) apply it to both
// endpoint sketches. Every vertex sketch uses the same seed (src/cc_sketch_alg.cpp:21), so the two
// endpoints get the same depths and the same checksum.
//
//   k_hash_sort_scatter  per tile of records: the two endpoint entries counting-sorted by gutter
//                        bin in shared memory, each record's C column depths hashed once into
//                        4-bit (or 3-bit) codes carried by both entries, the runs written out
//                        coalesced.
//   k_plane_update       per tile of W vertices: the tile's entries (filtered out of their gutter
//                        bin when a bin holds several tiles) XORed into bucket planes in shared
//                        memory that start at zero, then each vertex's rows XORed into its sketch
//                        in HBM. The checksum is hashed here, per entry.
// A coded entry is 128 bits: the C codes in bits 0 .. 4C - 1 (column c in bits 4c .. 4c + 3),
// then the neighbour shifted left by bin_shift bits OR the vertex's offset inside its gutter bin
// (the bin is known from where the entry lies). It is used when 4C + bin_shift + the neighbour's
// bits fit in 128 (every CameoSketch up to 2^18 vertices). Past that, codes of 3 bits (code 7 =
// depth 7 or more) fit larger graphs (3C + bin_shift + neighbour bits <= 128: 2^20 vertices and
// far beyond); an escaped column (1 in 128 column updates) is hashed again where the entry is
// applied, so the planes see the same 4-bit codes either way.
//
// Bucket planes. A warp takes 32 entries, one per lane. At step t = 0..31 lane l handles slot
// l ^ t of its entry: slot c < C is column c, slot C the deterministic bucket, higher slots are
// unused. A plane row is 32 words, so slot s is shared-memory bank s and the 32 lanes of a step hit
// 32 different banks whatever their vertices and depths: the red.shared.xor never conflict (the
// per-entry ordering, every lane on column c at once, concentrates lanes on a few banks because
// depth 0 takes half the updates). Each bucket is kept as three words,
//   A = XOR of (neighbour | 1 << 31) over the entries whose neighbour is above the vertex,
//   B = the same over the other entries,
//   G = XOR of their checksums,
// so one update XORs two words (A or B, and G) instead of three. With idx = (min << 32) | max
// (concat_pairing_fn, src/util.cpp:45-51) the bucket's alpha is recovered as
//   alpha low  = low31(A) ^ (top bit of B ? vertex : 0),
//   alpha high = low31(B) ^ (top bit of A ? vertex : 0),
// the top bits holding the parity of each kind's entry count (vertex ids are below 2^31).
// Rows hold depths 0 .. kPlaneRows - 2; the last row is scratch. Depths at or above it (2^-11 of
// the column updates) are XORed into the sketch in HBM with global atomics; those rows are never
// touched by the write-back, which rewrites only the rows the planes hold.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "gz_common.cuh"
#include "gz_device.cuh"
#include "gz_kernels.cuh"

namespace gz {

namespace {

using namespace gz::dev;

constexpr uint32_t kPlaneThr = kPlaneRows - 1;               // first depth not held in the planes
constexpr uint32_t kPlaneBytes = kPlaneRows * kPlaneSlots * 4;  // one plane of one vertex
// Planes of one vertex: A, its checksums GA, B, its checksums GB. Each checksum plane sits one
// plane after the plane it pairs with, so a slot step's second address is the first plus a
// constant (an immediate of the reduction) whichever of A and B the entry goes to; the sketch's
// checksum word is GA ^ GB.
constexpr uint32_t kVertBytes = 4 * kPlaneBytes;
constexpr uint32_t kQueueSlots = 64;                          // per-warp queue of filtered entries
constexpr uint32_t kWbWords = kQueueSlots * 4;                // per-warp buffer: the entry queue

// Depth codes of all C columns into the nibble words w (column c in bits 4(c % 8) of word c / 8;
// nibbles past C are zero); pm = premixed edge index. Every sketch has at least 18 columns: the
// first 18 are unrolled, the rest a loop of exactly C - 18 steps.
__device__ __forceinline__ void all_codes(uint64_t pm, const uint64_t *kcol, uint32_t C,
                                          uint32_t cap, uint32_t (&w)[4]) {
  w[0] = w[1] = 0;
#pragma unroll
  for (int c = 0; c < 16; ++c) w[c >> 3] |= depth_code(pm ^ kcol[c], cap) << (4 * (c & 7));
  uint64_t hiw = (uint64_t)depth_code(pm ^ kcol[16], cap) |
                 ((uint64_t)depth_code(pm ^ kcol[17], cap) << 4);
#pragma unroll 2
  for (uint32_t c = 18; c < C; ++c) hiw |= (uint64_t)depth_code(pm ^ kcol[c], cap) << (4 * (c - 16));
  w[2] = (uint32_t)hiw;
  w[3] = (uint32_t)(hiw >> 32);
}

// Coded entry of vertex a (neighbour b): the codes, then from bit 4C the payload
// (b << bin_shift) | (a & bin mask).
__device__ __forceinline__ uint4 pack_entry(const uint32_t (&w)[4], uint32_t a, uint32_t b,
                                            uint32_t C, uint32_t bin_shift) {
  const uint64_t pay = ((uint64_t)b << bin_shift) | (a & ((1u << bin_shift) - 1u));
  const uint64_t hi = (((uint64_t)w[3] << 32) | w[2]) | (pay << (4 * C - 64));
  return make_uint4(w[0], w[1], (uint32_t)hi, (uint32_t)(hi >> 32));
}

// Vertex, neighbour and codes of a coded entry lying in gutter bin `bin`.
__device__ __forceinline__ void unpack_entry(uint4 e, uint32_t bin, uint32_t C, uint32_t bin_shift,
                                             uint32_t &v, uint32_t &u, uint32_t (&w)[4]) {
  const uint64_t hi = ((uint64_t)e.w << 32) | e.z;
  const uint32_t sh = 4 * C - 64;
  const uint64_t pay = hi >> sh;
  const uint64_t codes_hi = hi & ((1ull << sh) - 1ull);
  v = (bin << bin_shift) | ((uint32_t)pay & ((1u << bin_shift) - 1u));
  u = (uint32_t)(pay >> bin_shift);
  w[0] = e.x;
  w[1] = e.y;
  w[2] = (uint32_t)codes_hi;
  w[3] = (uint32_t)(codes_hi >> 32);
}

// 3-bit codes (kEntryCoded3). Eight nibbles holding values <= 7 <-> their low 3 bits packed into
// 24 bits (nibble k at bits 3k .. 3k + 2), in three steps of pairs.
__device__ __forceinline__ uint32_t squeeze3(uint32_t w) {
  w = (w & 0x07070707u) | ((w >> 1) & 0x38383838u);
  w = (w & 0x003f003fu) | ((w >> 2) & 0x0fc00fc0u);
  return (w & 0x00000fffu) | ((w >> 4) & 0x00fff000u);
}
__device__ __forceinline__ uint32_t spread3(uint32_t x) {
  x = (x & 0x00000fffu) | ((x << 4) & 0x0fff0000u);
  x = (x & 0x003f003fu) | ((x << 2) & 0x3f003f00u);
  return (x & 0x07070707u) | ((x << 1) & 0x70707070u);
}

// Coded entry with 3-bit codes of vertex a (neighbour b): codes (each <= 7, as nibbles in w) in
// bits 0 .. 3C - 1, then from bit 3C the payload (b << bin_shift) | (a & bin mask). 3C >= 54.
__device__ __forceinline__ uint4 pack_entry3(const uint32_t (&w)[4], uint32_t a, uint32_t b,
                                             uint32_t C, uint32_t bin_shift) {
  const uint64_t z2 = squeeze3(w[2]);
  uint64_t lo = (uint64_t)squeeze3(w[0]) | ((uint64_t)squeeze3(w[1]) << 24) | (z2 << 48);
  uint64_t hi = (z2 >> 16) | ((uint64_t)squeeze3(w[3]) << 8);
  const uint64_t pay = ((uint64_t)b << bin_shift) | (a & ((1u << bin_shift) - 1u));
  const uint32_t sh = 3 * C;
  if (sh >= 64) {
    hi |= pay << (sh - 64);
  } else {
    lo |= pay << sh;
    hi |= pay >> (64 - sh);
  }
  return make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}

// Payload (bits from 3C on) of a 3-bit coded entry.
__device__ __forceinline__ uint64_t payload3(uint4 e, uint32_t C) {
  const uint64_t lo = ((uint64_t)e.y << 32) | e.x, hi = ((uint64_t)e.w << 32) | e.z;
  const uint32_t sh = 3 * C;
  return sh >= 64 ? hi >> (sh - 64) : (lo >> sh) | (hi << (64 - sh));
}

// Vertex, neighbour and codes (as nibbles, escapes = 7 left in place) of a 3-bit coded entry
// lying in gutter bin `bin`.
__device__ __forceinline__ void unpack_entry3(uint4 e, uint32_t bin, uint32_t C, uint32_t bin_shift,
                                              uint32_t &v, uint32_t &u, uint32_t (&w)[4]) {
  uint64_t lo = ((uint64_t)e.y << 32) | e.x, hi = ((uint64_t)e.w << 32) | e.z;
  const uint32_t sh = 3 * C;
  const uint64_t pay = sh >= 64 ? hi >> (sh - 64) : (lo >> sh) | (hi << (64 - sh));
  v = (bin << bin_shift) | ((uint32_t)pay & ((1u << bin_shift) - 1u));
  u = (uint32_t)(pay >> bin_shift);
  if (sh >= 64) {
    hi &= (1ull << (sh - 64)) - 1ull;
  } else {
    lo &= (1ull << sh) - 1ull;
    hi = 0;
  }
  w[0] = spread3((uint32_t)lo & 0xffffffu);
  w[1] = spread3((uint32_t)(lo >> 24) & 0xffffffu);
  w[2] = spread3((uint32_t)((lo >> 48) | (hi << 16)) & 0xffffffu);
  w[3] = spread3((uint32_t)(hi >> 8) & 0xffffffu);
}

// The 4-bit codes of a 3-bit coded entry: every escaped column (code 7: depth 7 or more) hashed
// again for min(depth, 15). Out of line: about one entry in five at 28 columns has an escape.
__device__ __noinline__ uint4 fix_escapes3(uint4 w4, uint64_t pm, const uint64_t *kcol, uint32_t cap) {
  uint32_t w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    // nibbles <= 7: adding 1 carries into bit 3 of a nibble exactly when it is 7
    for (uint32_t f = (w[g] + 0x11111111u) & 0x88888888u; f; f &= f - 1) {
      const uint32_t k = (__ffs(f) - 1) >> 2;  // nibble index in the word
      const uint32_t code = depth_code(pm ^ kcol[8 * g + k], cap);
      w[g] = (w[g] & ~(15u << (4 * k))) | (code << (4 * k));
    }
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// ------------------------------------------------------------------------------------------------
// hash sort-scatter (records in, coded entries out)
// ------------------------------------------------------------------------------------------------
// Per tile of rec_tile records: stage them (coalesced 128-bit loads), count their endpoint entries
// per bin, reserve one run per non-empty bin in the gutter (one global atomic each), hash every
// record's C columns once, place both entries (and their bins) in bin order in shared memory,
// and write the runs out.
// Exclusive scan over the threads of a block of NT threads (a multiple of 32, <= 1024).
template <int NT>
__device__ __forceinline__ uint32_t block_scan(uint32_t x, uint32_t *ws /*32*/) {
  if (NT == 1024) return block_scan_1024(x, ws);
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, inc, o);
    if (lane >= (uint32_t)o) inc += y;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < NT / 32 ? ws[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= (uint32_t)o) w += y;
    }
    ws[lane] = w;
  }
  __syncthreads();
  const uint32_t r = (warp ? ws[warp - 1] : 0u) + inc - x;
  __syncthreads();
  return r;
}

// C3: 3-bit codes (kEntryCoded3), else 4-bit (kEntryCoded).
template <int RPT, int NT, bool C3>
__global__ void __launch_bounds__(NT, 1024 / NT)
k_hash_sort_scatter(const uint8_t *__restrict__ rec, uint64_t n, GutterGeom g, PlaneHash ph,
                    uint32_t rec_tile, const uint64_t *__restrict__ base,
                    uint32_t *__restrict__ fill, uint4 *__restrict__ entries) {
  extern __shared__ __align__(16) uint8_t gsm[];
  __shared__ uint32_t ws[32];
  const uint32_t nb = g.nbins, nb4 = (nb + 3) & ~3u;
  uint32_t *s_cur = reinterpret_cast<uint32_t *>(gsm);  // counts, then placement cursors
  uint32_t *s_rel = s_cur + nb4;  // a bin's run: gutter position minus position in the tile
  uint4 *s_ent = reinterpret_cast<uint4 *>(s_rel + nb4);
  uint16_t *s_bin = reinterpret_cast<uint16_t *>(s_ent + 2 * (size_t)rec_tile);  // bin of each entry
  // the staged records share the entry area: they are parsed into registers before the first
  // entry is placed, and the next tile is staged only after the write-out
  uint8_t *s_rec = reinterpret_cast<uint8_t *>(s_ent);
  const uint32_t per_thread = (nb + NT - 1) / NT;  // bins per thread
  const uint32_t cap = 1u << min(ph.B, C3 ? kDepthEscape3 : kDepthEscape);
  for (uint64_t t0 = blockIdx.x * (uint64_t)rec_tile; t0 < n; t0 += (uint64_t)gridDim.x * rec_tile) {
    const uint32_t cnt = (uint32_t)(n - t0 < rec_tile ? n - t0 : rec_tile);
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s_cur[b] = 0u;
    const uint32_t shift = stage_records(rec, t0, cnt, s_rec);
    __syncthreads();
    // 1. this thread's records into registers, then their per-bin counts
    uint32_t ru[RPT], rv[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const uint32_t i = threadIdx.x + k * blockDim.x;
      ru[k] = rv[k] = 0xffffffffu;
      if (i < cnt) {
        parse_record(s_rec, shift, i, ru[k], rv[k]);
        if (ru[k] >= g.V || rv[k] >= g.V) ru[k] = 0xffffffffu;  // dropped (the count pass flags it)
      }
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        atomicAdd(&s_cur[ru[k] >> g.bin_shift], 1u);
        atomicAdd(&s_cur[rv[k] >> g.bin_shift], 1u);
      }
    __syncthreads();
    // 2. run offsets inside the tile (bins [tid*per_thread, +per_thread) per thread) and one run
    //    reserved per non-empty bin in the gutter
    uint32_t sum = 0;
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      sum += b < nb ? s_cur[b] : 0u;
    }
    uint32_t run = block_scan<NT>(sum, ws);
    for (uint32_t k = 0; k < per_thread; ++k) {
      const uint32_t b = threadIdx.x * per_thread + k;
      if (b < nb) {
        const uint32_t c = s_cur[b];
        s_rel[b] = c ? (uint32_t)base[b] + atomicAdd(&fill[b], c) - run : 0u;
        s_cur[b] = run;
        run += c;
      }
    }
    __syncthreads();
    // 3. slots claimed, each record hashed once, both endpoint entries placed in bin order
    uint32_t pu[RPT], pv[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        pu[k] = atomicAdd(&s_cur[ru[k] >> g.bin_shift], 1u);
        pv[k] = atomicAdd(&s_cur[rv[k] >> g.bin_shift], 1u);
      }
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (ru[k] != 0xffffffffu) {
        const uint32_t lo = max(ru[k], rv[k]), hi = min(ru[k], rv[k]);
        const uint64_t pm = xxh3_premix(((uint64_t)lo << 32) | hi);
        uint32_t w[4];
        all_codes(pm, ph.kcol, ph.C, cap, w);
        s_ent[pu[k]] = C3 ? pack_entry3(w, ru[k], rv[k], ph.C, g.bin_shift)
                          : pack_entry(w, ru[k], rv[k], ph.C, g.bin_shift);
        s_ent[pv[k]] = C3 ? pack_entry3(w, rv[k], ru[k], ph.C, g.bin_shift)
                          : pack_entry(w, rv[k], ru[k], ph.C, g.bin_shift);
        s_bin[pu[k]] = (uint16_t)(ru[k] >> g.bin_shift);
        s_bin[pv[k]] = (uint16_t)(rv[k] >> g.bin_shift);
      }
    __syncthreads();
    // 4. coalesced write-out of the runs
    const uint32_t total = s_cur[nb - 1];
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) entries[s_rel[s_bin[j]] + j] = s_ent[j];
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// bucket-plane sketch update
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void red_xor_shared(uint32_t addr, uint32_t v) {
  asm volatile("red.shared.xor.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// The same slot of the checksum plane that follows the plane of addr.
__device__ __forceinline__ void red_xor_shared_g(uint32_t addr, uint32_t v) {
  asm volatile("red.shared.xor.b32 [%0+%2], %1;" ::"r"(addr), "r"(v), "n"(kPlaneBytes) : "memory");
}

__device__ __forceinline__ uint32_t nibble_of(const uint32_t (&c4)[4], uint32_t c) {
  const uint32_t w = c < 16 ? (c < 8 ? c4[0] : c4[1]) : (c < 24 ? c4[2] : c4[3]);
  return (w >> (4 * (c & 7))) & 15u;
}

// Flags of the codes at or above the scratch row: per word, bit 4 of byte lane j flags nibble 2j
// and bit 5 flags nibble 2j + 1 (for a nibble n < 16, n + 5 carries into bit 4 of its byte lane
// exactly when n >= 11).
__device__ __forceinline__ uint32_t high_code_flags(uint32_t w) {
  static_assert(kPlaneThr == 11, "the byte-lane test below is written for threshold 11");
  const uint32_t lo = ((w & 0x0f0f0f0fu) + 0x05050505u) & 0x10101010u;
  const uint32_t hi = ((((w >> 4) & 0x0f0f0f0fu) + 0x05050505u) & 0x10101010u) << 1;
  return lo | hi;
}

// Bucket (c, d) of vertex v's sketch in HBM, three 32-bit atomics (alpha low, alpha high, gamma).
__device__ __forceinline__ void xor_bucket_global(uint32_t *sk, uint32_t bucket, uint32_t lo,
                                                  uint32_t hi, uint32_t chk) {
  uint32_t *p = sk + 3 * bucket;
  atomicXor(p, lo);
  atomicXor(p + 1, hi);
  atomicXor(p + 2, chk);
}

// Moves the codes at or above the scratch row into HBM (exact depth; code 15 means 15 or more
// and is recomputed) and points them at the scratch row. Rare per column (2^-11), so only the
// flagged nibbles are visited.
__device__ __noinline__ uint4 spill_high_codes(uint4 cw, uint4 fl, uint64_t pm, uint32_t lo,
                                               uint32_t hi, uint32_t chk, uint32_t *sk,
                                               const uint64_t *s_kcol, uint32_t B) {
  uint32_t c4[4] = {cw.x, cw.y, cw.z, cw.w};
  const uint32_t f4[4] = {fl.x, fl.y, fl.z, fl.w};
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    uint32_t f = f4[w];
    while (f) {
      const uint32_t bit = __ffs(f) - 1;  // 4 + 8j (nibble 2j) or 5 + 8j (nibble 2j + 1)
      f &= f - 1;
      const uint32_t nib = 2 * (bit >> 3) + (bit & 1u);  // nibble inside the word
      const uint32_t c = 8 * w + nib, sh = 4 * nib;
      const uint32_t code = (c4[w] >> sh) & 15u;
      const uint32_t d = code < kDepthEscape ? code : depth_exact(pm ^ s_kcol[c], B);
      if (d < B) xor_bucket_global(sk, c * B + d, lo, hi, chk);
      c4[w] = (c4[w] & ~(15u << sh)) | (kPlaneThr << sh);
    }
  }
  return make_uint4(c4[0], c4[1], c4[2], c4[3]);
}

// nibble t of the result = nibble t ^ lane of the input (5 index bits: half-byte, byte pair in
// the word, word)
__device__ __forceinline__ void permute_codes(uint32_t (&c4)[4], uint32_t lane) {
  if (lane & 1) {
#pragma unroll
    for (int w = 0; w < 4; ++w) c4[w] = ((c4[w] >> 4) & 0x0f0f0f0fu) | ((c4[w] & 0x0f0f0f0fu) << 4);
  }
  const uint32_t q = (lane >> 1) & 3u;
  const uint32_t sel = q | ((1u ^ q) << 4) | ((2u ^ q) << 8) | ((3u ^ q) << 12);
#pragma unroll
  for (int w = 0; w < 4; ++w) c4[w] = __byte_perm(c4[w], 0, sel);
  if (lane & 8) {
    uint32_t x = c4[0]; c4[0] = c4[1]; c4[1] = x;
    x = c4[2]; c4[2] = c4[3]; c4[3] = x;
  }
  if (lane & 16) {
    uint32_t x = c4[0]; c4[0] = c4[2]; c4[2] = x;
    x = c4[1]; c4[1] = c4[3]; c4[3] = x;
  }
}

struct PlaneCtx {
  uint32_t sp, tile_mask, sketch_words, C, B, cap, bin_shift;
  uint32_t *gsk;
  const uint64_t *s_kcol;
  uint64_t kchk;
};

// All codes of a plain {vertex, neighbour} entry (apply_update_batch), hashed where it is applied;
// out of line, so the coded path keeps its registers.
__device__ __noinline__ uint4 plain_codes(uint64_t pm, const uint64_t *kcol, uint32_t C, uint32_t cap) {
  uint32_t w[4];
  all_codes(pm, kcol, C, cap, w);
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// Vertex, neighbour and 4-bit codes of a gutter entry (kind) of bin `bin`: unpacked from a coded
// entry (3-bit codes: escapes hashed again), or hashed here for a plain {vertex, neighbour} entry
// (apply_update_batch).
__device__ __forceinline__ void decode_entry(uint4 e, uint32_t kind, uint32_t bin, const PlaneCtx &x,
                                             uint32_t &v, uint32_t &u, uint64_t &pm, uint32_t (&c4)[4]) {
  if (kind == kEntryCoded) {
    unpack_entry(e, bin, x.C, x.bin_shift, v, u, c4);
  } else if (kind == kEntryCoded3) {
    unpack_entry3(e, bin, x.C, x.bin_shift, v, u, c4);
  } else {
    v = e.x;
    u = e.y;
  }
  pm = xxh3_premix(((uint64_t)max(u, v) << 32) | min(u, v));  // idx = (min << 32) | max
  if (kind == kEntryCoded3) {
    const uint32_t esc = ((c4[0] + 0x11111111u) | (c4[1] + 0x11111111u) | (c4[2] + 0x11111111u) |
                          (c4[3] + 0x11111111u)) & 0x88888888u;
    if (esc) {
      const uint4 w = fix_escapes3(make_uint4(c4[0], c4[1], c4[2], c4[3]), pm, x.s_kcol, x.cap);
      c4[0] = w.x;
      c4[1] = w.y;
      c4[2] = w.z;
      c4[3] = w.w;
    }
  } else if (kind == kEntryPlain) {
    const uint4 w = plain_codes(pm, x.s_kcol, x.C, x.cap);
    c4[0] = w.x;
    c4[1] = w.y;
    c4[2] = w.z;
    c4[3] = w.w;
  }
}

// Vertex of a gutter entry of bin `bin` (for filtering a bin's entries by tile).
__device__ __forceinline__ uint32_t entry_vertex(uint4 e, uint32_t kind, uint32_t bin, const PlaneCtx &x) {
  if (kind == kEntryPlain) return e.x;
  const uint64_t pay = kind == kEntryCoded3 ? payload3(e, x.C)
                                            : (((uint64_t)e.w << 32) | e.z) >> (4 * x.C - 64);
  return (bin << x.bin_shift) | ((uint32_t)pay & ((1u << x.bin_shift) - 1u));
}

// One entry per lane into the tile's planes (invalid lanes XOR zeros into vertex 0 of the tile).
__device__ __forceinline__ void plane_entry(uint4 e, uint32_t kind, bool valid, uint32_t bin,
                                            uint32_t lane, const PlaneCtx &x) {
  uint32_t v, u, c4[4];
  uint64_t pm;
  decode_entry(e, kind, bin, x, v, u, pm, c4);
  const uint32_t lo = max(u, v), hi = min(u, v);
  const uint32_t chk = valid ? tail_lo32(pm ^ x.kchk) : 0u;
  const uint32_t val = valid ? (u | 0x80000000u) : 0u;
  const uint32_t p = u > v ? 0u : 1u;  // plane A or B
  if (!valid) c4[0] = c4[1] = c4[2] = c4[3] = 0;
  const uint4 fl = make_uint4(high_code_flags(c4[0]), high_code_flags(c4[1]), high_code_flags(c4[2]),
                              high_code_flags(c4[3]));
  if (fl.x | fl.y | fl.z | fl.w) {
    const uint4 y = spill_high_codes(make_uint4(c4[0], c4[1], c4[2], c4[3]), fl, pm, lo, hi, chk,
                                     x.gsk + (uint64_t)v * x.sketch_words, x.s_kcol, x.B);
    c4[0] = y.x;
    c4[1] = y.y;
    c4[2] = y.z;
    c4[3] = y.w;
  }
  permute_codes(c4, lane);
  // one byte per step: byte k of ev[w] (od[w]) = 8 x code of nibble 2k (2k + 1) of word w, so a
  // step takes its row offset with one byte extract
  uint32_t ev[4], od[4];
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    ev[w] = (c4[w] & 0x0f0f0f0fu) << 3;
    od[w] = ((c4[w] >> 4) & 0x0f0f0f0fu) << 3;
  }
  // bits 2..6 of base are the lane (sp is 128-byte aligned, the rest multiples of 128), and the
  // row offset (a multiple of 128) leaves them alone, so (base + row) ^ (t << 2) addresses slot
  // lane ^ t of the row
  const uint32_t base = x.sp + (v & x.tile_mask) * kVertBytes + p * 2 * kPlaneBytes + (lane << 2);
#pragma unroll
  for (int t = 0; t < 32; ++t) {
    const uint32_t w = (uint32_t)t >> 3, k = ((uint32_t)t & 7u) >> 1;
    const uint32_t d8 = __byte_perm((t & 1) ? od[w] : ev[w], 0, 0x4440u + k);
    const uint32_t a = (base + d8 * 16u) ^ (uint32_t)(t << 2);
    red_xor_shared(a, val);
    red_xor_shared_g(a, chk);
  }
}

// One entry applied straight to HBM (sparse tiles): deterministic bucket, then each column.
__device__ __forceinline__ void entry_in_place(uint4 e, uint32_t kind, uint32_t bin, uint32_t tile,
                                               uint32_t tile_shift, const PlaneCtx &x) {
  uint32_t v, u, c4[4];
  uint64_t pm;
  decode_entry(e, kind, bin, x, v, u, pm, c4);
  if ((v >> tile_shift) != tile) return;
  const uint32_t lo = max(u, v), hi = min(u, v);
  const uint32_t chk = tail_lo32(pm ^ x.kchk);
  uint32_t *sk = x.gsk + (uint64_t)v * x.sketch_words;
  xor_bucket_global(sk, x.C * x.B, lo, hi, chk);
  for (uint32_t c = 0; c < x.C; ++c) {
    const uint32_t code = nibble_of(c4, c);
    const uint32_t d = code < kDepthEscape ? code : depth_exact(pm ^ x.s_kcol[c], x.B);
    if (d < x.B) xor_bucket_global(sk, c * x.B + d, lo, hi, chk);
  }
}

__device__ __forceinline__ uint4 load_entry(const uint8_t *cb, uint32_t kind, uint32_t i) {
  if (kind != kEntryPlain) return reinterpret_cast<const uint4 *>(cb)[i];
  const uint2 k = reinterpret_cast<const uint2 *>(cb)[i];
  return make_uint4(k.x, k.y, 0, 0);
}

__global__ void __launch_bounds__(1024, 1)
k_plane_update(PlaneGeom g, PlaneHash ph, uint8_t *__restrict__ sketches,
               const uint8_t *__restrict__ gutter, ChunkTable chunks,
               const uint32_t *__restrict__ bin_off, int nchunks, uint32_t *work_counter) {
  extern __shared__ __align__(16) uint8_t dsm[];
  __shared__ uint64_t s_kcol[kPlaneMaxColumns];
  __shared__ uint32_t s_claim[2];
  const uint32_t W = 1u << g.tile_shift;
  const uint32_t nwarps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t per_bin = g.bin_shift - g.tile_shift;  // log2(tiles per bin)
  const uint32_t s0 = smem_u32(dsm);
  const uint32_t pad = (128u - (s0 & 127u)) & 127u;
  uint8_t *planes = dsm + pad;  // W vertices x planes A, GA, B, GB x kPlaneRows x 32 words
  uint32_t *wbuf = reinterpret_cast<uint32_t *>(planes + (size_t)W * kVertBytes) + warp * kWbWords;
  uint4 *queue = reinterpret_cast<uint4 *>(wbuf);  // the apply phase's per-warp entry queue
  for (uint32_t i = threadIdx.x; i < g.C; i += blockDim.x) s_kcol[i] = ph.kcol[i];
  PlaneCtx x;
  x.sp = s0 + pad;
  x.tile_mask = W - 1;
  x.sketch_words = g.sketch_words;
  x.C = g.C;
  x.B = g.B;
  x.cap = 1u << min(g.B, kDepthEscape);
  x.bin_shift = g.bin_shift;
  x.gsk = reinterpret_cast<uint32_t *>(sketches);
  x.s_kcol = s_kcol;
  x.kchk = ph.kchk;
  const uint32_t stride = g.nbins + 1;
  const uint32_t C = g.C, B = g.B;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(work_counter, 1u);
      uint32_t total = 0;
      if (t < g.ntiles) {
        const uint32_t bin = t >> per_bin;
        for (int k = 0; k < nchunks; ++k)
          total += bin_off[(uint64_t)k * stride + bin + 1] - bin_off[(uint64_t)k * stride + bin];
      }
      s_claim[0] = t;
      s_claim[1] = total;
    }
    __syncthreads();
    const uint32_t t = s_claim[0], total = s_claim[1];  // total: entries of the tile's bin
    if (t >= g.ntiles) break;
    const uint32_t bin = t >> per_bin;
    if (total == 0) {
      __syncthreads();
      continue;
    }
    if (total < (g.direct_max << per_bin)) {
      // few entries: updated in place in HBM (no planes to clear and write back)
      for (int k = 0; k < nchunks; ++k) {
        const uint32_t b = bin_off[(uint64_t)k * stride + bin], e = bin_off[(uint64_t)k * stride + bin + 1];
        const uint8_t *cb = gutter + chunks.base[k];
        const uint32_t kind = chunks.kind[k];
        for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x)
          entry_in_place(load_entry(cb, kind, i), kind, bin, t, g.tile_shift, x);
      }
      __syncthreads();
      continue;
    }
    {
      uint4 *pz = reinterpret_cast<uint4 *>(planes);
      const uint32_t n16 = W * (kVertBytes / 16);
      for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) pz[i] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();
    // an invalid lane carries an entry of vertex 0 of the tile with neighbour 0 and no codes
    const uint4 pad_entry = make_uint4(t << g.tile_shift, 0, 0, 0);
    for (int k = 0; k < nchunks; ++k) {
      const uint32_t b = bin_off[(uint64_t)k * stride + bin], e = bin_off[(uint64_t)k * stride + bin + 1];
      const uint8_t *cb = gutter + chunks.base[k];
      const uint32_t kind = chunks.kind[k];
      // each warp takes groups of 32 entries; the next group is loaded while this one is used
      uint32_t i0 = b + warp * 32;
      bool nvalid = i0 + lane < e;
      uint4 nx = nvalid ? load_entry(cb, kind, i0 + lane) : pad_entry;
      if (per_bin == 0) {
        // the bin is this tile: every entry applies
        for (; i0 < e; i0 += nwarps * 32) {
          const uint4 en = nx;
          const bool valid = nvalid;
          const uint32_t in = i0 + nwarps * 32 + lane;
          nvalid = in < e;
          if (nvalid) nx = load_entry(cb, kind, in);
          plane_entry(en, kind, valid, bin, lane, x);
        }
      } else {
        // the bin holds several tiles: each warp ballots its group, queues this tile's entries,
        // and applies full warps of queued entries; two groups are in flight ahead of the one
        // ballotted
        uint32_t qn = 0;
        const uint32_t step = nwarps * 32;
        bool nvalid2 = i0 + step + lane < e;
        uint4 nx2 = nvalid2 ? load_entry(cb, kind, i0 + step + lane) : pad_entry;
        for (; i0 < e; i0 += step) {
          const uint4 en = nx;
          const bool mine = nvalid && (entry_vertex(en, kind, bin, x) >> g.tile_shift) == t;
          nx = nx2;
          nvalid = nvalid2;
          const uint32_t in = i0 + 2 * step + lane;
          nvalid2 = in < e;
          if (nvalid2) nx2 = load_entry(cb, kind, in);
          const uint32_t m = __ballot_sync(kFull, mine);
          if (mine) queue[qn + __popc(m & ((1u << lane) - 1u))] = en;
          qn += __popc(m);
          __syncwarp();
          if (qn >= 32) {
            const uint4 q = queue[lane];
            __syncwarp();
            qn -= 32;
            if (lane < qn) queue[lane] = queue[32 + lane];
            __syncwarp();
            plane_entry(q, kind, true, bin, lane, x);
          }
        }
        const bool valid = lane < qn;
        const uint4 q = valid ? queue[lane] : pad_entry;
        __syncwarp();
        if (qn) plane_entry(q, kind, valid, bin, lane, x);
      }
    }
    __syncthreads();
    // write-back: one warp per vertex. The words of rows 0 .. R - 1 of every column (one run of
    // 3R words per column in the sketch) are taken as one list: word i of the list is column
    // i / 3R, row (i % 3R) / 3, word (i % 3R) % 3 of the bucket, converted from the planes, and
    // XORed into the sketch in HBM where it is not zero. Lane l takes words l, l + 32, ... (runs of
    // consecutive words: coalesced), eight read-modify-writes in flight at a time.
    const uint32_t R = min(B, kPlaneThr);
    const uint32_t runw = 3 * R, nwl = C * runw;
    for (uint32_t vl = warp; vl < W; vl += nwarps) {
      const uint32_t vg = (t << g.tile_shift) + vl;
      if (vg >= g.V) continue;
      const uint32_t *pa = reinterpret_cast<const uint32_t *>(planes + (size_t)vl * kVertBytes);
      const uint32_t *pga = pa + kPlaneRows * kPlaneSlots;
      const uint32_t *pb = pga + kPlaneRows * kPlaneSlots;
      const uint32_t *pgb = pb + kPlaneRows * kPlaneSlots;
      uint32_t *sk = x.gsk + (uint64_t)vg * g.sketch_words;
      // word (c, w) of lane l's current list position; w < runw
      uint32_t c = 0, w = lane;
      while (w >= runw) {
        w -= runw;
        ++c;
      }
      auto word = [&](uint32_t cc, uint32_t ww) -> uint32_t {
        const uint32_t r = (ww * 0xAAABu) >> 17;  // ww / 3 for ww < 2^15
        const uint32_t s = r * kPlaneSlots + cc, kk = ww - 3 * r;
        const uint32_t a = pa[s], bq = pb[s];
        return kk == 0 ? (a & 0x7fffffffu) ^ ((bq >> 31) ? vg : 0u)
             : kk == 1 ? (bq & 0x7fffffffu) ^ ((a >> 31) ? vg : 0u) : pga[s] ^ pgb[s];
      };
      for (uint32_t i0 = 0; i0 < nwl; i0 += 8 * 32) {
        uint32_t y[8], old[8], off[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const bool in = i0 + k * 32 + lane < nwl;
          y[k] = in ? word(c, w) : 0u;
          off[k] = 3 * c * B + w;
          old[k] = y[k] ? sk[off[k]] : 0u;
          w += 32;
          while (w >= runw) {
            w -= runw;
            ++c;
          }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (y[k]) sk[off[k]] = old[k] ^ y[k];
      }
      if (lane < 3) {  // deterministic bucket: slot C, row 0
        const uint32_t a = pa[C], bq = pb[C];
        const uint32_t y = lane == 0 ? (a & 0x7fffffffu) ^ ((bq >> 31) ? vg : 0u)
                         : lane == 1 ? (bq & 0x7fffffffu) ^ ((a >> 31) ? vg : 0u) : pga[C] ^ pgb[C];
        if (y) sk[3 * C * B + lane] ^= y;
      }
    }
    __syncthreads();
  }
}

// Register-only rate of the per-column hash above: eight independent chains per thread, each
// step a premixed input XOR a column constant, the rrmxmx tail and the depth code, the next input
// being this one XOR its code.
__global__ void k_plane_hash_peak(uint32_t iters, uint64_t *out) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t y[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) y[k] = xxh3_premix(tid * 8 + k);
  uint32_t acc = 0;
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t d = depth_code(y[k] ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(k + 1)), 1u << kDepthEscape);
      acc += d;
      y[k] ^= d;
    }
  }
  uint64_t r = acc;
#pragma unroll
  for (int k = 0; k < 8; ++k) r ^= y[k];
  out[tid] = r;
}

// Rate of the plane update's shared-memory step alone: 32 vertices of planes, each thread one
// synthetic entry per iteration (codes 0..3, random vertex and plane), 32 slot steps of two
// red.shared.xor each, addressed exactly as plane_entry does.
__global__ void __launch_bounds__(1024, 1) k_plane_update_peak(uint32_t iters, uint32_t *out) {
  extern __shared__ __align__(16) uint8_t dsm[];
  const uint32_t s0 = smem_u32(dsm);
  const uint32_t pad = (128u - (s0 & 127u)) & 127u;
  uint8_t *planes = dsm + pad;
  const uint32_t sp = s0 + pad, lane = threadIdx.x & 31;
  uint32_t *pw = reinterpret_cast<uint32_t *>(planes);
  for (uint32_t i = threadIdx.x; i < kPlaneMaxTile * kVertBytes / 4; i += blockDim.x) pw[i] = 0;
  __syncthreads();
  uint32_t z = fmix32_(blockIdx.x * 1024u + threadIdx.x);
  for (uint32_t it = 0; it < iters; ++it) {
    z = z * 1664525u + 1013904223u;
    uint32_t c4[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) c4[w] = fmix32_(z + (uint32_t)w) & 0x33333333u;
    const uint32_t v = z >> 27, p = (z >> 26) & 1u;
    const uint32_t val = z | 0x80000000u, chk = z * 747796405u;
    uint32_t ev[4], od[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      ev[w] = (c4[w] & 0x0f0f0f0fu) << 3;
      od[w] = ((c4[w] >> 4) & 0x0f0f0f0fu) << 3;
    }
    const uint32_t base = sp + v * kVertBytes + p * 2 * kPlaneBytes + (lane << 2);
#pragma unroll
    for (int t = 0; t < 32; ++t) {
      const uint32_t w = (uint32_t)t >> 3, k = ((uint32_t)t & 7u) >> 1;
      const uint32_t d8 = __byte_perm((t & 1) ? od[w] : ev[w], 0, 0x4440u + k);
      const uint32_t a = (base + d8 * 16u) ^ (uint32_t)(t << 2);
      red_xor_shared(a, val);
      red_xor_shared_g(a, chk);
    }
  }
  __syncthreads();
  uint32_t acc = 0;
  for (uint32_t i = threadIdx.x; i < kPlaneMaxTile * kVertBytes / 4; i += blockDim.x) acc ^= pw[i];
  out[blockIdx.x * 1024u + threadIdx.x] = acc;
}

}  // namespace

// ================================================================================================
// host wrappers
// ================================================================================================
PlaneHash plane_hash(uint64_t seed, uint32_t C, uint32_t B) {
  PlaneHash ph{};
  ph.C = C;
  ph.B = B;
  for (uint32_t c = 0; c < C && c < kPlaneMaxColumns; ++c)
    ph.kcol[c] = xxh3_premix(xxh3_flip(seed + 5ull * c));  // column_seed (include/sketch.h:175-176)
  ph.kchk = xxh3_premix(xxh3_flip(seed));                  // checksum_seed
  return ph;
}

constexpr int kHashSortMaxRpt = 6;
constexpr int kHashSortThreads = 1024;  // one CTA per SM (every register of the SM)

uint32_t hash_sort_tile(uint32_t nbins, size_t smem_budget) {
  const int nt = kHashSortThreads;
  const size_t fixed = (size_t)2 * ((nbins + 3) & ~3u) * 4 + 256;
  if (nbins > kSortBinsMax || fixed >= smem_budget) return 0;
  // 2 coded entries of 16 B per record, and their 2-byte bins
  const size_t t = std::min<size_t>((smem_budget - fixed) / 36, (size_t)kHashSortMaxRpt * nt);
  return (uint32_t)(t / nt * nt);
}

cudaError_t gutter_hash_sort(const void *d_rec, uint64_t n, GutterGeom g, const PlaneHash &ph,
                             uint32_t rec_tile, const uint64_t *base, uint32_t *fill,
                             uint4 *entries, uint32_t kind, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  constexpr int NT = kHashSortThreads;
  if (rec_tile < (uint32_t)NT || rec_tile > (uint32_t)(kHashSortMaxRpt * NT) || rec_tile % NT ||
      (kind != kEntryCoded && kind != kEntryCoded3))
    return cudaErrorInvalidValue;
  const size_t smem = (size_t)2 * ((g.nbins + 3) & ~3u) * 4 + (size_t)rec_tile * 36;
  const uint64_t tiles = (n + rec_tile - 1) / rec_tile;
  const uint8_t *rec = reinterpret_cast<const uint8_t *>(d_rec);
  auto launch = [&](auto kern) -> cudaError_t {
    cudaError_t e = smem_optin(kern);
    if (e != cudaSuccess) return e;
    const int G = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)num_sms(), tiles));
    kern<<<G, NT, smem, s>>>(rec, n, g, ph, rec_tile, base, fill, entries);
    add_launches(1);
    return cudaGetLastError();
  };
  auto by_rpt = [&](auto c3) -> cudaError_t {
    constexpr bool K = decltype(c3)::value;
    switch (rec_tile / NT) {
      case 1: return launch(k_hash_sort_scatter<1, NT, K>);
      case 2: return launch(k_hash_sort_scatter<2, NT, K>);
      case 3: return launch(k_hash_sort_scatter<3, NT, K>);
      case 4: return launch(k_hash_sort_scatter<4, NT, K>);
      case 5: return launch(k_hash_sort_scatter<5, NT, K>);
      default: return launch(k_hash_sort_scatter<6, NT, K>);
    }
  };
  return kind == kEntryCoded3 ? by_rpt(std::true_type{}) : by_rpt(std::false_type{});
}

size_t plane_update_smem(uint32_t tile_shift, int threads) {
  return 128 + ((size_t)kVertBytes << tile_shift) + (size_t)(threads / 32) * kWbWords * 4;
}

int plane_update_ctas_per_sm(uint32_t tile_shift, int threads) {
  int n = 0;
  if (smem_optin(k_plane_update) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_plane_update, threads,
                                                    plane_update_smem(tile_shift, threads)) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

cudaError_t plane_update(const PlaneGeom &g, const PlaneHash &ph, uint8_t *sketches,
                         const uint8_t *gutter, const ChunkTable &chunks, const uint32_t *bin_off,
                         int nchunks, uint32_t *work_counter, uint32_t * /*status*/, int grid,
                         int threads, cudaStream_t s) {
  if (g.C > kPlaneMaxColumns || g.C < 18 || g.tile_shift > 5 ||
      g.bin_shift < g.tile_shift || threads % 32 || threads < 32 || threads > 1024)
    return cudaErrorInvalidValue;
  cudaError_t e = smem_optin(k_plane_update);
  if (e != cudaSuccess) return e;
  k_plane_update<<<grid, threads, plane_update_smem(g.tile_shift, threads), s>>>(
      g, ph, sketches, gutter, chunks, bin_off, nchunks, work_counter);
  add_launches(1);
  return cudaGetLastError();
}

cudaError_t plane_hash_peak(uint32_t iters, int blocks, int threads, uint64_t *out, cudaStream_t s) {
  k_plane_hash_peak<<<blocks, threads, 0, s>>>(iters, out);
  add_launches(1);
  return cudaGetLastError();
}

cudaError_t plane_update_peak(uint32_t iters, int blocks, uint32_t *out, cudaStream_t s) {
  cudaError_t e = smem_optin(k_plane_update_peak);
  if (e != cudaSuccess) return e;
  k_plane_update_peak<<<blocks, 1024, 128 + kPlaneMaxTile * kVertBytes, s>>>(iters, out);
  add_launches(1);
  return cudaGetLastError();
}

}  // namespace gz
