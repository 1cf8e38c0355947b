// gz_device.cuh -- device-side building blocks shared by the ingest and query kernels.
//
// Hashing: XXH3_64bits_withSeed of one 8-byte little-endian value (xxHash 0.8.x, path
// XXH3_len_4to8_64b + XXH3_rrmxmx), which the reference calls through vec_hash / col_hash
// (include/types.h:8-9) for the bucket checksum (include/bucket.h:61-63) and the per-column depth
// (include/bucket.h:54-59). For an 8-byte input the seed only enters through one 64-bit constant
// ("flip" below), so the host precomputes flip for the checksum seed and for every column seed
// (seed + 5*col, include/sketch.h:175-176) and the device evaluates rrmxmx(swap32x2(idx) ^ flip).
#pragma once
#include <cstdint>

namespace gz {

// Bucket {u64 alpha; u32 gamma} packed to 12 bytes (include/bucket.h:7-12), seen as 3 words:
// w0 = low 32 bits of alpha, w1 = high 32 bits of alpha, w2 = gamma.
constexpr int kBucketBytes = 12;
constexpr int kMaxBktPerCol = 64;

// XXH3 default-secret words at byte offsets 8 and 16, and the rrmxmx multiplier.
constexpr uint64_t kSecret8 = 0x1cad21f72c81017cULL;
constexpr uint64_t kSecret16 = 0xdb979083e96dd4deULL;
constexpr uint64_t kPrimeMx2 = 0x9FB21C651E98DF25ULL;

// Seed-dependent constant of the 8-byte path: bitflip = (secret[8..16) ^ secret[16..24)) - seed',
// seed' = seed ^ (bswap32(lo32(seed)) << 32).
__host__ __device__ inline uint64_t xxh3_flip(uint64_t seed) {
  uint32_t lo = (uint32_t)seed;
  uint32_t sw = (lo >> 24) | ((lo >> 8) & 0xff00u) | ((lo << 8) & 0xff0000u) | (lo << 24);
  uint64_t s = seed ^ ((uint64_t)sw << 32);
  return (kSecret8 ^ kSecret16) - s;
}

__host__ __device__ inline uint64_t rrmxmx8(uint64_t h) {
  h ^= ((h << 49) | (h >> 15)) ^ ((h << 24) | (h >> 40));
  h *= kPrimeMx2;
  h ^= (h >> 35) + 8;
  h *= kPrimeMx2;
  return h ^ (h >> 28);
}

// Hash of edge index idx = (hi << 32) | lo. The 8-byte path reads the input as two LE32 words
// and recombines them swapped: input64 = (lo << 32) | hi.
__host__ __device__ inline uint64_t hash_idx(uint32_t lo, uint32_t hi, uint64_t flip) {
  return rrmxmx8((((uint64_t)lo << 32) | hi) ^ flip);
}

// Bucket_Boruvka::is_good (include/bucket.h:65-67): gamma == (u32) hash(alpha, checksum seed).
__host__ __device__ inline bool bucket_good(uint32_t w0, uint32_t w1, uint32_t w2,
                                            uint64_t flip_chk) {
  return w2 == (uint32_t)hash_idx(w0, w1, flip_chk);
}

#ifdef __CUDACC__
// depth = ctz(hash | 1 << B) (get_index_depth), B <= 64.
__device__ __forceinline__ uint32_t depth_of(uint64_t h, uint32_t B) {
  uint64_t x = h | (B < 64 ? (1ull << B) : 0ull);
  return (uint32_t)(__ffsll((long long)x) - 1);
}

// h ^= (h >> 35) + 8 on the 32-bit halves: (h >> 35) + 8 < 2^32 only changes the low word, and
// h >> 35 = hi >> 3 is taken as the high word of hi * 2^29 (an integer multiply-add, which
// measured 8% faster per hash on B200 than a shift and an add).
__device__ __forceinline__ uint64_t xorshift35_add8(uint64_t h) {
  const uint32_t lo = (uint32_t)h, hi = (uint32_t)(h >> 32);
  return ((uint64_t)hi << 32) | (lo ^ (__umulhi(hi, 1u << 29) + 8u));
}
// rrmxmx8 without its final xorshift, split into 32-bit halves: the final value is
// h ^ (h >> 28), whose low word needs both halves and whose high word is only ever needed when the
// low word is zero.
__device__ __forceinline__ void rrmxmx8_pre(uint64_t h, uint32_t &lo, uint32_t &hi) {
  h ^= ((h << 49) | (h >> 15)) ^ ((h << 24) | (h >> 40));
  h *= kPrimeMx2;
  h = xorshift35_add8(h);
  h *= kPrimeMx2;
  lo = (uint32_t)h;
  hi = (uint32_t)(h >> 32);
}
// low 32 bits of rrmxmx8(h): the bucket checksum
__device__ __forceinline__ uint32_t hash_lo32(uint64_t h) {
  uint32_t lo, hi;
  rrmxmx8_pre(h, lo, hi);
  return lo ^ __funnelshift_r(lo, hi, 28);
}
// depth_of(rrmxmx8(h), B) for B <= 63, computing the high word only when the low word is zero.
__device__ __forceinline__ uint32_t hash_depth(uint64_t h, uint32_t B) {
  uint32_t lo, hi;
  rrmxmx8_pre(h, lo, hi);
  const uint32_t flo = lo ^ __funnelshift_r(lo, hi, 28);
  if (B < 32) return __ffs(flo | (1u << B)) - 1;
  if (flo) return __ffs(flo) - 1;
  const uint32_t fhi = hi ^ (hi >> 28);
  return 31 + __ffs(fhi | (1u << (B - 32)));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
#endif

// The first step of rrmxmx, h ^ rotl(h, 49) ^ rotl(h, 24), is linear over GF(2). Hence
// rrmxmx8(in ^ flip) = rrmxmx8_tail(premix(in) ^ premix(flip)): premix of the record's input is
// computed once per record and premix(flip) once per column seed, which leaves two multiplies, a
// shift-add-xor and the final xorshift per column.
__host__ __device__ inline uint64_t xxh3_premix(uint64_t h) {
  return h ^ ((h << 49) | (h >> 15)) ^ ((h << 24) | (h >> 40));
}

#ifdef __CUDACC__
// rrmxmx8 after its premix step, without the final xorshift, as 32-bit halves.
__device__ __forceinline__ void rrmxmx8_tail_pre(uint64_t h, uint32_t &lo, uint32_t &hi) {
  h *= kPrimeMx2;
  h = xorshift35_add8(h);
  h *= kPrimeMx2;
  lo = (uint32_t)h;
  hi = (uint32_t)(h >> 32);
}
// low word of rrmxmx8 given the premixed input (the bucket checksum, and the low bits the depth
// is counted in)
__device__ __forceinline__ uint32_t tail_lo32(uint64_t pm) {
  uint32_t lo, hi;
  rrmxmx8_tail_pre(pm, lo, hi);
  return lo ^ __funnelshift_r(lo, hi, 28);
}
// Depth code of one column: min(depth, 15) where depth = ctz(hash | 1 << B); cap = 1 << min(B, 15).
// For B <= 15 this is the depth itself (depth <= B); for B > 15 the code 15 stands for "15 or
// more" and the exact depth is recomputed by depth_exact where it is needed.
__device__ __forceinline__ uint32_t depth_code(uint64_t pm, uint32_t cap) {
  return __clz(__brev(tail_lo32(pm) | cap));
}
// depth = ctz(hash | 1 << B), B <= 63, given the premixed input
__device__ __forceinline__ uint32_t depth_exact(uint64_t pm, uint32_t B) {
  uint32_t lo, hi;
  rrmxmx8_tail_pre(pm, lo, hi);
  const uint64_t r = (((uint64_t)(hi ^ (hi >> 28))) << 32) | (lo ^ __funnelshift_r(lo, hi, 28));
  return (uint32_t)(__ffsll((long long)(r | (1ull << B))) - 1);
}
#endif

}  // namespace gz
