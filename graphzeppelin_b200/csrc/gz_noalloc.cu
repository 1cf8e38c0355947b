// gz_noalloc.cu -- gz_ingest_records_noalloc: the record-ingest pipeline (device gutter +
// sketch update) for callers that cannot allocate GPU memory.
//
// Some callers of this library are not allowed to allocate device memory: plugins running inside
// a host framework that hands out all GPU memory from its own pool (a library-side cudaMalloc
// would bypass that pool's accounting and can fail or fragment it), and latency-critical service
// loops where cudaMalloc / cudaFree would synchronize the device and stall every other stream.
// For them this entry point takes the caller's sketches and records (both already in device
// memory) and allocates nothing: its scratch memory (gutter entries, bin counts and offsets,
// hash constants, status words) lives in one fixed, file-scope device array that every GPU which
// loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gz_b200.h"
#include "gz_device.cuh"
#include "gz_kernels.cuh"

// gz_capi.cu: stores the text gz_last_error() returns on this thread
void gz_internal_set_error(const std::string &msg);

namespace {

// Limits of one call, and the scratch layout they need.
constexpr uint64_t kNoAllocMaxRecords = 1ull << 21;  // 2,097,152 records per call
constexpr uint32_t kNoAllocMaxVertices = 1u << 22;   // 4,194,304 vertices
constexpr uint32_t kNoAllocMaxBins = 1u << 16;
constexpr uint32_t kNoAllocMaxColumns = 127;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffEntries = 0;
constexpr size_t kOffCounts = align256(kOffEntries + kNoAllocMaxRecords * 2 * 8);
constexpr size_t kOffCursor = align256(kOffCounts + (size_t)kNoAllocMaxBins * 8);
constexpr size_t kOffScanTmp = align256(kOffCursor + (size_t)kNoAllocMaxBins * 8);
constexpr size_t kOffTotal = align256(kOffScanTmp + 64 * 8);
constexpr size_t kOffBinOff = align256(kOffTotal + 8);
constexpr size_t kOffFill = align256(kOffBinOff + ((size_t)kNoAllocMaxBins + 1) * 4);
constexpr size_t kOffFlip = align256(kOffFill + (size_t)kNoAllocMaxBins * 4);
constexpr size_t kOffStatus = align256(kOffFlip + (kNoAllocMaxColumns + 1) * 8);
constexpr size_t kScratchBytes = align256(kOffStatus + 16);  // about 34 MiB

// The scratch array. Host code must not use this name as a device address: the address comes
// from cudaGetSymbolAddress, once per device (see scratch_for_current_device).
static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mtx;
uint8_t *g_noalloc_ptr[kMaxDevices] = {};

int noalloc_fail(int code, const std::string &msg) {
  gz_internal_set_error(msg);  // read back through gz_last_error()
  return code;
}

// Device address of the scratch array on the current device; looked up on the first call made
// on each device (that first call should therefore come before any stream capture).
int scratch_for_current_device(uint8_t **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(GZ_ERR_NO_DEVICE, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(GZ_ERR_INVALID, "device index too large");
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(GZ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<uint8_t *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return GZ_OK;
}

// The reference sizing (include/sketch.h:62-76, :181, :188-190), same double expressions.
void noalloc_params(uint32_t V, double f, uint32_t &C, uint32_t &B) {
  const uint64_t vec_len = (uint64_t)std::ceil(double(V) * (uint32_t)(V - 1) / 2);
  B = (uint32_t)(std::ceil(std::log2((double)vec_len)) + 1);
  const double num_samples_div = 1 - std::log2(2 - 0.8);
  const size_t s = (size_t)std::ceil(f * std::log2((double)V) / num_samples_div);
  C = (uint32_t)std::max<size_t>(18, s);
}

// Entries of the vertices past the last whole shared-memory tile ([tail_start, V), all inside
// one gutter bin) are folded into the caller's sketches with global atomicXor.
__global__ void k_noalloc_tail(uint32_t *sketches, const uint2 *entries, const uint32_t *bin_off,
                               uint32_t bin, uint32_t tail_start, uint32_t sketch_words,
                               uint32_t C, uint32_t B, const uint64_t *flip) {
  const uint32_t b = bin_off[bin], e = bin_off[bin + 1];
  const uint64_t flip_chk = flip[C];
  for (uint32_t i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) {
    const uint2 x = entries[i];
    if (x.x < tail_start) continue;
    const uint32_t lo = max(x.x, x.y), hi = min(x.x, x.y);
    const uint64_t in64 = ((uint64_t)lo << 32) | hi;
    const uint32_t chk = (uint32_t)gz::rrmxmx8(in64 ^ flip_chk);
    uint32_t *sk = sketches + (uint64_t)x.x * sketch_words;
    uint32_t *det = sk + 3 * C * B;
    atomicXor(det, lo);
    atomicXor(det + 1, hi);
    atomicXor(det + 2, chk);
    for (uint32_t c = 0; c < C; ++c) {
      const uint32_t d = gz::depth_of(gz::rrmxmx8(in64 ^ flip[c]), B);
      if (d < B) {
        uint32_t *bk = sk + 3 * (c * B + d);
        atomicXor(bk, lo);
        atomicXor(bk + 1, hi);
        atomicXor(bk + 2, chk);
      }
    }
  }
}

#define NA_CUDA(call)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return noalloc_fail(GZ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Once a call has queued work on its stream, every return waits for that work: the scratch array
// must be idle before the lock is released, or the next call (on any stream) would overwrite the
// regions the queued kernels still use. Declared after the lock guard, so it runs first.
struct StreamDrain {
  cudaStream_t s;
  bool armed = false;
  ~StreamDrain() {
    if (armed) cudaStreamSynchronize(s);
  }
};

}  // namespace

extern "C" {

int gz_ingest_records_noalloc(void *d_sketches, uint32_t num_vertices, uint64_t seed,
                              double sketches_factor, const void *d_records, size_t n_records,
                              void *stream_ptr) {
  if (!d_sketches || (n_records && !d_records)) return noalloc_fail(GZ_ERR_INVALID, "null argument");
  if (num_vertices < 2 || num_vertices > kNoAllocMaxVertices)
    return noalloc_fail(GZ_ERR_INVALID, "num_vertices must be in [2, " +
                                            std::to_string(kNoAllocMaxVertices) + "] for this entry point");
  if (n_records > kNoAllocMaxRecords)
    return noalloc_fail(GZ_ERR_INVALID, "at most " + std::to_string(kNoAllocMaxRecords) +
                                            " records per call (the fixed scratch holds no more); "
                                            "split the stream");
  const double f = sketches_factor > 0 ? sketches_factor : 1;
  uint32_t C = 0, B = 0;
  noalloc_params(num_vertices, f, C, B);
  if (C > kNoAllocMaxColumns || B > 63)
    return noalloc_fail(GZ_ERR_INVALID, "sketch has too many columns for this entry point");
  if (n_records == 0) return GZ_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);

  std::lock_guard<std::mutex> lk(g_noalloc_mtx);
  StreamDrain drain{s};
  uint8_t *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != GZ_OK) return rc;

  // geometry: the default tiling rule of the handle path
  const uint32_t nb = C * B + 1;
  const uint64_t sketch_bytes = (uint64_t)nb * 12;
  int dev = 0, smem_optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem_optin <= 0) smem_optin = 227 * 1024;
  const size_t budget = (size_t)smem_optin - 64 - gz::kQueueBytes;
  const size_t flip_bytes = (size_t)(C + 1) * 8;
  uint32_t shift = 2;
  const uint64_t want = std::max<uint64_t>(4, num_vertices / (2ull * gz::num_sms()));
  while (shift < 6 && (1ull << (shift + 1)) <= want && (sketch_bytes << (shift + 1)) + flip_bytes <= budget)
    ++shift;
  if ((sketch_bytes << shift) + flip_bytes > budget)
    return noalloc_fail(GZ_ERR_INVALID, "sketch too large to stage 4 vertices in shared memory");
  uint32_t bshift = shift;
  while (((num_vertices + (1u << bshift) - 1) >> bshift) > 4096 && (1u << (bshift - shift)) < 16)
    ++bshift;
  const uint32_t nbins = (num_vertices + (1u << bshift) - 1) >> bshift;
  if (nbins > kNoAllocMaxBins) return noalloc_fail(GZ_ERR_INVALID, "too many gutter bins");
  const uint32_t full_tiles = num_vertices >> shift;
  const uint32_t tail_start = full_tiles << shift;

  // scratch regions
  uint2 *entries = reinterpret_cast<uint2 *>(scratch + kOffEntries);
  uint64_t *counts = reinterpret_cast<uint64_t *>(scratch + kOffCounts);
  uint64_t *cursor = reinterpret_cast<uint64_t *>(scratch + kOffCursor);
  uint64_t *scan_tmp = reinterpret_cast<uint64_t *>(scratch + kOffScanTmp);
  uint64_t *total = reinterpret_cast<uint64_t *>(scratch + kOffTotal);
  uint32_t *bin_off = reinterpret_cast<uint32_t *>(scratch + kOffBinOff);
  uint32_t *fill = reinterpret_cast<uint32_t *>(scratch + kOffFill);
  uint64_t *flip = reinterpret_cast<uint64_t *>(scratch + kOffFlip);
  uint32_t *status = reinterpret_cast<uint32_t *>(scratch + kOffStatus);  // [0] bits, [1] work

  // the array keeps the previous call's contents: reset what must start at zero
  uint64_t hflip[kNoAllocMaxColumns + 1];
  for (uint32_t c = 0; c < C; ++c) hflip[c] = gz::xxh3_flip(seed + 5ull * c);
  hflip[C] = gz::xxh3_flip(seed);
  drain.armed = true;
  NA_CUDA(cudaMemcpyAsync(flip, hflip, flip_bytes, cudaMemcpyHostToDevice, s));
  NA_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint64_t) * nbins, s));
  NA_CUDA(cudaMemsetAsync(fill, 0, sizeof(uint32_t) * nbins, s));
  NA_CUDA(cudaMemsetAsync(status, 0, 16, s));

  const gz::GutterGeom gg{num_vertices, bshift, nbins};
  const int G = (int)std::max<uint64_t>(
      1, std::min<uint64_t>(2ull * gz::num_sms(), (n_records + gz::kRecTile - 1) / gz::kRecTile));
  NA_CUDA(gz::gutter_count(gz::kInputRecords, d_records, n_records, gg, G, counts, status, s));
  NA_CUDA(gz::scan_exclusive_u64(counts, nbins, total, scan_tmp, s));
  NA_CUDA(gz::gutter_bin_offsets(counts, 1, nbins, total, bin_off, s));
  const uint32_t tile = gz::sort_scatter_tile(gz::kInputRecords, gg, (size_t)smem_optin - 1024);
  if (tile >= 1024) {
    NA_CUDA(gz::gutter_sort_scatter(gz::kInputRecords, d_records, n_records, gg, tile, counts, fill,
                                    entries, s));
  } else {
    NA_CUDA(gz::copy_u64(counts, cursor, nbins, s));
    NA_CUDA(gz::gutter_scatter_global(gz::kInputRecords, d_records, n_records, gg, G, cursor,
                                      entries, s));
  }
  if (full_tiles) {
    gz::SketchGeom g;
    g.V = num_vertices;
    g.C = C;
    g.B = B;
    g.sketch_words = nb * 3;
    g.tile_shift = shift;
    g.ntiles = full_tiles;  // whole tiles only: the tail never leaves the caller's buffer
    g.bin_shift = bshift;
    g.nbins = nbins;
    NA_CUDA(gz::sketch_update_prepare(g, 1024));
    gz::ChunkTable chunks{};
    chunks.base[0] = 0;
    chunks.kind[0] = gz::kEntryPlain;
    const int grid = (int)std::min<uint64_t>(full_tiles, (uint64_t)gz::num_sms() *
                                                             gz::sketch_update_ctas_per_sm(g, 1024));
    NA_CUDA(gz::sketch_update(g, static_cast<uint8_t *>(d_sketches),
                              reinterpret_cast<const uint8_t *>(entries), chunks, bin_off, 1, flip,
                              status + 1, status, grid, 1024, s));
  }
  if (tail_start < num_vertices) {
    k_noalloc_tail<<<std::max(1, gz::num_sms()), 256, 0, s>>>(
        static_cast<uint32_t *>(d_sketches), entries, bin_off, tail_start >> bshift, tail_start,
        nb * 3, C, B, flip);
    NA_CUDA(cudaGetLastError());
  }
  uint32_t st = 0;
  NA_CUDA(cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  if (st & gz::kStatusTimeout) return noalloc_fail(GZ_ERR_TIMEOUT, "a bounded device wait timed out");
  if (st & gz::kStatusBadVertex)
    return noalloc_fail(GZ_ERR_BAD_VERTEX, "a record named a vertex id >= V; it was dropped");
  return GZ_OK;
}

}  // extern "C"
