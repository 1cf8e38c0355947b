// gz_kernels.cuh -- launch interface of the sm_100a kernels (implemented in gz_kernels.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gz {

// Status bits a kernel may raise in the handle's device status word.
enum : uint32_t {
  kStatusBadVertex = 1u << 0,
  kStatusTimeout = 1u << 1,
  kStatusBadSample = 1u << 2,
};

enum GutterInput : int {
  kInputRecords = 0,  // packed 9-byte records {u8 type, u32 src, u32 dst}: 2 endpoint entries
  kInputEntries = 1,  // uint2 {vertex, neighbour}: 1 endpoint entry
};

// Geometry shared by the gutter kernels. A gutter bin groups 1 << bin_shift consecutive
// vertices; it is coarser than the shared-memory tile of the sketch-update kernel so the scatter
// has few enough destinations for its partial lines to stay in L2.
struct GutterGeom {
  uint32_t V;
  uint32_t bin_shift;  // bin of a vertex = v >> bin_shift
  uint32_t nbins;
};

// Maximum number of gutter chunks buffered before the sketches must be updated.
constexpr int kMaxChunks = 128;
// Entry kinds of a gutter chunk.
enum EntryKind : uint8_t {
  kEntryPlain = 0,   // uint2 {vertex, neighbour}: hashed where it is applied
  kEntryCoded = 1,   // 128 bits: the 4-bit depth codes of all C columns, computed once per
                     // record (column c in bits 4c .. 4c + 3), then from bit 4C the neighbour
                     // shifted left by bin_shift OR the vertex's offset inside its gutter bin
  kEntryCoded3 = 2,  // the same with 3-bit codes (column c in bits 3c .. 3c + 2; the payload from
                     // bit 3C): code 7 = "7 or more", recomputed where the entry is applied
};
constexpr uint32_t kDepthEscape = 15;  // depth code for "15 or more"
constexpr uint32_t kDepthEscape3 = 7;  // 3-bit depth code for "7 or more"
inline uint32_t neighbour_bits(uint32_t V) {
  uint32_t ubits = 1;
  while (ubits < 32 && (1ull << ubits) < V) ++ubits;  // bits of a neighbour id (< V)
  return ubits;
}
// Whether coded entries hold the codes of C columns for V vertices in bins of 2^bin_shift
// (code_bits = 4 or 3).
inline bool coded_entry_fits(uint32_t V, uint32_t C, uint32_t bin_shift, uint32_t code_bits = 4) {
  return C >= 18 && code_bits * C + bin_shift + neighbour_bits(V) <= 128;
}
struct ChunkTable {
  uint64_t base[kMaxChunks];  // byte offset of the chunk's entries in the gutter buffer
  uint8_t kind[kMaxChunks];
};

struct SketchGeom {
  uint32_t V;
  uint32_t C;                  // columns
  uint32_t B;                  // buckets per column
  uint32_t sketch_words;       // (C*B+1)*3 32-bit words per vertex sketch
  uint32_t tile_shift;         // vertices staged together in shared memory = 1 << tile_shift
  uint32_t ntiles;
  uint32_t bin_shift;          // gutter bin (>= tile_shift); a bin holds 1 << (bin - tile) tiles
  uint32_t nbins;
  uint32_t cube = 0;           // CubeSketch update rule (every depth 0..d) instead of CameoSketch
  uint32_t direct_max = 0;     // one tile per bin only: a tile with fewer plain entries than this
                               // is updated in place in HBM (global atomics) instead of staged
  uint32_t nbuf = 2;           // tile buffers of the pipelined kernel (2..4)
};

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum, once per kernel
// and device. One fixed maximum, instead of each launch's own size set just before it, leaves no
// window in which another host thread lowers the limit between that set and the launch.
cudaError_t smem_optin_fn(const void *kernel);
template <class K>
cudaError_t smem_optin(K kernel) {
  return smem_optin_fn(reinterpret_cast<const void *>(kernel));
}

// Records per staging tile of the gutter kernels, and the largest bin count for which the
// per-CTA histogram lives in shared memory.
constexpr int kRecTile = 4096;
constexpr uint32_t kSmemBinsMax = 12288;
// Largest bin count handled by the shared-memory sort-scatter (above it: global cursors).
constexpr uint32_t kSortBinsMax = 8192;

// ---- scan -------------------------------------------------------------------------------------
// Exclusive prefix sum over n u64 values, in place; writes the total to *d_total. `tmp` must
// hold scan_tmp_words(n) u64.
size_t scan_tmp_words(uint64_t n);
cudaError_t scan_exclusive_u64(uint64_t *d_data, uint64_t n, uint64_t *d_total, uint64_t *tmp,
                               cudaStream_t s);

// ---- device gutter ----------------------------------------------------------------------------
// counts[b] += endpoint entries of bin b (counts zeroed by the caller); flags bad vertex ids.
cudaError_t gutter_count(int input, const void *d_in, uint64_t n, GutterGeom g, int G,
                         uint64_t *counts, uint32_t *status, cudaStream_t s);
// Inputs per tile of the shared-memory sort-scatter for this geometry (0: not applicable).
uint32_t sort_scatter_tile(int input, GutterGeom g, size_t smem_budget);
// Entries of bin b go to entries[base[b] + ...]; fill (nbins u32) must start at zero.
cudaError_t gutter_sort_scatter(int input, const void *d_in, uint64_t n, GutterGeom g,
                                uint32_t rec_tile, const uint64_t *base, uint32_t *fill,
                                uint2 *entries, cudaStream_t s);
// Fallback for many bins: one global atomic cursor per bin (cursor = copy of base).
cudaError_t gutter_scatter_global(int input, const void *d_in, uint64_t n, GutterGeom g, int G,
                                  uint64_t *cursor, uint2 *entries, cudaStream_t s);

// ---- coded entries and bucket planes (gz_planes.cu) ---------------------------------------
// A vertex sketch is accumulated in shared memory as four planes of kPlaneRows rows x
// kPlaneSlots 32-bit slots: slot c < C is column c, slot C the deterministic bucket (row 0).
// Row d of a column holds depth d; the last row is scratch (depth codes at or above it are
// handled in HBM). Plane A XORs (neighbour | 1 << 31) of the entries whose neighbour is above
// the vertex, plane B of the others; planes GA and GB their checksums.
constexpr uint32_t kPlaneSlots = 32;
constexpr uint32_t kPlaneRows = 12;
constexpr uint32_t kPlaneMaxColumns = kPlaneSlots - 1;
constexpr uint32_t kPlaneMaxTile = 32;     // vertices per shared-memory tile
struct PlaneHash {
  uint32_t C, B;
  uint64_t kcol[kPlaneMaxColumns];  // xxh3_premix(flip of column seed c)
  uint64_t kchk;                    // xxh3_premix(flip of the checksum seed)
};
struct PlaneGeom {
  uint32_t V, C, B, sketch_words;
  uint32_t tile_shift;  // W = 1 << tile_shift vertices per tile
  uint32_t ntiles;
  uint32_t bin_shift;   // gutter bin (>= tile_shift): a bin holds 1 << (bin - tile) tiles
  uint32_t nbins;
  uint32_t direct_max;  // a tile with fewer entries is updated in place in HBM
};
PlaneHash plane_hash(uint64_t seed, uint32_t C, uint32_t B);
// Records per tile of the hash sort-scatter for this bin count (0: the bins do not fit).
uint32_t hash_sort_tile(uint32_t nbins, size_t smem_budget);
// Hash every record once (all C columns) and write its two coded endpoint entries,
// counting-sorted by bin, to entries[base[b] + ...]; fill (nbins u32) starts at zero.
// kind = kEntryCoded or kEntryCoded3.
cudaError_t gutter_hash_sort(const void *d_rec, uint64_t n, GutterGeom g, const PlaneHash &ph,
                             uint32_t rec_tile, const uint64_t *base, uint32_t *fill,
                             uint4 *entries, uint32_t kind, cudaStream_t s);
// Applies every buffered chunk (coded or plain entries) tile by tile through bucket planes.
size_t plane_update_smem(uint32_t tile_shift, int threads);
int plane_update_ctas_per_sm(uint32_t tile_shift, int threads);
cudaError_t plane_update(const PlaneGeom &g, const PlaneHash &ph, uint8_t *sketches,
                         const uint8_t *gutter, const ChunkTable &chunks, const uint32_t *bin_off,
                         int nchunks, uint32_t *work_counter, uint32_t *status, int grid,
                         int threads, cudaStream_t s);
// Register-only rate of the per-column hash of this ingest: premixed input XOR a premixed
// column constant, rrmxmx tail, depth code (blocks x threads x iters x 8 hashes).
cudaError_t plane_hash_peak(uint32_t iters, int blocks, int threads, uint64_t *out, cudaStream_t s);
// Rate of the bucket-plane update's shared-memory step without hashing or global traffic:
// blocks x 1024 threads x iters entries, each 32 slot steps of two red.shared.xor.
cudaError_t plane_update_peak(uint32_t iters, int blocks, uint32_t *out, cudaStream_t s);

// bin_off[b] = scanned[b * stride], bin_off[nbins] = *total  (u32, relative to chunk base)
cudaError_t gutter_bin_offsets(const uint64_t *scanned, uint32_t stride, uint32_t nbins,
                               const uint64_t *total, uint32_t *bin_off, cudaStream_t s);
// gutter_scatter_1d consumes cursors; copy scanned counts into them first.
cudaError_t copy_u64(const uint64_t *src, uint64_t *dst, uint64_t n, cudaStream_t s);

// ---- sketch update -------------------------------------------------------------------------------
// Per-warp queues (64 entries x 32 warps) that compact the entries of a bin belonging to this
// CTA's tile into full warps.
constexpr size_t kQueueBytes = 64 * 4 * 32;
size_t sketch_update_smem_bytes(SketchGeom g);
cudaError_t sketch_update_prepare(SketchGeom g, int threads);
// CTAs of the sketch-update kernel that fit on one SM at this geometry.
int sketch_update_ctas_per_sm(SketchGeom g, int threads);
// Applies every buffered entry of `nchunks` chunks: for each tile whose bin has entries, stage
// its sketches in shared memory with bulk async copies, XOR in the bin entries that belong to
// the tile, write the tile back.
// Tile pipeline with g.nbuf buffers (one tile per bin, plain CameoSketch entries only): 1024 threads
// (31 consumer warps + a producer warp), one CTA per SM.
size_t sketch_update_pipe_smem_bytes(SketchGeom g);
cudaError_t sketch_update_pipe(SketchGeom g, uint8_t *sketches, const uint8_t *gutter,
                               const ChunkTable &chunks, const uint32_t *bin_off, int nchunks,
                               const uint64_t *flip, uint32_t *work_counter, uint32_t *status,
                               int grid, cudaStream_t s);
cudaError_t sketch_update(SketchGeom g, uint8_t *sketches, const uint8_t *gutter,
                          const ChunkTable &chunks, const uint32_t *bin_off, int nchunks,
                          const uint64_t *flip, uint32_t *work_counter, uint32_t *status,
                          int grid, int threads, cudaStream_t s);
// XOR num_buckets raw buckets (device) into the sketch of vertex v.
// Updates applied in place in HBM, without staging (sketches too large for a shared-memory tile
// of 4 vertices): records are hashed once and XORed into both endpoints' sketches, entries
// {vertex, neighbour} into their vertex's sketch.
cudaError_t apply_in_place(int input, const void *d_in, uint64_t n, SketchGeom g, uint8_t *sketches,
                           const uint64_t *flip, uint32_t *status, cudaStream_t s);
cudaError_t sketch_xor_raw(uint8_t *sketches, uint32_t sketch_words, uint32_t v,
                           const uint32_t *raw, cudaStream_t s);

// ---- Boruvka -----------------------------------------------------------------------------------
struct BoruvkaBufs {
  uint32_t *parent;      // V   DSU parents
  uint32_t *label;       // V   root per vertex for the current round
  uint32_t *cnt;         // V   members per root
  uint32_t *fill;        // V   scatter cursors
  uint32_t *minv;        // V   smallest member per root (trace keys)
  uint64_t *packed;      // V   (cnt | has_members << 32), scanned in place
  uint64_t *scan_total;  // 1
  uint64_t *scan_tmp;
  uint32_t *order;       // V   vertices grouped by component
  uint32_t *order_comp;  // V   component index of each grouped position
  uint32_t *comp_start;  // V+1
  uint32_t *comp_key;    // V
  uint32_t *ncomp;       // 1
  uint32_t *acc;         // (V / span + 2) * (B+1) * 3 words: merged buckets of each component
                         // crossing a span edge, at slot (its first grouped position / span)
  uint32_t *part;        // per merge warp: its members' XOR when one component covers its span
  uint32_t *part_comp;   // per merge warp: that component, or ~0
  uint32_t *big;         // 1   the component holding more than half the vertices, or ~0
  uint32_t *round;       // 1   the current round (device-driven loop)
  uint32_t *ctl;         // 3   after the loop: rounds run, out of samples (0/1); go on (0/1)
  uint32_t *flags;       // [0] modified (k_bv_query: [round % 3])
  uint32_t *cross;       // V / span + 1  components crossing a span edge (sampled from acc)
  uint32_t *ncross;      // 1
  uint32_t *qbar;        // 1   arrivals at the grid barriers of k_bv_query
  uint64_t *btot;        // kBvQueryMaxBlocks  per-block totals of k_bv_query's scan
  uint64_t *forest;      // V   spanning-forest edge indices
  uint32_t *forest_n;    // 1
  void *trace;           // gz_trace_rec_t[trace_cap] or null
  uint32_t *trace_n;     // 1
  uint32_t trace_cap;
  uint32_t *status;
};

// Bytes allocated past the last vertex sketch of any sketch buffer a query reads: its bulk copies
// read 16-byte-aligned supersets of bucket runs, up to 15 bytes beyond the last sketch.
constexpr size_t kSketchTail = 256;

// Blocks of the one-launch query (k_bv_query), at most: per-block scan totals are kept for
// each, and each block scans all of them in shared memory.
constexpr uint32_t kBvQueryMaxBlocks = 1184;

// Grouped members XOR-merged by one warp per Boruvka round (the per-warp partial slots are
// sized by it).
constexpr uint32_t kBoruvkaSpan = 32;

struct BoruvkaGeom {
  uint32_t V, C, B, sketch_words;
  uint64_t flip_chk;
  uint32_t span;     // members merged per warp
  uint32_t cps = 1;  // columns per sample: round r merges and scans columns r*cps .. r*cps+cps-1
  // Every update reached both endpoint sketches (records, gz_update), so the XOR of all vertex
  // sketches is zero and a component's merged sketch equals the XOR over all other vertices:
  // the largest component (over half the vertices) is merged from its complement.
  uint32_t complement = 0;
};

// XOR of every vertex sketch, word by word, into total[sketch_words] (zeroed by the caller).
cudaError_t sketch_total_xor(const uint8_t *sketches, uint32_t V, uint32_t sketch_words,
                             uint32_t *total, cudaStream_t s);

cudaError_t boruvka_reset(const BoruvkaGeom &g, const BoruvkaBufs &b, cudaStream_t s);
cudaError_t boruvka_round0(const BoruvkaGeom &g, const uint8_t *sketches, const BoruvkaBufs &b,
                           cudaStream_t s);
// one round >= 1; the round number is read from b.round
cudaError_t boruvka_round(const BoruvkaGeom &g, const uint8_t *sketches, const BoruvkaBufs &b,
                          cudaStream_t s);
// parent_out[v] = root of v; *ncc = number of roots (device pointers)
cudaError_t boruvka_final(const BoruvkaGeom &g, const BoruvkaBufs &b, uint32_t *labels_out,
                          uint32_t *ncc, cudaStream_t s);

// boruvka_emulation (src/cc_sketch_alg.cpp:464-513) as one CUDA graph: round 0, then a
// conditional while node whose body is one round plus a check kernel that ends the loop when a
// round neither FAILs nor merges, or when the next round would exceed `samples` (b.ctl then
// holds the rounds and the out-of-samples flag), then the labels (labels_out, *ncc). No host
// round trip between rounds.
struct BoruvkaGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  uint32_t fixed_kernels = 0, round_kernels = 0;  // kernel nodes outside / inside the loop body
  // what the graph was built for
  BoruvkaGeom g{};
  BoruvkaBufs b{};
  const uint8_t *sketches = nullptr;
  uint32_t *labels = nullptr, *ncc = nullptr, samples = 0;
};
cudaError_t boruvka_graph_launch(BoruvkaGraph &q, const BoruvkaGeom &g, uint32_t samples,
                                 const uint8_t *sketches, const BoruvkaBufs &b, uint32_t *labels_out,
                                 uint32_t *ncc, cudaStream_t s);
void boruvka_graph_free(BoruvkaGraph &q);
// The same kernels with the loop run from the host (a device-to-host copy and a synchronize per
// round; for profilers that do not see kernels inside conditional graphs). Leaves b.ctl[0..1]
// as the graph does; pin is pinned host memory of at least 3 words.
// boruvka_emulation in one cooperative kernel launch (all rounds on the device, grid barriers
// between the phases of a round): the same answer, rounds, samples and trace as the graph and the
// host loop. b.ctl then holds the rounds and the out-of-samples flag.
cudaError_t boruvka_query_launch(const BoruvkaGeom &g, uint32_t samples, const uint8_t *sketches,
                                 const BoruvkaBufs &b, uint32_t *labels_out, uint32_t *ncc,
                                 cudaStream_t s);
cudaError_t boruvka_host_loop(const BoruvkaGeom &g, uint32_t samples, const uint8_t *sketches,
                              const BoruvkaBufs &b, uint32_t *labels_out, uint32_t *ncc,
                              uint32_t *pin, cudaStream_t s);

int num_sms();
// columns C and buckets per column B of one vertex sketch for V vertices and sketches factor f
void sketch_sizing(uint32_t V, double f, uint32_t &C, uint32_t &B);
// samples, columns per sample and B of CameoSketch (cube = false: C = samples) or CubeSketch
void sketch_sizing_alg(uint32_t V, double f, bool cube, uint32_t &samples, uint32_t &cps, uint32_t &B);

// Kernel launches issued by the host wrappers of this file (monotonic, process-wide).
uint64_t launch_count();
// kernels launched by a CUDA graph (counted by its owner once the graph has run)
void add_launches(uint64_t n);

}  // namespace gz
