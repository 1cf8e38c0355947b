// Chunk plan of host-record ingest (gz_ingest_records): how a call's records are cut into
// host->device copies and when the gutter is folded into the sketches. Host-only C++, shared by
// the library and its CPU unit test.
//
// The copies run on a second stream into kStageBuffers device buffers while the gutter and the
// sketch update run on the handle's stream. A long call is cut so that the sketch update overlaps
// the copies from start to end: the first chunk is kFirstChunk records and the chunks double up to
// kStageRecords, every chunk is folded into the sketches as soon as it lands (a wave of its own),
// and the last chunk is kLastChunk records, so little is left to sort and apply once the last
// copy has landed. A wave re-reads and re-writes every vertex sketch it touches, so this shape is
// used only while all sketches together are at most kShapeSketchBytes (a pass over them then costs
// a fraction of a millisecond, and a chunk's sketch update keeps pace with the copy of the next);
// other calls copy kStageRecords-record chunks and fold one wave per kWaveEntries endpoint updates.
#pragma once

#include <algorithm>
#include <cstdint>

namespace gz {

constexpr uint64_t kStageRecords = 1ull << 24;  // records per host->device copy, at most
constexpr int kStageBuffers = 4;                 // device staging buffers of the copy pipeline
constexpr uint64_t kWaveEntries = 1ull << 26;    // endpoint updates per wave of an unshaped call
constexpr uint64_t kFirstChunk = 1ull << 23;
constexpr uint64_t kLastChunk = 1ull << 23;
constexpr uint64_t kShapeSketchBytes = 3ull << 29;
static_assert(kFirstChunk <= kStageRecords && kLastChunk <= kStageRecords, "shaped chunks fit a stage");

struct IngestPlan {
  uint64_t n = 0;       // records of the call
  uint64_t chunk = 0;   // largest chunk (= the staging buffers' capacity in records)
  uint64_t ramp = 0;    // size of the next chunk before the end-of-call rule
  bool shaped = false;  // doubling first chunks, a wave per chunk, a short last chunk

  // in_place: the handle applies records straight to the sketches (no gutter, no waves);
  // sketch_bytes_total: every vertex sketch of the handle together.
  IngestPlan(uint64_t n_, bool in_place, uint64_t sketch_bytes_total)
      : n(n_), chunk(std::min<uint64_t>(kStageRecords, n_)) {
    shaped = n > 2 * kStageRecords && !in_place && sketch_bytes_total <= kShapeSketchBytes;
    ramp = shaped ? std::min(kFirstChunk, chunk) : chunk;
  }

  // Records of the chunk that starts at record off (off < n); at least 1, at most chunk.
  uint64_t next(uint64_t off) {
    const uint64_t left = n - off;
    uint64_t m = std::min(ramp, left);
    if (shaped && left > kLastChunk && left - m < kLastChunk) m = left - kLastChunk;
    ramp = std::min(2 * ramp, chunk);
    return m;
  }

  // Whether to fold the gutter into the sketches after the chunk that ends at record end, with
  // pending endpoint updates buffered. The last chunk is left to the next flush or query.
  bool wave_after(uint64_t end, uint64_t pending) const {
    return end < n && (shaped || pending >= kWaveEntries);
  }
};

}  // namespace gz
