// Chunk plan of host-record ingest (gz_ingest_records): how a call's records are cut into
// host->device copies and when the gutter is folded into the sketches. Host-only C++, shared by
// the library and its CPU unit test.
//
// The copies run on a second stream into kStageBuffers device buffers while the gutter and the
// sketch update run on the handle's stream. A long call is cut so that the sketch update overlaps
// the copies from start to end: the first chunk is kFirstChunk records and the chunks double up to
// kStageRecords, and every chunk is folded into the sketches as soon as it lands (a wave of its
// own). The last kTailRecords records come as a tail of halving chunks (about 8, 4 and 2 Mi
// records) with no wave of their own: a wave re-reads and re-writes every vertex sketch it
// touches, which costs more than a small chunk's copy, so their gutter passes keep pace with the
// copies and one wave folds the whole tail at the next flush or query, when the last and
// smallest chunk has landed. This shape is used only while all sketches together are at most
// kShapeSketchBytes (a pass over them then costs a fraction of a millisecond, and a chunk's
// sketch update keeps pace with the copy of the next); other calls copy kStageRecords-record
// chunks and fold one wave per kWaveEntries endpoint updates.
#pragma once

#include <algorithm>
#include <cstdint>

namespace gz {

constexpr uint64_t kStageRecords = 1ull << 24;  // records per host->device copy, at most
constexpr int kStageBuffers = 4;                 // device staging buffers of the copy pipeline
constexpr uint64_t kWaveEntries = 1ull << 26;    // endpoint updates per wave of an unshaped call
constexpr uint64_t kFirstChunk = 1ull << 23;
constexpr uint64_t kLastChunk = 1ull << 21;                       // the tail's last chunk
constexpr uint64_t kTailRecords = (1ull << 23) + (1ull << 22) + kLastChunk;  // the tail
constexpr uint64_t kShapeSketchBytes = 3ull << 29;
static_assert(kFirstChunk <= kStageRecords && kTailRecords <= kStageRecords, "shaped chunks fit a stage");

struct IngestPlan {
  uint64_t n = 0;       // records of the call
  uint64_t chunk = 0;   // largest chunk (= the staging buffers' capacity in records)
  uint64_t ramp = 0;    // size of the next chunk before the end-of-call rule
  bool shaped = false;  // doubling first chunks, a wave per chunk, a tail of halving chunks

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
    if (shaped) {
      if (left > kTailRecords) {
        m = std::min(m, left - kTailRecords);  // the full chunks end where the tail starts
      } else {
        // the tail: what is left above 2 Mi + 4 Mi, then 4 Mi, then 2 Mi
        const uint64_t rest = kLastChunk + (kLastChunk << 1);
        m = left > rest ? left - rest : left > kLastChunk ? left - kLastChunk : left;
      }
    }
    ramp = std::min(2 * ramp, chunk);
    return m;
  }

  // Whether to fold the gutter into the sketches after the chunk that ends at record end, with
  // pending endpoint updates buffered. The last chunk (and in the shaped form the whole tail) is
  // left to the next flush or query.
  bool wave_after(uint64_t end, uint64_t pending) const {
    if (shaped) return n - end >= kTailRecords && end < n;
    return end < n && pending >= kWaveEntries;
  }
};

}  // namespace gz
