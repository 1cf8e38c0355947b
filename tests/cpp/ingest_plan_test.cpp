// Properties of the host-record ingest chunk plan (graphzeppelin_b200/csrc/gz_ingest_plan.h) over
// many call lengths: the chunks tile [0, n) exactly, fit the staging buffers, take the shaped form
// (doubling first chunks, a wave after every chunk before a tail of 8, 4 and 2 Mi records that
// has none) exactly when it applies, and otherwise keep full chunks with one wave per kWaveEntries
// endpoint updates.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gz_ingest_plan.h"

static int failures = 0;
#define CHECK(c, ...)                                  \
  do {                                                 \
    if (!(c)) {                                        \
      ++failures;                                      \
      std::printf("FAIL %s:%d: %s  ", __FILE__, __LINE__, #c); \
      std::printf(__VA_ARGS__);                        \
      std::printf("\n");                               \
    }                                                  \
  } while (0)

static void check(uint64_t n, bool in_place, uint64_t sketch_total) {
  using namespace gz;
  IngestPlan plan(n, in_place, sketch_total);
  const bool want_shaped = n > 2 * kStageRecords && !in_place && sketch_total <= kShapeSketchBytes;
  CHECK(plan.shaped == want_shaped, "n=%llu", (unsigned long long)n);
  CHECK(plan.chunk >= 1 && plan.chunk <= kStageRecords && plan.chunk <= n, "n=%llu", (unsigned long long)n);
  std::vector<uint64_t> m;
  std::vector<bool> wave;
  uint64_t pending = 0, off = 0, max_pending = 0;
  while (off < n && m.size() < 100000) {
    const uint64_t c = plan.next(off);
    CHECK(c >= 1 && c <= plan.chunk && c <= n - off, "n=%llu off=%llu c=%llu", (unsigned long long)n,
          (unsigned long long)off, (unsigned long long)c);
    if (c == 0) return;
    pending += 2 * c;
    max_pending = pending > max_pending ? pending : max_pending;
    const bool w = plan.wave_after(off + c, pending);
    if (w) pending = 0;
    m.push_back(c);
    wave.push_back(w);
    off += c;
  }
  CHECK(off == n, "n=%llu covered %llu", (unsigned long long)n, (unsigned long long)off);
  CHECK(!wave.back(), "n=%llu: the last chunk is left to the flush", (unsigned long long)n);
  const size_t k = m.size();
  if (plan.shaped) {
    CHECK(m[0] == kFirstChunk, "n=%llu first=%llu", (unsigned long long)n, (unsigned long long)m[0]);
    CHECK(k >= 4, "n=%llu k=%zu", (unsigned long long)n, k);
    // the tail: 8, 4 and 2 Mi records, no wave after any of them; a wave after every other chunk
    CHECK(m[k - 1] == kLastChunk && m[k - 2] == 2 * kLastChunk && m[k - 3] == 4 * kLastChunk,
          "n=%llu tail %llu %llu %llu", (unsigned long long)n, (unsigned long long)m[k - 3],
          (unsigned long long)m[k - 2], (unsigned long long)m[k - 1]);
    for (size_t i = 0; i + 3 < k; ++i) CHECK(wave[i], "n=%llu chunk %zu has no wave", (unsigned long long)n, i);
    for (size_t i = k - 3; i < k; ++i) CHECK(!wave[i], "n=%llu tail chunk %zu has a wave", (unsigned long long)n, i);
    // doubling up to full chunks, then full chunks, then at most one shortened chunk and the tail
    size_t i = 1;
    while (i < k && m[i] == 2 * m[i - 1] && m[i] <= kStageRecords) ++i;
    while (i + 4 < k) {
      CHECK(m[i] == kStageRecords, "n=%llu chunk %zu = %llu", (unsigned long long)n, i, (unsigned long long)m[i]);
      ++i;
    }
    CHECK(k <= (n + kStageRecords - 1) / kStageRecords + 5, "n=%llu k=%zu", (unsigned long long)n, k);
  } else {
    for (size_t i = 0; i + 1 < k; ++i)
      CHECK(m[i] == plan.chunk, "n=%llu chunk %zu = %llu", (unsigned long long)n, i, (unsigned long long)m[i]);
    CHECK(max_pending < kWaveEntries + 2 * plan.chunk, "n=%llu pending %llu", (unsigned long long)n,
          (unsigned long long)max_pending);
  }
}

int main() {
  using namespace gz;
  const uint64_t small_sk = 1285029888ull, big_sk = 14ull << 30;
  std::vector<uint64_t> ns = {1, 2, 9, 1000, kLastChunk - 1, kLastChunk, kLastChunk + 1, kStageRecords - 1,
                              kStageRecords, kStageRecords + 1, 2 * kStageRecords, 2 * kStageRecords + 1,
                              2 * kStageRecords + kLastChunk, 3 * kStageRecords - 1, 139997155ull,
                              127926272ull, 1ull << 30, 10000000000ull};
  uint64_t x = 88172645463325252ull;
  for (int i = 0; i < 2000; ++i) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    ns.push_back(1 + x % (40 * kStageRecords));
  }
  for (uint64_t n : ns) {
    check(n, false, small_sk);
    check(n, true, small_sk);
    check(n, false, big_sk);
    check(n, false, kShapeSketchBytes);
    check(n, false, kShapeSketchBytes + 1);
  }
  // the dense headline stream: 1.4e8 records over 1.285 GB of sketches
  IngestPlan plan(139997155ull, false, small_sk);
  std::printf("dense plan:");
  for (uint64_t off = 0, m = 0; off < plan.n; off += m) {
    m = plan.next(off);
    std::printf(" %.2f", m / 1048576.0);
  }
  std::printf(" (Mi records)\n");
  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("ingest plan ok: %zu lengths\n", ns.size());
  return 0;
}
