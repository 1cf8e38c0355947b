// ref_harness.cpp -- project-written driver around the UNMODIFIED reference sources
// (src/sketch.cpp, src/util.cpp, src/cc_sketch_alg.cpp, src/return_types.cpp,
// src/cc_alg_configuration.cpp), compiled by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement (gz_oracle.c) to the reference's own
// code and serves as the timed CPU baseline. It replaces tools/process_stream.cpp, which
// cannot be built here (GutterTree / StreamingUtilities are not vendored) and which seeds
// from the wall clock (tools/process_stream.cpp:15-18).
//
// The GutteringSystem is not available, so a stand-in gutter buffers every endpoint update
// per vertex (parallel counting sort) and hands batches of get_desired_updates_per_batch()
// to apply_update_batch from `threads` worker threads, which is the driver contract of
// include/graph_sketch_driver.h:28-69 / :205-209.
//
// Modes:
//   ingest <stream> <seed> <sketches_factor> <threads> <max_records|0> <dump|-> <labels|->
//       CCSketchAlg ingest + connected_components(); JSON line on stdout with timings.
//   trace <dump> <trace_out> <labels_out>
//       loads a write_binary dump into reference Sketch objects and runs Boruvka round by round
//       with the reference's Sketch::range_merge / Sketch::sample, logging every sampled
//       component as {u32 round, u32 key, u32 result, u32 0, u64 idx}.
//   params <sketches_factor> <V>...
//       the reference's sizing functions (include/sketch.h:62-76, :181) for each V.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "cc_sketch_alg.h"

namespace {

struct Stream {
  uint32_t V = 0;
  uint64_t n = 0;
  std::vector<uint8_t> rec;  // n * 9 bytes
};

bool read_stream(const char *path, uint64_t max_records, Stream &s) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  if (fread(&s.V, 4, 1, f) != 1 || fread(&s.n, 8, 1, f) != 1) { fclose(f); return false; }
  if (max_records && max_records < s.n) s.n = max_records;
  s.rec.resize(s.n * 9);
  size_t got = fread(s.rec.data(), 1, s.rec.size(), f);
  fclose(f);
  if (got != s.rec.size()) return false;
  return true;
}

inline uint32_t le32(const uint8_t *p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int run_ingest(int argc, char **argv) {
  if (argc < 9) return 2;
  const char *path = argv[2];
  size_t seed = strtoull(argv[3], nullptr, 10);
  double factor = atof(argv[4]);
  int threads = atoi(argv[5]);
  uint64_t max_records = strtoull(argv[6], nullptr, 10);
  std::string dump = argv[7], labels_out = argv[8];
  if (threads < 1) threads = 1;

  Stream s;
  if (!read_stream(path, max_records, s)) {
    fprintf(stderr, "cannot read stream %s\n", path);
    return 1;
  }
  const uint32_t V = s.V;
  for (uint64_t i = 0; i < s.n; ++i) {
    if (le32(&s.rec[9 * i + 1]) >= V || le32(&s.rec[9 * i + 5]) >= V) {
      fprintf(stderr, "record %llu names a vertex >= %u\n", (unsigned long long)i, V);
      return 1;
    }
  }

  CCAlgConfiguration cfg;
  cfg.sketches_factor(factor);
  CCSketchAlg alg(V, seed, cfg);
  alg.allocate_worker_memory(threads);
  const size_t batch = alg.get_desired_updates_per_batch();

  // ---- timed ingest: stand-in gutter (counting sort by endpoint) + workers ----
  double t0 = now_s();
  std::vector<std::vector<uint32_t>> local_cnt(threads, std::vector<uint32_t>(V, 0));
  auto slice = [&](int t, uint64_t &b, uint64_t &e) {
    b = s.n * t / threads;
    e = s.n * (t + 1) / threads;
  };
  {
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
      th.emplace_back([&, t] {
        uint64_t b, e;
        slice(t, b, e);
        auto &cnt = local_cnt[t];
        for (uint64_t i = b; i < e; ++i) {
          const uint8_t *r = &s.rec[9 * i];
          GraphUpdate upd;
          upd.edge.src = le32(r + 1);
          upd.edge.dst = le32(r + 5);
          upd.type = static_cast<UpdateType>(r[0]);
          alg.pre_insert(upd, t);  // eager-DSU hook, called per update by the driver
          ++cnt[upd.edge.src];
          ++cnt[upd.edge.dst];
        }
      });
    for (auto &x : th) x.join();
  }
  // offsets: vertex-major, thread-minor so each thread scatters into its own sub-ranges
  std::vector<uint64_t> vstart(V + 1, 0);
  std::vector<std::vector<uint64_t>> cursor(threads, std::vector<uint64_t>(V, 0));
  {
    uint64_t acc = 0;
    for (uint32_t v = 0; v < V; ++v) {
      vstart[v] = acc;
      for (int t = 0; t < threads; ++t) {
        cursor[t][v] = acc;
        acc += local_cnt[t][v];
      }
    }
    vstart[V] = acc;
  }
  std::vector<uint32_t> nbr(vstart[V]);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
      th.emplace_back([&, t] {
        uint64_t b, e;
        slice(t, b, e);
        auto &cur = cursor[t];
        for (uint64_t i = b; i < e; ++i) {
          const uint8_t *r = &s.rec[9 * i];
          uint32_t u = le32(r + 1), v = le32(r + 5);
          nbr[cur[u]++] = v;
          nbr[cur[v]++] = u;
        }
      });
    for (auto &x : th) x.join();
  }
  {
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
      th.emplace_back([&, t] {
        std::vector<node_id_t> dsts;
        dsts.reserve(batch);
        for (;;) {
          uint32_t v0 = next.fetch_add(64);
          if (v0 >= V) break;
          uint32_t v1 = v0 + 64 < V ? v0 + 64 : V;
          for (uint32_t v = v0; v < v1; ++v) {
            for (uint64_t i = vstart[v]; i < vstart[v + 1]; i += batch) {
              uint64_t j = std::min<uint64_t>(vstart[v + 1], i + batch);
              dsts.assign(nbr.begin() + i, nbr.begin() + j);
              alg.apply_update_batch(t, v, dsts);
            }
          }
        }
      });
    for (auto &x : th) x.join();
  }
  double t1 = now_s();
  const int cached = alg.has_cached_query(CONNECTIVITY) ? 1 : 0;  // before the query
  // ---- timed query ----
  ConnectedComponents cc = alg.connected_components();
  double t2 = now_s();

  if (dump != "-") alg.write_binary(dump);
  if (labels_out != "-") {
    std::vector<uint32_t> lab(V);
    for (auto &set : cc.get_component_sets()) {
      uint32_t k = *set.begin();
      for (auto v : set) lab[v] = k;
    }
    FILE *f = fopen(labels_out.c_str(), "wb");
    fwrite(lab.data(), 4, V, f);
    fclose(f);
  }
#ifdef NO_EAGER_DSU
  const int eager = 0;
#else
  const int eager = 1;
#endif
  printf("{\"V\": %u, \"updates\": %llu, \"threads\": %d, \"eager_dsu\": %d, \"batch\": %zu, "
         "\"ingest_s\": %.6f, \"query_s\": %.6f, \"num_cc\": %u, \"rounds\": %zu, "
         "\"cached_before_query\": %d}\n",
         V, (unsigned long long)s.n, threads, eager, batch, t1 - t0, t2 - t1, (unsigned)cc.size(),
         alg.last_query_rounds, cached);
  return 0;
}

int run_trace(int argc, char **argv) {
  if (argc < 5) return 2;
  std::ifstream in(argv[2], std::ios::binary);
  if (!in) return 1;
  size_t seed;
  node_id_t V;
  double factor;
  in.read((char *)&seed, sizeof(seed));
  in.read((char *)&V, sizeof(V));
  in.read((char *)&factor, sizeof(factor));
  const vec_t len = Sketch::calc_vector_length(V);
  const size_t samples = Sketch::calc_cc_samples(V, factor);
  std::vector<Sketch *> sk(V);
  for (node_id_t v = 0; v < V; ++v) sk[v] = new Sketch(len, seed, in, samples);

  struct Rec {
    uint32_t round, key, result, pad;
    uint64_t idx;
  };
  std::vector<Rec> trace;
  DisjointSetUnion<node_id_t> dsu(V);
  std::vector<node_id_t> root(V), key(V);
  size_t round = 0;
  int status = 0;
  Sketch local(len, seed, samples);
  for (;;) {
    if (round >= samples) {
      status = 3;  // OutOfSamplesException would be thrown by the next Sketch::sample
      break;
    }
    for (node_id_t v = 0; v < V; ++v) root[v] = dsu.find_root(v);
    std::vector<std::vector<node_id_t>> members(V);
    for (node_id_t v = 0; v < V; ++v) members[root[v]].push_back(v);
    std::vector<SketchSample> got;
    std::vector<node_id_t> keys;
    for (node_id_t v = 0; v < V; ++v) {
      if (members[root[v]].empty() || members[root[v]][0] != v) continue;
      local.zero_contents();
      for (node_id_t m : members[root[v]]) local.range_merge(*sk[m], round, 1);
      got.push_back(local.sample());
      keys.push_back(v);
    }
    bool modified = false;
    for (size_t i = 0; i < got.size(); ++i) {
      trace.push_back({(uint32_t)round, keys[i], (uint32_t)got[i].result, 0u, got[i].idx});
      if (got[i].result == FAIL) modified = true;
      if (got[i].result == GOOD) {
        Edge e = inv_concat_pairing_fn(got[i].idx);
        if (e.src >= V || e.dst >= V) { status = 5; continue; }
        if (dsu.merge(e.src, e.dst).merged) modified = true;
      }
    }
    if (status || !modified) break;
    ++round;
  }
  FILE *f = fopen(argv[3], "wb");
  fwrite(trace.data(), sizeof(Rec), trace.size(), f);
  fclose(f);
  std::vector<uint32_t> lab(V, UINT32_MAX), mn(V, UINT32_MAX);
  for (node_id_t v = 0; v < V; ++v) {
    node_id_t r = dsu.find_root(v);
    if (mn[r] == UINT32_MAX) mn[r] = v;
    lab[v] = mn[r];
  }
  f = fopen(argv[4], "wb");
  fwrite(lab.data(), 4, V, f);
  fclose(f);
  for (auto p : sk) delete p;
  printf("{\"V\": %u, \"rounds\": %zu, \"status\": %d, \"samples\": %zu}\n", V, round, status,
         trace.size());
  return 0;
}

// params <sketches_factor> <V>...: the reference's own sizing functions, one JSON line per V.
int run_params(int argc, char **argv) {
  if (argc < 4) return 2;
  double factor = atof(argv[2]);
  for (int i = 3; i < argc; ++i) {
    node_id_t V = (node_id_t)strtoul(argv[i], nullptr, 10);
    vec_t len = Sketch::calc_vector_length(V);
    size_t samples = Sketch::calc_cc_samples(V, factor);
    Sketch sk(len, 0, samples);
    CCAlgConfiguration cfg;
    cfg.sketches_factor(factor);
    printf("{\"V\": %u, \"vector_len\": %llu, \"num_columns\": %zu, \"bkt_per_col\": %zu, "
           "\"num_buckets\": %zu, \"sketch_bytes\": %zu}\n",
           V, (unsigned long long)len, sk.get_columns(), Sketch::calc_bkt_per_col(len),
           sk.get_buckets(), sk.bucket_array_bytes());
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc >= 2 && !strcmp(argv[1], "ingest")) return run_ingest(argc, argv);
  if (argc >= 2 && !strcmp(argv[1], "trace")) return run_trace(argc, argv);
  if (argc >= 2 && !strcmp(argv[1], "params")) return run_params(argc, argv);
  fprintf(stderr,
          "usage: %s ingest <stream> <seed> <sketches_factor> <threads> <max_records|0> "
          "<dump|-> <labels|->\n       %s trace <dump> <trace_out> <labels_out>\n",
          argv[0], argv[0]);
  return 2;
}
