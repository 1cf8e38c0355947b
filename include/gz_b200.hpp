// gz_b200.hpp -- header-only C++ facade over the C ABI (gz_b200.h) with the reference's class
// surface, so C++ code written against GraphZeppelin's CCSketchAlg / GraphSketchDriver
// (include/cc_sketch_alg.h, include/graph_sketch_driver.h) compiles against the B200 path by
// switching includes and linking libgz_b200.so. Status codes become the reference's exceptions.
#pragma once

#include <cstdint>
#include <cstdio>
#include <exception>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gz_b200.h"

namespace gzb200 {

typedef uint32_t node_id_t;
typedef uint64_t edge_id_t;

// ---- exceptions (include/sketch.h:193-204, include/cc_sketch_alg.h:25-29,
//      include/graph_sketch_driver.h:13-21) ---------------------------------------------------
class GZException : public std::runtime_error {
 public:
  GZException(int status, const std::string &msg) : std::runtime_error(msg), status(status) {}
  int status;
};
class OutOfSamplesException : public GZException {
 public:
  explicit OutOfSamplesException(const std::string &m) : GZException(GZ_ERR_OUT_OF_SAMPLES, m) {}
};
class UpdateLockedException : public GZException {
 public:
  UpdateLockedException()
      : GZException(GZ_ERR_LOCKED,
                    "Cannot update the algorithm: Connected components currently running") {}
};
class DriverException : public std::exception {
 public:
  explicit DriverException(std::string m) : msg(std::move(m)) {}
  const char *what() const noexcept override { return msg.c_str(); }

 private:
  std::string msg;
};

inline void check(int rc) {
  if (rc == GZ_OK) return;
  const std::string msg = std::string(gz_status_string(rc)) + ": " + gz_last_error();
  if (rc == GZ_ERR_OUT_OF_SAMPLES) throw OutOfSamplesException(msg);
  if (rc == GZ_ERR_LOCKED) throw UpdateLockedException();
  throw GZException(rc, msg);
}

// ---- plain types -----------------------------------------------------------------------------
enum QueryCode { CONNECTIVITY = GZ_CONNECTIVITY, KSPANNINGFORESTS = GZ_KSPANNINGFORESTS };
enum SampleResult { GOOD = GZ_SAMPLE_GOOD, ZERO = GZ_SAMPLE_ZERO, FAIL = GZ_SAMPLE_FAIL };
enum UpdateType { INSERT = 0, DELETE = 1, BREAKPOINT = 2 };
struct Edge {
  node_id_t src = 0;
  node_id_t dst = 0;
};
struct GraphUpdate {
  Edge edge;
  UpdateType type;
};

// concat_pairing_fn / inv_concat_pairing_fn (src/util.cpp:45-57)
inline edge_id_t concat_pairing_fn(node_id_t i, node_id_t j) {
  if (i > j) std::swap(i, j);
  return ((edge_id_t)i << 32) | j;
}
inline Edge inv_concat_pairing_fn(edge_id_t idx) {
  Edge e;
  e.src = (node_id_t)(idx >> 32);
  e.dst = (node_id_t)(idx & 0xFFFFFFFFu);
  return e;
}

// include/cc_alg_configuration.h
class CCAlgConfiguration {
 public:
  CCAlgConfiguration &disk_dir(std::string d) {
    disk_dir_ = std::move(d);
    return *this;
  }
  CCAlgConfiguration &sketches_factor(double f) {
    sketches_factor_ = f > 0 ? f : 1;
    return *this;
  }
  CCAlgConfiguration &batch_factor(double f) {
    batch_factor_ = f > 0 ? f : 1;
    return *this;
  }
  std::string get_disk_dir() const { return disk_dir_; }
  double get_sketches_factor() const { return sketches_factor_; }
  double get_batch_factor() const { return batch_factor_; }

 private:
  std::string disk_dir_ = ".";
  double sketches_factor_ = 1, batch_factor_ = 1;
};

// include/return_types.h
class ConnectedComponents {
 public:
  ConnectedComponents(std::vector<node_id_t> parent, node_id_t num_cc)
      : parent_(std::move(parent)), num_cc_(num_cc) {}
  node_id_t size() const { return num_cc_; }
  bool is_connected(node_id_t a, node_id_t b) const { return parent_[a] == parent_[b]; }
  std::vector<std::set<node_id_t>> get_component_sets() const {
    std::map<node_id_t, std::set<node_id_t>> tmp;
    for (node_id_t i = 0; i < parent_.size(); ++i) tmp[parent_[i]].insert(i);
    std::vector<std::set<node_id_t>> out;
    out.reserve(tmp.size());
    for (auto &kv : tmp) out.push_back(std::move(kv.second));
    return out;
  }
  const std::vector<node_id_t> &parents() const { return parent_; }

 private:
  std::vector<node_id_t> parent_;
  node_id_t num_cc_;
};

class SpanningForest {
 public:
  explicit SpanningForest(std::vector<Edge> e) : edges_(std::move(e)) {}
  const std::vector<Edge> &get_edges() const { return edges_; }

 private:
  std::vector<Edge> edges_;
};

// ---- CCSketchAlg (include/cc_sketch_alg.h:69-258) ---------------------------------------------
class CCSketchAlg {
 public:
  CCSketchAlg(node_id_t num_vertices, size_t seed, CCAlgConfiguration config = CCAlgConfiguration())
      : config_(config) {
    check(gz_create(num_vertices, seed, config.get_sketches_factor(), config.get_batch_factor(),
                    &h_));
    check(gz_get_params(h_, &p_));
  }
  ~CCSketchAlg() { gz_destroy(h_); }
  CCSketchAlg(const CCSketchAlg &) = delete;
  CCSketchAlg &operator=(const CCSketchAlg &) = delete;

  static CCSketchAlg *construct_from_serialized_data(
      const std::string &input_file, CCAlgConfiguration config = CCAlgConfiguration()) {
    gz_alg_t *h = nullptr;
    check(gz_create_from_serialized(input_file.c_str(), config.get_batch_factor(), &h));
    return new CCSketchAlg(h, config);
  }

  size_t get_desired_updates_per_batch() { return (size_t)p_.desired_updates_per_batch; }
  void pre_insert(GraphUpdate upd, int thr_id = 0) {
    check(gz_pre_insert(h_, upd.edge.src, upd.edge.dst, upd.type, thr_id));
  }
  void allocate_worker_memory(size_t num_workers) {
    check(gz_allocate_worker_memory(h_, num_workers));
  }
  void apply_update_batch(int thr_id, node_id_t src_vertex,
                          const std::vector<node_id_t> &dst_vertices) {
    check(gz_apply_update_batch(h_, thr_id, src_vertex, dst_vertices.data(), dst_vertices.size()));
  }
  bool has_cached_query(int query_code) {
    int out = 0;
    check(gz_has_cached_query(h_, query_code, &out));
    return out != 0;
  }
  void print_configuration() {
    std::printf("Connected Components Algorithm Configuration:\n"
                " Sketching algorithm   = CameoSketch\n"
                " Using Eager DSU       = False\n"
                " Num sketches factor   = %g\n"
                " Batch size factor     = %g\n"
                " On disk data location = %s\n",
                config_.get_sketches_factor(), config_.get_batch_factor(),
                config_.get_disk_dir().c_str());
  }
  void apply_raw_buckets_update(node_id_t src_vertex, const void *raw_buckets) {
    check(gz_apply_raw_buckets_update(h_, src_vertex, raw_buckets));
  }
  void update(GraphUpdate upd) { check(gz_update(h_, upd.edge.src, upd.edge.dst, upd.type)); }

  ConnectedComponents connected_components() {
    std::vector<node_id_t> parent(p_.num_vertices);
    uint32_t n = 0;
    check(gz_connected_components(h_, parent.data(), &n));
    return ConnectedComponents(std::move(parent), n);
  }
  bool point_query(node_id_t a, node_id_t b) {
    int out = 0;
    check(gz_point_query(h_, a, b, &out));
    return out != 0;
  }
  SpanningForest calc_spanning_forest() {
    size_t n = 0;
    check(gz_spanning_forest(h_, nullptr, 0, &n));
    std::vector<uint32_t> buf(2 * (n ? n : 1));
    check(gz_spanning_forest(h_, buf.data(), n, &n));
    std::vector<Edge> e(n);
    for (size_t i = 0; i < n; ++i) {
      e[i].src = buf[2 * i];
      e[i].dst = buf[2 * i + 1];
    }
    return SpanningForest(std::move(e));
  }
  void write_binary(const std::string &filename) { check(gz_write_binary(h_, filename.c_str())); }

  size_t last_query_rounds() const {
    size_t r = 0;
    check(gz_last_query_rounds(h_, &r));
    return r;
  }
  node_id_t get_num_vertices() const { return p_.num_vertices; }
  size_t get_seed() const { return (size_t)p_.seed; }
  size_t max_rounds() const { return (size_t)p_.max_rounds; }

  // device-native additions: whole-stream ingest through the device gutter
  void ingest_records(const void *records, size_t n) { check(gz_ingest_records(h_, records, n)); }
  void ingest_records_device(const void *d_records, size_t n) {
    check(gz_ingest_records_device(h_, d_records, n));
  }
  void flush() { check(gz_flush(h_)); }
  gz_alg_t *handle() { return h_; }

 private:
  CCSketchAlg(gz_alg_t *h, CCAlgConfiguration config) : h_(h), config_(config) {
    check(gz_get_params(h_, &p_));
    config_.sketches_factor(p_.sketches_factor);
  }
  gz_alg_t *h_ = nullptr;
  gz_params_t p_{};
  CCAlgConfiguration config_;
};

// ---- streams + driver (include/graph_sketch_driver.h:70-229) -----------------------------------
// Reader of the binary stream format (4-byte num_nodes, 8-byte num_updates, 9-byte records).
class BinaryFileStream {
 public:
  explicit BinaryFileStream(const std::string &file_name) {
    FILE *f = std::fopen(file_name.c_str(), "rb");
    if (!f) throw DriverException("cannot open " + file_name);
    uint64_t n = 0;
    if (std::fread(&V_, 4, 1, f) != 1 || std::fread(&n, 8, 1, f) != 1) {
      std::fclose(f);
      throw DriverException("truncated stream header");
    }
    rec_.resize(n * 9);
    const size_t got = std::fread(rec_.data(), 1, rec_.size(), f);
    std::fclose(f);
    if (got != rec_.size()) throw DriverException("truncated stream");
    n_ = n;
    break_ = n;
  }
  node_id_t vertices() const { return V_; }
  edge_id_t edges() const { return n_; }
  bool set_break_point(edge_id_t idx) {
    if (idx > n_) idx = n_;
    if (idx < pos_) return false;
    break_ = idx;
    return true;
  }
  bool get_update_is_thread_safe() const { return true; }
  // records from the current position up to the break point
  const uint8_t *take(size_t *n) {
    const uint8_t *p = rec_.data() + pos_ * 9;
    *n = (size_t)(break_ - pos_);
    pos_ = break_;
    return p;
  }

 private:
  node_id_t V_ = 0;
  uint64_t n_ = 0, pos_ = 0, break_ = 0;
  std::vector<uint8_t> rec_;
};

static constexpr edge_id_t END_OF_STREAM = (edge_id_t)-1;

class DriverConfiguration {
 public:
  DriverConfiguration &worker_threads(size_t n) {
    workers_ = n ? n : 1;
    return *this;
  }
  DriverConfiguration &disk_dir(std::string d) {
    disk_dir_ = std::move(d);
    return *this;
  }
  size_t get_worker_threads() const { return workers_; }
  std::string get_disk_dir() const { return disk_dir_; }

 private:
  size_t workers_ = 1;
  std::string disk_dir_ = ".";
};

// The GutteringSystem and worker threads are replaced by the device gutter: records go to the
// GPU as they are, prep_query folds the gutter into the sketches.
template <class Alg>
class GraphSketchDriver {
 public:
  GraphSketchDriver(Alg *alg, BinaryFileStream *stream,
                    DriverConfiguration config = DriverConfiguration(),
                    size_t num_stream_threads = 1)
      : alg_(alg), stream_(stream) {
    (void)num_stream_threads;
    alg_->allocate_worker_memory(config.get_worker_threads());
  }
  void process_stream_until(edge_id_t break_edge_idx) {
    if (!stream_->set_break_point(break_edge_idx))
      throw DriverException("Could not correctly set breakpoint: " +
                            std::to_string(break_edge_idx));
    size_t n = 0;
    const uint8_t *rec = stream_->take(&n);
    if (n) alg_->ingest_records(rec, n);
    total_updates_ += 2 * n;
  }
  void prep_query(int query_code) {
    if (alg_->has_cached_query(query_code)) return;
    alg_->flush();
  }
  void batch_callback(int thr_id, node_id_t src_vertex, const std::vector<node_id_t> &dsts) {
    total_updates_ += dsts.size();
    alg_->apply_update_batch(thr_id, src_vertex, dsts);
  }
  size_t get_total_updates() const { return total_updates_; }

 private:
  Alg *alg_;
  BinaryFileStream *stream_;
  size_t total_updates_ = 0;
};

}  // namespace gzb200
