// Project-written stand-in for StreamingUtilities' graph_zeppelin_common.h, which the
// reference fetches at build time (CMakeLists.txt:54-60) and which is not vendored.
// Only the typedefs the reference's sketch / CC sources use are declared. Widths follow
// the reference's packed Bucket (include/bucket.h:7-12, sizeof == 12): vec_t is 64-bit,
// vec_hash_t is 32-bit; node ids are 32-bit (src/util.cpp:239 shifts by 8*sizeof(node_id_t)).
// Used only to compile the reference into oracle/_ref for parity checks.
#pragma once
#include <cstdint>

typedef uint32_t node_id_t;
typedef uint64_t edge_id_t;
typedef uint64_t vec_t;
typedef uint32_t vec_hash_t;

struct Edge {
  node_id_t src = 0;
  node_id_t dst = 0;
};

enum UpdateType { INSERT = 0, DELETE = 1, BREAKPOINT = 2 };
