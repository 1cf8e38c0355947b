// C++ use of the reference-shaped facade (include/gz_b200.hpp), mirroring the reference tests
// test/cc_alg_test.cpp SmallGraphConnectivity (78 components on the multiples graph),
// TestPointQuery and TestCorrectnessOfReheating. Usage: facade_test <multiples stream file>
#include <cstdio>
#include <vector>

#include "gz_b200.hpp"

using namespace gzb200;

#define EXPECT(c)                                                  \
  do {                                                             \
    if (!(c)) {                                                    \
      std::fprintf(stderr, "FAILED %s at line %d\n", #c, __LINE__); \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  BinaryFileStream stream(argv[1]);
  const node_id_t num_nodes = stream.vertices();
  CCSketchAlg cc_alg{num_nodes, 777};
  GraphSketchDriver<CCSketchAlg> driver(&cc_alg, &stream, DriverConfiguration());
  driver.process_stream_until(END_OF_STREAM);
  driver.prep_query(CONNECTIVITY);
  EXPECT(driver.get_total_updates() == 2 * stream.edges());
  auto cc = cc_alg.connected_components();
  EXPECT(cc.size() == 78);

  // point queries agree with the component sets
  auto sets = cc.get_component_sets();
  std::vector<size_t> ccid(num_nodes);
  for (size_t i = 0; i < sets.size(); ++i)
    for (node_id_t v : sets[i]) ccid[v] = i;
  for (node_id_t i = 0; i < 10; ++i)
    for (node_id_t j = 0; j < 10; ++j) EXPECT(cc_alg.point_query(i, j) == (ccid[i] == ccid[j]));

  // reheat from a checkpoint
  cc_alg.write_binary(argv[2]);
  CCSketchAlg *re = CCSketchAlg::construct_from_serialized_data(argv[2]);
  EXPECT(!re->has_cached_query(CONNECTIVITY));
  EXPECT(re->connected_components().size() == 78);
  delete re;

  // the driver's worker contract: apply_update_batch of both directions
  CCSketchAlg alg2{num_nodes, 777};
  alg2.apply_update_batch(0, 2, {4, 6});
  alg2.apply_update_batch(1, 4, {2});
  alg2.apply_update_batch(1, 6, {2});
  EXPECT(alg2.connected_components().size() == num_nodes - 2);
  EXPECT(alg2.point_query(4, 6));
  bool locked = false;
  try {
    alg2.apply_update_batch(0, num_nodes, {1});
  } catch (const GZException &e) {
    locked = e.status == GZ_ERR_BAD_VERTEX;
  }
  EXPECT(locked);
  std::printf("facade ok: %u components, %zu rounds\n", cc.size(), cc_alg.last_query_rounds());
  return 0;
}
