"""CubeSketch handles (the reference built with -DL0_SAMPLING): sketch bytes, partition, rounds and
per-round sample traces equal the oracle's (pinned to the compiled reference in
test_cube_oracle.py), through the shared-memory tile path and, for sketches too large to stage,
the in-place path."""
import numpy as np
import pytest

from _golden import canonical

pytestmark = pytest.mark.gpu


def _streams():
    from graphzeppelin_b200 import streams as S
    return [
        (64, S.erdos_renyi_stream(64, 0.08, seed=4, churn_fraction=0.2)),
        (300, S.planted_partition_stream(300, 3, 5, mean_degree=6, churn_fraction=0.1)[0]),
        (1024, S.edges_to_stream(1024, S.multiples_graph_edges(1024), 3)),
    ]


@pytest.mark.parametrize("idx", range(3))
def test_cube_tile_path_matches_oracle(gz, oracle_mod, idx):
    V, st = _streams()[idx]
    alg = gz.CCSketchAlg(V, 77, sketch_algorithm="cube")
    p = alg.params
    samples, cps, B = oracle_mod.params_alg(V, 1.0, cube=True)
    assert (p.cols_per_sample, p.num_columns, p.bkt_per_col, p.max_rounds) == (7, samples * 7, B, samples)
    assert p.in_place == 0
    alg.set_trace(True)
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, 77, cube=True)
    osk.apply_records(st.raw())
    assert alg.dump_sketches().tobytes() == osk.data.tobytes()
    cc = alg.connected_components()
    rc, lab, rounds, tr = osk.boruvka()
    assert rc == 0 and cc.size() == len(set(lab.tolist())) and alg.last_query_rounds == rounds
    assert (canonical(cc.parent_arr) == lab).all()
    got = alg.get_trace()
    assert got.size == tr.size and (got["result"] == tr["result"]).all() and (got["idx"] == tr["idx"]).all()
    alg.close()


def test_cube_in_place_path_matches_oracle(gz, oracle_mod):
    """V = 2^14: four CubeSketch vertex sketches (56 KB each) exceed a shared-memory tile, so
    records are hashed once and XORed into both endpoints in HBM."""
    from graphzeppelin_b200 import streams as S
    V = 1 << 14
    st, _ = S.planted_partition_stream(V, 6, 9, mean_degree=3, churn_fraction=0.1)
    alg = gz.CCSketchAlg(V, 5, sketch_algorithm="cube")
    assert alg.params.in_place == 1
    half = st.num_updates // 2
    alg.ingest_records(st.records[:half])
    # the per-update paths too: a record through update(), a batch through apply_update_batch()
    r = st.records[half]
    alg.update(gz.GraphUpdate((int(r["src"]), int(r["dst"])), int(r["type"])))
    rest = st.records[half + 1:]
    alg.ingest_records(rest)
    extra_src, extra_dst = 3, np.array([7, 11, 9000], np.uint32)
    alg.apply_update_batch(0, extra_src, extra_dst)
    alg.apply_update_batch(0, int(extra_dst[0]), [extra_src])  # the other endpoint of (3, 7)
    osk = oracle_mod.OracleSketches(V, 5, cube=True)
    osk.apply_records(st.raw())
    extra = S.make_records(np.array([3], np.uint32), np.array([7], np.uint32))
    osk.apply_records(extra.view(np.uint8).reshape(-1))
    for d in (11, 9000):  # one endpoint only, as apply_update_batch does
        one = S.make_records(np.array([3], np.uint32), np.array([d], np.uint32))
        filt = np.zeros(V, np.uint8)
        filt[3] = 1
        osk.apply_records(one.view(np.uint8).reshape(-1), filt)
    assert alg.dump_sketches().tobytes() == osk.data.tobytes()
    cc = alg.connected_components()
    rc, lab, rounds, _ = osk.boruvka(with_trace=False)
    assert rc == 0 and alg.last_query_rounds == rounds and (canonical(cc.parent_arr) == lab).all()
    alg.close()


def test_cube_out_of_samples_and_checkpoint(gz, oracle_mod, tmp_path):
    V, seed = 16, 7
    osk = oracle_mod.OracleSketches(V, seed, cube=True)
    rng = np.random.default_rng(1)
    osk.data[:] = rng.integers(0, 256, osk.data.size, dtype=np.uint8)
    rc, _, rounds, _ = osk.boruvka()
    assert rc == 3
    p = str(tmp_path / "cube.bin")
    open(p, "wb").write(osk.dump_bytes())
    alg = gz.CCSketchAlg.construct_from_serialized_data(p, sketch_algorithm="cube")
    assert alg.dump_sketches().tobytes() == osk.data.tobytes()
    with pytest.raises(gz.OutOfSamplesException):
        alg.connected_components()
    assert alg.last_query_rounds == rounds == alg.params.max_rounds
    alg.close()
