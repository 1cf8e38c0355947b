"""GPU tests of the reference-facing surface: edge cases and error behaviour the reference's own
tests exercise (test/cc_alg_test.cpp, test/sketch_test.cpp), through the C ABI."""
import numpy as np
import pytest

from _golden import canonical, load_case

pytestmark = pytest.mark.gpu


def test_fresh_alg_has_singletons_and_cached_answer(gz):
    alg = gz.CCSketchAlg(100, 1)
    assert alg.has_cached_query(gz.CONNECTIVITY)
    cc = alg.connected_components()
    assert cc.size() == 100
    assert alg.last_query_rounds == 0


def test_empty_stream_and_full_cancellation(gz):
    from graphzeppelin_b200 import streams as S
    alg = gz.CCSketchAlg(256, 9)
    alg.ingest_records(np.zeros(0, S.RECORD_DTYPE))
    st = S.erdos_renyi_stream(256, 0.05, seed=2)
    alg.ingest_records(st)
    alg.ingest_records(st)  # every edge toggled twice: empty graph
    assert not alg.dump_sketches().any()
    cc = alg.connected_components()
    assert cc.size() == 256
    assert alg.last_query_rounds == 0


def test_self_loops_cancel(gz):
    from graphzeppelin_b200 import streams as S
    recs = S.make_records(np.arange(50, dtype=np.uint32), np.arange(50, dtype=np.uint32))
    alg = gz.CCSketchAlg(64, 3)
    alg.ingest_records(recs)
    assert not alg.dump_sketches().any()
    assert alg.connected_components().size() == 64


def test_bad_vertex_is_reported_and_dropped(gz, oracle_mod):
    from graphzeppelin_b200 import streams as S
    alg = gz.CCSketchAlg(64, 3)
    with pytest.raises(gz.BadVertexError):
        alg.apply_update_batch(0, 64, [1])
    with pytest.raises(gz.BadVertexError):
        alg.update(gz.GraphUpdate((1, 70)))
    good = S.make_records(np.array([1, 2], np.uint32), np.array([2, 3], np.uint32))
    bad = S.make_records(np.array([5], np.uint32), np.array([640], np.uint32))
    alg.ingest_records(np.concatenate([good, bad, good[:1]]))
    with pytest.raises(gz.BadVertexError):
        alg.flush()
    # the bad record is dropped, the good ones are kept
    osk = oracle_mod.OracleSketches(64, 3)
    osk.apply_records(np.concatenate([good, good[:1]]).view(np.uint8).reshape(-1))
    assert (alg.dump_sketches() == osk.data).all()


def test_point_query_matches_components(gz):
    """TestPointQuery (test/cc_alg_test.cpp:149-176)."""
    c, st, labels, _ = load_case("mult_v1024")
    alg = gz.CCSketchAlg(1024, c["seed"])
    alg.ingest_records(st)
    sets = alg.connected_components().get_component_sets()
    assert len(sets) == 78
    ccid = np.zeros(1024, int)
    for i, s in enumerate(sets):
        for v in s:
            ccid[v] = i
    for i in range(10):
        for j in range(10):
            assert alg.point_query(i, j) == (ccid[i] == ccid[j])
    # point queries on a fresh update run Boruvka again
    alg.update(gz.GraphUpdate((2, 1019)))
    assert not alg.has_cached_query(gz.CONNECTIVITY)
    assert alg.point_query(0, 0)


def test_reheat_from_serialized(gz, tmp_path):
    """TestCorrectnessOfReheating (test/cc_alg_test.cpp:97-125)."""
    c, st, labels, _ = load_case("cl_v2048")
    alg = gz.CCSketchAlg(2048, c["seed"])
    alg.ingest_records(st)
    p = str(tmp_path / "ckpt.bin")
    alg.write_binary(p)
    orig = alg.connected_components()
    re = gz.CCSketchAlg.construct_from_serialized_data(p)
    assert not re.has_cached_query(gz.CONNECTIVITY)
    assert re.get_seed() == c["seed"] and re.get_num_vertices() == 2048
    rcc = re.connected_components()
    assert rcc.size() == orig.size() == c["num_cc"]
    assert (canonical(rcc.parent_arr) == labels).all()
    assert (re.dump_sketches() == alg.dump_sketches()).all()


def test_spanning_forest_is_a_forest_of_the_graph(gz):
    c, st, labels, _ = load_case("c0_v1024")
    alg = gz.CCSketchAlg(1024, c["seed"])
    alg.ingest_records(st)
    sf = alg.calc_spanning_forest().get_edges()
    final = set(map(int, st.final_edges()))
    assert len(sf) == 1024 - c["num_cc"]
    parent = list(range(1024))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for e in sf:
        assert ((min(e) << 32) | max(e)) in final
        a, b = find(e.src), find(e.dst)
        assert a != b  # no cycles
        parent[a] = b
    got = np.array([find(v) for v in range(1024)])
    assert (canonical(got) == labels).all()


def test_raw_bucket_update_cancels(gz, oracle_mod):
    """TestRawBucketUpdate (test/sketch_test.cpp:423-458) at the CCSketchAlg level."""
    c, st, _, _ = load_case("er_v64")
    alg = gz.CCSketchAlg(64, c["seed"])
    alg.ingest_records(st)
    dump = alg.dump_sketches()
    sb = alg.params.sketch_bytes
    for v in range(64):
        alg.apply_raw_buckets_update(v, dump[v * sb:(v + 1) * sb])
    assert not alg.dump_sketches().any()


def test_out_of_samples_then_locked(gz, oracle_mod, tmp_path):
    """A sketch that never yields a good bucket FAILs every round: OutOfSamplesException after
    num_columns rounds, and (as in the reference, whose update_locked stays set) updates are
    refused afterwards."""
    V, seed = 16, 7
    osk = oracle_mod.OracleSketches(V, seed)
    rng = np.random.default_rng(0)
    osk.data[:] = rng.integers(0, 256, osk.data.size, dtype=np.uint8)
    p = str(tmp_path / "junk.bin")
    open(p, "wb").write(osk.dump_bytes())
    rc, _, rounds, tr = osk.boruvka()
    assert rc == 3
    alg = gz.CCSketchAlg.construct_from_serialized_data(p)
    alg.set_trace(True)
    with pytest.raises(gz.OutOfSamplesException):
        alg.connected_components()
    got = alg.get_trace()
    assert got.size == tr.size and (got["result"] == tr["result"]).all() and \
        (got["idx"] == tr["idx"]).all()
    with pytest.raises(gz.UpdateLockedException):
        alg.update(gz.GraphUpdate((0, 1)))


def test_profile_counters(gz):
    c, st, _, _ = load_case("c0_v1024")
    alg = gz.CCSketchAlg(1024, c["seed"])
    alg.set_profiling(True)
    alg.ingest_records(st)
    alg.connected_components()
    p = alg.get_profile()
    assert p["sketch_update_launches"] >= 1 and p["gutter_launches"] >= 1
    assert p["entries_applied"] == 2 * st.num_updates
    assert p["sketch_update_ms"] > 0 and p["query_ms"] > 0


def test_handles_of_different_geometry_interleave(gz, oracle_mod):
    """Two live handles with different sketch sizes: launches of one must not be limited by
    the shared-memory setting made for the other."""
    from graphzeppelin_b200 import streams as S
    big_st = S.erdos_renyi_stream(1 << 14, 0.001, seed=41)
    small_st = S.erdos_renyi_stream(256, 0.05, seed=42)
    big = gz.CCSketchAlg(1 << 14, 5)
    small = gz.CCSketchAlg(256, 6)
    for part_b, part_s in zip(np.array_split(big_st.records, 3), np.array_split(small_st.records, 3)):
        big.ingest_records(part_b)
        big.flush()
        small.ingest_records(part_s)
        small.flush()
    ob = oracle_mod.OracleSketches(1 << 14, 5)
    ob.apply_records(big_st.raw())
    os_ = oracle_mod.OracleSketches(256, 6)
    os_.apply_records(small_st.raw())
    assert (big.dump_sketches() == ob.data).all()
    assert (small.dump_sketches() == os_.data).all()
