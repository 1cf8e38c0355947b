"""Coded entries and bucket planes, the default ingest of CameoSketch handles up to 2^18 vertices
(every record hashed once; entries XORed into shared-memory bucket planes; the planes' rows XORed
into the sketches in HBM). Edge cases the golden cases do not reach, bit-exact against the oracle,
and the reference's own stream fixture with the queries its test makes."""
import os

import numpy as np
import pytest

from _golden import GOLDEN, canonical, load_case

pytestmark = pytest.mark.gpu


def _alg(gz, V, seed, form=2):
    a = gz.CCSketchAlg(V, seed)
    a.set_tuning(0, 0, 0, form)
    assert a.params.entry_form == form
    return a


def _check(gz, oracle_mod, V, seed, recs, form=2):
    from graphzeppelin_b200 import streams as S
    st = S.Stream(V, recs)
    alg = _alg(gz, V, seed, form)
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    n, exact = oracle_mod.exact_cc(V, st.raw())
    cc = alg.connected_components()
    assert cc.size() == n
    assert (canonical(cc.parent_arr) == exact).all()
    rc, lab, rounds, _ = osk.boruvka(with_trace=False)
    assert alg.last_query_rounds == rounds
    return alg


def test_default_entry_form(gz):
    """Coded entries by default up to 2^18 vertices (gutter bins of one tile of 32 vertices)."""
    a = gz.CCSketchAlg(1 << 18, 1)
    assert a.params.entry_form == 2
    assert a.params.vertices_per_tile == 32 and a.params.vertices_per_bin == 32
    a.close()
    assert gz.CCSketchAlg((1 << 18) + 1, 1).params.entry_form == 1
    a = gz.CCSketchAlg(1024, 1)
    a.set_pipeline(1)
    assert a.params.entry_form == 1  # the staged-tile kernels take plain entries
    a.set_pipeline(-1)
    assert a.params.entry_form == 2


@pytest.mark.parametrize("form", [1, 2, 3])
def test_reference_stream_fixture_with_queries(gz, oracle_mod, form):
    """The reference's test/res/multiples_graph_1024_stream.data, unchanged, as its
    MTStreamWithMultipleQueries test reads it (test/cc_alg_test.cpp:300-350): a query after each
    tenth of the stream, each partition equal to the exact one of the prefix; 78 components at
    the end (test/cc_alg_test.cpp:56)."""
    c, st, labels, _ = load_case("ref_mult_v1024")
    assert st.num_updates == 8528
    V = st.num_vertices
    alg = _alg(gz, V, c["seed"], form)
    driver = gz.GraphSketchDriver(alg, gz.BinaryFileStream(os.path.join(GOLDEN, c["stream"])),
                                  gz.DriverConfiguration(), 4)
    per = st.num_updates // 10
    raw = st.raw()
    for q in range(10):
        end = st.num_updates if q == 9 else per * (q + 1)
        driver.process_stream_until(end if q < 9 else gz.END_OF_STREAM)
        driver.prep_query(gz.CONNECTIVITY)
        cc = alg.connected_components()
        n, exact = oracle_mod.exact_cc(V, raw[:end * 9])
        assert cc.size() == n, q
        assert (canonical(cc.parent_arr) == exact).all(), q
    assert cc.size() == 78
    assert (canonical(cc.parent_arr) == labels).all()


def test_self_loops_cancel(gz, oracle_mod):
    """A record (v, v) reaches v's sketch twice with the same index, so it cancels (the
    reference's update XORs it into sketches[src] and sketches[dst], src/cc_sketch_alg.cpp:127-133)."""
    from graphzeppelin_b200 import streams as S
    rng = np.random.default_rng(3)
    V = 700
    src = rng.integers(0, V, 20000, dtype=np.uint32)
    dst = rng.integers(0, V, 20000, dtype=np.uint32)
    dst[::7] = src[::7]  # one record in seven is a self-loop
    _check(gz, oracle_mod, V, 91, S.make_records(src, dst))


@pytest.mark.parametrize("form", [1, 2, 3])
def test_star_vertex(gz, oracle_mod, form):
    """One vertex adjacent to every other: its 4095 entries land in one tile, all of them in
    the same bucket rows of its sketch."""
    from graphzeppelin_b200 import streams as S
    V = 4096
    leaves = np.arange(1, V, dtype=np.uint32)
    src = np.concatenate([np.zeros(V - 1, np.uint32), leaves[::3]])
    dst = np.concatenate([leaves, np.zeros(leaves[::3].size, np.uint32)])  # some deleted again
    _check(gz, oracle_mod, V, 5150, S.make_records(src, dst), form)


@pytest.mark.parametrize("V", [2, 3, 17, 31, 45, 46, 100, 1000, 1001])
def test_vertex_counts(gz, oracle_mod, V):
    """Tiles past the last vertex, and bucket counts below, at and above the planes' rows
    (V = 17: 9 buckets per column; 45: 11; 46: 12)."""
    from graphzeppelin_b200 import streams as S
    rng = np.random.default_rng(V)
    n = 40 * V
    src = rng.integers(0, V, n, dtype=np.uint32)
    dst = rng.integers(0, V, n, dtype=np.uint32)
    _check(gz, oracle_mod, V, 1000 + V, S.make_records(src, dst))


@pytest.mark.parametrize("form", [2, 3])
def test_deep_depths_of_a_dense_graph(gz, oracle_mod, form):
    """2^12 vertices and 3e6 records: about 2^-11 of the column updates go to depths past the
    planes' rows (XORed into HBM), and a few per million to depths of 15 or more (code 15,
    recomputed); with 3-bit codes, 1 in 128 column updates is an escape (code 7) hashed again."""
    from graphzeppelin_b200 import streams as S
    V = 1 << 12
    st, _ = S.planted_partition_stream_fast(V, 4, seed=9, mean_degree=1400, min_size=256,
                                            churn_fraction=0.1)
    assert st.num_updates > 2_500_000
    alg = _alg(gz, V, 0xDEC0DE, form)
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, 0xDEC0DE)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert alg.num_connected_components() == 4


def test_coded_and_plain_equal_across_flushes(gz, oracle_mod):
    """The same stream in uneven parts with flushes between (sparse launches go in place, dense
    ones through the planes): both entry forms give the oracle's bytes."""
    c, st, labels, _ = load_case("cl_v2048")
    rec = st.records
    cuts = [0, 3, 50, 1000, 1001, 4000, rec.size]
    dumps = []
    for form in (1, 2, 3):
        alg = _alg(gz, 2048, c["seed"], form)
        for a, b in zip(cuts[:-1], cuts[1:]):
            alg.ingest_records(rec[a:b])
            alg.flush()
        dumps.append(alg.dump_sketches())
        assert (canonical(alg.connected_components().parent_arr) == labels).all()
    osk = oracle_mod.OracleSketches(2048, c["seed"])
    osk.apply_records(st.raw())
    for d in dumps:
        assert (d == osk.data).all()


@pytest.mark.parametrize("tiles_per_bin", [1, 4])
def test_three_bit_codes_with_multi_tile_bins(gz, oracle_mod, tiles_per_bin):
    """3-bit coded entries at 2^17 vertices (24 columns: the payload starts past bit 64), in bins
    of one and of four tiles (each tile filters its bin's entries): the oracle's bytes and the
    exact partition."""
    from graphzeppelin_b200 import streams as S
    V = 1 << 17
    rng = np.random.default_rng(70 + tiles_per_bin)
    src = rng.integers(0, V, 400_000, dtype=np.uint32)
    dst = (src + rng.integers(1, 2000, src.size, dtype=np.uint32)) % V
    st = S.Stream(V, S.make_records(src, dst))
    alg = gz.CCSketchAlg(V, 4321)
    alg.set_tuning(0, 0, tiles_per_bin, 3)
    assert alg.params.entry_form == 3
    assert alg.params.vertices_per_bin == 32 * tiles_per_bin
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, 4321)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    n, exact = oracle_mod.exact_cc(V, st.raw())
    cc = alg.connected_components()
    assert cc.size() == n and (canonical(cc.parent_arr) == exact).all()


def test_three_bit_codes_chosen_past_2_19_vertices(gz, oracle_mod):
    """2^19 + 1 vertices (26 columns, 20-bit neighbours): coded entries asked for take 3-bit codes
    (4-bit ones do not fit 16 bytes) in bins of two tiles; the bytes equal the oracle's."""
    from graphzeppelin_b200 import streams as S
    V = (1 << 19) + 1
    rng = np.random.default_rng(19)
    src = rng.integers(0, V, 1_000_000, dtype=np.uint32)
    dst = rng.integers(0, V, src.size, dtype=np.uint32)
    st = S.Stream(V, S.make_records(src, dst))
    alg = gz.CCSketchAlg(V, 1919)
    alg.set_tuning(0, 0, 0, 2)
    assert alg.params.entry_form == 3
    assert alg.params.num_bins <= 8192
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, 1919)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    del osk
    n, exact = oracle_mod.exact_cc(V, st.raw())
    cc = alg.connected_components()
    assert cc.size() == n and (canonical(cc.parent_arr) == exact).all()
    alg.close()
