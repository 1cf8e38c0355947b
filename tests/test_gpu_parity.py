"""GPU path vs the golden vectors from the reference and vs the C oracle (bit-exact).

Every check goes through the C ABI (libgz_b200.so) via the Python mirror of CCSketchAlg."""
import hashlib
import os

import numpy as np
import pytest

from _golden import canonical, case_names, load_case

pytestmark = pytest.mark.gpu


def _alg(gz, V, seed, factor=1.0):
    return gz.CCSketchAlg(V, seed, gz.CCAlgConfiguration().sketches_factor(factor))


def _header(seed, V, factor):
    return (np.array([seed], "<u8").tobytes() + np.array([V], "<u4").tobytes()
            + np.array([factor], "<f8").tobytes())


@pytest.mark.parametrize("form", [1, 2, 3])
@pytest.mark.parametrize("name", case_names())
def test_golden_case_bit_exact(gz, name, form, tmp_path):
    c, st, labels, trace = load_case(name)
    V, seed, f = c["num_vertices"], c["seed"], c["sketches_factor"]
    alg = _alg(gz, V, seed, f)
    alg.set_tuning(0, 0, 0, form)
    alg.set_trace(True)
    alg.ingest_records(st)
    dump = alg.dump_sketches()
    assert hashlib.sha256(_header(seed, V, f) + dump.tobytes()).hexdigest() == c["dump_sha256"]
    path = str(tmp_path / "dump.bin")
    alg.write_binary(path)
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == c["dump_sha256"]
    cc = alg.connected_components()
    assert cc.size() == c["num_cc"]
    assert (canonical(cc.parent_arr) == labels).all()
    assert alg.last_query_rounds == c["rounds"]
    tr = alg.get_trace()
    assert tr.size == trace.size
    for fld in ("round", "key", "result", "idx"):
        assert (tr[fld] == trace[fld]).all(), fld


@pytest.mark.parametrize("name", ["c0_v1024", "mult_v1024", "cl_v2048"])
def test_apply_update_batch_path_equals_records_path(gz, oracle_mod, name):
    """apply_update_batch (one endpoint per call, the driver's worker contract) must give the
    same bytes as the record path and as the oracle's apply_batch."""
    c, st, labels, _ = load_case(name)
    V, seed = c["num_vertices"], c["seed"]
    r = st.records
    src = np.concatenate([r["src"], r["dst"]])
    dst = np.concatenate([r["dst"], r["src"]])
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    alg = _alg(gz, V, seed)
    osk = oracle_mod.OracleSketches(V, seed)
    bounds = np.flatnonzero(np.diff(src)) + 1
    batch = alg.get_desired_updates_per_batch()
    for s_, d_ in zip(np.split(src, bounds), np.split(dst, bounds)):
        for k in range(0, d_.size, batch):
            alg.apply_update_batch(0, int(s_[0]), d_[k:k + batch])
            osk.apply_batch(int(s_[0]), d_[k:k + batch])
    assert (alg.dump_sketches() == osk.data).all()
    cc = alg.connected_components()
    assert (canonical(cc.parent_arr) == labels).all()


def test_update_path_equals_oracle(gz, oracle_mod):
    c, st, labels, _ = load_case("er_v64")
    alg = _alg(gz, 64, c["seed"])
    for rec in st.records:
        alg.update(gz.GraphUpdate((int(rec["src"]), int(rec["dst"])), int(rec["type"])))
    osk = oracle_mod.OracleSketches(64, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


@pytest.mark.parametrize("offset", [0, 1, 3, 7, 8, 12, 15])
def test_device_ingest_any_alignment(gz, oracle_mod, offset):
    torch = pytest.importorskip("torch")
    c, st, labels, _ = load_case("c0_v1024")
    raw = st.raw()
    buf = torch.zeros(raw.size + 32, dtype=torch.uint8, device="cuda")
    buf[offset:offset + raw.size] = torch.from_numpy(raw).cuda()
    torch.cuda.synchronize()
    alg = _alg(gz, 1024, c["seed"])
    alg.ingest_records_device(buf.data_ptr() + offset, st.num_updates)
    cc = alg.connected_components()
    osk = oracle_mod.OracleSketches(1024, c["seed"])
    osk.apply_records(raw)
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(cc.parent_arr) == labels).all()


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("cap", [2, 1000, 4097, 65536])
def test_small_gutter_many_chunks(gz, oracle_mod, cap, form):
    """A tiny device gutter forces many partial applications; bytes must not change."""
    c, st, labels, _ = load_case("cl_v2048")
    alg = _alg(gz, 2048, c["seed"])
    alg.set_tuning(0, 0, 0, form)
    alg.set_gutter_capacity(cap)
    for part in np.array_split(st.records, 7):
        alg.ingest_records(part)
    osk = oracle_mod.OracleSketches(2048, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


def test_tile_that_does_not_fit_is_rejected(gz):
    alg = _alg(gz, 1024, 1)
    with pytest.raises(gz.GZError):
        alg.set_tuning(64, 1024)  # 64 * 4332 bytes > shared memory per block


@pytest.mark.parametrize("vpt,threads,tpb", [(4, 128, 1), (8, 256, 2), (16, 1024, 8), (32, 512, 4),
                                             (32, 1024, 1), (4, 1024, 64), (16, 640, 16)])
def test_tile_shapes_bit_exact(gz, oracle_mod, vpt, threads, tpb):
    """Plain entries through the staged-tile kernel: tiles, bins and block sizes."""
    c, st, labels, _ = load_case("c0_v1024")
    alg = _alg(gz, 1024, c["seed"])
    alg.set_tuning(vpt, threads, tpb, 1)
    assert alg.params.vertices_per_tile == vpt
    assert alg.params.vertices_per_bin == vpt * tpb
    assert alg.params.entry_form == 1
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(1024, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()


@pytest.mark.parametrize("vpt,threads", [(4, 64), (8, 256), (16, 640), (32, 1024), (32, 96),
                                         (16, 1024)])
def test_plane_tile_shapes_bit_exact(gz, oracle_mod, vpt, threads):
    """Coded entries through the bucket planes: every tile size and block size (several warps per
    vertex, or several vertices per warp in the write-back)."""
    c, st, labels, _ = load_case("c0_v1024")
    alg = _alg(gz, 1024, c["seed"])
    alg.set_tuning(vpt, threads, 1, 2)
    assert alg.params.vertices_per_tile == alg.params.vertices_per_bin == vpt
    assert alg.params.entry_form == 2
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(1024, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


@pytest.mark.parametrize("vpt,tpb", [(32, 2), (32, 4), (16, 8), (8, 4)])
def test_plane_tiles_per_bin_bit_exact(gz, oracle_mod, vpt, tpb):
    """Coded entries in gutter bins of several tiles: each tile filters its entries out of the
    bin (per-warp queues), coded and plain chunks alike."""
    c, st, labels, _ = load_case("cl_v2048")
    alg = _alg(gz, 2048, c["seed"])
    alg.set_tuning(vpt, 1024, tpb, 2)
    assert alg.params.vertices_per_tile == vpt
    assert alg.params.vertices_per_bin == vpt * tpb
    half = st.num_updates // 2
    alg.ingest_records(st.records[:half])
    for r in st.records[half:half + 200]:  # plain entries in the same bins
        alg.apply_update_batch(0, int(r["src"]), [int(r["dst"])])
        alg.apply_update_batch(1, int(r["dst"]), [int(r["src"])])
    alg.ingest_records(st.records[half + 200:])
    osk = oracle_mod.OracleSketches(2048, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


def test_coded_entries_reject_bad_shapes(gz):
    alg = _alg(gz, 1024, 5)
    with pytest.raises(gz.GZError):
        alg.set_tuning(8, 1024, 16, 2)
    with pytest.raises(gz.GZError):
        alg.set_tuning(64, 1024, 1, 2)
    assert alg.params.entry_form == 2  # the handle keeps its tiling after a rejected request


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("factor", [0.0, 1.0, 1e9])
@pytest.mark.parametrize("vpt", [4, 16])
def test_direct_route_bit_exact(gz, oracle_mod, vpt, factor, form):
    """Sparse tiles updated in place in HBM (global atomics) instead of staged (plain entries) or
    run through the bucket planes (coded entries): 0 never goes in place, 1e9 sends every tile in
    place, 1 mixes the two by entry count. Bytes must not move."""
    c, st, labels, _ = load_case("c0_v1024")
    alg = _alg(gz, 1024, c["seed"])
    alg.set_tuning(vpt, 1024, 1, form)
    alg.set_direct_factor(factor)
    half = st.num_updates // 2
    rec = st.records
    alg.ingest_records(rec[:half])
    alg.flush()
    alg.ingest_records(rec[half:half + 500])  # a sparse launch: most tiles get few entries
    alg.flush()
    alg.ingest_records(rec[half + 500:])
    osk = oracle_mod.OracleSketches(1024, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    cc = alg.connected_components()
    assert cc.size() == c["num_cc"]
    assert (canonical(cc.parent_arr) == labels).all()


@pytest.mark.parametrize("mode", [1, 3, 4])
@pytest.mark.parametrize("name", ["c0_v1024", "cl_v2048", "mult_v1024"])
def test_pipelined_sketch_update_bit_exact(gz, oracle_mod, name, mode):
    """The pipelined sketch-update kernel (gz_set_pipeline: default, 3 and 4 tile buffers):
    staged tiles, in-place tiles of a sparse launch, several gutter chunks per launch; bytes and
    answer as the reference's."""
    c, st, labels, _ = load_case(name)
    V, seed = c["num_vertices"], c["seed"]
    alg = _alg(gz, V, seed, c["sketches_factor"])
    alg.set_pipeline(mode)
    assert alg.params.vertices_per_bin == alg.params.vertices_per_tile
    alg.set_gutter_capacity(4096)  # many chunks per launch
    rec = st.records
    half = len(rec) // 2
    alg.ingest_records(rec[:half])
    alg.flush()
    alg.ingest_records(rec[half:half + 300])  # a sparse launch: tiles go in place
    alg.flush()
    alg.ingest_records(rec[half + 300:])
    osk = oracle_mod.OracleSketches(V, seed, c["sketches_factor"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    cc = alg.connected_components()
    assert cc.size() == c["num_cc"]
    assert (canonical(cc.parent_arr) == labels).all()


def test_queries_during_stream(gz, oracle_mod):
    """TestQueryDuringStream / MTStreamWithMultipleQueries: 10 queries at stream breakpoints."""
    c, st, _, _ = load_case("c0_v1024")
    V, seed = 1024, c["seed"]
    alg = _alg(gz, V, seed)
    alg.set_trace(True)
    driver = gz.GraphSketchDriver(alg, gz.BinaryFileStream(stream=st))
    n = st.num_updates
    tenth = n // 10
    for q in range(10):
        end = n if q == 9 else tenth * (q + 1)
        driver.process_stream_until(end if q < 9 else gz.END_OF_STREAM)
        driver.prep_query(gz.CONNECTIVITY)
        cc = alg.connected_components()
        osk = oracle_mod.OracleSketches(V, seed)
        osk.apply_records(st.records[:end].view(np.uint8).reshape(-1))
        rc, lab, rounds, tr = osk.boruvka()
        assert rc == 0
        assert (canonical(cc.parent_arr) == lab).all(), q
        assert alg.last_query_rounds == rounds
        got = alg.get_trace()
        assert got.size == tr.size and (got["idx"] == tr["idx"]).all() and \
            (got["result"] == tr["result"]).all()
        ex_n, ex = oracle_mod.exact_cc(V, st.records[:end].view(np.uint8).reshape(-1))
        assert cc.size() == ex_n
    assert driver.get_total_updates() == 2 * n


@pytest.mark.parametrize("path", ["records", "update_batch", "loaded"])
def test_giant_component_merge_paths(gz, oracle_mod, path, tmp_path):
    """A component holding over half the vertices is merged from the XOR of all other vertex
    sketches when every update reached both endpoints (records; a loaded file whose sketches XOR
    to zero), and by the plain merge once apply_update_batch has made the sketches one-sided.
    Labels, rounds and every round's samples equal the oracle's on all three."""
    from graphzeppelin_b200 import streams as S
    V, seed = 3000, 91
    st = S.erdos_renyi_stream(V, 0.0025, seed=7, churn_fraction=0.3)
    alg = _alg(gz, V, seed)
    if path == "update_batch":
        r = st.records
        for a, b_ in zip(r["src"].tolist(), r["dst"].tolist()):
            alg.apply_update_batch(0, a, [b_])
            alg.apply_update_batch(0, b_, [a])
    else:
        alg.ingest_records(st)
    if path == "loaded":
        f = str(tmp_path / "sk.bin")
        alg.write_binary(f)
        alg.close()
        alg = gz.CCSketchAlg.construct_from_serialized_data(f)
    alg.set_trace(True)
    cc = alg.connected_components()
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    rc, lab, rounds, tr = osk.boruvka()
    assert rc == 0
    assert np.bincount(lab).max() * 2 > V  # the case has a giant component
    assert (canonical(cc.parent_arr) == lab).all()
    assert alg.last_query_rounds == rounds
    got = alg.get_trace()
    assert got.size == tr.size
    for fld in ("round", "key", "result", "idx"):
        assert (got[fld] == tr[fld]).all(), fld
    n, exact = oracle_mod.exact_cc(V, st.raw())
    assert cc.size() == n


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("name", ["c0_v1024", "mult_v1024", "cl_v2048"])
def test_per_phase_query_modes(gz, name, mode):
    """gz_set_query_graph(1) runs the Boruvka rounds as a CUDA graph of per-phase kernels, (0) the
    same kernels with the round loop on the host; the default (2) is one cooperative kernel. In
    every mode labels, rounds and every round's samples equal the golden answer of the
    reference."""
    c, st, labels, trace = load_case(name)
    alg = _alg(gz, c["num_vertices"], c["seed"], c["sketches_factor"])
    alg.set_query_graph(mode)
    alg.set_trace(True)
    alg.ingest_records(st)
    cc = alg.connected_components()
    assert cc.size() == c["num_cc"]
    assert (canonical(cc.parent_arr) == labels).all()
    assert alg.last_query_rounds == c["rounds"]
    tr = alg.get_trace()
    assert tr.size == trace.size
    for fld in ("round", "key", "result", "idx"):
        assert (tr[fld] == trace[fld]).all(), fld
    t = alg.query_submit()
    cc2, rounds = alg.query_wait(t)
    assert (cc2.parent_arr == cc.parent_arr).all() and rounds == c["rounds"]


def test_query_modes_past_the_size_switch(gz, oracle_mod):
    """2^18 + 5 vertices, past the size where the default query switches from the one-launch
    kernel to the graph of per-phase kernels: both (and the host loop) give the exact partition
    and the same rounds."""
    from graphzeppelin_b200 import streams as S
    V = (1 << 18) + 5
    rng = np.random.default_rng(41)
    src = rng.integers(0, V, 600000, dtype=np.uint32)
    dst = (src + rng.integers(1, 64, src.size, dtype=np.uint32)) % V  # local edges: many components
    st = S.Stream(V, S.make_records(src, dst))
    n, exact = oracle_mod.exact_cc(V, st.raw())
    rounds = set()
    for mode in (-1, 2, 1, 0):
        alg = gz.CCSketchAlg(V, 777)
        alg.set_query_graph(mode)
        alg.ingest_records(st)
        cc = alg.connected_components()
        assert cc.size() == n, mode
        assert (canonical(cc.parent_arr) == exact).all(), mode
        rounds.add(alg.last_query_rounds)
        alg.close()
    assert len(rounds) == 1


@pytest.mark.parametrize("V", [2, 3, 5, 17, 100, 301])
def test_odd_vertex_counts(gz, oracle_mod, V):
    from graphzeppelin_b200 import streams as S
    st = S.erdos_renyi_stream(V, 0.3, seed=V, churn_fraction=0.5)
    alg = _alg(gz, V, 4242 + V)
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(V, 4242 + V)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    rc, lab, rounds, _ = osk.boruvka(with_trace=False)
    cc = alg.connected_components()
    assert (canonical(cc.parent_arr) == lab).all()
    assert alg.last_query_rounds == rounds


def test_sampled_vertices_of_a_large_graph(gz, oracle_mod):
    """V = 2^17: bytes of 48 random vertex sketches vs the oracle, partition vs exact CC."""
    from graphzeppelin_b200 import streams as S
    V = 1 << 17
    st, planted = S.planted_partition_stream(V, 64, seed=17, mean_degree=40, min_size=256,
                                             churn_fraction=0.1)
    seed = 0xC0FFEE
    alg = _alg(gz, V, seed)
    alg.ingest_records(st)
    dump = alg.dump_sketches()
    rng = np.random.default_rng(1)
    pick = rng.choice(V, 48, replace=False)
    filt = np.zeros(V, np.uint8)
    filt[pick] = 1
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw(), vertex_filter=filt)
    sb = osk.sketch_bytes
    for v in pick:
        assert (dump[v * sb:(v + 1) * sb] == osk.sketch(v)).all(), v
    cc = alg.connected_components()
    n, exact = oracle_mod.exact_cc(V, st.raw())
    assert cc.size() == n >= 64  # small planted components may split at this degree
    assert (canonical(cc.parent_arr) == exact).all()


@pytest.mark.parametrize("vpt,tpb", [(4, 1), (4, 2), (8, 8)])
def test_many_bins_gutter_paths(gz, oracle_mod, vpt, tpb):
    """20000 vertices at 4 vertices per bin exceed the shared-memory sort's bin limit (global
    cursor scatter); coarser bins take the sort-scatter path. Bytes must not depend on it."""
    from graphzeppelin_b200 import streams as S
    V = 20000
    st = S.erdos_renyi_stream(V, 0.0004, seed=21, churn_fraction=0.2)
    alg = _alg(gz, V, 77)
    alg.set_tuning(vpt, 1024, tpb, 1)
    alg.ingest_records(st)
    rng = np.random.default_rng(5)
    pick = rng.choice(V, 64, replace=False)
    filt = np.zeros(V, np.uint8)
    filt[pick] = 1
    osk = oracle_mod.OracleSketches(V, 77)
    osk.apply_records(st.raw(), vertex_filter=filt)
    dump = alg.dump_sketches()
    sb = osk.sketch_bytes
    for v in pick:
        assert (dump[v * sb:(v + 1) * sb] == osk.sketch(v)).all(), v
    n, exact = oracle_mod.exact_cc(V, st.raw())
    cc = alg.connected_components()
    assert cc.size() == n
    assert (canonical(cc.parent_arr) == exact).all()


def test_records_with_more_than_31_columns_use_plain_entries(gz, oracle_mod):
    """sketches_factor 3 gives 41 columns: records are hashed per endpoint (plain entries)."""
    c, st, _, _ = load_case("c0_v1024")
    alg = _alg(gz, 1024, 99, 3.0)
    assert alg.params.num_columns == 41
    assert alg.params.entry_form == 1
    alg.ingest_records(st)
    osk = oracle_mod.OracleSketches(1024, 99, 3.0)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    rc, lab, rounds, _ = osk.boruvka(with_trace=False)
    assert (canonical(alg.connected_components().parent_arr) == lab).all()
    assert alg.last_query_rounds == rounds


def test_coded_entries_at_the_bin_limit(gz, oracle_mod):
    """65536 vertices at 8 per tile: 8192 bins, the most the hash sort-scatter takes (8 bins per
    thread in its scan); 4 per tile (16384 bins) is refused for coded entries."""
    from graphzeppelin_b200 import streams as S
    V = 1 << 16
    st = S.erdos_renyi_stream(V, 0.0002, seed=23, churn_fraction=0.1)
    alg = _alg(gz, V, 31)
    with pytest.raises(gz.GZError):
        alg.set_tuning(4, 1024, 1, 2)
    alg.set_tuning(8, 1024, 1, 2)
    assert alg.params.num_bins == 8192
    alg.ingest_records(st)
    rng = np.random.default_rng(8)
    pick = rng.choice(V, 64, replace=False)
    filt = np.zeros(V, np.uint8)
    filt[pick] = 1
    osk = oracle_mod.OracleSketches(V, 31)
    osk.apply_records(st.raw(), vertex_filter=filt)
    dump = alg.dump_sketches()
    sb = osk.sketch_bytes
    for v in pick:
        assert (dump[v * sb:(v + 1) * sb] == osk.sketch(v)).all(), v
    n, exact = oracle_mod.exact_cc(V, st.raw())
    assert (canonical(alg.connected_components().parent_arr) == exact).all()


def test_mixed_coded_and_plain_chunks(gz, oracle_mod):
    """Records (coded entries) and apply_update_batch (plain entries, hashed where the planes
    apply them) buffered together."""
    c, st, labels, _ = load_case("cl_v2048")
    alg = _alg(gz, 2048, c["seed"])
    alg.set_tuning(0, 0, 1, 2)
    half = st.num_updates // 2
    alg.ingest_records(st.records[:half])
    rest = st.records[half:]
    for r in rest:
        alg.apply_update_batch(0, int(r["src"]), [int(r["dst"])])
        alg.apply_update_batch(1, int(r["dst"]), [int(r["src"])])
    osk = oracle_mod.OracleSketches(2048, c["seed"])
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


def test_host_ingest_waves_match_device_ingest(gz, oracle_mod):
    """4e7 host records cross many wave boundaries (the gutter is folded into the sketches while
    later records are still being copied; the call is cut into a doubling first chunk, full chunks
    and a short last chunk); bytes must equal one device-resident ingest."""
    torch = pytest.importorskip("torch")
    from graphzeppelin_b200 import streams as S
    V = 1 << 14
    st, _ = S.planted_partition_stream_fast(V, 8, seed=3, mean_degree=4900, min_size=256,
                                            churn_fraction=0.1)
    assert st.num_updates > (1 << 25)
    a = _alg(gz, V, 99)
    a.set_gutter_capacity(2 * st.num_updates + 16)
    a.ingest_records(st)
    b = _alg(gz, V, 99)
    b.set_gutter_capacity(2 * st.num_updates + 16)
    d = torch.from_numpy(st.raw()).cuda()
    b.ingest_records_device(d.data_ptr(), st.num_updates)
    da, db = a.dump_sketches(), b.dump_sketches()
    assert (da == db).all()
    pick = np.random.default_rng(2).choice(V, 16, replace=False)
    filt = np.zeros(V, np.uint8)
    filt[pick] = 1
    osk = oracle_mod.OracleSketches(V, 99)
    osk.apply_records(st.raw(), vertex_filter=filt)
    sb = osk.sketch_bytes
    for v in pick:
        assert (da[v * sb:(v + 1) * sb] == osk.sketch(v)).all()
    assert a.num_connected_components() == 8
