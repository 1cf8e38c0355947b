"""gz_ingest_records_noalloc: record ingest for callers that may not allocate GPU memory (a plugin
inside a framework that owns every device byte through its own pool, or a latency-critical loop
where cudaMalloc / cudaFree would synchronize the device). Its scratch is a fixed device array
inside the library, so the test checks that two calls in a row leave the caller's sketches
byte-identical (the tolerance of every parity test here) to what a handle produces with
gz_ingest_records_device + gz_flush and to the oracle, that a call at the record limit is
exact, and that oversize calls are refused.

This file is collected last on purpose, and passes alone in a fresh process as well as after the
other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_sk, V, seed, factor, d_rec, n):
    return lib.gz_ingest_records_noalloc(ctypes.c_void_p(d_sk), V, seed, factor,
                                         ctypes.c_void_p(d_rec), n, None)


@pytest.mark.parametrize("name,V", [("cl_v2048", 2048), ("sparse_v300", 300), ("er_v64", 64)])
def test_noalloc_matches_handle_on_two_calls(name, V, oracle_mod):
    torch = pytest.importorskip("torch")
    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import _lib
    from _golden import load_case
    c, st, _, _ = load_case(name)
    assert c["num_vertices"] == V
    seed = c["seed"]
    lib = _lib.load()
    ref = gz.CCSketchAlg(V, seed)
    sb = ref.params.sketch_bytes
    d_sk = torch.zeros(V * sb, dtype=torch.uint8, device="cuda")
    half = st.num_updates // 2
    for part in (st.records[:half], st.records[half:]):  # two calls in a row
        raw = np.ascontiguousarray(part).view(np.uint8).reshape(-1)
        d_rec = torch.from_numpy(raw.copy()).cuda()
        torch.cuda.synchronize()
        rc = _noalloc(lib, d_sk.data_ptr(), V, seed, 1.0, d_rec.data_ptr(), part.size)
        assert rc == 0, _lib.last_error()
        ref.ingest_records_device(d_rec.data_ptr(), part.size)
        ref.flush()
        assert (d_sk.cpu().numpy() == ref.dump_sketches()).all()
    ref.close()
    # and directly against the oracle (the CPU restatement of Sketch::update)
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw())
    assert (d_sk.cpu().numpy() == osk.data).all()


def test_noalloc_call_at_the_record_limit(oracle_mod):
    """One call of exactly 2,097,152 records (the entries region of the scratch array filled to
    the last byte), after a small call that left other contents in the array."""
    torch = pytest.importorskip("torch")
    from graphzeppelin_b200 import _lib
    from graphzeppelin_b200 import streams as S
    V, seed = 1 << 15, 777
    st, _ = S.planted_partition_stream_fast(V, 8, seed=4, mean_degree=160, min_size=256,
                                            churn_fraction=0.1)
    assert st.num_updates >= 1 << 21
    recs = st.records[:1 << 21]
    lib = _lib.load()
    _, _, _, sb = oracle_mod.params(V, 1.0)
    d_sk = torch.zeros(V * sb, dtype=torch.uint8, device="cuda")
    small = np.ascontiguousarray(st.records[-1000:]).view(np.uint8).reshape(-1)
    d_small = torch.from_numpy(small.copy()).cuda()
    d_rec = torch.from_numpy(np.ascontiguousarray(recs).view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    assert _noalloc(lib, d_sk.data_ptr(), V, seed, 1.0, d_small.data_ptr(), 1000) == 0, _lib.last_error()
    assert _noalloc(lib, d_sk.data_ptr(), V, seed, 1.0, d_rec.data_ptr(), 1 << 21) == 0, _lib.last_error()
    pick = np.random.default_rng(6).choice(V, 48, replace=False)
    filt = np.zeros(V, np.uint8)
    filt[pick] = 1
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(small, vertex_filter=filt)
    osk.apply_records(np.ascontiguousarray(recs).view(np.uint8).reshape(-1), vertex_filter=filt)
    got = d_sk.cpu().numpy()
    for v in pick:
        assert (got[v * sb:(v + 1) * sb] == osk.sketch(v)).all(), v


@pytest.mark.parametrize("V", [1001, 3])
def test_noalloc_partial_last_tile(V):
    """Vertex counts that leave a partial shared-memory tile (1001 = 250 tiles of 4 + 1; 3 is all
    tail): those vertices take the tail path, the caller's buffer holds exactly V sketches."""
    torch = pytest.importorskip("torch")
    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import _lib
    from graphzeppelin_b200 import streams as S
    st = S.erdos_renyi_stream(V, 0.5 if V < 10 else 0.01, seed=V, churn_fraction=0.3)
    lib = _lib.load()
    ref = gz.CCSketchAlg(V, 4321)
    d_sk = torch.zeros(V * ref.params.sketch_bytes, dtype=torch.uint8, device="cuda")
    half = st.num_updates // 2
    for part in (st.records[:half], st.records[half:]):
        raw = np.ascontiguousarray(part).view(np.uint8).reshape(-1)
        d_rec = torch.from_numpy(raw.copy()).cuda()
        torch.cuda.synchronize()
        assert _noalloc(lib, d_sk.data_ptr(), V, 4321, 1.0, d_rec.data_ptr(), part.size) == 0, \
            _lib.last_error()
        ref.ingest_records_device(d_rec.data_ptr(), part.size)
        ref.flush()
        assert (d_sk.cpu().numpy() == ref.dump_sketches()).all()
    ref.close()


def test_noalloc_rejects_oversize_calls():
    torch = pytest.importorskip("torch")
    from graphzeppelin_b200 import _lib
    lib = _lib.load()
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = _noalloc(lib, d.data_ptr(), 1024, 1, 1.0, d.data_ptr(), (1 << 21) + 1)
    assert rc == _lib.GZ_ERR_INVALID and "records per call" in _lib.last_error()
    rc = _noalloc(lib, d.data_ptr(), (1 << 22) + 1, 1, 1.0, d.data_ptr(), 1)
    assert rc == _lib.GZ_ERR_INVALID
    assert not d.any()
