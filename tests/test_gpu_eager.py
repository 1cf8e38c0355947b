"""Eager DSU on the device handle: the cached answer survives exactly as the oracle's restatement
of the reference's pre_insert says (pinned to the compiled reference in test_eager_dsu.py), and
every answer -- cached or from Boruvka -- is the exact partition."""
import numpy as np
import pytest

from test_eager_dsu import _streams

pytestmark = pytest.mark.gpu


def _canon(labels):
    from _golden import canonical
    return canonical(labels)


@pytest.mark.parametrize("name,V,recs", _streams(), ids=[s[0] for s in _streams()])
@pytest.mark.parametrize("path", ["records", "updates"])
def test_eager_cache_matches_oracle(gz, oracle_mod, name, V, recs, path):
    raw = recs.view(np.uint8).reshape(-1)
    pos, _ = oracle_mod.eager_dsu(V, raw)
    alg = gz.CCSketchAlg(V, 11)
    alg.set_eager_dsu(True)
    if path == "records":
        alg.ingest_records(recs)
    else:
        for r in recs:
            alg.update(gz.GraphUpdate((int(r["src"]), int(r["dst"])), int(r["type"])))
    assert alg.has_cached_query(gz.CONNECTIVITY) == (pos is None), name
    cc = alg.connected_components()
    n, exact = oracle_mod.exact_cc(V, raw)
    assert cc.size() == n and (_canon(cc.parent_arr) == exact).all()
    if pos is None:
        assert alg.last_query_rounds == 0  # answered from the DSU: no Boruvka ran
    alg.close()


def test_eager_across_queries(gz, oracle_mod):
    """cached -> invalidated by a forest-edge toggle -> Boruvka re-seeds the DSU -> cached again;
    point queries and the spanning forest come from the DSU while it is valid."""
    from graphzeppelin_b200 import streams as S
    V = 2000
    st, _ = S.planted_partition_stream(V, 6, 5, mean_degree=8)
    recs = st.records
    a, b = recs[: len(recs) // 2], recs[len(recs) // 2:]
    alg = gz.CCSketchAlg(V, 3)
    alg.set_eager_dsu(True)
    alg.ingest_records(a)
    assert alg.has_cached_query(gz.CONNECTIVITY)
    n, exact = oracle_mod.exact_cc(V, a.view(np.uint8).reshape(-1))
    cc = alg.connected_components()
    assert cc.size() == n and (_canon(cc.parent_arr) == exact).all() and alg.last_query_rounds == 0
    forest = alg.calc_spanning_forest().get_edges()
    assert len(forest) == V - n
    # toggle one forest edge: the cache is gone, the next query runs Boruvka
    e = forest[0]
    alg.update(gz.GraphUpdate((e.src, e.dst), 1))
    assert not alg.has_cached_query(gz.CONNECTIVITY)
    toggle = S.make_records(np.array([e.src], np.uint32), np.array([e.dst], np.uint32), np.array([1], np.uint8))
    so_far = np.concatenate([a, toggle])
    n, exact = oracle_mod.exact_cc(V, so_far.view(np.uint8).reshape(-1))
    cc = alg.connected_components()
    assert cc.size() == n and (_canon(cc.parent_arr) == exact).all() and alg.last_query_rounds > 0
    assert alg.has_cached_query(gz.CONNECTIVITY)
    # inserts after the query keep the DSU valid and extend it
    alg.ingest_records(b)
    full = np.concatenate([so_far, b])
    pos, _ = oracle_mod.eager_dsu(V, full.view(np.uint8).reshape(-1))
    n, exact = oracle_mod.exact_cc(V, full.view(np.uint8).reshape(-1))
    cc = alg.connected_components()
    assert cc.size() == n and (_canon(cc.parent_arr) == exact).all()
    for u, v in [(0, 1), (5, 1999), (17, 400)]:
        assert alg.point_query(u, v) == (exact[u] == exact[v])
    alg.close()


def test_eager_device_records_invalidate(gz):
    import torch
    from graphzeppelin_b200 import streams as S
    st = S.erdos_renyi_stream(500, 0.01, seed=2)
    alg = gz.CCSketchAlg(500, 9)
    alg.set_eager_dsu(True)
    assert alg.has_cached_query(gz.CONNECTIVITY)
    d = torch.from_numpy(st.raw().copy()).cuda()
    alg.ingest_records_device(d.data_ptr(), st.num_updates)
    alg.flush()
    assert not alg.has_cached_query(gz.CONNECTIVITY)
    alg.connected_components()
    assert alg.has_cached_query(gz.CONNECTIVITY)
    alg.close()
