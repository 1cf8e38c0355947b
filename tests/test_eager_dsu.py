"""Eager DSU (the reference's default build): the oracle's sequential restatement agrees with
the compiled reference on whether the cached answer survives a stream, and on its partition."""
import os
import tempfile

import numpy as np
import pytest

from graphzeppelin_b200 import streams as S


def _streams():
    one = S.edge_index(np.array([0, 1], np.uint64), np.array([1, 2], np.uint64))
    toggled = S.make_records(np.array([0, 1, 0], np.uint32), np.array([1, 2, 1], np.uint32))
    cycle_del = S.make_records(np.array([0, 1, 0, 0], np.uint32), np.array([1, 2, 2, 2], np.uint32))
    return [
        ("insert_only_planted", 600, S.planted_partition_stream(600, 5, 3, mean_degree=6)[0].records),
        ("planted_churn", 600, S.planted_partition_stream(600, 5, 4, mean_degree=6, churn_fraction=0.2)[0].records),
        ("multiples", 1024, S.edges_to_stream(1024, S.multiples_graph_edges(1024), 9).records),
        ("forest_edge_toggled", 8, toggled),
        ("cycle_edge_toggled", 8, cycle_del),
        ("chain", 4, S.edges_to_stream(4, one, 1).records),
    ]


@pytest.mark.parametrize("name,V,recs", _streams(), ids=[s[0] for s in _streams()])
def test_eager_oracle_matches_reference(oracle_mod, name, V, recs):
    if not oracle_mod.have_reference():
        pytest.skip("the reference is not compiled here")
    raw = recs.view(np.uint8).reshape(-1)
    pos, labels = oracle_mod.eager_dsu(V, raw)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "s.gzs")
        S.Stream(V, recs).write(p)
        lab = os.path.join(td, "lab.bin")
        r = oracle_mod.ref_ingest(p, 7, 1.0, threads=1, eager=True, labels_path=lab)
        ref_labels = np.fromfile(lab, np.uint32)
    assert r["eager_dsu"] == 1
    assert r["cached_before_query"] == (1 if pos is None else 0), name
    n_cc, exact = oracle_mod.exact_cc(V, raw)
    assert (ref_labels == exact).all() and r["num_cc"] == n_cc
    if pos is None:
        # while valid, the eager partition is the exact one
        assert (labels == exact).all()


def test_eager_oracle_known_cases(oracle_mod):
    toggled = S.make_records(np.array([0, 1, 0], np.uint32), np.array([1, 2, 1], np.uint32))
    assert oracle_mod.eager_dsu(8, toggled.view(np.uint8))[0] == 2
    cyc = S.make_records(np.array([0, 1, 0, 0], np.uint32), np.array([1, 2, 2, 2], np.uint32))
    pos, lab = oracle_mod.eager_dsu(8, cyc.view(np.uint8))
    assert pos is None and lab[2] == 0 and lab[3] == 3  # deleting a cycle edge keeps the DSU
