"""CubeSketch (the reference built with -DL0_SAMPLING): the oracle's restatement -- sizing,
update rule, multi-column samples and Boruvka -- against the compiled reference."""
import json
import os
import subprocess
import tempfile

import pytest

from graphzeppelin_b200 import streams as S


def _ref(oracle_mod):
    if not oracle_mod.have_cube_reference():
        pytest.skip("the reference is not compiled here")


def test_cube_sizing_matches_reference(oracle_mod):
    _ref(oracle_mod)
    Vs = [2, 3, 64, 300, 1024, 1 << 14, 1 << 17, 1 << 20]
    for f in (1.0, 0.5, 2.0):
        out = subprocess.run([oracle_mod.REF_CUBE, "params", repr(f)] + [str(v) for v in Vs],
                             check=True, capture_output=True, text=True).stdout
        for V, line in zip(Vs, out.strip().splitlines()):
            r = json.loads(line)
            samples, cps, B = oracle_mod.params_alg(V, f, cube=True)
            assert cps == 7 and r["num_columns"] == samples * cps and r["bkt_per_col"] == B


@pytest.mark.parametrize("V,make", [
    (64, lambda: S.erdos_renyi_stream(64, 0.08, seed=4, churn_fraction=0.2)),
    (300, lambda: S.planted_partition_stream(300, 3, 5, mean_degree=6, churn_fraction=0.1)[0]),
    (1024, lambda: S.edges_to_stream(1024, S.multiples_graph_edges(1024), 3)),
])
def test_cube_dump_labels_trace_match_reference(oracle_mod, V, make):
    _ref(oracle_mod)
    st = make()
    raw = st.raw()
    osk = oracle_mod.OracleSketches(V, 77, cube=True)
    osk.apply_records(raw)
    with tempfile.TemporaryDirectory() as td:
        sp, dp = os.path.join(td, "s.gzs"), os.path.join(td, "d.bin")
        st.write(sp)
        r = oracle_mod.ref_ingest(sp, 77, 1.0, threads=1, dump_path=dp, cube=True)
        dump = open(dp, "rb").read()
        assert dump == osk.dump_bytes()
        info, labels, trace = oracle_mod.ref_trace(dp, cube=True)
    rc, lab, rounds, tr = osk.boruvka()
    assert rc == 0 and info["status"] == 0 and rounds == info["rounds"] == r["rounds"]
    n, exact = oracle_mod.exact_cc(V, raw)
    assert r["num_cc"] == n and (labels == exact).all() and (lab == exact).all()
    assert tr.size == trace.size and (tr["result"] == trace["result"]).all()
    assert (tr["idx"] == trace["idx"]).all()
