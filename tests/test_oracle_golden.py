"""The C restatement (oracle/gz_oracle.c) against the golden vectors made from the reference:
xxHash outputs, sizing, write_binary dump bytes, partitions, Boruvka rounds and traces."""
import hashlib
import os

import numpy as np
import pytest

from _golden import case_names, load_case, params_table, xxh3_vectors


def test_xxh3_matches_libxxhash(oracle_mod):
    vecs = xxh3_vectors()
    assert len(vecs) >= 200
    for v in vecs:
        assert oracle_mod.xxh3_8b(v["value"], v["seed"]) == v["hash"], v


def test_params_match_reference_sizing(oracle_mod):
    for row in params_table():
        C, B, nb, sb = oracle_mod.params(row["V"], row["sketches_factor"])
        assert (C, B, nb, sb) == (row["num_columns"], row["bkt_per_col"], row["num_buckets"],
                                  row["sketch_bytes"]), row


def test_concat_pairing_roundtrip():
    # util_test.cpp TestConcatPairingFn
    from graphzeppelin_b200 import concat_pairing_fn, inv_concat_pairing_fn
    for i in range(0, 200, 7):
        for j in range(0, 200, 3):
            if i == j:
                continue
            e = inv_concat_pairing_fn(concat_pairing_fn(i, j))
            assert (e.src, e.dst) == (min(i, j), max(i, j))


@pytest.mark.parametrize("name", case_names())
def test_oracle_reproduces_reference(oracle_mod, name):
    c, st, labels, trace = load_case(name)
    sk = oracle_mod.OracleSketches(c["num_vertices"], c["seed"], c["sketches_factor"])
    assert sk.apply_records(st.raw()) == 0
    dump = sk.dump_bytes()
    assert len(dump) == c["dump_bytes"]
    assert hashlib.sha256(dump).hexdigest() == c["dump_sha256"]
    rc, lab, rounds, tr = sk.boruvka()
    assert rc == 0
    assert rounds == c["rounds"]
    assert (lab == labels).all()
    assert len(np.unique(lab)) == c["num_cc"]
    assert tr.size == trace.size and (tr == trace).all()
    n, exact = oracle_mod.exact_cc(c["num_vertices"], st.raw())
    assert n == c["exact_num_cc"] == c["num_cc"]
    assert (exact == labels).all()


def test_multiples_graph_has_78_components(oracle_mod):
    # known answer of test/cc_alg_test.cpp:56 and test/util/graph_verifier_test.cpp:30
    from graphzeppelin_b200 import streams as S
    e = S.multiples_graph_edges(1024)
    assert e.size == 5206
    st = S.edges_to_stream(1024, e, seed=9)
    n, _ = oracle_mod.exact_cc(1024, st.raw())
    assert n == 78
    for seed in (1, 2, 3):
        sk = oracle_mod.OracleSketches(1024, seed)
        sk.apply_records(st.raw())
        rc, lab, rounds, _ = sk.boruvka(with_trace=False)
        assert rc == 0 and len(np.unique(lab)) == 78


def test_insert_delete_cancels_to_zero(oracle_mod):
    # sketch_test.cpp TestRawBucketUpdate: merging a sketch into itself cancels to ZERO
    from graphzeppelin_b200 import streams as S
    st = S.erdos_renyi_stream(128, 0.2, seed=3)
    sk = oracle_mod.OracleSketches(128, 5)
    sk.apply_records(st.raw())
    sk.apply_records(st.raw())
    assert not sk.data.any()


def test_out_of_samples_when_every_round_fails(oracle_mod):
    # a component whose sketch never yields a good bucket FAILs every round until the columns
    # run out: Sketch::sample throws OutOfSamplesException (src/sketch.cpp:95-97)
    sk = oracle_mod.OracleSketches(16, 7)
    rng = np.random.default_rng(0)
    sk.data[:] = rng.integers(0, 256, sk.data.size, dtype=np.uint8)
    rc, _, rounds, tr = sk.boruvka()
    assert rc == 3
    assert rounds == sk.C


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "gz_ref_noeager")),
                    reason="oracle/_ref not built (reference tree absent)")
def test_oracle_vs_live_reference_random_streams(oracle_mod, tmp_path):
    from graphzeppelin_b200 import streams as S
    for seed in range(3):
        st = S.erdos_renyi_stream(200, 0.02 + 0.02 * seed, seed=100 + seed, churn_fraction=0.3)
        p = str(tmp_path / f"s{seed}.gzs")
        st.write(p)
        dump = str(tmp_path / f"d{seed}")
        info = oracle_mod.ref_ingest(p, 1000 + seed, threads=3, dump_path=dump)
        sk = oracle_mod.OracleSketches(200, 1000 + seed)
        sk.apply_records(st.raw())
        assert open(dump, "rb").read() == sk.dump_bytes()
        rc, lab, rounds, _ = sk.boruvka(with_trace=False)
        assert rounds == info["rounds"] and len(np.unique(lab)) == info["num_cc"]
