"""Queries on a snapshot while ingest resumes (the interleaved-query workload): every answer is
the exact partition of the stream prefix at submission, identical to a blocking query on a
handle fed only that prefix (same roots, same rounds)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_snapshot_queries_interleaved_with_ingest(gz, oracle_mod):
    from graphzeppelin_b200 import streams as S
    V = 3000
    st = S.chung_lu_stream_fast(V, 2.1, 12, 300, seed=4)
    recs = st.records
    cuts = np.linspace(0, len(recs), 6).astype(int)
    alg = gz.CCSketchAlg(V, 21)
    tickets = []
    for k in range(5):
        alg.ingest_records(recs[cuts[k]:cuts[k + 1]])
        tickets.append(alg.query_submit())
        if k >= 1:  # collect the previous answer after more ingest was queued behind it
            cc, rounds = alg.query_wait(tickets[k - 1])
            prefix = recs[:cuts[k]]
            ref = gz.CCSketchAlg(V, 21)
            ref.ingest_records(prefix)
            rcc = ref.connected_components()
            assert (cc.parent_arr == rcc.parent_arr).all() and rounds == ref.last_query_rounds
            n, exact = oracle_mod.exact_cc(V, prefix.view(np.uint8).reshape(-1))
            assert cc.size() == n
            ref.close()
    cc, rounds = alg.query_wait(tickets[-1])
    n, _ = oracle_mod.exact_cc(V, recs.view(np.uint8).reshape(-1))
    assert cc.size() == n == alg.num_connected_components()
    with pytest.raises(gz.GZError):
        alg.query_wait(tickets[-1])  # already collected
    alg.close()


def test_snapshot_query_out_of_samples(gz, oracle_mod, tmp_path):
    V, seed = 16, 7
    osk = oracle_mod.OracleSketches(V, seed)
    rng = np.random.default_rng(3)
    osk.data[:] = rng.integers(0, 256, osk.data.size, dtype=np.uint8)
    p = str(tmp_path / "junk.bin")
    open(p, "wb").write(osk.dump_bytes())
    alg = gz.CCSketchAlg.construct_from_serialized_data(p)
    t = alg.query_submit()
    with pytest.raises(gz.OutOfSamplesException):
        alg.query_wait(t)
    alg.update(gz.GraphUpdate((0, 1)))  # a failed snapshot query does not lock updates
    alg.close()


def test_several_queries_in_flight(gz):
    """Tickets need not be collected in order: three queries are queued between ingest calls,
    then collected last to first; each answer is its own prefix's."""
    from graphzeppelin_b200 import streams as S
    V = 2000
    st = S.chung_lu_stream_fast(V, 2.3, 10, 200, seed=9)
    recs = st.records
    cuts = np.linspace(0, len(recs), 4).astype(int)
    alg = gz.CCSketchAlg(V, 5)
    tickets = []
    for k in range(3):
        alg.ingest_records(recs[cuts[k]:cuts[k + 1]])
        tickets.append(alg.query_submit())
    for k in reversed(range(3)):
        cc, rounds = alg.query_wait(tickets[k])
        ref = gz.CCSketchAlg(V, 5)
        ref.ingest_records(recs[:cuts[k + 1]])
        rcc = ref.connected_components()
        assert (cc.parent_arr == rcc.parent_arr).all() and rounds == ref.last_query_rounds
        ref.close()
    alg.close()
