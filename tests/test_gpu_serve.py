"""Serving: every tenant of a SketchServer answers exactly as a CCSketchAlg with its V and seed
fed the same updates -- whatever else the server holds or applies in the same call -- and a
query answers for the state at submission even when ingestion continues before it is read."""
import numpy as np
import pytest

from _golden import canonical

pytestmark = pytest.mark.gpu


def _streams():
    from graphzeppelin_b200 import streams as S
    one_edge = S.edges_to_stream(2, S.edge_index(np.array([0], np.uint64), np.array([1], np.uint64)), 5)
    return [
        (300, 11, S.erdos_renyi_stream(300, 0.02, seed=1, churn_fraction=0.2).records),
        (1024, 12, S.planted_partition_stream(1024, 5, 2, mean_degree=12, churn_fraction=0.1)[0].records),
        (4000, 13, S.chung_lu_stream(4000, 2.3, 10, 300, seed=3).records),
        (2, 14, one_edge.records),
    ]


def _single(gz, V, seed, recs):
    a = gz.CCSketchAlg(V, seed)
    if len(recs):
        a.ingest_records(recs)
    cc = a.connected_components()
    return a, cc


def test_server_tenants_match_single_graph(gz):
    from graphzeppelin_b200.serve import SketchServer
    specs = _streams()
    with SketchServer(1 << 30, 1 << 28) as srv:
        ids = [srv.admit(V, seed) for V, seed, _ in specs]
        # each tenant's stream in three chunks, spread over calls with different tenant subsets
        chunks = [np.array_split(r, 3) for _, _, r in specs]
        calls = [[(0, 0), (1, 0)], [(2, 0), (3, 0), (0, 1)], [(1, 1), (2, 1)],
                 [(0, 2), (1, 2), (2, 2), (3, 1)], [(3, 2)]]
        for call in calls:
            srv.ingest([ids[k] for k, _ in call], [chunks[k][c] for k, c in call])
        out = srv.connected_components(ids)
        for k, (V, seed, recs) in enumerate(specs):
            a, cc = _single(gz, V, seed, recs)
            lab, ncc, rounds, status = out[k]
            assert status == 0 and ncc == cc.size() and rounds == a.last_query_rounds
            assert (lab == cc.parent_arr).all()
            assert srv.dump_sketches(ids[k]).tobytes() == a.dump_sketches().tobytes()
            a.close()


def test_server_query_is_a_snapshot(gz):
    """Ingest continues after a query is submitted: the answer is the submitted state's."""
    from graphzeppelin_b200.serve import SketchServer
    from graphzeppelin_b200 import streams as S
    st, _ = S.planted_partition_stream(2000, 3, 9, mean_degree=10)
    recs = st.records
    first, rest = recs[: len(recs) // 4], recs[len(recs) // 4:]
    with SketchServer(1 << 28, 1 << 28) as srv:
        t = srv.admit(2000, 99)
        srv.ingest([t], [first])
        ticket = srv.query_submit([t])
        srv.ingest([t], [rest])  # proceeds while the query runs
        lab, ncc, rounds, _ = srv.query_wait(ticket, [t])[0]
        a, cc = _single(gz, 2000, 99, first)
        assert ncc == cc.size() and (lab == cc.parent_arr).all() and rounds == a.last_query_rounds
        a.close()
        lab2, ncc2, _, _ = srv.connected_components([t])[0]
        b, cc2 = _single(gz, 2000, 99, recs)
        assert ncc2 == cc2.size() and (lab2 == cc2.parent_arr).all()
        b.close()


def test_server_in_place_queries_and_merged_jobs(gz):
    """Queries that read the sketches in place answer for the state at submission: an ingest or
    an eviction naming a queried tenant waits for the query. Queries queued back to back are
    answered by merged batched runs, each exactly as the tenant's own CCSketchAlg."""
    from graphzeppelin_b200.serve import SketchServer
    specs = _streams()
    halves = [np.array_split(r, 2) for _, _, r in specs]
    with SketchServer(1 << 30, 1 << 26) as srv:
        srv.set_query_snapshot(False)
        ids = [srv.admit(V, seed) for V, seed, _ in specs]
        srv.ingest(ids, [h[0] for h in halves])
        tickets = [srv.query_submit([i]) for i in ids]
        t_all = srv.query_submit(ids[::-1])
        srv.ingest(ids, [h[1] for h in halves])  # waits for the queries above
        out_all = srv.query_wait(t_all, ids[::-1])[::-1]
        for k, (V, seed, _) in enumerate(specs):
            a, cc = _single(gz, V, seed, halves[k][0])
            for lab, ncc, rounds, status in (srv.query_wait(tickets[k], [ids[k]])[0], out_all[k]):
                assert status == 0 and ncc == cc.size() and rounds == a.last_query_rounds
                assert (lab == cc.parent_arr).all()
            a.close()
        final = srv.connected_components(ids)
        tk = srv.query_submit([ids[2]])
        srv.evict(ids[2])  # waits for the query reading its sketches
        lab_e, ncc_e, _, _ = srv.query_wait(tk, [ids[2]])[0]
        for k, (V, seed, recs) in enumerate(specs):
            a, cc = _single(gz, V, seed, recs)
            lab, ncc, rounds, status = final[k]
            assert status == 0 and ncc == cc.size() and rounds == a.last_query_rounds
            assert (lab == cc.parent_arr).all()
            if k == 2:
                assert ncc_e == cc.size() and (lab_e == cc.parent_arr).all()
            a.close()


def test_server_budget_admission_and_eviction(gz):
    from graphzeppelin_b200.serve import BudgetExhausted, SketchServer, tenant_bytes
    c = tenant_bytes(5000)
    with SketchServer(3 * c + 1000, 1 << 27) as srv:
        ids = [srv.admit(5000, s) for s in range(3)]
        used, budget, n = srv.usage()
        assert n == 3 and used == 3 * c and budget >= 3 * c
        with pytest.raises(BudgetExhausted):
            srv.admit(5000, 7)
        srv.evict(ids[1])
        assert srv.usage()[2] == 2
        t = srv.admit(5000, 8)  # reuses the freed range
        srv.ingest([t], [np.zeros(0, np.uint8)])
        lab, ncc, rounds, _ = srv.connected_components([t])[0]
        assert ncc == 5000 and rounds == 0
        with pytest.raises(gz.GZError):
            srv.ingest([ids[1]], [np.zeros(9, np.uint8)])  # evicted


def test_server_bad_vertex_and_duplicates(gz):
    from graphzeppelin_b200.serve import SketchServer
    from graphzeppelin_b200 import streams as S
    with SketchServer(1 << 26, 1 << 26) as srv:
        t = srv.admit(100, 1)
        bad = S.make_records(np.array([5], np.uint32), np.array([100], np.uint32))
        with pytest.raises(gz.BadVertexError):
            srv.ingest([t], [bad.view(np.uint8)])
        with pytest.raises(gz.GZError):
            srv.ingest([t, t], [bad.view(np.uint8), bad.view(np.uint8)])


def test_serving_replay_batched_equals_plain_and_alone(gz, oracle_mod):
    """A small serving trace: the batched server and the plain per-tenant path give the same
    answer to every request; tenants replayed alone answer as they did in the mix; and a tenant's
    sketches equal the oracle's for its full stream."""
    from graphzeppelin_b200 import serve as SV
    tr = SV.serving_trace(24, 5, log2_v_min=8, log2_v_max=12, requests_per_tenant=6,
                          batch_min=200, batch_max=4000, tenant_rate=400.0, request_rate=200.0,
                          mix=(0.6, 0.3, 0.1))
    budget = 6 * SV.tenant_bytes(1 << 12)  # some tenants must wait for others to leave
    b = SV.replay(tr, "batched", budget, time_scale=4.0)
    p = SV.replay(tr, "plain", budget, time_scale=4.0)
    assert len(b.answers) == tr.time.size == len(p.answers)
    assert b.answers == p.answers
    # queries on snapshots, pageable records and one-batch ticks answer the same
    bs = SV.replay(tr, "batched", budget, time_scale=4.0, query_snapshot=True, pin=False,
                   max_tick_updates=1)
    assert bs.answers == p.answers
    assert b.admitted == 24 and b.max_resident < 24 and b.gpu_queries >= 1
    # alone vs in the mix
    for t in (0, 7, 19):
        idx = np.flatnonzero(tr.tenant == t)
        sub = SV.ServingTrace(tr.num_vertices[t:t + 1], tr.seeds[t:t + 1], tr.time[idx],
                              np.zeros(idx.size, np.int64), tr.kind[idx],
                              np.concatenate([[0], np.cumsum(np.diff(tr.rec_off)[idx])]),
                              np.concatenate([tr.records(i) for i in idx] or [np.zeros(0, np.uint8)]),
                              tr.point[idx], np.array([idx.size - 1]))
        alone = SV.replay(sub, "batched", budget, time_scale=4.0)
        assert [alone.answers[k] for k in range(idx.size)] == [b.answers[i] for i in idx]
    # the oracle on one tenant's whole stream
    t = 3
    idx = np.flatnonzero((tr.tenant == t) & (tr.kind == SV.UPDATE))
    raw = np.concatenate([tr.records(i) for i in idx])
    with SV.SketchServer(1 << 28, 1 << 26) as srv:
        sid = srv.admit(int(tr.num_vertices[t]), int(tr.seeds[t]))
        srv.ingest([sid], [raw])
        osk = oracle_mod.OracleSketches(int(tr.num_vertices[t]), int(tr.seeds[t]))
        osk.apply_records(raw)
        assert srv.dump_sketches(sid).tobytes() == osk.data.tobytes()


def test_server_checkpoint_and_readmission(gz, tmp_path):
    """A tenant checkpointed by the server, evicted and re-admitted keeps its sketches and
    answers; files move both ways between the server and CCSketchAlg."""
    from graphzeppelin_b200.serve import SketchServer
    from graphzeppelin_b200 import streams as S
    st, _ = S.planted_partition_stream(1500, 4, 8, mean_degree=7, churn_fraction=0.1)
    recs = st.records
    with SketchServer(1 << 28, 1 << 27) as srv:
        t = srv.admit(1500, 77)
        srv.ingest([t], [recs[: len(recs) // 2]])
        before = srv.dump_sketches(t).tobytes()
        p = str(tmp_path / "tenant.bin")
        srv.write_binary(t, p)
        srv.evict(t)
        t2 = srv.admit_serialized(p)
        assert srv.dump_sketches(t2).tobytes() == before
        srv.ingest([t2], [recs[len(recs) // 2:]])
        lab, ncc, rounds, _ = srv.connected_components([t2])[0]
        a = gz.CCSketchAlg.construct_from_serialized_data(p)
        a.ingest_records(recs[len(recs) // 2:])
        cc = a.connected_components()
        assert ncc == cc.size() and (lab == cc.parent_arr).all() and rounds == a.last_query_rounds
        q = str(tmp_path / "alg.bin")
        a.write_binary(q)
        t3 = srv.admit_serialized(q)
        assert srv.dump_sketches(t3).tobytes() == srv.dump_sketches(t2).tobytes()
        a.close()
