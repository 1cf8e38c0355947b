"""Many graphs on one GPU: every graph of a CCSketchBatch must give exactly what a CCSketchAlg with
the same V and seed gives on the same records -- sketch bytes, partition (the same roots),
component count, last_query_rounds and out-of-samples outcome."""
import hashlib

import numpy as np
import pytest

from _golden import canonical, load_case

pytestmark = pytest.mark.gpu


def _mixed_streams():
    from graphzeppelin_b200 import streams as S
    specs = [
        (2, lambda: S.edges_to_stream(2, S.edge_index(np.array([0], np.uint64),
                                                       np.array([1], np.uint64)), 3)),
        (3, lambda: S.erdos_renyi_stream(3, 0.9, seed=5)),
        (1000, lambda: S.planted_partition_stream(1000, 7, 11, p=0.05, churn_fraction=0.1)[0]),
        (257, lambda: S.erdos_renyi_stream(257, 0.02, seed=13, churn_fraction=0.2)),
        (4096, lambda: S.planted_partition_stream(4096, 3, 17, mean_degree=24, churn_fraction=0.1)[0]),
        (64, None),  # no records at all: V singletons
        (1023, lambda: S.chung_lu_stream(1023, 2.5, 12, 200, seed=19)),
        (5000, lambda: S.planted_partition_stream(5000, 12, 23, mean_degree=8, min_size=20)[0]),
        (130, lambda: S.erdos_renyi_stream(130, 0.5, seed=29, churn_fraction=0.5)),
    ]
    Vs, sts = [], []
    for V, mk in specs:
        Vs.append(V)
        sts.append(mk().records if mk else np.zeros(0, dtype=S.RECORD_DTYPE))
    return Vs, sts


def _single(gz, V, seed, records):
    alg = gz.CCSketchAlg(V, seed)
    if len(records):
        alg.ingest_records(records)
    cc = alg.connected_components()
    return alg, cc


def _check_graph(gz, batch, res, g, V, seed, records):
    alg, cc = _single(gz, V, seed, records)
    assert batch.dump_sketches(g).tobytes() == alg.dump_sketches().tobytes(), f"graph {g} sketches"
    assert int(res.num_cc[g]) == cc.size(), f"graph {g} components"
    assert int(res.rounds[g]) == alg.last_query_rounds, f"graph {g} rounds"
    assert (res.labels[g] == cc.parent_arr).all(), f"graph {g} roots"
    alg.close()


def test_batch_matches_single_graph_handles(gz):
    Vs, sts = _mixed_streams()
    seeds = [1000 + 7 * i for i in range(len(Vs))]
    with gz.CCSketchBatch(Vs, seeds) as b:
        for g, V in enumerate(Vs):
            p = b.params[g]
            alg = gz.CCSketchAlg(V, seeds[g])
            assert (p.num_columns, p.bkt_per_col, p.sketch_bytes) == \
                (alg.params.num_columns, alg.params.bkt_per_col, alg.params.sketch_bytes)
            alg.close()
        b.ingest(sts)
        res = b.connected_components()
        assert (res.status == 0).all()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])


def test_batch_golden_cases(gz, oracle_mod):
    """Every committed golden case as one graph of a single batch: each graph's sketches equal
    the oracle's bytes, and its partition, component count and rounds equal the reference's."""
    from _golden import case_names
    cases = [load_case(n) for n in case_names()]
    for factor in sorted({c.get("sketches_factor", 1.0) for c, _, _, _ in cases}):
        group = [(c, st, lab) for c, st, lab, _ in cases if c.get("sketches_factor", 1.0) == factor]
        Vs = [c["num_vertices"] for c, _, _ in group]
        seeds = [c["seed"] for c, _, _ in group]
        with gz.CCSketchBatch(Vs, seeds, sketches_factor=factor) as b:
            b.ingest([st.records for _, st, _ in group])
            res = b.connected_components()
            for g, (c, st, labels) in enumerate(group):
                osk = oracle_mod.OracleSketches(c["num_vertices"], c["seed"], factor)
                osk.apply_records(st.raw())
                assert b.dump_sketches(g).tobytes() == osk.data.tobytes(), c["name"]
                assert (canonical(res.labels[g]) == canonical(labels)).all(), c["name"]
                assert int(res.num_cc[g]) == c["num_cc"], c["name"]
                assert int(res.rounds[g]) == c["rounds"], c["name"]


def test_batch_streamed_in_pieces_and_cleared(gz):
    """Several ingest calls (records of a graph split across calls, some graphs absent from a
    call), a query between them, then clear and a second stream."""
    Vs, sts = _mixed_streams()
    seeds = [31 * i + 3 for i in range(len(Vs))]
    with gz.CCSketchBatch(Vs, seeds) as b:
        first = [s[: len(s) // 3] for s in sts]
        rest = [s[len(s) // 3:] for s in sts]
        b.ingest(first)
        mid = b.connected_components()
        for g, V in enumerate(Vs):
            alg, cc = _single(gz, V, seeds[g], first[g])
            assert (mid.labels[g] == cc.parent_arr).all() and int(mid.rounds[g]) == alg.last_query_rounds
            alg.close()
        b.ingest(rest)
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])
        b.clear()
        b.ingest(rest)
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], rest[g])


def test_batch_device_records_and_tiles(gz):
    """Records already on the device at an odd byte offset, and explicit per-graph tile sizes
    (every graph's tile and bin geometry differs from the default one)."""
    import torch
    Vs, sts = _mixed_streams()
    seeds = [9 * i + 1 for i in range(len(Vs))]
    vpt = [4, 4, 8, 16, 16, 4, 16, 8, 32]
    raw = np.concatenate([s.view(np.uint8).reshape(-1) for s in sts])
    off = np.concatenate([[0], np.cumsum([len(s) for s in sts])]).astype(np.uint64)
    dev = torch.zeros(raw.size + 16, dtype=torch.uint8, device="cuda")
    dev[5:5 + raw.size] = torch.from_numpy(raw).cuda()
    torch.cuda.synchronize()
    with gz.CCSketchBatch(Vs, seeds, vertices_per_tile=vpt) as b:
        for g in range(len(Vs)):
            assert b.params[g].vertices_per_tile == vpt[g]
        b.ingest_device(dev.data_ptr() + 5, off)
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])


def test_batch_out_of_samples_is_per_graph(gz, oracle_mod):
    """One graph's sketches are junk (no good bucket anywhere): that graph alone ends
    out-of-samples after num_columns rounds, as the oracle does; the others answer normally."""
    from graphzeppelin_b200 import streams as S
    V, seed = 16, 7
    osk = oracle_mod.OracleSketches(V, seed)
    rng = np.random.default_rng(0)
    osk.data[:] = rng.integers(0, 256, osk.data.size, dtype=np.uint8)
    rc, _, rounds, _ = osk.boruvka()
    assert rc == 3
    good, _ = S.planted_partition_stream(500, 4, 3, mean_degree=10)
    with gz.CCSketchBatch([500, V, 40], [11, seed, 12]) as b:
        b.load_sketches(1, osk.data)
        b.ingest([good.records, np.zeros(0, S.RECORD_DTYPE),
                  S.erdos_renyi_stream(40, 0.2, seed=4).records])
        res = b.connected_components()
        assert res.out_of_samples(1) and int(res.rounds[1]) == rounds
        with pytest.raises(gz.OutOfSamplesException):
            res.connected_components(1)
        assert not res.out_of_samples(0) and not res.out_of_samples(2)
        alg, cc = _single(gz, 500, 11, good.records)
        assert (res.labels[0] == cc.parent_arr).all()
        alg.close()


def test_batch_bad_vertex(gz):
    from graphzeppelin_b200 import streams as S
    bad = S.make_records(np.array([1], np.uint32), np.array([50], np.uint32))
    with gz.CCSketchBatch([100, 40], [1, 2]) as b:
        with pytest.raises(gz.BadVertexError):
            b.ingest([np.zeros(0, S.RECORD_DTYPE), bad])


def test_batch_many_graphs(gz):
    """512 graphs of uneven size (V log-uniform in [2^6, 2^12]) in one ingest and one query."""
    from graphzeppelin_b200 import streams as S
    rng = np.random.default_rng(2024)
    G = 512
    Vs = np.exp2(rng.uniform(6, 12, G)).astype(int)
    seeds = rng.integers(0, 2**63, G)
    sts = [S.planted_partition_stream(int(V), int(rng.integers(1, 17)), int(s) & 0xffff,
                                      mean_degree=float(rng.uniform(4, 16)), churn_fraction=0.1)[0].records
           for V, s in zip(Vs, seeds)]
    with gz.CCSketchBatch(Vs, seeds) as b:
        b.ingest(sts)
        res = b.connected_components()
        for g in rng.choice(G, 24, replace=False):
            _check_graph(gz, b, res, int(g), int(Vs[g]), int(seeds[g]), sts[g])
        h = hashlib.sha256()
        for g in range(G):
            h.update(res.labels[g].tobytes())
        # repeat: the answer is deterministic
        res2 = b.connected_components()
        h2 = hashlib.sha256()
        for g in range(G):
            h2.update(res2.labels[g].tobytes())
        assert h.digest() == h2.digest() and (res.rounds == res2.rounds).all()


@pytest.mark.parametrize("threads,ctas", [(512, 2), (256, 4), (1024, 1), (384, 1)])
def test_batch_tuning_keeps_results(gz, threads, ctas):
    """Every launch shape and tile choice gives the same bytes; retuning keeps the sketches."""
    Vs, sts = _mixed_streams()
    seeds = [5 * i + 2 for i in range(len(Vs))]
    with gz.CCSketchBatch(Vs, seeds) as b:
        half = [s[: len(s) // 2] for s in sts]
        b.ingest(half)
        b.set_tuning(threads, ctas)
        b.ingest([s[len(s) // 2:] for s in sts])
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])
        with pytest.raises(gz.GZError):
            b.set_tuning(1024, 3)


def test_batch_rejects_oversized_tile(gz):
    with gz.CCSketchBatch([1 << 16, 100], [1, 2]) as b:
        with pytest.raises(gz.GZError):
            b.set_tuning(1024, 1, [64, 4])
        assert b.params[0].vertices_per_tile <= 16


def test_batch_autotune_keeps_sketches_and_results(gz):
    """The autotuner retiles the batch (one vertices-per-tile per size class) without touching
    the sketches; ingest after tuning still matches the single-graph path."""
    Vs, sts = _mixed_streams()
    seeds = [3 * i + 11 for i in range(len(Vs))]
    with gz.CCSketchBatch(Vs, seeds) as b:
        half = [s[: len(s) // 2] for s in sts]
        b.ingest(half)
        before = [b.dump_sketches(g).tobytes() for g in range(len(Vs))]
        vpt = b.autotune(32)
        assert all(v in (4, 8, 16, 32, 64) for v in vpt)
        assert [b.dump_sketches(g).tobytes() for g in range(len(Vs))] == before
        classes = {}
        for g in range(len(Vs)):
            p = b.params[g]
            assert p.vertices_per_tile == vpt[g]
            classes.setdefault((p.num_columns, p.bkt_per_col), set()).add(int(vpt[g]))
        assert all(len(v) == 1 for v in classes.values())
        b.ingest([s[len(s) // 2:] for s in sts])
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])


def test_batch_sparse_ingest_in_place_and_staged(gz):
    """Calls with only a few entries per tile update sketches in place in HBM; calls with many
    stage tiles in shared memory; the two mix within a launch and across calls."""
    from graphzeppelin_b200 import streams as S
    Vs = [4096, 1000, 300, 20000]
    seeds = [21, 22, 23, 24]
    full = [S.erdos_renyi_stream(V, min(1.0, 40.0 / V), seed=V).records for V in Vs]
    with gz.CCSketchBatch(Vs, seeds) as b:
        # sparse calls: a few hundred records per graph, then one dense call with the rest
        cuts = [np.linspace(0, len(r) // 4, 6).astype(int) for r in full]
        for k in range(5):
            b.ingest([r[c[k]:c[k + 1]] for r, c in zip(full, cuts)])
        b.ingest([r[c[-1]:] for r, c in zip(full, cuts)])
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], full[g])


@pytest.mark.parametrize("route", [0.0, 1.0, 1e30])
def test_batch_routes_agree(gz, route):
    """Always staged, the cost model's choice, and always in place give the same bytes."""
    Vs, sts = _mixed_streams()
    seeds = [13 * i + 5 for i in range(len(Vs))]
    with gz.CCSketchBatch(Vs, seeds) as b:
        b.set_route(route)
        parts = [np.array_split(s, 4) for s in sts]
        for k in range(4):
            b.ingest([p[k] for p in parts])
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], sts[g])


def test_batch_hub_bins(gz):
    """Star hubs put up to 40k entries of one call into a single tile's bin, next to tiles of a
    few entries: every graph's bytes and answers equal the single-graph handle's, over several
    calls."""
    from graphzeppelin_b200 import streams as S
    Vs = [10000, 3000, 40000, 700]
    seeds = [31, 32, 33, 34]
    hubs, rests = [], []
    for V in Vs:
        hubs.append(S.edges_to_stream(V, S.edge_index(np.zeros(V - 1, np.uint64),
                                                      np.arange(1, V, dtype=np.uint64)), V).records)
        rests.append(S.erdos_renyi_stream(V, min(1.0, 6.0 / V), seed=V + 1, churn_fraction=0.2).records)
    full = [np.concatenate([h, r]) for h, r in zip(hubs, rests)]
    with gz.CCSketchBatch(Vs, seeds) as b:
        b.ingest(hubs)  # the hubs' bins: 9999 and 39999 entries in one call
        parts = [np.array_split(r, 2) for r in rests]
        for k in range(2):
            b.ingest([p[k] for p in parts])
        res = b.connected_components()
        for g, V in enumerate(Vs):
            _check_graph(gz, b, res, g, V, seeds[g], full[g])
