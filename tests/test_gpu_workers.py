"""Concurrent callers through the boundary. The driver contract calls apply_update_batch from
its worker threads at once (include/graph_sketch_driver.h:28-69; the reference's MultipleWorkers
test runs 8 workers, test/cc_alg_test.cpp:128-147), and stream reader threads hand it records
concurrently. Sketches are XOR sums, so any interleaving must give the oracle's bytes."""
import threading

import numpy as np
import pytest

from _golden import canonical, load_case

pytestmark = pytest.mark.gpu


def _batches(st, batch):
    r = st.records
    src = np.concatenate([r["src"], r["dst"]])
    dst = np.concatenate([r["dst"], r["src"]])
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    bounds = np.flatnonzero(np.diff(src)) + 1
    out = []
    for s_, d_ in zip(np.split(src, bounds), np.split(dst, bounds)):
        for k in range(0, d_.size, batch):
            out.append((int(s_[0]), d_[k:k + batch]))
    return out


def _run_threads(n, fn):
    errs = []

    def wrap(k):
        try:
            fn(k)
        except Exception as e:  # surfaced after join
            errs.append(e)
    ts = [threading.Thread(target=wrap, args=(k,)) for k in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs


@pytest.mark.parametrize("name", ["cl_v2048", "ref_mult_v1024"])
def test_eight_workers_apply_update_batch(gz, oracle_mod, name):
    c, st, labels, _ = load_case(name)
    V, seed = c["num_vertices"], c["seed"]
    alg = gz.CCSketchAlg(V, seed)
    alg.allocate_worker_memory(8)
    # small batches interleave the workers' vertices finely
    batches = _batches(st, max(1, alg.get_desired_updates_per_batch() // 16))
    _run_threads(8, lambda k: [alg.apply_update_batch(k, s, d) for s, d in batches[k::8]])
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    assert (canonical(alg.connected_components().parent_arr) == labels).all()


def test_stream_threads_ingest_records_concurrently(gz, oracle_mod):
    """Four reader threads each hand their own segments of the stream to ingest_records while
    four workers call apply_update_batch on the other half of the stream."""
    c, st, labels, _ = load_case("c0_v1024")
    V, seed = c["num_vertices"], c["seed"]
    alg = gz.CCSketchAlg(V, seed)
    rec = st.records
    half = rec.size // 2
    segs = np.array_split(np.arange(half), 64)
    from graphzeppelin_b200 import streams as S
    tail = S.Stream(V, rec[half:])
    batches = _batches(tail, 64)

    def job(k):
        if k < 4:
            for idx in segs[k::4]:
                alg.ingest_records(rec[idx[0]:idx[-1] + 1])
        else:
            for s, d in batches[k - 4::4]:
                alg.apply_update_batch(k, s, d)
    _run_threads(8, job)
    osk = oracle_mod.OracleSketches(V, seed)
    osk.apply_records(st.raw())
    assert (alg.dump_sketches() == osk.data).all()
    cc = alg.connected_components()
    assert cc.size() == c["num_cc"]
    assert (canonical(cc.parent_arr) == labels).all()
