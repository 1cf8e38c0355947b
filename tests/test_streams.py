"""Stream format and the seeded workload generators."""
import numpy as np

from graphzeppelin_b200 import streams as S


def test_record_layout_and_file_roundtrip(tmp_path):
    r = S.make_records(np.array([1, 7], np.uint32), np.array([2, 3], np.uint32),
                       np.array([0, 1], np.uint8))
    st = S.Stream(10, r)
    raw = st.raw()
    assert raw.size == 18
    assert bytes(raw[:9]) == bytes([0, 1, 0, 0, 0, 2, 0, 0, 0])
    assert bytes(raw[9:]) == bytes([1, 7, 0, 0, 0, 3, 0, 0, 0])
    p = str(tmp_path / "s.bin")
    st.write(p)
    data = open(p, "rb").read()
    assert data[:4] == (10).to_bytes(4, "little") and data[4:12] == (2).to_bytes(8, "little")
    back = S.read_stream(p)
    assert back.num_vertices == 10 and (back.records == r).all()
    assert S.read_stream(p, max_updates=1).num_updates == 1


def test_planted_partition_final_graph_is_planted():
    st, comp = S.planted_partition_stream(512, 4, seed=3, p=0.2, churn_fraction=0.2,
                                          uniform_assignment=True)
    fe = st.final_edges()
    u, v = (fe >> np.uint64(32)).astype(np.int64), (fe & np.uint64(0xFFFFFFFF)).astype(np.int64)
    assert (comp[u] == comp[v]).all()
    # every churn pair appears twice, insert before delete
    idx = S.edge_index(st.records["src"], st.records["dst"])
    uniq, first, cnt = np.unique(idx, return_index=True, return_counts=True)
    assert set(cnt.tolist()) <= {1, 2}
    assert (st.records["type"][first] == 0).all()
    assert (cnt == 2).sum() == round(0.2 * fe.size)


def test_generators_are_deterministic():
    a, _ = S.planted_partition_stream(256, 3, seed=5, p=0.1, churn_fraction=0.1)
    b, _ = S.planted_partition_stream(256, 3, seed=5, p=0.1, churn_fraction=0.1)
    assert (a.records == b.records).all()
    c1 = S.chung_lu_stream(1000, 2.1, 10, 100, seed=1)
    c2 = S.chung_lu_stream(1000, 2.1, 10, 100, seed=1)
    assert (c1.records == c2.records).all()


def test_multiples_graph():
    e = S.multiples_graph_edges(1024)
    assert e.size == 5206
    assert ((e >> np.uint64(32)) < (e & np.uint64(0xFFFFFFFF))).all()


def test_chung_lu_delete_reinsert_semantics():
    st = S.chung_lu_stream(2000, 2.1, 20, 200, seed=4, delete_fraction=0.15, reinsert_fraction=0.5)
    t = st.records["type"]
    ins = (t == 0).sum()
    dele = (t == 1).sum()
    # inserts = E + reinserts, deletes = 15% of E, reinserts = half the deletes
    E = ins - dele // 2
    assert abs(dele - int(0.15 * E)) <= 1
    final = st.final_edges()
    assert final.size == E - dele + dele // 2
