"""The serving trace generator and the server's admission cost (host only, no GPU)."""
import numpy as np

from graphzeppelin_b200 import serve as SV
from graphzeppelin_b200.streams import RECORD_DTYPE


def test_trace_shape_and_consistency():
    tr = SV.serving_trace(30, 1, log2_v_min=8, log2_v_max=11, requests_per_tenant=8,
                          batch_min=100, batch_max=1500)
    N = tr.time.size
    assert (np.diff(tr.time) >= 0).all()
    assert tr.rec_off.size == N + 1 and tr.rec_off[-1] * 9 == tr.raw.size
    # every tenant's first request is an update batch; queries carry no records
    for t in range(30):
        idx = np.flatnonzero(tr.tenant == t)
        assert idx.size >= 1 and tr.kind[idx[0]] == SV.UPDATE and tr.last_request[t] == idx[-1]
    for i in range(N):
        n = tr.rec_off[i + 1] - tr.rec_off[i]
        assert (n > 0) == (tr.kind[i] == SV.UPDATE)
    # deletions only remove edges the tenant inserted before and still holds
    for t in range(30):
        live = {}
        for i in np.flatnonzero(tr.tenant == t):
            r = tr.records(i).view(RECORD_DTYPE)
            V = tr.num_vertices[t]
            assert (r["src"] < V).all() and (r["dst"] < V).all() and (r["src"] != r["dst"]).all()
            for typ, u, v in zip(r["type"], r["src"], r["dst"]):
                e = (min(u, v), max(u, v))
                if typ == 1:
                    assert live.get(e, 0) > 0
                    live[e] -= 1
                else:
                    live[e] = live.get(e, 0) + 1


def test_trace_mix_and_batch_sizes():
    tr = SV.serving_trace(400, 2, log2_v_min=8, log2_v_max=9, requests_per_tenant=10,
                          batch_min=64, batch_max=128)
    frac = np.bincount(tr.kind, minlength=3) / tr.kind.size
    # the first request of each tenant is forced to be an update batch
    assert abs(frac[1] - 0.08) < 0.02 and abs(frac[2] - 0.02) < 0.01
    n = np.diff(tr.rec_off)[tr.kind == SV.UPDATE]
    assert n.min() >= 1 and n.max() <= 128


def test_trace_is_seeded():
    a = SV.serving_trace(10, 4, log2_v_min=8, log2_v_max=9, batch_min=10, batch_max=20)
    b = SV.serving_trace(10, 4, log2_v_min=8, log2_v_max=9, batch_min=10, batch_max=20)
    assert (a.raw == b.raw).all() and (a.time == b.time).all()


def test_tenant_bytes_is_the_padded_sketch_size(gz, oracle_mod):
    for V in (2, 300, 1024, 5000, 1 << 18):
        C, B, nb, sb = oracle_mod.params(V)
        pad = (V + 63) // 64 * 64
        assert SV.tenant_bytes(V) == (pad * sb + 255) // 256 * 256
