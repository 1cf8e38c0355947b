"""Graph update streams in the reference's 9-byte binary format, and seeded generators.

Format (reference README.md "Binary Stream Format"): a 4-byte little-endian ``num_nodes``,
an 8-byte ``num_updates``, then ``num_updates`` records of 9 bytes each:
``u8 type`` (0 insert, 1 delete), ``u32 src``, ``u32 dst``. The sketches treat insert and
delete identically (an XOR toggle, src/cc_sketch_alg.cpp:127-133), so only the parity of the
number of times a pair appears matters for the final graph.

The generators build the synthetic workloads used by the tests and the benchmark. Each takes
an explicit integer seed and is deterministic for it.
"""
from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass

import numpy as np

RECORD_DTYPE = np.dtype([("type", "u1"), ("src", "<u4"), ("dst", "<u4")])
assert RECORD_DTYPE.itemsize == 9
HEADER_BYTES = 12
INSERT, DELETE = 0, 1


@dataclass
class Stream:
    """An update stream held in memory: ``records`` is a packed (n,) RECORD_DTYPE array."""

    num_vertices: int
    records: np.ndarray

    @property
    def num_updates(self) -> int:
        return int(self.records.shape[0])

    def raw(self) -> np.ndarray:
        """The records as a flat uint8 view (n * 9 bytes), as passed to ingest_records."""
        return self.records.view(np.uint8).reshape(-1)

    def to_bytes(self) -> bytes:
        head = np.array([self.num_vertices], "<u4").tobytes() + np.array(
            [self.num_updates], "<u8").tobytes()
        return head + self.records.tobytes()

    def write(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(np.array([self.num_vertices], "<u4").tobytes())
            f.write(np.array([self.num_updates], "<u8").tobytes())
            self.records.tofile(f)

    def final_edges(self) -> np.ndarray:
        """Sorted u64 edge indices ((min << 32) | max) present after the whole stream."""
        return final_edge_set(self.records)


def read_stream(path: str, max_updates: int | None = None) -> Stream:
    """Read a binary stream file (the BinaryFileStream format)."""
    with open(path, "rb") as f:
        head = f.read(HEADER_BYTES)
        if len(head) != HEADER_BYTES:
            raise ValueError(f"{path}: truncated header")
        v = int(np.frombuffer(head[:4], "<u4")[0])
        n = int(np.frombuffer(head[4:], "<u8")[0])
        if max_updates is not None:
            n = min(n, max_updates)
        recs = np.fromfile(f, dtype=RECORD_DTYPE, count=n)
    if recs.shape[0] != n:
        raise ValueError(f"{path}: header says {n} updates, file holds {recs.shape[0]}")
    return Stream(v, recs)


def make_records(src: np.ndarray, dst: np.ndarray, types: np.ndarray | None = None) -> np.ndarray:
    recs = np.empty(src.shape[0], RECORD_DTYPE)
    recs["type"] = INSERT if types is None else types
    recs["src"] = src
    recs["dst"] = dst
    return recs


def edge_index(u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """concat_pairing_fn (src/util.cpp:45-51): (min << 32) | max, as uint64."""
    u = u.astype(np.uint64)
    v = v.astype(np.uint64)
    return (np.minimum(u, v) << np.uint64(32)) | np.maximum(u, v)


def final_edge_set(records: np.ndarray) -> np.ndarray:
    idx = edge_index(records["src"], records["dst"])
    uniq, cnt = np.unique(idx, return_counts=True)
    return uniq[(cnt & 1) == 1]


# ---------------------------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------------------------

def _tri_decode(k: np.ndarray):
    """Triangular index k -> (i, j) with 0 <= i < j, k = j*(j-1)/2 + i."""
    k = k.astype(np.int64)
    j = ((1.0 + np.sqrt(1.0 + 8.0 * k.astype(np.float64))) / 2.0).astype(np.int64)
    j -= (j * (j - 1) // 2 > k)
    j += ((j + 1) * j // 2 <= k)
    i = k - j * (j - 1) // 2
    return i, j


def _planted_edges(rng: np.random.Generator, sizes: np.ndarray, p: float, perm: np.ndarray):
    """Bernoulli(p) edges inside each planted component; returns uint64 edge indices."""
    out = []
    off = 0
    chunk = 1 << 24
    for s in sizes.tolist():
        members = perm[off:off + s]
        off += s
        pairs = s * (s - 1) // 2
        for base in range(0, pairs, chunk):
            cnt = min(chunk, pairs - base)
            hit = np.flatnonzero(rng.random(cnt) < p) + base
            if hit.size == 0:
                continue
            i, j = _tri_decode(hit)
            out.append(edge_index(members[i], members[j]))
    return np.concatenate(out) if out else np.zeros(0, np.uint64)


def _random_nonedges(rng, num_vertices: int, count: int, edges_sorted: np.ndarray):
    """`count` distinct uniform vertex pairs that are neither self-loops nor in edges_sorted."""
    got = np.zeros(0, np.uint64)
    while got.size < count:
        need = int((count - got.size) * 1.2) + 16
        u = rng.integers(0, num_vertices, need, dtype=np.uint64)
        v = rng.integers(0, num_vertices, need, dtype=np.uint64)
        keep = u != v
        idx = edge_index(u[keep], v[keep])
        if edges_sorted.size:
            pos = np.searchsorted(edges_sorted, idx)
            pos = np.minimum(pos, edges_sorted.size - 1)
            idx = idx[edges_sorted[pos] != idx]
        got = np.unique(np.concatenate([got, idx]))
    return rng.permutation(got)[:count]


def _churn_stream(rng, edges: np.ndarray, churn: np.ndarray) -> np.ndarray:
    """Shuffle edge inserts together with insert-then-delete pairs for each churn index."""
    n = edges.size + 2 * churn.size
    keys = np.empty(n, np.uint64)
    types = np.zeros(n, np.uint8)
    keys[:edges.size] = edges
    keys[edges.size:edges.size + churn.size] = churn
    keys[edges.size + churn.size:] = churn
    types[edges.size + churn.size:] = DELETE
    order = rng.permutation(n)
    keys, types = keys[order], types[order]
    # make every churn delete come after its insert: the first occurrence is the insert
    if churn.size:
        is_churn = np.zeros(n, bool)
        is_churn[np.isin(keys, churn)] = True
        ck = keys[is_churn]
        first = np.zeros(ck.size, bool)
        _, first_pos = np.unique(ck, return_index=True)
        first[first_pos] = True
        ct = np.where(first, INSERT, DELETE).astype(np.uint8)
        types[is_churn] = ct
    src = (keys >> np.uint64(32)).astype(np.uint32)
    dst = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    # present each update with a random endpoint order, as a stream would
    flip = rng.random(n) < 0.5
    s2 = np.where(flip, dst, src)
    d2 = np.where(flip, src, dst)
    return make_records(s2, d2, types)


def planted_partition_stream(num_vertices: int, num_components: int, seed: int, *,
                             p: float | None = None, mean_degree: float | None = None,
                             min_size: int = 1, churn_fraction: float = 0.0,
                             uniform_assignment: bool = False):
    """Planted-components graph streamed as shuffled inserts plus insert-then-delete churn.

    Vertices go to ``num_components`` components, either by an independent uniform draw per
    vertex (``uniform_assignment``) or as a random partition with uniform random sizes of at
    least ``min_size``. Each intra-component pair is an edge with probability ``p`` (or the
    single p giving ``mean_degree``). ``churn_fraction * edges`` extra vertex pairs that are not
    edges (inter-component pairs included) are inserted and later deleted, so the final graph
    is the planted one. Returns (Stream, planted component label per vertex).
    """
    rng = np.random.default_rng(seed)
    V, k = num_vertices, num_components
    if uniform_assignment:
        comp = rng.integers(0, k, V)
        perm = np.argsort(comp, kind="stable").astype(np.uint64)
        sizes = np.bincount(comp, minlength=k)
    else:
        extra = V - k * min_size
        cuts = np.sort(rng.integers(0, extra + 1, k - 1))
        sizes = np.diff(np.concatenate([[0], cuts, [extra]])) + min_size
        perm = rng.permutation(V).astype(np.uint64)
    if p is None:
        pairs = float((sizes * (sizes - 1) // 2).sum())
        p = min(1.0, (mean_degree or 0) * V / 2.0 / pairs)
    edges = np.sort(_planted_edges(rng, sizes, p, perm))
    churn = _random_nonedges(rng, V, int(round(churn_fraction * edges.size)), edges)
    recs = _churn_stream(rng, edges, churn)
    label = np.empty(V, np.int64)
    off = 0
    for c, s in enumerate(sizes.tolist()):
        label[perm[off:off + s].astype(np.int64)] = c
        off += s
    return Stream(V, recs), label


def multiples_graph_edges(num_vertices: int = 1024) -> np.ndarray:
    """Edges {i, k*i} for i, k >= 2, k*i < num_vertices: the graph of the reference's fixture
    test/res/multiples_graph_1024.txt (5206 edges, 78 components at 1024 vertices)."""
    out = []
    for i in range(2, num_vertices):
        ks = np.arange(2, (num_vertices - 1) // i + 1, dtype=np.uint64)
        if ks.size:
            out.append(edge_index(np.full(ks.size, i, np.uint64), ks * np.uint64(i)))
    return np.sort(np.concatenate(out))


def edges_to_stream(num_vertices: int, edges: np.ndarray, seed: int,
                    churn_fraction: float = 0.0) -> Stream:
    rng = np.random.default_rng(seed)
    edges = np.sort(edges.astype(np.uint64))
    churn = _random_nonedges(rng, num_vertices, int(round(churn_fraction * edges.size)), edges)
    return Stream(num_vertices, _churn_stream(rng, edges, churn))


def erdos_renyi_stream(num_vertices: int, p: float, seed: int, churn_fraction: float = 0.0):
    rng = np.random.default_rng(seed)
    pairs = num_vertices * (num_vertices - 1) // 2
    m = int(rng.binomial(pairs, p))
    if pairs <= (1 << 26):
        k = rng.choice(pairs, m, replace=False)
    else:
        k = np.unique(rng.integers(0, pairs, int(m * 1.05) + 8))[:m]
    i, j = _tri_decode(k)
    edges = edge_index(i.astype(np.uint64), j.astype(np.uint64))
    return edges_to_stream(num_vertices, edges, seed + 1, churn_fraction)


def chung_lu_stream(num_vertices: int, exponent: float, mean_degree: float, max_degree: int,
                    seed: int, delete_fraction: float = 0.15, reinsert_fraction: float = 0.5):
    """Chung-Lu power-law graph: shuffled inserts, then deletes of a seeded fraction of the
    inserted edges, then re-inserts of a fraction of those (each after its delete)."""
    rng = np.random.default_rng(seed)
    V = num_vertices
    w = np.arange(1, V + 1, dtype=np.float64) ** (-1.0 / (exponent - 1.0))
    w *= mean_degree * V / w.sum()
    w = np.minimum(w, max_degree)
    m = int(w.sum() / 2)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    ids = rng.permutation(V).astype(np.uint64)
    u = ids[np.searchsorted(cdf, rng.random(m))]
    v = ids[np.searchsorted(cdf, rng.random(m))]
    keep = u != v
    edges = rng.permutation(np.unique(edge_index(u[keep], v[keep])))
    nd = int(delete_fraction * edges.size)
    dele = edges[:nd]
    rein = dele[:int(reinsert_fraction * nd)]
    ins_order = rng.permutation(edges)
    # deletes land after all inserts of the first pass, re-inserts after their deletes
    keys = np.concatenate([ins_order, rng.permutation(dele), rng.permutation(rein)])
    types = np.concatenate([np.zeros(edges.size, np.uint8), np.ones(nd, np.uint8),
                            np.zeros(rein.size, np.uint8)])
    src = (keys >> np.uint64(32)).astype(np.uint32)
    dst = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    return Stream(V, make_records(src, dst, types))


# ---------------------------------------------------------------------------------------------
# fast generator (libgz_gen.so): the same planted-partition workload at benchmark scale
# ---------------------------------------------------------------------------------------------

_gen = None


def _genlib():
    global _gen
    if _gen is None:
        import ctypes
        from . import build as _build
        path = _build.build_gen()
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.gzg_planted_edges.restype = ctypes.c_uint64
        L.gzg_planted_edges.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, vp]
        L.gzg_planted_nonedges.restype = None
        L.gzg_planted_nonedges.argtypes = [ctypes.c_uint32, vp, vp, ctypes.c_double,
                                           ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, vp]
        L.gzg_chung_lu_stream.restype = ctypes.c_uint64
        L.gzg_chung_lu_stream.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_uint64, vp]
        L.gzg_shuffle_stream.restype = None
        L.gzg_shuffle_stream.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_uint64, ctypes.c_uint64, vp]
        _gen = L
    return _gen


def planted_partition_stream_fast(num_vertices: int, num_components: int, seed: int, *,
                                  p: float | None = None, mean_degree: float | None = None,
                                  min_size: int = 1, churn_fraction: float = 0.0,
                                  uniform_assignment: bool = False, out: np.ndarray | None = None):
    """Planted-components stream of the same shape as planted_partition_stream, built by the
    multithreaded C generator (counter-based randomness + Feistel shuffle): seconds for 1e8
    records. Returns (Stream, planted component label per vertex). ``out`` may be a
    preallocated uint8 buffer (e.g. pinned memory) of at least 9 * num_updates bytes."""
    L = _genlib()
    rng = np.random.default_rng(seed)
    V, k = num_vertices, num_components
    if uniform_assignment:
        comp = rng.integers(0, k, V).astype(np.uint32)
    else:
        extra = V - k * min_size
        cuts = np.sort(rng.integers(0, extra + 1, k - 1))
        sizes = np.diff(np.concatenate([[0], cuts, [extra]])) + min_size
        comp = np.repeat(np.arange(k, dtype=np.uint32), sizes)[rng.permutation(V)]
    order = np.argsort(comp, kind="stable")
    members = order.astype(np.uint32)
    sizes = np.bincount(comp, minlength=k).astype(np.uint64)
    comp_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    pos = np.empty(V, np.uint32)
    pos[order] = (np.arange(V, dtype=np.uint64) - comp_off[comp[order]]).astype(np.uint32)
    if p is None:
        pairs = float((sizes * (sizes - 1) // 2).sum())
        p = min(1.0, (mean_degree or 0) * V / 2.0 / pairs)
    gseed = int(rng.integers(0, 2**63))
    E = L.gzg_planted_edges(members.ctypes.data, comp_off.ctypes.data, k, p, gseed, None)
    edges = np.empty(E, np.uint64)
    L.gzg_planted_edges(members.ctypes.data, comp_off.ctypes.data, k, p, gseed, edges.ctypes.data)
    nc = int(round(churn_fraction * E))
    cand = np.empty(int(nc * 1.02) + 64, np.uint64)
    L.gzg_planted_nonedges(V, comp.ctypes.data, pos.ctypes.data, p, gseed,
                           int(rng.integers(0, 2**63)), cand.size, cand.ctypes.data)
    _, first = np.unique(cand, return_index=True)
    churn = cand[np.sort(first)][:nc]
    n = E + 2 * churn.size
    buf = out if out is not None else np.empty(n * 9, np.uint8)
    assert buf.size >= n * 9
    L.gzg_shuffle_stream(edges.ctypes.data, E, churn.ctypes.data, churn.size,
                         int(rng.integers(0, 2**63)), buf.ctypes.data)
    recs = buf[:n * 9].view(RECORD_DTYPE)
    return Stream(V, recs), comp.astype(np.int64)


def cached_stream(cache_dir: str, name: str, builder) -> Stream:
    """Build a stream once and keep it as a file under cache_dir (keyed by name)."""
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, hashlib.sha1(name.encode()).hexdigest()[:16] + ".gzs")
    if os.path.exists(path):
        return read_stream(path)
    s = builder()
    tmp = path + f".tmp{os.getpid()}"
    s.write(tmp)
    os.replace(tmp, path)
    return s


def many_graph_streams(num_graphs: int, seed: int, *, log2_v_min: float = 8.0,
                       log2_v_max: float = 16.0, degree_min: float = 8.0,
                       degree_max: float = 256.0, max_components: int = 16,
                       churn_fraction: float = 0.10):
    """Independent planted-components streams of uneven size, one per graph: V log-uniform in
    [2^log2_v_min, 2^log2_v_max], 1..max_components planted components, intra-component edge
    probability set for a mean degree uniform in [degree_min, degree_max], churn as in
    planted_partition_stream. Built by the C generator. Returns (num_vertices, sketch seeds,
    packed records of all graphs back to back as one uint8 array, record offsets (G + 1))."""
    rng = np.random.default_rng(seed)
    Vs = np.exp2(rng.uniform(log2_v_min, log2_v_max, num_graphs)).astype(np.int64)
    Vs = np.maximum(Vs, 2)
    ks = rng.integers(1, max_components + 1, num_graphs)
    degs = rng.uniform(degree_min, degree_max, num_graphs)
    stream_seeds = rng.integers(0, 2**31, num_graphs)
    sketch_seeds = rng.integers(0, 2**63, num_graphs, dtype=np.int64).astype(np.uint64)
    parts = []
    for V, k, d, s in zip(Vs, ks, degs, stream_seeds):
        k = int(min(k, V))
        st, _ = planted_partition_stream_fast(int(V), k, int(s), mean_degree=float(d),
                                              churn_fraction=churn_fraction)
        parts.append(st.records.view(np.uint8).reshape(-1))
    counts = np.array([p.size // 9 for p in parts], np.uint64)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    raw = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    return Vs.astype(np.uint32), sketch_seeds, raw, offsets


def chung_lu_stream_fast(num_vertices: int, exponent: float, mean_degree: float, max_degree: int,
                         seed: int, delete_fraction: float = 0.15, reinsert_fraction: float = 0.5,
                         out: np.ndarray | None = None) -> Stream:
    """Chung-Lu power-law stream from the multithreaded C generator: vertex weights
    (rank)^(-1/(exponent-1)) scaled to mean_degree and capped at max_degree (vertex ids a seeded
    permutation of the ranks), V * mean_degree / 2 inserts of weight-drawn endpoint pairs, then
    deletes of a delete_fraction of them, then re-inserts of a reinsert_fraction of those.
    Repeated pairs toggle, like any repeated update. ``out``: optional preallocated uint8 buffer."""
    L = _genlib()
    rng = np.random.default_rng(seed)
    V = num_vertices
    w = np.arange(1, V + 1, dtype=np.float64) ** (-1.0 / (exponent - 1.0))
    for _ in range(100):  # scale so that the mean degree after the cap is mean_degree
        f = mean_degree * V / np.minimum(w, max_degree).sum()
        w *= f
        if abs(f - 1.0) < 1e-12:
            break
    w = np.minimum(w, max_degree)
    m = int(w.sum() / 2)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    cdf[-1] = 1.0
    ids = rng.permutation(V).astype(np.uint32)
    gseed = int(rng.integers(0, 2**63))
    n = L.gzg_chung_lu_stream(cdf.ctypes.data, ids.ctypes.data, V, m, delete_fraction,
                              reinsert_fraction, gseed, None)
    buf = out if out is not None else np.empty(n * 9, np.uint8)
    assert buf.size >= n * 9
    L.gzg_chung_lu_stream(cdf.ctypes.data, ids.ctypes.data, V, m, delete_fraction,
                          reinsert_fraction, gseed, buf.ctypes.data)
    return Stream(V, buf[:n * 9].view(RECORD_DTYPE))
