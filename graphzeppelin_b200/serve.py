"""Serving many tenants' connectivity sketches on one GPU.

A tenant is one CCSketchAlg (include/cc_sketch_alg.h:69) with its own vertex count and seed.
``SketchServer`` wraps the gz_server_* entry points: tenants are admitted while their sketch bytes
fit a device budget, update batches of many tenants are applied by one batched ingest, and
connectivity queries run on a device snapshot (or on the sketches in place, the tenant's ingest
held until the answer) while later ingests proceed.

``serving_trace`` builds a seeded request trace (tenant arrivals and per-tenant requests on
Poisson processes; update batches with deletions of live edges; connectivity and point queries),
and ``replay`` runs a trace against either the batched server or the plain path -- one
CCSketchAlg per tenant, each request handled on its own -- recording throughput, query latency,
admissions and every answer, so the two can be compared answer for answer.
"""
from __future__ import annotations

import ctypes
import gc
import hashlib
import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np

from . import _lib
from .cc import CCSketchAlg, GZError, _as_raw, _check, _ptr
from .streams import RECORD_DTYPE

UPDATE, CONNECTIVITY_QUERY, POINT_QUERY = 0, 1, 2


class BudgetExhausted(GZError):
    """The server's sketch-byte budget has no room for the tenant (GZ_ERR_BUDGET)."""


def _check_srv(rc: int):
    if rc == _lib.GZ_ERR_BUDGET:
        raise BudgetExhausted(rc, _lib.last_error())
    _check(rc)


def tenant_bytes(num_vertices: int, sketches_factor: float = 1.0) -> int:
    """Device bytes one tenant's sketches take from a server budget."""
    lib = _lib.load()
    out = ctypes.c_uint64()
    _check(lib.gz_server_tenant_bytes(num_vertices, sketches_factor, ctypes.byref(out)))
    return int(out.value)


class SketchServer:
    def __init__(self, budget_bytes: int, snapshot_bytes: int, sketches_factor: float = 1.0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        _check(self.lib.gz_server_create(int(budget_bytes), int(snapshot_bytes), sketches_factor,
                                         ctypes.byref(h)))
        self._h = h
        self.num_vertices: Dict[int, int] = {}
        self._sizes: Dict[int, List[int]] = {}  # ticket -> V of each queried tenant

    def close(self):
        if getattr(self, "_h", None):
            self.lib.gz_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, num_vertices: int, seed: int) -> int:
        t = ctypes.c_uint32()
        _check_srv(self.lib.gz_server_admit(self._h, num_vertices, int(seed) & (2**64 - 1),
                                            ctypes.byref(t)))
        self.num_vertices[t.value] = int(num_vertices)
        return int(t.value)

    def evict(self, tenant: int) -> None:
        _check(self.lib.gz_server_evict(self._h, tenant))
        self.num_vertices.pop(tenant, None)

    def set_route(self, sparse_factor: float) -> None:
        """Per-call routing between in-place and staged ingest (gz_server_set_route)."""
        _check(self.lib.gz_server_set_route(self._h, float(sparse_factor)))

    def set_query_snapshot(self, snapshot: bool) -> None:
        """True (the default): queries copy their tenants' sketches to a snapshot, so ingest of
        those tenants may go on at once. False: queries read the sketches in place; an ingest or
        eviction naming a tenant with an unfinished query waits for it."""
        _check(self.lib.gz_server_set_query_snapshot(self._h, int(bool(snapshot))))

    def usage(self):
        used, budget, n = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        _check(self.lib.gz_server_usage(self._h, ctypes.byref(used), ctypes.byref(budget),
                                        ctypes.byref(n)))
        return int(used.value), int(budget.value), int(n.value)

    def params(self, tenant: int):
        p = _lib.gz_params_t()
        _check(self.lib.gz_server_get_params(self._h, tenant, ctypes.byref(p)))
        return p

    def ingest(self, tenants: Sequence[int], raws: Sequence[np.ndarray]) -> None:
        """Apply one update batch per listed tenant (each a packed 9-byte record buffer)."""
        if not tenants:
            return
        ids = np.ascontiguousarray(tenants, dtype=np.uint32)
        raws = [_as_raw(r) for r in raws]
        off = np.zeros(len(raws) + 1, np.uint64)
        off[1:] = np.cumsum([r.size // 9 for r in raws])
        buf = np.concatenate(raws)
        _check(self.lib.gz_server_ingest(self._h, ids.size, _ptr(ids),
                                         _ptr(buf) if buf.size else None, _ptr(off)))

    def ingest_segments(self, tenants: Sequence[int], segments: Sequence[np.ndarray]) -> None:
        """Apply update batches given as segments (tenants[k]'s records in segments[k]; a
        tenant's segments consecutive). Each segment is copied to the device once, straight
        from its memory (pinned memory copies fastest)."""
        if not tenants:
            return
        segs = [_as_raw(r) for r in segments]
        ids = np.ascontiguousarray(tenants, dtype=np.uint32)
        ptrs = (ctypes.c_void_p * len(segs))(*[r.ctypes.data if r.size else None for r in segs])
        counts = np.array([r.size // 9 for r in segs], np.uint64)
        _check(self.lib.gz_server_ingest_segments(self._h, ids.size, _ptr(ids), ptrs, _ptr(counts)))
        del segs

    def query_submit(self, tenants: Sequence[int]) -> int:
        ids = np.ascontiguousarray(tenants, dtype=np.uint32)
        t = ctypes.c_uint64()
        _check(self.lib.gz_server_query_submit(self._h, ids.size, _ptr(ids), ctypes.byref(t)))
        # the answer's layout, kept with the ticket: a tenant may be evicted before it is read
        self._sizes[int(t.value)] = [self.num_vertices[int(k)] for k in ids]
        return int(t.value)

    def query_ready(self, ticket: int) -> bool:
        """Whether query_wait(ticket, ...) would return at once (gz_server_query_ready)."""
        out = ctypes.c_int()
        _check(self.lib.gz_server_query_ready(self._h, int(ticket), ctypes.byref(out)))
        return bool(out.value)

    def query_wait(self, ticket: int, tenants: Sequence[int]):
        """Per tenant (labels, num_cc, rounds, status) of a submitted query."""
        sizes = self._sizes.pop(int(ticket), None)
        if sizes is None or len(sizes) != len(tenants):
            raise GZError(_lib.GZ_ERR_INVALID, "unknown ticket, or not the tenants it was submitted for")
        labels = np.empty(sum(sizes), np.uint32)
        ncc = np.zeros(len(tenants), np.uint32)
        rounds = np.zeros(len(tenants), np.uint32)
        status = np.zeros(len(tenants), np.int32)
        _check(self.lib.gz_server_query_wait(self._h, ticket, _ptr(labels), _ptr(ncc),
                                             _ptr(rounds), _ptr(status)))
        out, o = [], 0
        for i, n in enumerate(sizes):
            out.append((labels[o:o + n], int(ncc[i]), int(rounds[i]), int(status[i])))
            o += n
        return out

    def connected_components(self, tenants: Sequence[int]):
        return self.query_wait(self.query_submit(tenants), tenants)

    def write_binary(self, tenant: int, path: str) -> None:
        """Checkpoint a tenant in CCSketchAlg::write_binary's format."""
        _check(self.lib.gz_server_write_binary(self._h, tenant, path.encode()))

    def admit_serialized(self, path: str) -> int:
        """Admit a tenant from a write_binary file (its V, seed and sketches)."""
        t = ctypes.c_uint32()
        _check_srv(self.lib.gz_server_admit_serialized(self._h, path.encode(), ctypes.byref(t)))
        self.num_vertices[t.value] = int(self.params(t.value).num_vertices)
        return int(t.value)

    def dump_sketches(self, tenant: int) -> np.ndarray:
        p = self.params(tenant)
        buf = np.empty(p.sketch_bytes * p.num_vertices, np.uint8)
        _check(self.lib.gz_server_dump_sketches(self._h, tenant, _ptr(buf), buf.size))
        return buf


# ------------------------------------------------------------------------------------------------
# request trace
# ------------------------------------------------------------------------------------------------
@dataclass
class ServingTrace:
    num_vertices: np.ndarray   # (T,) per tenant
    seeds: np.ndarray          # (T,) sketch seed per tenant
    time: np.ndarray           # (N,) arrival time of each request, seconds, non-decreasing
    tenant: np.ndarray         # (N,)
    kind: np.ndarray           # (N,) UPDATE / CONNECTIVITY_QUERY / POINT_QUERY
    rec_off: np.ndarray        # (N + 1,) record range of each request in raw (empty for queries)
    raw: np.ndarray            # packed 9-byte records of every update batch, in request order
    point: np.ndarray          # (N, 2) endpoints of point queries
    last_request: np.ndarray   # (T,) index of each tenant's last request

    @property
    def num_updates(self) -> int:
        return int(self.rec_off[-1])

    def records(self, i: int) -> np.ndarray:
        return self.raw[9 * int(self.rec_off[i]):9 * int(self.rec_off[i + 1])]


def _chung_lu_endpoints(rng, V: int, n: int, a: float) -> np.ndarray:
    """n vertex draws with P(i) proportional to (i + 1)^-a (inverse of the continuous CDF)."""
    u = rng.random(n)
    b = 1.0 - a
    z = ((V + 1.0) ** b - 1.0) / b
    x = (u * z * b + 1.0) ** (1.0 / b) - 1.0
    return np.minimum(x.astype(np.int64), V - 1).astype(np.uint32)


def serving_trace(num_tenants: int = 2000, seed: int = 7, *, log2_v_min: float = 10.0,
                  log2_v_max: float = 18.0, exponent: float = 2.3,
                  requests_per_tenant: float = 6.0, batch_min: int = 1024,
                  batch_max: int = 65536, delete_fraction: float = 0.2,
                  mix=(0.90, 0.08, 0.02), tenant_rate: float = 100.0,
                  request_rate: float = 4.0) -> ServingTrace:
    """Seeded serving trace. Tenants arrive as a Poisson process (tenant_rate per second), each
    with V log-uniform in [2^log2_v_min, 2^log2_v_max] and 1 + Poisson(requests_per_tenant - 1)
    requests arriving as a Poisson process (request_rate per second) after it. The first request
    is an update batch; the rest are update batches / connectivity queries / point queries with
    probabilities `mix`. An update batch has U[batch_min, batch_max] records: (1 -
    delete_fraction) of them insert an edge whose endpoints are drawn from the tenant's Chung-Lu
    weights (i + 1)^(-1/(exponent - 1)), the rest delete live edges of the tenant. Each tenant's
    requests follow its own stream in order."""
    rng = np.random.default_rng(seed)
    T = num_tenants
    Vs = np.exp2(rng.uniform(log2_v_min, log2_v_max, T)).astype(np.int64).clip(2, None)
    seeds = rng.integers(0, 2**63, T, dtype=np.int64).astype(np.uint64)
    arrive = np.cumsum(rng.exponential(1.0 / tenant_rate, T))
    a = 1.0 / (exponent - 1.0)
    times, tenants, kinds, counts, points, parts = [], [], [], [], [], []
    for t in range(T):
        V = int(Vs[t])
        R = 1 + int(rng.poisson(max(requests_per_tenant - 1.0, 0.0)))
        k = rng.choice(3, R, p=mix)
        k[0] = UPDATE
        ts = arrive[t] + np.cumsum(rng.exponential(1.0 / request_rate, R))
        tr = np.random.default_rng([seed, t])
        eu = np.zeros(0, np.uint32)
        ev = np.zeros(0, np.uint32)
        alive = np.zeros(0, bool)
        for r in range(R):
            pu = pv = 0
            cnt = 0
            if k[r] == UPDATE:
                n = int(tr.integers(batch_min, batch_max + 1))
                n_alive = int(alive.sum())
                nd = min(int(round(delete_fraction * n)), n_alive)
                ni = n - nd
                u = _chung_lu_endpoints(tr, V, ni, a)
                v = _chung_lu_endpoints(tr, V, ni, a)
                keep = u != v
                u, v = u[keep], v[keep]
                recs_i = np.empty(u.size, RECORD_DTYPE)
                recs_i["type"], recs_i["src"], recs_i["dst"] = 0, u, v
                if nd:
                    live_idx = np.flatnonzero(alive)
                    pick = tr.choice(live_idx, nd, replace=False)
                    alive[pick] = False
                    recs_d = np.empty(nd, RECORD_DTYPE)
                    recs_d["type"], recs_d["src"], recs_d["dst"] = 1, eu[pick], ev[pick]
                else:
                    recs_d = np.empty(0, RECORD_DTYPE)
                eu = np.concatenate([eu, u])
                ev = np.concatenate([ev, v])
                alive = np.concatenate([alive, np.ones(u.size, bool)])
                recs = np.concatenate([recs_i, recs_d])
                recs = recs[tr.permutation(recs.size)]
                parts.append(recs.view(np.uint8).reshape(-1))
                cnt = recs.size
            elif k[r] == POINT_QUERY:
                pu, pv = (int(x) for x in tr.integers(0, V, 2))
            times.append(ts[r])
            tenants.append(t)
            kinds.append(int(k[r]))
            counts.append(cnt)
            points.append((pu, pv))
    order = np.argsort(np.asarray(times), kind="stable")
    times = np.asarray(times)[order]
    tenants = np.asarray(tenants, np.int64)[order]
    kinds = np.asarray(kinds, np.int8)[order]
    counts = np.asarray(counts, np.int64)
    points = np.asarray(points, np.uint32).reshape(-1, 2)[order]
    # records in request order
    part_of = np.full(len(counts), -1, np.int64)
    part_of[np.flatnonzero(counts)] = np.arange(int((counts > 0).sum()))
    ordered = [parts[part_of[i]] for i in order if part_of[i] >= 0]
    raw = np.concatenate(ordered) if ordered else np.zeros(0, np.uint8)
    rec_off = np.zeros(len(order) + 1, np.int64)
    rec_off[1:] = np.cumsum(counts[order])
    last = np.zeros(T, np.int64)
    last[tenants] = np.arange(len(order))  # the last write per tenant wins: its last request
    return ServingTrace(Vs.astype(np.uint32), seeds, times, tenants, kinds, rec_off, raw,
                        points, last)


# ------------------------------------------------------------------------------------------------
# replay
# ------------------------------------------------------------------------------------------------
@dataclass
class ServingResult:
    mode: str
    seconds: float = 0.0
    updates: int = 0
    latencies_ms: List[float] = field(default_factory=list)  # one per query, request order
    # the same measured from when the query could first be served: its release, or its tenant's
    # admission when the tenant was still waiting for budget
    service_ms: List[float] = field(default_factory=list)
    query_req: List[int] = field(default_factory=list)  # request index of each latency
    answers: Dict[int, tuple] = field(default_factory=dict)  # request index -> answer
    admitted: int = 0
    max_resident: int = 0
    max_used_bytes: int = 0
    ticks: int = 0
    gpu_queries: int = 0
    rejected: int = 0
    waited: set = field(default_factory=set)  # tenants that waited for budget before admission
    max_waiting: int = 0                      # longest queue of tenants waiting for budget
    phase_s: Dict[str, float] = field(default_factory=dict)  # wall seconds per loop phase

    def _add(self, phase: str, t0: float) -> None:
        self.phase_s[phase] = self.phase_s.get(phase, 0.0) + time.perf_counter() - t0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        svc = np.asarray(self.service_ms) if self.service_ms else np.zeros(1)
        return {"mode": self.mode, "seconds": self.seconds, "updates": self.updates,
                "updates_per_s": self.updates / max(self.seconds, 1e-9),
                "queries": len(self.latencies_ms),
                "query_p50_ms": float(np.percentile(lat, 50)),
                "query_p99_ms": float(np.percentile(lat, 99)),
                "service_p50_ms": float(np.percentile(svc, 50)),
                "service_p99_ms": float(np.percentile(svc, 99)),
                "admitted_tenants": self.admitted, "max_resident_tenants": self.max_resident,
                "max_used_bytes": self.max_used_bytes, "ticks": self.ticks,
                "gpu_query_batches": self.gpu_queries, "rejected_tenants": self.rejected,
                "tenants_waited_for_budget": len(self.waited), "max_waiting_tenants": self.max_waiting,
                "phase_s": {k: round(v, 4) for k, v in self.phase_s.items()}}


def _cc_answer(labels: np.ndarray, ncc: int) -> tuple:
    """(components, digest of the canonical partition: each vertex labelled by the smallest member
    of its component)."""
    p = labels.astype(np.int64)
    mn = np.empty(p.size, np.int64)
    # repeated indices keep the last value assigned: in descending vertex order, the smallest
    mn[p[::-1]] = np.arange(p.size - 1, -1, -1)
    canon = mn[p].astype(np.uint32)
    return (ncc, hashlib.sha1(canon.tobytes()).hexdigest())


def _digest_answers(answers: Dict[int, tuple]) -> None:
    """Connectivity answers are kept as ("cc", labels, ncc) while requests are served; their
    digests are taken once the replay is over, outside the latencies."""
    done = {}
    for i, a in answers.items():
        if a and a[0] == "cc":
            key = id(a[1])
            if key not in done:
                done[key] = _cc_answer(a[1], a[2])
            answers[i] = done[key]


class pinned_host:
    """Page-locks a host buffer (gz_host_register) for the life of the ``with`` block, so record
    copies from it run at full host-link speed. A serving process keeps its incoming update
    batches in such buffers; a pageable buffer is copied through the driver's staging, several
    times slower."""

    def __init__(self, buf: np.ndarray):
        self.buf = buf
        self.ptr = None

    def __enter__(self):
        # a buffer that is page-locked already (or cannot be) is used as it is: only the copy
        # speed depends on it
        if self.buf.nbytes and _lib.load().gz_host_register(self.buf.ctypes.data, self.buf.nbytes) == 0:
            self.ptr = self.buf.ctypes.data
        return self.buf

    def __exit__(self, *exc):
        if self.ptr is not None:
            _check(_lib.load().gz_host_unregister(self.ptr))
            self.ptr = None


def plan_tick(resident, pending: Dict[int, deque], queued_q: Dict[int, int], busy, kind: np.ndarray,
              rec_off: np.ndarray, max_records: int):
    """The requests one tick of the batched replay takes, in order; taken requests leave
    `pending`, and `queued_q` (released queries not yet taken, per tenant) counts down.

    Tenants with a query waiting come first (their updates up to that query), then the others by
    their oldest request; a tenant in `busy` (its query still running) is skipped. A tenant's
    update batches are taken while the tick has records left (the last one may overshoot
    max_records), and its first query ends its part of the tick: an `early` query needs no update
    of this tick (it can go out before the tick's ingest), a `late` one comes after this tick's
    updates of its tenant. Returns (updates, early, late), lists of (request, tenant)."""
    updates, early, late = [], [], []
    left = max_records
    end = len(kind)
    for t in sorted(resident, key=lambda x: (not queued_q.get(x), pending[x][0] if pending.get(x) else end)):
        q = pending.get(t)
        if not q or t in busy:
            continue
        took = False
        while q:
            i = q[0]
            if kind[i] == UPDATE:
                if left <= 0:
                    break
                left -= int(rec_off[i + 1] - rec_off[i])
                updates.append((i, t))
                took = True
                q.popleft()
            else:
                (late if took else early).append((i, t))
                q.popleft()
                queued_q[t] -= 1
                break
    return updates, early, late


# records one tick of a batched replay ingests at most: with queries taken first, it bounds how
# long a query released during a tick waits for that tick's ingest
REPLAY_TICK_RECORDS = 1 << 19


def replay(trace: ServingTrace, mode: str, budget_bytes: int, *, snapshot_bytes: int = 0,
           time_scale: float = 1.0, sketches_factor: float = 1.0,
           max_tick_updates: int = REPLAY_TICK_RECORDS, route: float | None = None,
           pin: bool = True, query_snapshot: bool = False) -> ServingResult:
    """Serve every request of `trace`. mode "batched": the gz_server path (continuous batching:
    each tick submits the queries that need no update of this tick, applies the arrived update
    batches of all admitted tenants, up to max_tick_updates records, in one ingest, then submits
    the queries behind those updates; a collector thread takes each answer as soon as its query
    finishes). mode "plain": one CCSketchAlg per tenant, every request handled on its own in
    arrival order. Requests are released at trace time / time_scale after the start; tenants are
    admitted in arrival order while their sketch bytes fit the budget and leave after their last
    request. pin: the trace's records are page-locked for the replay (both modes), as a server's
    receive buffers would be; the page-locking is outside the timed replay. query_snapshot:
    whether the batched server copies a query's tenants to a snapshot; by default it reads them in
    place, which is safe here because a tenant's later requests wait until its answer is in."""
    if pin and trace.raw.nbytes:
        with pinned_host(trace.raw):
            return replay(trace, mode, budget_bytes, snapshot_bytes=snapshot_bytes,
                          time_scale=time_scale, sketches_factor=sketches_factor,
                          max_tick_updates=max_tick_updates, route=route, pin=False,
                          query_snapshot=query_snapshot)
    res = ServingResult(mode)
    N = trace.time.size
    T = trace.num_vertices.size
    cost = {}
    pending: Dict[int, deque] = {}
    waiting: deque = deque()
    resident = set()
    state = {}          # plain: CCSketchAlg; batched: server tenant id
    used = [0]
    served = np.zeros(T, np.int64)      # requests answered per tenant
    total = np.bincount(trace.tenant, minlength=T)
    server = None
    snap_job_bytes = 0
    if mode == "batched":
        snap = snapshot_bytes or max(budget_bytes // 4, 1 << 26)
        server = SketchServer(budget_bytes, snap, sketches_factor)
        if route is not None:
            server.set_route(route)
        server.set_query_snapshot(query_snapshot)
        # with snapshots, jobs of at most half the pool, so one runs while the next is copied
        snap_job_bytes = snap // 2 if query_snapshot else 1 << 62
    cache = {}          # batched: tenant -> (labels, ncc, version it answers for)
    version = np.zeros(T, np.int64)  # update batches applied per tenant
    queued_q: Dict[int, int] = {}     # batched: released queries not yet taken, per tenant
    inflight = []       # batched: submitted jobs not yet taken in, (ticket, tenants, ids, reqs, versions)
    done_jobs: deque = deque()  # batched: (job, per-tenant results, answers, seconds) from the collector
    jobs_in: deque = deque()    # batched: jobs for the collector, in submission order
    wake = threading.Condition()
    collector_error = []
    # a cyclic garbage collection pass can stall the loop for many milliseconds in a process that
    # holds many objects: one pass now, none while requests are served
    gc_on = gc.isenabled()
    gc.collect()
    t0 = time.perf_counter()
    nxt = 0

    def now_trace():
        return (time.perf_counter() - t0) * time_scale

    admitted_at = {}    # tenant -> wall seconds since start of its admission

    def finish(i, t, answer, at=None):
        res.answers[i] = answer
        if trace.kind[i] != UPDATE:
            now = (time.perf_counter() if at is None else at) - t0
            release = trace.time[i] / time_scale
            res.latencies_ms.append((now - release) * 1e3)
            res.service_ms.append((now - max(release, admitted_at.get(t, 0.0))) * 1e3)
            res.query_req.append(i)
        served[t] += 1
        if served[t] == total[t]:
            depart(t)

    def depart(t):
        ts = time.perf_counter()
        resident.discard(t)
        used[0] -= cost[t]
        if mode == "batched":
            server.evict(state.pop(t))
            cache.pop(t, None)
        else:
            state.pop(t).close()
        res._add("evict", ts)

    def admit():
        while waiting:
            t = waiting[0]
            c = cost.setdefault(t, tenant_bytes(int(trace.num_vertices[t]), sketches_factor))
            if c > budget_bytes:  # can never fit: refused, its requests are dropped
                waiting.popleft()
                res.rejected += 1
                dropped = pending.pop(t, deque())
                served[t] = total[t]
                for i in dropped:
                    res.answers[i] = ("rejected",)
                continue
            if used[0] + c > budget_bytes:
                res.waited.update(waiting)
                res.max_waiting = max(res.max_waiting, len(waiting))
                return
            ts = time.perf_counter()
            if mode == "batched":
                try:
                    state[t] = server.admit(int(trace.num_vertices[t]), int(trace.seeds[t]))
                except BudgetExhausted:
                    res.waited.update(waiting)
                    res.max_waiting = max(res.max_waiting, len(waiting))
                    return
            else:
                a = CCSketchAlg(int(trace.num_vertices[t]), int(trace.seeds[t]))
                a.set_gutter_capacity(1 << 18)
                state[t] = a
            res._add("admit", ts)
            admitted_at[t] = time.perf_counter() - t0
            waiting.popleft()
            used[0] += c
            resident.add(t)
            res.admitted += 1
            res.max_resident = max(res.max_resident, len(resident))
            res.max_used_bytes = max(res.max_used_bytes, used[0])

    def _answer(i, lab, ncc):
        if trace.kind[i] == CONNECTIVITY_QUERY:
            return ("cc", lab, ncc)  # digested after the replay
        u, v = trace.point[i]
        return (bool(lab[u] == lab[v]),)

    def collector():
        # waits for each submitted query in submission order and hands its answers back with the
        # time they were ready; the wait releases the interpreter lock, so ingest calls of the
        # main loop proceed meanwhile
        try:
            while True:
                with wake:
                    while not jobs_in:
                        wake.wait()
                    job = jobs_in.popleft()
                if job is None:
                    return
                ticket, tens, ids, reqs, vers = job
                out = server.query_wait(ticket, ids)
                got = {t: (lab.copy(), ncc, v) for t, (lab, ncc, rounds, status), v in zip(tens, out, vers)}
                answers = [(i, t, _answer(i, got[t][0], got[t][1])) for i, t in reqs]
                done_jobs.append((job, got, answers, time.perf_counter()))
        except BaseException as e:  # re-raised by the main loop
            collector_error.append(e)

    def take_answers():
        while done_jobs:
            job, got, answers, at = done_jobs.popleft()
            inflight.remove(job)
            cache.update(got)
            for i, t, answer in answers:
                finish(i, t, answer, at)
        if collector_error:
            raise collector_error[0]

    def submit(fresh):
        groups, cur, cur_bytes = [], [], 0
        for t in sorted({t for _, t in fresh}):
            if cur and cur_bytes + cost[t] > snap_job_bytes:
                groups.append(cur)
                cur, cur_bytes = [], 0
            cur.append(t)
            cur_bytes += cost[t]
        groups.append(cur)
        for tens in groups:
            members = set(tens)
            ids = [state[t] for t in tens]
            ts = time.perf_counter()
            ticket = server.query_submit(ids)
            res._add("query_submit", ts)
            res.gpu_queries += 1
            job = (ticket, tens, ids, [(i, t) for i, t in fresh if t in members],
                   [int(version[t]) for t in tens])
            inflight.append(job)
            with wake:
                jobs_in.append(job)
                wake.notify()

    def queries(qreq):
        # cached answers at once, the rest on the device
        fresh = []
        for i, t in qreq:
            c = cache.get(t)
            if c is not None and c[2] == version[t]:  # nothing applied since: cached answer
                finish(i, t, _answer(i, c[0], c[1]))
            else:
                fresh.append((i, t))
        if fresh:
            submit(fresh)

    thread = None
    if mode == "batched":
        thread = threading.Thread(target=collector, daemon=True)
        thread.start()
    gc.disable()
    try:
        while True:
            tnow = now_trace()
            while nxt < N and trace.time[nxt] <= tnow:
                t = int(trace.tenant[nxt])
                if t not in pending:
                    pending[t] = deque()
                    waiting.append(t)
                pending[t].append(nxt)
                if trace.kind[nxt] != UPDATE:
                    queued_q[t] = queued_q.get(t, 0) + 1
                nxt += 1
            admit()
            if mode == "plain":
                # oldest released request of a resident tenant first
                best = None
                for t in resident:
                    q = pending.get(t)
                    if q and (best is None or q[0] < best[0]):
                        best = (q[0], t)
                if best is None:
                    if nxt >= N and not resident and not waiting:
                        break
                    if nxt < N:
                        time.sleep(max(0.0, min(0.0005, (trace.time[nxt] - tnow) / time_scale)))
                    continue
                i, t = best
                pending[t].popleft()
                a = state[t]
                ts = time.perf_counter()
                if trace.kind[i] == UPDATE:
                    a.ingest_records(trace.records(i))
                    res._add("ingest", ts)
                    res.updates += int(trace.rec_off[i + 1] - trace.rec_off[i])
                    finish(i, t, ())
                elif trace.kind[i] == CONNECTIVITY_QUERY:
                    cc = a.connected_components()
                    res._add("query", ts)
                    finish(i, t, ("cc", cc.parent_arr.copy(), cc.size()))
                else:
                    u, v = trace.point[i]
                    finish(i, t, (bool(a.point_query(int(u), int(v))),))
                continue
            # batched: one tick. Answers that are ready go out first.
            take_answers()
            busy = {t for job in inflight for t in job[1]}
            ing_req, early, late = plan_tick(resident, pending, queued_q, busy, trace.kind,
                                             trace.rec_off, max_tick_updates)
            ing_t = [state[t] for _, t in ing_req]
            ing_seg = [trace.records(i) for i, _ in ing_req]
            for t in {t for _, t in ing_req}:
                version[t] += 1
            if not ing_t and not early and not late:
                if nxt >= N and not resident and not waiting:
                    break
                wait = 0.0005 if nxt >= N else min(0.0005, (trace.time[nxt] - tnow) / time_scale)
                time.sleep(max(0.0, wait) if not inflight else min(max(0.0, wait), 0.0002))
                continue
            res.ticks += 1
            if early:
                queries(early)
            if ing_t:
                ts = time.perf_counter()
                server.ingest_segments(ing_t, ing_seg)
                res._add("ingest", ts)
                for i, t in ing_req:
                    res.updates += int(trace.rec_off[i + 1] - trace.rec_off[i])
                    finish(i, t, ())
            if late:
                queries(late)
    finally:
        if thread is not None:
            with wake:
                jobs_in.append(None)
                wake.notify()
            thread.join()
        res.seconds = time.perf_counter() - t0
        if gc_on:
            gc.enable()
        for t in list(state):
            if mode == "plain":
                state.pop(t).close()
        if server is not None:
            server.close()
    _digest_answers(res.answers)
    return res
