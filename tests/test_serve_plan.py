"""The batched replay's tick policy (serve.plan_tick), on the host: tenants with a query waiting go
first, the record cap bounds the tick's updates, a query that needs none of the tick's updates is
early, a tenant whose query is still running is skipped, and each tenant's requests keep their
order."""
from collections import deque

import numpy as np

from graphzeppelin_b200.serve import CONNECTIVITY_QUERY, POINT_QUERY, UPDATE, plan_tick


def _requests(spec):
    """spec: list of (tenant, kind, records). Returns kind, rec_off, pending, queued_q."""
    kind = np.array([k for _, k, _ in spec], np.uint8)
    sizes = [n if k == UPDATE else 0 for _, k, n in spec]
    rec_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    pending, queued = {}, {}
    for i, (t, k, _) in enumerate(spec):
        pending.setdefault(t, deque()).append(i)
        if k != UPDATE:
            queued[t] = queued.get(t, 0) + 1
    return kind, rec_off, pending, queued


def test_queried_tenants_first_and_early_late():
    spec = [(0, UPDATE, 100), (0, UPDATE, 100),        # tenant 0: oldest, updates only
            (1, UPDATE, 50), (1, CONNECTIVITY_QUERY, 0),  # tenant 1: updates, then a query
            (2, POINT_QUERY, 0), (2, UPDATE, 10)]        # tenant 2: a query at the head
    kind, rec_off, pending, queued = _requests(spec)
    updates, early, late = plan_tick({0, 1, 2}, pending, queued, set(), kind, rec_off, 1 << 20)
    # tenants 1 and 2 (a query waiting) before tenant 0; tenant 2's update stays behind its query
    assert updates == [(2, 1), (0, 0), (1, 0)]
    assert early == [(4, 2)] and late == [(3, 1)]
    assert list(pending[2]) == [5] and not pending[0] and not pending[1]
    assert queued[1] == 0 and queued[2] == 0


def test_record_cap_and_queries_past_it():
    spec = [(0, UPDATE, 300), (0, UPDATE, 300), (0, UPDATE, 300),
            (1, CONNECTIVITY_QUERY, 0), (1, UPDATE, 5),
            (2, UPDATE, 300), (2, CONNECTIVITY_QUERY, 0)]
    kind, rec_off, pending, queued = _requests(spec)
    updates, early, late = plan_tick({0, 1, 2}, pending, queued, set(), kind, rec_off, 400)
    # queried tenants first: 1 (query at its head: early, no records), then 2 (300 records, its
    # query late), then tenant 0 takes one more batch (400 - 300 > 0) and stops at the cap
    assert early == [(3, 1)]
    assert late == [(6, 2)]
    assert updates == [(5, 2), (0, 0)]
    assert list(pending[0]) == [1, 2] and list(pending[1]) == [4]
    # the cap spent: another tick with no room still sends queries at a tenant's head
    spec2 = [(0, UPDATE, 10), (1, CONNECTIVITY_QUERY, 0)]
    kind, rec_off, pending, queued = _requests(spec2)
    updates, early, late = plan_tick({0, 1}, pending, queued, set(), kind, rec_off, 0)
    assert updates == [] and early == [(1, 1)] and late == []


def test_busy_tenants_and_order():
    spec = [(0, UPDATE, 10), (0, CONNECTIVITY_QUERY, 0), (0, UPDATE, 10),
            (1, UPDATE, 10), (1, UPDATE, 10), (1, POINT_QUERY, 0), (1, UPDATE, 10)]
    kind, rec_off, pending, queued = _requests(spec)
    updates, early, late = plan_tick({0, 1}, pending, queued, {0}, kind, rec_off, 1 << 20)
    assert updates == [(3, 1), (4, 1)] and late == [(5, 1)] and early == []
    assert list(pending[0]) == [0, 1, 2] and list(pending[1]) == [6]
    assert queued[0] == 1 and queued[1] == 0
    # not resident: untouched
    updates, early, late = plan_tick({1}, pending, queued, set(), kind, rec_off, 1 << 20)
    assert updates == [(6, 1)] and list(pending[0]) == [0, 1, 2]
