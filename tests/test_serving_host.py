"""Host-side scheduling of the serving loop (no GPU): admission by memory
budget, passing over busy diagrams, eviction of idle diagrams into the reuse
pool, failures delivered through the futures."""
import collections
import threading
from concurrent.futures import Future

import numpy as np
import pytest

from integer_delauney_b200 import serving
from integer_delauney_b200.serving import SEED_HEADROOM, _Diagram, _Pooled, _Request, estimate_bytes


def make_server(budget):
    srv = object.__new__(serving.Server)
    srv.budget = budget
    srv.padding = 16
    srv._cv = threading.Condition()
    srv._queue = collections.deque()
    srv._diagrams = {}
    srv._pool = []
    srv._used = 0
    srv._closed = True          # _next returns None instead of waiting when nothing is left
    srv.stats = collections.Counter()
    return srv


def new_req(srv, rid, did, W=200, H=150, n=100):
    seeds = np.zeros((n, 2), np.int32)
    need = estimate_bytes(*serving._class_dims(W, H), n + SEED_HEADROOM, 16)
    srv._diagrams[did] = _Diagram(did, pins=1)
    r = _Request(rid, "new", 0.0, Future(), did, W, H, seeds, False, need)
    srv._queue.append(r)
    return r


def ins_req(srv, rid, did):
    srv._diagrams[did].pins += 1
    r = _Request(rid, "insert", 0.0, Future(), did, seeds=np.zeros((1, 2), np.int32))
    srv._queue.append(r)
    return r


def test_estimate_grows_with_canvas_and_seeds():
    assert estimate_bytes(256, 256, 1000, 16) < estimate_bytes(512, 256, 1000, 16) < \
        estimate_bytes(512, 256, 100000, 16)
    assert estimate_bytes(256, 256, 1000, 0) < estimate_bytes(256, 256, 1000, 16)
    assert serving._class_dims(1, 129) == (128, 256)
    # reuse is decided by areas, as the C reset rule decides it
    cap = serving._capacity(512, 256, 1000, 16)
    assert serving._fits(cap, 256, 512, 1000, 16) and serving._fits(cap, 300, 300, 900, 16)
    assert not serving._fits(cap, 600, 300, 1000, 16) and not serving._fits(cap, 256, 256, 1001, 16)


def test_busy_diagram_is_passed_over():
    srv = make_server(1 << 40)
    srv._diagrams[7] = _Diagram(7, obj=object(), bytes=10, busy=True)
    ins = ins_req(srv, 0, 7)
    new = new_req(srv, 1, 8)
    with srv._cv:
        kind, items = srv._next([])
    assert kind == "new" and items == [(new, None)] and srv._used == new.need
    assert list(srv._queue) == [ins] and srv._diagrams[8].busy


def test_insert_waits_for_its_diagram_creation():
    srv = make_server(1 << 40)
    new = new_req(srv, 0, 3)
    ins = ins_req(srv, 1, 3)
    with srv._cv:
        kind, items = srv._next([])
    assert kind == "new" and items[0][0] is new
    srv._diagrams[3].busy = True       # still being created: the insert is not admissible
    srv._queue.append(new_req(srv, 2, 4))
    with srv._cv:
        kind, items = srv._next([])
    assert items[0][0].diagram_id == 4 and ins in srv._queue


def test_idle_diagram_evicted_and_its_object_reused():
    need = estimate_bytes(256, 256, 100 + SEED_HEADROOM, 16)
    srv = make_server(need + need // 2)
    obj = object()
    srv._diagrams[1] = _Diagram(1, obj=obj, bytes=need, last_used=1.0,
                                cap=serving._capacity(256, 256, 100 + SEED_HEADROOM, 16))
    srv._used = need
    new = new_req(srv, 0, 2, W=200, H=200)
    with srv._cv:
        kind, items = srv._next([])
    (req, pooled), = items
    assert req is new and pooled is not None and pooled.obj is obj
    assert 1 not in srv._diagrams and srv.stats["evicted"] == 1 and srv._used == need


def test_pool_dropped_when_nothing_fits():
    need = estimate_bytes(256, 256, 100 + SEED_HEADROOM, 16)
    srv = make_server(2 * need)
    srv._pool.append(_Pooled(object(), 2 * need - 10, serving._capacity(128, 128, 10, 16)))   # too small
    srv._used = 2 * need - 10
    free = []
    new = new_req(srv, 0, 2, W=200, H=200)
    with srv._cv:
        kind, items = srv._next(free)
    assert items == [(new, None)] and len(free) == 1 and srv.stats["freed_objects"] == 1


def test_failures_reach_the_futures():
    srv = make_server(1000)
    big = new_req(srv, 0, 1, W=4096, H=4096)
    ins = ins_req(srv, 1, 1)
    with srv._cv:
        assert srv._next([]) is None
    with pytest.raises(MemoryError):
        big.future.result(timeout=1)
    with pytest.raises(KeyError):
        ins.future.result(timeout=1)


def test_new_diagrams_queued_together_share_one_group():
    srv = make_server(1 << 40)
    a = new_req(srv, 0, 1)
    srv._diagrams[9] = _Diagram(9, obj=object(), bytes=10)
    ins = ins_req(srv, 1, 9)
    b = new_req(srv, 2, 2, W=300, H=100)
    huge = new_req(srv, 3, 3, W=4096, H=4096)      # would overflow the group's canvas limit
    with srv._cv:
        kind, items = srv._next([])
    assert kind == "new" and [r for r, _ in items] == [a, b]
    assert list(srv._queue) == [ins, huge] and all(srv._diagrams[i].busy for i in (1, 2))
    with srv._cv:
        kind, items = srv._next([])
    assert kind == "insert" and items[0][0] is ins


def test_request_that_can_never_fit_fails_instead_of_waiting():
    srv = make_server(1 << 30)
    srv._used = (1 << 30) - 1000            # reserved workspaces leave too little, nothing to evict
    r1 = new_req(srv, 0, 1)
    r2 = new_req(srv, 1, 2)
    assert r1.need < srv.budget
    with srv._cv:
        assert srv._next([]) is None        # both failed; the queue is empty and the server closed
    for r in (r1, r2):
        with pytest.raises(MemoryError):
            r.future.result(timeout=1)
