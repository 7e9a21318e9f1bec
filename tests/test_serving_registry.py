"""Resident-model registry of the serving loop (CPU, no device).

The registry logic -- least-recently-used eviction against the HBM budget,
packs freed as a unit, in-flight groups never freed under a running re-solve
-- is host code; these tests drive it with stand-in device models.
"""
import threading

import pytest

from jf_2026_05_25_b200 import serving as S


class FakeDM:
    """Stand-in for lib.DeviceModel: the registry only sizes and frees it."""

    def __init__(self, factor_bytes):
        self.factor_bytes = factor_bytes
        self.ndof = 0
        self.closed = 0

    def symbolic_info(self):
        return {"factor_bytes": self.factor_bytes}

    def sizes(self):
        return 0, 0, 0

    def close(self):
        self.closed += 1


@pytest.fixture
def server():
    srv = S.SolveServer(slots=0, hbm_budget_bytes=100.0)
    yield srv
    srv.close()


def _group(srv, n_members, nbytes):
    dm = FakeDM(nbytes / 1.6)
    keys = srv._register(dm, {}, None, [object()] * n_members)
    return dm, keys


def test_eviction_skips_a_busy_pack_and_frees_whole_groups(server):
    dm_a, keys_a = _group(server, 2, 50.0)     # a pack of two models
    dm_b, keys_b = _group(server, 1, 50.0)
    assert server.resident_bytes == pytest.approx(100.0)
    res_a = server._lookup(keys_a[0])
    server._lookup(keys_b[0])                  # b is now the most recently used
    # a re-solve holds pack a's lock while a new model needs room: a is the
    # least recently used but busy, so b goes instead
    with res_a.lock:
        server._admit(50.0)
        assert dm_a.closed == 0 and dm_b.closed == 1
        assert all(k in server.registry for k in keys_a)
        assert keys_b[0] not in server.registry
        assert server.resident_bytes == pytest.approx(50.0)
    # once idle the pack is freed as one unit and its bytes released once
    server._admit(60.0)
    assert dm_a.closed == 1
    assert not any(k in server.registry for k in keys_a)
    assert server.resident_bytes == pytest.approx(0.0)


def test_resolve_after_eviction_raises_key_error(server):
    dm_a, keys_a = _group(server, 2, 60.0)
    res = server._lookup(keys_a[1])            # looked up before the eviction
    server._admit(80.0)
    assert dm_a.closed == 1
    with res.lock:
        with pytest.raises(KeyError):
            server._check_live(res, keys_a[1])
    with pytest.raises(KeyError):
        server._lookup(keys_a[0])


def test_eviction_waits_for_nothing_when_every_group_is_busy(server):
    dm_a, keys_a = _group(server, 1, 90.0)
    res = server._lookup(keys_a[0])
    done = threading.Event()
    with res.lock:
        t = threading.Thread(target=lambda: (server._admit(50.0), done.set()))
        t.start()
        assert done.wait(5.0), "admission blocked on a busy group"
        t.join()
    assert dm_a.closed == 0 and keys_a[0] in server.registry


def test_second_stage_admission_does_not_wait_on_its_own_reservation():
    """A model holds its upload estimate and asks for the rest once its
    analysis exists.  With nothing resident and only its own bytes reserved,
    nothing can be freed: it is admitted over budget at once instead of
    waiting for the timeout."""
    import time
    srv = S.SolveServer(slots=0, hbm_budget_bytes=1.0)
    srv.wait_s = 30.0
    try:
        srv._admit(10.0, wait=True)            # upload estimate, over budget: admitted (empty server)
        t0 = time.perf_counter()
        srv._admit(40.0, wait=True, own=10.0)  # the exact figure
        assert time.perf_counter() - t0 < 2.0
        assert srv.reserved == pytest.approx(50.0)
        assert srv.waiting_reserved == pytest.approx(0.0)
    finally:
        srv.close()


def test_two_second_stage_admissions_do_not_wait_on_each_other():
    """Two requests each hold an estimate and both ask for more with nothing
    resident: the one that finds every reservation held by waiters goes
    ahead at once; the other goes once the first's bytes are released."""
    import time
    srv = S.SolveServer(slots=0, hbm_budget_bytes=1.0)
    srv.wait_s = 30.0
    try:
        srv._admit(10.0)                       # two upload estimates, admitted over budget
        srv._admit(10.0)
        ths = [threading.Thread(target=srv._admit, args=(5.0,), kwargs={"wait": True, "own": 10.0})
               for _ in range(2)]
        for t in ths:
            t.start()
        t0 = time.perf_counter()
        while all(t.is_alive() for t in ths) and time.perf_counter() - t0 < 5.0:
            time.sleep(0.05)
        assert sum(not t.is_alive() for t in ths) == 1
        srv._release(15.0)                     # the first one's model is done and gone
        for t in ths:
            t.join(timeout=5)
        assert all(not t.is_alive() for t in ths)
        assert time.perf_counter() - t0 < 10.0
        assert srv.reserved == pytest.approx(15.0)
    finally:
        srv.close()


class _Mesh:
    """Stand-in model: a mesh key from its connectivity, a size above the
    pack limit (single-model requests)."""

    def __init__(self, tag, ndof=100000):
        import numpy as np
        self.n_nodes = ndof // 6
        self.ndof = ndof
        self.q4_nodes = np.full((4, 4), tag, np.int32)
        self.t10_nodes = np.zeros((0, 10), np.int32)


def test_dispatch_defers_a_model_whose_mesh_is_being_prepared(server):
    """Two new models of one mesh queued together: the second is not taken
    while the first is being prepared (it would repeat the pattern build and
    the analysis); other work goes first, and once the first is registered
    as a resident of that mesh the second is taken."""
    a1, a2, b = _Mesh(1), _Mesh(1), _Mesh(2)
    server.submit(S.Request("solve", model=a1))
    server.submit(S.Request("solve", model=a2))
    server.submit(S.Request("solve", model=b))
    w1 = server._take()
    assert w1[0].model is a1
    mk = w1[0].mesh
    assert mk is not None and server.preparing == {mk: 1}
    w2 = server._take()                       # a2 is deferred: b goes first
    assert w2[0].model is b
    assert server.deferred == 1
    # a1 registered as the mesh's resident: a2 may go (and will share)
    server.meshes[mk] = "k0"
    w3 = server._take()
    assert w3[0].model is a2 and w3[0].was_deferred


def test_dispatch_waits_when_only_deferred_work_is_queued(server):
    """With only a deferred model queued, a slot waits; the end of the
    preparing slot's request releases it."""
    a1, a2 = _Mesh(3), _Mesh(3)
    server.submit(S.Request("solve", model=a1))
    server.submit(S.Request("solve", model=a2))
    w1 = server._take()
    got = []
    t = threading.Thread(target=lambda: got.append(server._take()))
    t.start()
    t.join(timeout=1.2)
    assert t.is_alive() and not got          # still waiting on the deferred a2
    with server.plock:                       # what _worker does when a1's request ends
        server.preparing.pop(w1[0].mesh)
        server.plock.notify_all()
    t.join(timeout=5)
    assert got and got[0][0].model is a2


def test_admission_keeps_the_pinned_structure_donor(server):
    """A new model pins the resident model whose structure it will take over
    before its admission: room is made by freeing other groups, never the
    donor, and with only the donor left the request is admitted over budget
    at once instead of waiting for it."""
    dm_a, keys_a = _group(server, 1, 50.0)     # the donor (least recently used)
    dm_b, keys_b = _group(server, 1, 50.0)
    server._lookup(keys_b[0])
    donor = server.registry[keys_a[0]]
    with donor.pin:
        server._admit(50.0, wait=True, keep=id(dm_a))
        assert dm_a.closed == 0 and dm_b.closed == 1
        assert keys_a[0] in server.registry
        import time as _t
        t0 = _t.perf_counter()
        server._admit(80.0, wait=True, keep=id(dm_a))   # nothing else to free
        assert _t.perf_counter() - t0 < 1.0
        assert dm_a.closed == 0
    server._release(130.0)
