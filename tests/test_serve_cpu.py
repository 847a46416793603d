"""CPU: the continuous-batching server's host logic (admission against the byte
budget, lookahead past a head request that does not fit, a request larger than
the budget running alone, failure isolation, statistics) with fake slots in
place of CUDA streams and events.  The device side is covered by
tests/test_gpu_serve.py."""

import pytest

from nufftax_b200 import serve


class _FakeEvent:
    def __init__(self):
        self.is_done = False

    def query(self):
        return self.is_done

    def record(self, stream=None):
        self.is_done = True


class _FakeSlot:
    def __init__(self, device):
        self.stream = None
        self.reqs = []
        self.done = _FakeEvent()
        self.grids = []
        self.held = []
        self.ws = None


@pytest.fixture
def server_factory(monkeypatch):
    monkeypatch.setattr(serve, "_Slot", _FakeSlot)
    monkeypatch.setattr(serve, "estimate_bytes", lambda req: req.M)  # bytes = M, for readable budgets

    def make(slots=4, budget=100, lookahead=16, fail_kinds=(), **kw):
        srv = serve.NufftServer("cpu", slots=slots, hbm_budget=budget, lookahead=lookahead, **kw)
        srv.started = []
        srv.waves = []

        def fake_run(req, slot):
            if req.kind in fail_kinds:
                raise ValueError("bad request")
            slot.done = _FakeEvent()
            srv.started.append(req)

        def fake_wave(reqs, slot):
            if any(r.kind in fail_kinds for r in reqs):
                raise ValueError("bad request")
            slot.done = _FakeEvent()
            srv.started.extend(reqs)
            srv.waves.append(list(reqs))

        srv._run = fake_run
        srv._run_wave = fake_wave
        return srv

    return make


def _req(M, kind=1, dim=2, eps=1e-6):
    return serve.Request(kind=kind, dim=dim, n_modes=(16,) * dim, M=M, eps=eps)


def _finish(srv, req):
    for s in srv.slots:
        if req in s.reqs:
            s.done.is_done = True
    srv.step()


def test_budget_and_lookahead(server_factory):
    srv = server_factory(budget=100, wave_max_points=0)
    r = [_req(60), _req(60), _req(30), _req(10)]
    for q in r:
        srv.submit(q)
    srv.step()
    # the second 60 does not fit next to the first; the two behind it do
    assert srv.started == [r[0], r[2], r[3]] and srv.in_use == 100
    assert list(srv.pending) == [r[1]]
    _finish(srv, r[0])
    assert srv.started[-1] is r[1] and srv.in_use == 100
    for q in (r[1], r[2], r[3]):
        _finish(srv, q)
    assert srv.in_use == 0 and not srv.busy() and len(srv.completed) == 4


def test_head_of_line_without_lookahead(server_factory):
    srv = server_factory(budget=100, lookahead=1, wave_max_points=0)
    r = [_req(60), _req(60), _req(30)]
    for q in r:
        srv.submit(q)
    srv.step()
    assert srv.started == [r[0]]  # the head that does not fit blocks the rest
    _finish(srv, r[0])
    assert srv.started == [r[0], r[1], r[2]]  # then both fit (60 + 30)


def test_request_larger_than_budget_runs_alone(server_factory):
    srv = server_factory(budget=100, wave_max_points=0)
    big, small = _req(500), _req(10)
    srv.submit(big)
    srv.submit(small)
    srv.step()
    assert srv.started == [big] and srv.in_use == 500
    _finish(srv, big)
    assert srv.started == [big, small]


def test_slots_bound_concurrency(server_factory):
    srv = server_factory(slots=2, budget=10**9, wave_max_points=0)
    r = [_req(1) for _ in range(5)]
    for q in r:
        srv.submit(q)
    srv.step()
    assert len(srv.started) == 2 and len(srv.pending) == 3


def test_failure_isolated_and_excluded_from_stats(server_factory):
    srv = server_factory(budget=100, fail_kinds=(3,), wave_max_points=0)
    good, bad = _req(20), _req(20, kind=3)
    srv.submit(bad)
    srv.submit(good)
    srv.step()
    assert bad.error is not None and bad.error.startswith("ValueError")
    assert srv.started == [good]
    srv.step()  # the failed request's slot completes through its event
    _finish(srv, good)
    assert srv.in_use == 0 and len(srv.completed) == 2
    st = srv.stats()
    assert st["requests"] == 1 and st["points"] == good.points()


def test_shape_state_is_bounded(monkeypatch):
    """Per-shape options of the one-call path are kept least recently used out
    (host structs only; runs without a GPU on the CPU device)."""
    monkeypatch.setattr(serve, "_Slot", _FakeSlot)
    srv = serve.NufftServer("cpu", slots=1)
    srv.keep_shapes = 3
    reqs = [serve.Request(kind=1, dim=2, n_modes=(16 + 2 * i, 16), M=10) for i in range(5)]
    for r in reqs[:3]:
        srv._shape(r, 0)
    srv._shape(reqs[0], 0)  # touch: most recently used
    srv._shape(reqs[3], 0)
    srv._shape(reqs[4], 0)
    kept = {k[1] for k in srv.shapes}
    assert len(srv.shapes) == 3 and (16, 16) in kept and (18, 16) not in kept
    sh = srv._shape(reqs[4], 0)
    assert sh.nf == tuple(nb_grid(n) for n in (24, 16)) and sh.sign == 1


def nb_grid(n):
    from nufftax_b200.grid import compute_grid_size
    from nufftax_b200.kernel import compute_kernel_params

    return compute_grid_size(n, 2.0, compute_kernel_params(1e-6).nspread)


def test_small_requests_form_waves_by_key(server_factory):
    """A backlog of small type-1/2 requests larger than the free slots is packed
    into waves of one dimension, eps and precision (one slot each, at most
    wave_size requests); larger ones, type 3 and other keys run alone."""
    srv = server_factory(slots=4, budget=10**9, wave_max_points=100, wave_size=3)
    small2 = [_req(10, kind=1 + i % 2) for i in range(9)]
    small3 = [_req(10, dim=3)]
    big = _req(1000)
    t3 = _req(10, kind=3)
    for q in small2 + small3 + [big, t3]:
        srv.submit(q)
    srv.step()
    # 10 small requests over 4 free slots: waves of up to 3
    assert srv.waves[0] == small2[:3] and srv.waves[1] == small2[3:6]
    assert all(len(w) <= 3 for w in srv.waves)
    assert sum(len(w) for w in srv.waves) + sum(1 for r in srv.started if r not in sum(srv.waves, [])) == \
        len(srv.started)
    assert len(srv.started) == 3 * 3 + 1 or len(srv.started) == 10  # 4 slots used
    for s in srv.slots:
        s.done.is_done = True
    srv.step()
    for s in srv.slots:
        s.done.is_done = True
    srv.step()
    assert all(q in srv.started for q in small2 + small3 + [big, t3])


def test_few_small_requests_spread_over_slots(server_factory):
    """Fewer small requests than free slots: each runs alone on its own slot."""
    srv = server_factory(slots=4, budget=10**9, wave_max_points=100, wave_size=8)
    reqs = [_req(10, kind=1 + i % 2) for i in range(3)]
    for q in reqs:
        srv.submit(q)
    srv.step()
    assert srv.waves == [] and srv.started == reqs


def test_wave_failure_fails_every_member(server_factory):
    """An exception from a wave's launch fails every member of that wave."""
    srv = server_factory(slots=1, budget=10**9, wave_max_points=100, fail_kinds=(2,))
    good, bad = _req(10, kind=1), _req(10, kind=2)
    srv.submit(good)
    srv.submit(bad)
    srv.step()
    assert good.error is not None and bad.error is not None
    srv.step()
    assert srv.in_use == 0 and len(srv.completed) == 2
