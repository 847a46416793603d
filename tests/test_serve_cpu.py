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
        self.req = None
        self.done = _FakeEvent()
        self.grids = []
        self.ws = None


@pytest.fixture
def server_factory(monkeypatch):
    monkeypatch.setattr(serve, "_Slot", _FakeSlot)
    monkeypatch.setattr(serve, "estimate_bytes", lambda req: req.M)  # bytes = M, for readable budgets

    def make(slots=4, budget=100, lookahead=16, fail_kinds=()):
        srv = serve.NufftServer("cpu", slots=slots, hbm_budget=budget, lookahead=lookahead)
        srv.started = []

        def fake_run(req, slot):
            if req.kind in fail_kinds:
                raise ValueError("bad request")
            slot.done = _FakeEvent()
            srv.started.append(req)

        srv._run = fake_run
        return srv

    return make


def _req(M, kind=1):
    return serve.Request(kind=kind, dim=2, n_modes=(16, 16), M=M)


def _finish(srv, req):
    for s in srv.slots:
        if s.req is req:
            s.done.is_done = True
    srv.step()


def test_budget_and_lookahead(server_factory):
    srv = server_factory(budget=100)
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
    srv = server_factory(budget=100, lookahead=1)
    r = [_req(60), _req(60), _req(30)]
    for q in r:
        srv.submit(q)
    srv.step()
    assert srv.started == [r[0]]  # the head that does not fit blocks the rest
    _finish(srv, r[0])
    assert srv.started == [r[0], r[1], r[2]]  # then both fit (60 + 30)


def test_request_larger_than_budget_runs_alone(server_factory):
    srv = server_factory(budget=100)
    big, small = _req(500), _req(10)
    srv.submit(big)
    srv.submit(small)
    srv.step()
    assert srv.started == [big] and srv.in_use == 500
    _finish(srv, big)
    assert srv.started == [big, small]


def test_slots_bound_concurrency(server_factory):
    srv = server_factory(slots=2, budget=10**9)
    r = [_req(1) for _ in range(5)]
    for q in r:
        srv.submit(q)
    srv.step()
    assert len(srv.started) == 2 and len(srv.pending) == 3


def test_failure_isolated_and_excluded_from_stats(server_factory):
    srv = server_factory(budget=100, fail_kinds=(3,))
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
