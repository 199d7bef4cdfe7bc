"""GPU: the serving loop (ge_server) -- continuous batching under an HBM budget.

Requests (2D disks and 3D Plummer spheres with their own step counts) run
in two pools that are sized once from the budget.  Checks: every result is
bit-identical to the same request run alone on a context with the same
parameters; requests that arrive while others run are admitted as room frees
up, so with a small budget some must wait and all still finish; the pools
hold no more device memory than the budget; a request larger than its pool
is refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS2 = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")
KEYS3 = KEYS2 + ("z", "vz", "az")


def _params(ge, dims, precision):
    soft = 0.01
    return ge.default_params(dims, G=1.0, theta=0.6 if dims == 2 else 0.5, softening=soft,
                             dt=1e-3, precision=precision)


def _alone(ge, p, st, steps):
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(steps)
        return s.download()


def _requests(ics):
    reqs = []
    for k, (dims, n, steps) in enumerate([(2, 5000, 3), (3, 3000, 5), (2, 20000, 1),
                                          (2, 1500, 7), (3, 9000, 2), (2, 4097, 4)]):
        st = ics.disk2d(n, seed=70 + k, center=(k, -k)) if dims == 2 else ics.plummer3d(n, seed=70 + k)
        reqs.append((dims, st, steps))
    return reqs


@pytest.mark.parametrize("precision", [0, 2], ids=["fast", "mixed"])
def test_serving_results_equal_alone(ge, ics, precision):
    p2, p3 = _params(ge, 2, precision), _params(ge, 3, precision)
    reqs = _requests(ics)
    with ge.Server(2 << 30, p2, p3, frac_2d=0.5, max_sims=64) as srv:
        ids = [srv.submit(st, steps) for _, st, steps in reqs]
        while srv.stats().completed < len(ids):
            srv.poll()
        outs = [srv.take(r) for r in ids]
        s = srv.stats()
        assert s.failed == 0 and s.queued == 0 and s.running == 0
        assert sum(s.pool_bytes) <= 2 << 30
    for (dims, st, steps), out in zip(reqs, outs):
        ref = _alone(ge, p2 if dims == 2 else p3, st, steps)
        for k in (KEYS2 if dims == 2 else KEYS3):
            assert np.array_equal(out[k], ref[k]), (dims, steps, k)


def test_serving_budget_admission_and_arrivals(ge, ics):
    """A budget that holds only a few requests at once: the worker thread runs
    while requests keep arriving; some must queue, all finish, and results are
    those of the requests run alone."""
    import time
    p2, p3 = _params(ge, 2, 0), _params(ge, 3, 0)
    n = 20000
    per2 = ge.estimate_bytes(p2, 3 * n, 4)
    per3 = ge.estimate_bytes(p3, 2 * n, 4)
    budget = per2 + per3
    sts = [ics.disk2d(n, seed=90 + k) for k in range(8)] + \
          [ics.plummer3d(n, seed=90 + k) for k in range(4)]
    steps = [3 + (k % 4) for k in range(len(sts))]
    with ge.Server(budget, p2, p3, frac_2d=per2 / budget, max_sims=4) as srv:
        st = srv.stats()
        assert sum(st.pool_bytes) <= budget
        assert st.pool_capacity[0] >= 3 * n - 16 and st.pool_capacity[0] < 4 * n
        srv.start()
        ids = []
        max_running = 0
        for k, s in enumerate(sts):
            ids.append(srv.submit(s, steps[k]))
            time.sleep(0.002)
            max_running = max(max_running, srv.stats().running)
        for r in ids:
            srv.wait(r, 300.0)
        srv.stop()
        s = srv.stats()
        assert s.completed == len(ids) and s.failed == 0
        assert s.iterations >= max(steps)
        lat = [srv.status(r)[2] for r in ids]
        assert all(v > 0 for v in lat)
        outs = [srv.take(r) for r in ids]
    assert max_running <= 3 + 2
    for k in (0, 7, 8, 11):
        p = p2 if k < 8 else p3
        ref = _alone(ge, p, sts[k], steps[k])
        for key in (KEYS2 if k < 8 else KEYS3):
            assert np.array_equal(outs[k][key], ref[key]), (k, key)


def test_serving_rejects_oversize(ge, ics):
    p2, p3 = _params(ge, 2, 0), _params(ge, 3, 0)
    with ge.Server(ge.estimate_bytes(p2, 1000, 2) * 2, p2, p3, frac_2d=0.5, max_sims=2) as srv:
        cap = srv.stats().pool_capacity[0]
        assert 900 <= cap < 2000
        with pytest.raises(ge.GeError) as ei:
            srv.submit(ics.disk2d(cap + 1, seed=1), 1)
        assert ei.value.code == 4
