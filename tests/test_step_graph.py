"""GPU: ge_step replays pairs of steps as a captured CUDA graph.

The graph holds exactly the launches two plain steps make, so every frame
must equal the plain path's (params.no_graph = 1) bit for bit, whatever the
step counts of the calls (odd counts finish with a plain step and flip the
buffer roles), and a change of parameters, particle count or simulations
between calls must be seen by the next call (the graph is recaptured).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS2 = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")
KEYS3 = KEYS2 + ("z", "vz", "az")


def _pair(ge, p):
    q = ge.Params.from_buffer_copy(p)
    q.no_graph = 1
    return ge.Simulation(p), ge.Simulation(q)


def _same(a, b, keys, what):
    for k in keys:
        assert np.array_equal(a[k], b[k]), (what, k)


@pytest.mark.parametrize("dims,precision,kw", [(2, 0, {}), (3, 1, {}), (2, 2, dict(group_size=64)),
                                               (3, 2, dict(group_size=32)), (2, 2, {})])
def test_graph_steps_equal_plain_steps(ge, ics, dims, precision, kw):
    n = 30000 if dims == 2 else 20000
    st = ics.disk2d(n, seed=3) if dims == 2 else ics.plummer3d(n, seed=3)
    p = ge.default_params(dims, G=1.0, theta=0.7, softening=0.01, dt=1e-3, leaf_cap=4,
                          precision=precision, **kw)
    keys = KEYS2 if dims == 2 else KEYS3
    a, b = _pair(ge, p)
    with a, b:
        a.upload(st)
        b.upload(st)
        for calls, k in enumerate([2, 3, 1, 4, 5, 2]):
            a.step(k)
            b.step(k)
            _same(a.download(), b.download(), keys, (calls, k))


def test_parameter_and_particle_changes_between_calls(ge, ics):
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, leaf_cap=4,
                          precision=ge.PREC_EXACT)
    a, b = _pair(ge, p)
    with a, b:
        for s in (a, b):
            s.upload(ics.disk2d(12000, seed=5))
            s.step(4)
        # a new theta and time step: the next pair must use them
        for s, nog in ((a, 0), (b, 1)):
            q = ge.default_params(2, G=1.0, theta=0.5, softening=0.01, dt=2e-3, leaf_cap=4,
                                  precision=ge.PREC_EXACT)
            q.no_graph = nog
            s.set_params(q)
            s.step(4)
        _same(a.download(), b.download(), KEYS2, "params")
        # a different particle count: new buffers, new launches
        for s in (a, b):
            s.upload(ics.disk2d(7000, seed=6))
            s.step(6)
        _same(a.download(), b.download(), KEYS2, "upload")


def test_batch_with_direct_and_walked_simulations(ge, ics):
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, leaf_cap=4,
                          precision=ge.PREC_FAST, direct_below=5000)
    sizes = [3000, 9000, 700, 20000]
    sts = [ics.disk2d(n, seed=60 + k, center=(3.0 * k, 0.0)) for k, n in enumerate(sizes)]
    a, b = _pair(ge, p)
    with a, b:
        ha = [a.add_sim(s) for s in sts]
        hb = [b.add_sim(s) for s in sts]
        a.step(4)
        b.step(4)
        a.remove_sims([ha[1]])
        b.remove_sims([hb[1]])
        a.step(6)
        b.step(6)
        for x, y in zip((ha[0], ha[2], ha[3]), (hb[0], hb[2], hb[3])):
            _same(a.download_sim(x), b.download_sim(y), KEYS2, "batch")
