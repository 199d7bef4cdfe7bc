"""GPU: many independent simulations stepped together in one context.

The batch keeps every simulation in its own particle range with its own root
box, Morton order, tree and walk, so a simulation's result must not depend on
what else is in the batch: after the same number of steps its state is
bit-identical to the same simulation stepped alone in its own context, in
both precision modes, in 2D and 3D, across additions and removals and across
the reallocations that growth causes.  Sizes are chosen so that simulations
straddle the 4096-particle sort tiles and the box kernel's block tiles, and
include simulations of 1 to 3 particles.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS2 = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")
KEYS3 = KEYS2 + ("z", "vz", "az")


def _params(ge, dims, precision, leaf_cap=4):
    soft = 0.01
    return ge.default_params(dims, G=1.0, theta=0.7, softening=soft, leaf_cap=leaf_cap,
                             dt=1e-3, precision=precision)


def _ic(ics, dims, n, seed):
    if dims == 2:
        return ics.disk2d(n, seed=seed, center=(3.0 * (seed % 5), -2.0 * (seed % 3)))
    return ics.plummer3d(n, seed=seed)


def _alone(ge, p, st, steps):
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(steps)
        return s.download()


def _same(a, b, keys):
    for k in keys:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("dims,precision", [(2, 1), (2, 0), (3, 0), (3, 1)])
def test_batch_equals_alone(ge, ics, dims, precision):
    p = _params(ge, dims, precision)
    sizes = [1024, 3000, 1, 20000, 2, 5000, 4097, 3, 70001] if dims == 2 else \
            [1024, 7000, 2, 30000, 4095]
    ics_list = [_ic(ics, dims, n, seed) for seed, n in enumerate(sizes)]
    steps = 3
    keys = KEYS2 if dims == 2 else KEYS3
    with ge.Simulation(p) as b:
        handles = [b.add_sim(st) for st in ics_list]
        assert b.sims() == handles
        b.step(steps)
        for h, st, n in zip(handles, ics_list, sizes):
            assert b.query(h) == (n, int(np.sum(sizes[: handles.index(h)])), steps)
            _same(b.download_sim(h), _alone(ge, p, st, steps), keys)


def test_batch_add_remove_midway(ge, ics):
    p = _params(ge, 2, 1)
    sizes = [5000, 1500, 9000, 4096, 12345]
    st = [_ic(ics, 2, n, 10 + k) for k, n in enumerate(sizes)]
    with ge.Simulation(p) as b:
        h = [b.add_sim(s) for s in st[:3]]
        b.step(2)
        b.remove_sim(h[1])                    # middle one goes; the others move down
        h.append(b.add_sim(st[3]))            # joins after two steps
        b.step(1)
        b.remove_sim(h[0])                    # the first one goes
        h.append(b.add_sim(st[4]))
        b.step(2)
        assert b.sims() == [h[2], h[3], h[4]]
        assert [b.query(k)[2] for k in (h[2], h[3], h[4])] == [5, 3, 2]
        _same(b.download_sim(h[2]), _alone(ge, p, st[2], 5), KEYS2)
        _same(b.download_sim(h[3]), _alone(ge, p, st[3], 3), KEYS2)
        _same(b.download_sim(h[4]), _alone(ge, p, st[4], 2), KEYS2)
        with pytest.raises(ge.GeError):
            b.download_sim(h[1])


def test_batch_growth_keeps_state(ge, ics):
    """Adding simulations one at a time reallocates several times; the state
    of the earlier ones survives every reallocation."""
    p = _params(ge, 2, 0)
    sizes = [int(v) for v in ics.batch_sizes(count=24, lo=1024, hi=40000, seed=5)]
    st = [_ic(ics, 2, n, 100 + k) for k, n in enumerate(sizes)]
    with ge.Simulation(p) as b:
        h = []
        for k, s in enumerate(st):
            h.append(b.add_sim(s))
            b.step(1)
        for k in (0, 7, 23):
            _same(b.download_sim(h[k]), _alone(ge, p, st[k], len(st) - k), KEYS2)


def test_batch_matches_oracle_exact(ge, ics, O):
    """One simulation inside a batch, EXACT mode, against the oracle frame."""
    p = _params(ge, 2, 1)
    st = [_ic(ics, 2, n, 40 + k) for k, n in enumerate([2048, 3001, 1500])]
    with ge.Simulation(p) as b:
        h = [b.add_sim(s) for s in st]
        b.step(1)
        got = b.download_sim(h[1])
    fr = {k: np.array(v, copy=True) for k, v in st[1].items()}
    fr["ax"] = np.zeros(len(fr["x"]), np.float32)
    fr["ay"] = np.zeros(len(fr["x"]), np.float32)
    O.frame(O.make_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, leaf_cap=4), fr)
    for k in ("x", "y", "vx", "vy", "ax", "ay", "m", "id"):
        assert np.array_equal(got[k], fr[k]), k


def test_batch_tree_and_diagnostics(ge, ics):
    p = _params(ge, 2, 1)
    st = [_ic(ics, 2, n, 60 + k) for k, n in enumerate([3000, 1, 7000])]
    with ge.Simulation(p) as b:
        h = [b.add_sim(s) for s in st]
        b.build_tree()
        tb = b.export_tree()
        idx = np.array([0, 2999, 3000, 3001, 9001], np.uint32)
        ab = b.direct_sum_f64(idx)
    nodes = 0
    for k, s in enumerate(st):
        with ge.Simulation(p) as a:
            a.upload(s)
            a.build_tree()
            ta = a.export_tree()
            nodes += len(ta["mass"])
            if k == 2:
                aa = a.direct_sum_f64(np.array([0, 6000], np.uint32))
            if k == 0:
                a0 = a.direct_sum_f64(np.array([0, 2999], np.uint32))
                first = ta
    assert len(tb["mass"]) == nodes
    # the first simulation's tree is the first block of the export
    m = len(first["mass"])
    for key in ("size", "com", "mass", "start", "end", "next"):
        assert np.array_equal(tb[key][:m], first[key]), key
    ab = np.stack(ab[:2], 1)
    assert np.array_equal(ab[[0, 1]], np.stack(a0[:2], 1))
    assert np.all(ab[2] == 0.0)                # the one-particle simulation feels nothing
    assert np.array_equal(ab[[3, 4]], np.stack(aa[:2], 1))
