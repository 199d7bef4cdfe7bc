"""GPU: the direct sum the application runs for small simulations.

Below 5000 particles (or with myVar.naive) the frame takes its accelerations
from Physics::naiveGravity (physics.cpp:392-434) / naiveGravity3D
(physics3D.cpp:416-469) instead of the tree walk (globalLogic.cpp:1321-1346,
3D :1677-1702): every pair in the particles' (Morton) order, softening added
un-squared, the acceleration itself (no division by the particle's mass), no
heat exchange.  params.direct_below selects it per simulation.  EXACT frames
are bit-identical to the oracle frame with the same dispatch (the oracle's
scalar direct sum), alone and inside a batch whose other simulations walk;
FAST frames agree within the plain-path tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS2 = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")
KEYS3 = KEYS2 + ("z", "vz", "az")
SOFT = 0.01


def _params(ge, dims, precision, below, **kw):
    return ge.default_params(dims, G=1.0, theta=0.7, softening=SOFT, dt=1e-3, leaf_cap=4,
                             precision=precision, direct_below=below, **kw)


def _oracle(O, st, dims, steps, below, periodic=False, domain=(0.0, 0.0, 0.0)):
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        fr[k] = np.zeros(len(fr["x"]), np.float32)
    eps2 = SOFT * SOFT if dims == 2 else SOFT
    p = O.make_params(dims, G=1.0, theta=0.7, eps2=eps2, dt=1e-3, leaf_cap=4,
                      naive_soft=SOFT, direct_below=below, periodic=periodic, domain=domain)
    for _ in range(steps):
        O.frame(p, fr, walk_kind=0)
    return fr


def _gpu(ge, st, p, steps):
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(steps)
        return s.download()


@pytest.mark.parametrize("dims,n,periodic", [(2, 3000, False), (2, 4999, False),
                                             (3, 2048, False), (2, 2500, True),
                                             (3, 1500, True)])
def test_direct_exact_matches_oracle(ge, ics, O, dims, n, periodic):
    if dims == 2:
        st = ics.disk2d(n, seed=n, center=(10.0, 10.0) if periodic else (0.0, 0.0))
    else:
        st = ics.plummer3d(n, seed=n)
        if periodic:
            st = dict(st)
            for k in ("x", "y", "z"):
                st[k] = (st[k] + np.float32(4.0)).astype(np.float32)
    domain = (20.0, 20.0, 20.0) if dims == 2 else (8.0, 8.0, 8.0)
    kw = dict(periodic=1, domain=domain) if periodic else {}
    keys = KEYS2 if dims == 2 else KEYS3
    got = _gpu(ge, st, _params(ge, dims, ge.PREC_EXACT, 5000, **kw), 3)
    ref = _oracle(O, st, dims, 3, 5000, periodic=periodic, domain=domain if periodic else (0, 0, 0))
    for k in keys:
        assert np.array_equal(got[k], ref[k]), k
    # it is the direct sum, not the walk: the walk's frame differs
    walk = _oracle(O, st, dims, 3, 0, periodic=periodic, domain=domain if periodic else (0, 0, 0))
    assert not np.array_equal(walk["ax"], ref["ax"])


def test_threshold_is_strict(ge, ics, O):
    """A simulation of exactly direct_below particles walks."""
    st = ics.disk2d(3000, seed=4)
    got = _gpu(ge, st, _params(ge, 2, ge.PREC_EXACT, 3000), 2)
    ref = _oracle(O, st, 2, 2, 0)
    for k in KEYS2:
        assert np.array_equal(got[k], ref[k]), k


def test_direct_fast_within_tolerance(ge, ics, O):
    st = ics.disk2d(4000, seed=8)
    got = _gpu(ge, st, _params(ge, 2, ge.PREC_FAST, 5000), 1)
    ref = _oracle(O, st, 2, 1, 5000)
    assert np.array_equal(got["id"], ref["id"])
    a = np.hypot(ref["ax"], ref["ay"])
    err = np.hypot(got["ax"] - ref["ax"], got["ay"] - ref["ay"]) / a
    assert np.median(err) <= 1e-5
    assert np.percentile(err, 99) <= 1e-4


@pytest.mark.parametrize("dims,precision", [(2, 1), (3, 1), (2, 0)])
def test_batch_mixes_direct_and_walk(ge, ics, O, dims, precision):
    """Simulations below the threshold take the direct sum, the others walk,
    in one batch; each equals the same simulation alone."""
    sizes = [3000, 7000, 1, 1500, 5000, 4097] if dims == 2 else [2048, 6000, 700]
    sts = [ics.disk2d(n, seed=20 + k, center=(2.0 * k, 0.0)) if dims == 2
           else ics.plummer3d(n, seed=20 + k) for k, n in enumerate(sizes)]
    p = _params(ge, dims, precision, 5000)
    keys = KEYS2 if dims == 2 else KEYS3
    with ge.Simulation(p) as b:
        hs = [b.add_sim(s) for s in sts]
        b.step(2)
        got = [b.download_sim(h) for h in hs]
    for st, g in zip(sts, got):
        alone = _gpu(ge, st, p, 2)
        for k in keys:
            assert np.array_equal(g[k], alone[k]), k
    if precision == 1:
        for st, g in zip(sts, got):
            ref = _oracle(O, st, dims, 2, 5000)
            for k in keys:
                assert np.array_equal(g[k], ref[k]), k


def test_switch_on_a_live_context(ge, ics, O):
    """direct_below changed between steps applies from the next step."""
    st = ics.disk2d(2500, seed=31)
    p = _params(ge, 2, ge.PREC_EXACT, 0)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)
        p.direct_below = 5000
        s.set_params(p)
        s.step(1)
        got = s.download()
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    fr["ax"] = np.zeros(len(fr["x"]), np.float32)
    fr["ay"] = np.zeros(len(fr["x"]), np.float32)
    O.frame(O.make_params(2, G=1.0, theta=0.7, eps2=SOFT * SOFT, dt=1e-3, leaf_cap=4), fr)
    O.frame(O.make_params(2, G=1.0, theta=0.7, eps2=SOFT * SOFT, dt=1e-3, leaf_cap=4,
                          naive_soft=SOFT, direct_below=5000), fr)
    for k in KEYS2:
        assert np.array_equal(got[k], fr[k]), k


def test_direct_keeps_temperatures(ge, ics):
    """The direct sum exchanges no heat (naiveGravity has no temperature
    term): with heat exchange on, a small simulation's temperatures only
    follow their particles."""
    st = ics.disk2d(3000, seed=6)
    t0 = np.random.default_rng(6).uniform(100.0, 5000.0, 3000).astype(np.float32)
    p = _params(ge, 2, ge.PREC_EXACT, 5000, temp_enabled=1)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.upload_temp(t0)
        s.step(2)
        out = s.download()
        t = s.download_temp()
    assert np.array_equal(t, t0[out["id"]])


def test_direct_refusals(ge):
    with pytest.raises(ge.GeError) as ei:
        ge.Simulation(_params(ge, 2, ge.PREC_MIXED, 5000))
    assert ei.value.code == 8
    p = _params(ge, 2, ge.PREC_EXACT, 5000)
    p.direct_eps2 = 0.0
    with pytest.raises(ge.GeError) as ei:
        ge.Simulation(p)
    assert ei.value.code == 1
    p = _params(ge, 2, ge.PREC_EXACT, -1)
    with pytest.raises(ge.GeError) as ei:
        ge.Simulation(p)
    assert ei.value.code == 1
