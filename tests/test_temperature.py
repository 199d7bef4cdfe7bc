"""GPU: heat exchange inside the walk (myVar.isTempEnabled).

The reference walk moves heat between a particle and every accepted node
(by the node's average temperature) and every other particle of an opened
leaf: temp_i += globalHeatConductivity * (T - temp_i) / distance * dt
(physics.cpp:145-158, 183-191; physics3D.cpp:190-201, 230-237).  It updates
temp_i in place while other OpenMP threads read it, so the oracle and the
device both use one fixed order: the others' temperatures (and the node
sums, taken at build time) as they were before the walk.  EXACT frames are
then bit-identical to the oracle frame, temperatures included, over several
steps; FAST frames agree within the plain-path tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "vx", "vy", "ax", "ay", "m", "id", "temp")


def _state(ics, dims, n, seed):
    st = ics.disk2d(n, seed=seed) if dims == 2 else ics.plummer3d(n, seed=seed)
    st = {k: np.array(v, copy=True) for k, v in st.items()}
    st["temp"] = np.random.default_rng(seed).uniform(100.0, 5000.0, n).astype(np.float32)
    return st


def _oracle(O, st, dims, steps, theta, eps2, leaf_cap, heat):
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        fr[k] = np.zeros(len(fr["x"]), np.float32)
    p = O.make_params(dims, G=1.0, theta=theta, eps2=eps2, dt=1e-3, leaf_cap=leaf_cap,
                      temp_enabled=True, heat_cond=heat)
    for _ in range(steps):
        O.frame(p, fr, walk_kind=0)
    return fr


def _gpu(ge, st, dims, steps, theta, eps2, leaf_cap, heat, precision):
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, dt=1e-3, leaf_cap=leaf_cap,
                          precision=precision, temp_enabled=1, heat_cond=heat)
    with ge.Simulation(p) as s:
        s.upload({k: v for k, v in st.items() if k != "temp"})
        s.upload_temp(st["temp"])
        s.step(steps)
        out = s.download()
        out["temp"] = s.download_temp()
    return out


@pytest.mark.parametrize("dims,n,steps", [(2, 3000, 1), (2, 5000, 4), (3, 2048, 3)])
def test_heat_exchange_exact_matches_oracle(ge, ics, O, dims, n, steps):
    st = _state(ics, dims, n, seed=11 + n)
    eps2 = 1e-4 if dims == 2 else 0.01
    keys = KEYS + (("z", "vz", "az") if dims == 3 else ())
    ref = _oracle(O, st, dims, steps, 0.7, eps2, 4, 0.045)
    got = _gpu(ge, st, dims, steps, 0.7, eps2, 4, 0.045, ge.PREC_EXACT)
    assert not np.array_equal(ref["temp"][np.argsort(ref["id"])], st["temp"])   # heat moved
    for k in keys:
        assert np.array_equal(got[k], ref[k]), k


def test_heat_exchange_fast_within_tolerance(ge, ics, O):
    st = _state(ics, 2, 8000, seed=3)
    ref = _oracle(O, st, 2, 1, 0.7, 1e-4, 4, 0.045)
    got = _gpu(ge, st, 2, 1, 0.7, 1e-4, 4, 0.045, ge.PREC_FAST)
    assert np.array_equal(got["id"], ref["id"])
    rel = np.abs(got["temp"] - ref["temp"]) / np.abs(ref["temp"])
    assert rel.max() <= 1e-5


def test_heat_exchange_off_leaves_temperatures(ge, ics):
    """With the exchange off the temperatures only follow their particles."""
    st = _state(ics, 2, 3000, seed=5)
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, precision=ge.PREC_EXACT)
    with ge.Simulation(p) as s:
        s.upload({k: v for k, v in st.items() if k != "temp"})
        s.upload_temp(st["temp"])
        s.step(2)
        out = s.download()
        t = s.download_temp()
    assert np.array_equal(t, st["temp"][out["id"]])


def test_heat_exchange_refused_in_mixed_mode(ge):
    p = ge.default_params(2, precision=ge.PREC_MIXED, temp_enabled=1)
    with pytest.raises(ge.GeError) as ei:
        ge.Simulation(p)
    assert ei.value.code == 8
