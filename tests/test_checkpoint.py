"""GPU: checkpoint / resume (ge_download_state, ge_upload_state).

A run split in two -- k steps, a snapshot of every term the next step reads,
a new context restored from it, m more steps -- must give the same state bit
for bit as k + m steps in one context.  In GE_PREC_MIXED that needs the
Kahan compensation terms of positions and velocities (ge_download /
ge_upload alone drop them; the test shows the difference); in the other modes
it covers prevVel, pin flags and temperatures.  The reference's scene files
(SaveSystem, saveSystem.cpp:285-410) keep none of the compensation terms.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _straight_and_split(ge, p, st, k, m, extra=None):
    with ge.Simulation(p) as s:
        s.upload(st)
        if extra:
            extra(s)
        s.step(k + m)
        straight = s.download_state()
    with ge.Simulation(p) as s:
        s.upload(st)
        if extra:
            extra(s)
        s.step(k)
        snap = s.download_state()
    with ge.Simulation(p) as s:
        s.upload_state(snap)
        s.step(m)
        split = s.download_state()
    return straight, split, snap


@pytest.mark.parametrize("dims", [2, 3])
def test_mixed_mode_resumes_bit_for_bit(ge, ics, dims):
    if dims == 2:
        st = ics.two_disks2d(1 << 16, seed=3)
        p = ge.default_params(2, G=1.0, theta=0.7, softening=0.005, dt=1e-3,
                              precision=ge.PREC_MIXED, group_size=64, leaf_cap=8)
    else:
        st = ics.plummer3d(1 << 15, seed=3)
        p = ge.default_params(3, G=1.0, theta=0.5, eps2=0.01, dt=5e-4, precision=ge.PREC_MIXED,
                              group_size=32, leaf_cap=8)
    straight, split, snap = _straight_and_split(ge, p, st, 3, 4)
    assert np.any(snap["kx"] != 0) and np.any(snap["kvx"] != 0)   # the terms are live
    for key in straight:
        assert np.array_equal(straight[key], split[key]), key
    # without the compensation terms the resumed run departs
    lossy = {k: v for k, v in snap.items() if not k.startswith("k")}
    with ge.Simulation(p) as s:
        s.upload_state(lossy)
        s.step(4)
        out = s.download_state()
    assert not all(np.array_equal(out[k], straight[k]) for k in ("x", "y", "vx", "vy"))


def test_fast_mode_with_pins_temperatures_and_prev_vel(ge, ics):
    st = ics.disk2d(20000, seed=4)
    n = len(st["x"])
    rng = np.random.default_rng(1)
    pinned = (rng.random(n) < 0.02).astype(np.uint8)
    temp = rng.uniform(100.0, 500.0, n).astype(np.float32)
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, precision=ge.PREC_FAST,
                          track_prev_vel=1, temp_enabled=1)

    def extra(s):
        s.upload_pinned(pinned)
        s.upload_temp(temp)

    straight, split, snap = _straight_and_split(ge, p, st, 2, 3, extra)
    assert np.any(snap["pinned"]) and np.any(snap["pvx"] != 0)
    for key in straight:
        assert np.array_equal(straight[key], split[key]), key


def test_compensation_terms_are_refused_outside_the_mixed_mode(ge, ics):
    import ctypes as C
    st = ics.disk2d(1000, seed=5)
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, precision=ge.PREC_FAST)
    arrs = {k: np.ascontiguousarray(v) for k, v in st.items()}
    kx = np.zeros(1000, np.float32)
    with ge.Simulation(p) as s:
        sa = ge.StateArrays(*[arrs[k].ctypes.data if k in arrs else
                              (kx.ctypes.data if k == "kx" else None) for k in ge.STATE_KEYS])
        rc = ge.lib().ge_upload_state(s._h, 1000, C.byref(sa))
        assert rc == 5   # GE_ERR_STATE
