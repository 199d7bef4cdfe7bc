"""GPU: ge_frame_host, the drop-in frame on host arrays, over consecutive frames.

From its second frame on the same simulation, ge_frame_host overlaps the
copies with the step (masses and ids go up beside the kick, box, keys and
sort; positions, masses and ids come back beside the build and the walk).
The frames must be the same as the serial path's (upload, one step,
download) bit for bit in every mode, and, in EXACT mode, the oracle's
frames (the reference's frame order, globalLogic.cpp:1155-1370).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS2 = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")
KEYS3 = KEYS2 + ("z", "vz", "az")


def _start(ics, dims, n, seed):
    st = ics.disk2d(n, seed=seed) if dims == 2 else ics.plummer3d(n, seed=seed)
    st = {k: np.ascontiguousarray(v) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        st[k] = np.zeros(n, np.float32)
    return st


def _params(ge, dims, precision, **kw):
    return ge.default_params(dims, G=1.0, theta=0.7, softening=0.01, dt=1e-3, leaf_cap=4,
                             precision=precision, **kw)


@pytest.mark.parametrize("dims", [2, 3])
def test_frames_match_the_oracle(ge, ics, O, dims):
    st = _start(ics, dims, 6000, seed=dims)
    ref = {k: np.array(v, copy=True) for k, v in st.items()}
    eps2 = 1e-4 if dims == 2 else 0.01
    prm = O.make_params(dims, G=1.0, theta=0.7, eps2=eps2, dt=1e-3, leaf_cap=4)
    keys = KEYS2 if dims == 2 else KEYS3
    with ge.Simulation(_params(ge, dims, ge.PREC_EXACT)) as s:
        for f in range(4):
            s.frame_host(st)
            O.frame(prm, ref, walk_kind=0, nthreads=os.cpu_count() or 8)
            for k in keys:
                assert np.array_equal(st[k], ref[k]), (f, k)


@pytest.mark.parametrize("dims,precision,kw", [(2, 0, {}), (2, 2, dict(group_size=64)),
                                               (3, 2, dict(group_size=32)),
                                               (2, 0, dict(track_prev_vel=1))])
def test_frames_match_the_serial_path(ge, ics, dims, precision, kw):
    st = _start(ics, dims, 20000, seed=10 + dims)
    ser = {k: np.array(v, copy=True) for k, v in st.items()}
    keys = KEYS2 if dims == 2 else KEYS3
    p = _params(ge, dims, precision, **kw)
    with ge.Simulation(p) as a, ge.Simulation(p) as b:
        for f in range(3):
            a.frame_host(st)
            b.upload(ser)
            b.step(1)
            ser = b.download()
            for k in keys:
                assert np.array_equal(st[k], ser[k]), (f, k)
        if kw.get("track_prev_vel"):
            assert np.array_equal(a.download_prev_vel()[0], b.download_prev_vel()[0])
