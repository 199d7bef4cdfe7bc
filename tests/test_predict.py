"""GPU: trajectory preview on the resident tree (ge_predict_trajectory).

ParticlesSpawning::predictTrajectory (particlesSpawning.cpp:443-500, 3D
:1000-1060) steps a probe particle against the frame's tree, which is not
rebuilt, with the older walk (physics.cpp:4-90, physics3D.cpp:49-120).  The
device runs many probes at once with the reference's rounding; every path is
bit-identical to the oracle's statement on the same tree (which is the
device's tree, bit for bit).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probes(rng, dims, k, spread):
    pos = rng.uniform(-spread, spread, (k, dims)).astype(np.float32)
    vel = rng.normal(0.0, 0.3, (k, dims)).astype(np.float32)
    mass = rng.uniform(1e-3, 1.0, k).astype(np.float32)
    return pos, vel, mass


@pytest.mark.parametrize("dims,periodic", [(2, False), (3, False), (2, True)])
def test_predict_matches_oracle(ge, ics, O, dims, periodic):
    rng = np.random.default_rng(7)
    if dims == 2:
        st = ics.disk2d(5000, seed=2, center=(10.0, 10.0) if periodic else (0.0, 0.0))
        eps2_walk, eps2_pred = 1e-4, 1e-4
    else:
        st = ics.plummer3d(3000, seed=2)
        eps2_walk, eps2_pred = 0.1, 0.01   # the preview walk squares the softening in 3D too
    domain = (20.0, 20.0, 20.0) if periodic else (0.0, 0.0, 0.0)
    kw = dict(periodic=1, domain=domain) if periodic else {}
    p = ge.default_params(dims, G=1.0, theta=0.7, eps2=eps2_walk, dt=1e-3, leaf_cap=4,
                          precision=ge.PREC_EXACT, **kw)
    pos, vel, mass = _probes(rng, dims, 24, 3.0)
    if periodic:
        pos += 10.0
    steps = 150
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(2)
        out = s.download()
        got = s.predict_trajectory(pos, vel, mass, steps, eps2_pred)
    z = out.get("z")
    bb = O.bbox(out["x"], out["y"], z)
    tree = O.build_tree(out["x"], out["y"], out["m"], bb, z=z, leaf_cap=4, holder=True)
    op = O.make_params(dims, G=1.0, theta=0.7, eps2=eps2_walk, dt=1e-3, leaf_cap=4,
                       periodic=periodic, domain=domain)
    ref = O.predict_trajectory(out["x"], out["y"], tree, op, eps2_pred, pos, vel, mass, steps,
                               z=z)
    assert got.shape == (24, steps, dims)
    assert np.all(np.isfinite(got))
    assert np.array_equal(got, ref)
    moved = np.abs(got[:, -1] - got[:, 0]).max()
    assert moved > 1e-3


def test_predict_refused_in_mixed_mode(ge, ics):
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, precision=ge.PREC_MIXED)
    with ge.Simulation(p) as s:
        s.upload(ics.disk2d(2048, seed=1))
        s.step(1)
        with pytest.raises(ge.GeError) as ei:
            s.predict_trajectory(np.zeros(2), np.zeros(2), np.ones(1), 5, 1e-4)
        assert ei.value.code == 8
