"""GPU: the warp-cooperative FAST walk (params.walk_kind = 1).

The 32 particles of a warp walk the tree together: every node is decided for
the whole warp against its bounding box with the reference's own rounding,
undecided subtrees are walked particle by particle.  Each particle's set of
interactions must therefore be exactly the reference's
(physics.cpp:91-205, physics3D.cpp:131-253):

  * accelerations within 1e-4 (per particle, relative) of the strict oracle
    walk on the same state and tree;
  * the interaction count equal to the oracle's, summed over particles;
  * a simulation's result bit-identical alone and in a batch (its warps are
    counted from its own first particle);
  * theta = 0 opens every node, so the warp's shared-memory stack overflows
    and every warp takes the per-particle fallback: still within 1e-4.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-4
NT = os.cpu_count() or 8
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
IDS = [os.path.basename(c)[:-4] for c in CASES]


def _rel_err(out, ref, dims):
    num = sum((out[a] - ref[a]).astype(np.float64) ** 2 for a in range(dims))
    den = sum(ref[a].astype(np.float64) ** 2 for a in range(dims))
    return np.sqrt(num / np.maximum(den, 1e-300))


def _params(ge, dims, theta, eps2, leaf_cap, dt):
    return ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=leaf_cap, dt=dt,
                             precision=ge.PREC_FAST, walk_kind=1)


def _forces(ge, st, dims, theta, eps2, leaf_cap, dt):
    """Sort, build and walk once (stage calls) with the warp walk; returns
    the sorted state, the accelerations and the interaction count."""
    with ge.Simulation(_params(ge, dims, theta, eps2, leaf_cap, dt)) as s:
        s.upload(st)
        s.compute_morton_keys()
        s.sort_particles_by_morton_key()
        s.build_tree()
        s.count_interactions(True)
        s.calculate_force_from_grid()
        out = s.download()
        inter = s.stats().interactions
        bb = s.bounding_box()
    return out, inter, bb


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_goldens(ge, path):
    g = dict(np.load(path))
    dims, theta, eps2, leaf_cap, dt, _ = g["meta"]
    dims, leaf_cap = int(dims), int(leaf_cap)
    if not eps2 > 0:
        pytest.skip("the warp walk needs eps2 > 0")
    st = {k[3:]: v for k, v in g.items() if k.startswith("in_")}
    out, inter, _ = _forces(ge, st, dims, float(theta), float(eps2), leaf_cap, float(dt))
    ax = ("ax", "ay", "az")[:dims]
    err = _rel_err([out[a] for a in ax], [g["walk_" + a] for a in ax], dims)
    assert err.max() <= FAST_TOL, err.max()
    assert inter == int(g["walk_inter"].astype(np.int64).sum())


def _oracle_check(O, out, bb, dims, theta, eps2, leaf_cap, inter):
    z = out.get("z")
    h = O.build_tree(out["x"], out["y"], out["m"], bb, z=z, leaf_cap=leaf_cap, holder=True)
    prm = O.make_params(dims=dims, theta=theta, eps2=eps2, leaf_cap=leaf_cap)
    res = O.walk(out["x"], out["y"], out["m"], h, prm, z=z, nthreads=NT, want_counts=True)
    ref, cnt = res[:dims], res[dims]
    ax = ("ax", "ay", "az")[:dims]
    err = _rel_err([out[a] for a in ax], ref, dims)
    assert err.max() <= FAST_TOL, err.max()
    assert inter == int(cnt.astype(np.int64).sum())


@pytest.mark.parametrize("theta", [0.5, 0.7, 1.0])
def test_two_disks_1m(ge, ics, O, theta):
    st = ics.two_disks2d(1 << 20, seed=0)
    eps2 = 0.005 ** 2
    out, inter, bb = _forces(ge, st, 2, theta, eps2, 4, 1e-3)
    _oracle_check(O, out, bb, 2, theta, eps2, 4, inter)


def test_plummer_3d(ge, ics, O):
    st = ics.plummer3d(1 << 16, seed=1)
    out, inter, bb = _forces(ge, st, 3, 0.5, 0.01, 4, 5e-4)
    _oracle_check(O, out, bb, 3, 0.5, 0.01, 4, inter)


def test_theta_zero_overflows_into_the_fallback(ge, ics, O):
    st = ics.disk2d(4096, seed=3)
    out, inter, bb = _forces(ge, st, 2, 0.0, 1e-4, 4, 1e-3)
    _oracle_check(O, out, bb, 2, 0.0, 1e-4, 4, inter)
    assert inter == 4096 * 4095


@pytest.mark.parametrize("dims", [2, 3])
def test_batch_equals_alone(ge, ics, dims):
    keys = ("x", "y", "vx", "vy", "ax", "ay", "m", "id") + (("z", "vz", "az") if dims == 3 else ())
    p = _params(ge, dims, 0.7, 1e-4 if dims == 2 else 0.01, 4, 1e-3)
    p.direct_below = 2000
    p.direct_eps2 = 0.01
    sizes = [1024, 3000, 1, 20000, 1500, 4097, 3, 70001] if dims == 2 else [1024, 7000, 2, 30000, 4095]
    sims = [(ics.disk2d(n, seed=k, center=(3.0 * (k % 5), -2.0 * (k % 3))) if dims == 2
             else ics.plummer3d(n, seed=k)) for k, n in enumerate(sizes)]
    with ge.Simulation(p) as b:
        handles = [b.add_sim(st) for st in sims]
        b.step(3)
        got = [b.download_sim(h) for h in handles]
    for st, out in zip(sims, got):
        with ge.Simulation(p) as s:
            s.upload(st)
            s.step(3)
            alone = s.download()
        for k in keys:
            assert np.array_equal(out[k], alone[k]), k


def test_step_with_the_warp_walk_stays_with_the_per_particle_walk(ge, ics):
    """Ten frames of the 16K disk: the two walks keep the same trajectory to
    within the FAST tolerance (they differ only in the order of the terms)."""
    st = ics.disk2d(16384, seed=0)
    outs = []
    for wk in (0, 1):
        p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, leaf_cap=1, dt=1e-3,
                              precision=ge.PREC_FAST, walk_kind=wk)
        with ge.Simulation(p) as s:
            s.upload(st)
            s.step(10)
            outs.append(s.download())
    a, b = outs
    oa, ob = np.argsort(a["id"]), np.argsort(b["id"])
    err = _rel_err([b["ax"][ob], b["ay"][ob]], [a["ax"][oa], a["ay"][oa]], 2)
    assert np.median(err) < 1e-5 and err.max() < 1e-3, (np.median(err), err.max())
