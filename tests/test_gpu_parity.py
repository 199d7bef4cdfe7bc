"""GPU parity: every stage of the CUDA path, through the C ABI, against the
oracle (golden fixtures plus live oracle runs at full size).

Tolerances:
  * bounding box, keys, permutation, tree topology, masses and centres of mass:
    bit-exact (integer/index work, and float sums made in the reference's order
    with the reference's rounding);
  * accelerations, GE_PREC_EXACT: bit-exact against the strict oracle;
  * accelerations, GE_PREC_FAST: per-particle relative error <= 1e-4 (the
    plain-path bound) against the strict oracle.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TREE_KEYS = ["pos", "size", "com", "mass", "start", "end", "next", "child"]
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
IDS = [os.path.basename(c)[:-4] for c in CASES]
FAST_TOL = 1e-4


def _case(path):
    g = dict(np.load(path))
    dims, theta, eps2, leaf_cap, dt, _ = g["meta"]
    return g, int(dims), float(theta), float(eps2), int(leaf_cap), float(dt)


def _inputs(g, dims):
    st = {k[3:]: v for k, v in g.items() if k.startswith("in_")}
    return st


def _sim(ge, dims, theta, eps2, leaf_cap, dt, precision, **kw):
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=leaf_cap, dt=dt,
                          precision=precision, **kw)
    return ge.Simulation(p)


def _rel_err(ax, ay, bx, by, az=None, bz=None):
    num = (ax - bx) ** 2 + (ay - by) ** 2
    den = bx.astype(np.float64) ** 2 + by.astype(np.float64) ** 2
    if az is not None:
        num = num + (az - bz) ** 2
        den = den + bz.astype(np.float64) ** 2
    return np.sqrt(num / np.maximum(den, 1e-300))


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_bbox_keys_sort_bit_exact(ge, path):
    g, dims, theta, eps2, leaf_cap, dt = _case(path)
    st = _inputs(g, dims)
    with _sim(ge, dims, theta, eps2, leaf_cap, dt, ge.PREC_EXACT) as s:
        s.upload(st)
        assert np.array_equal(s.bounding_box(), g["bbox"])
        assert np.array_equal(s.compute_morton_keys(), g["keys"])
        perm = s.sort_particles_by_morton_key()
        assert np.array_equal(perm, g["perm"])
        out = s.download()
        for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id"):
            if k in st:
                assert np.array_equal(out[k], st[k][g["perm"]]), k


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_tree_bit_exact(ge, path):
    g, dims, theta, eps2, leaf_cap, dt = _case(path)
    st = _inputs(g, dims)
    for tag, lc, sort in (("tc", leaf_cap, True), ("t4", 4, True), ("tu", 4, False)):
        with _sim(ge, dims, theta, eps2, lc, dt, ge.PREC_EXACT) as s:
            s.upload(st)
            if sort:
                s.compute_morton_keys()
                s.sort_particles_by_morton_key()
            s.build_tree()
            t = s.export_tree()
            for a in TREE_KEYS:
                assert np.array_equal(t[a], g[f"{tag}_{a}"]), (tag, a)


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_forces_exact_mode_bit_exact(ge, path):
    g, dims, theta, eps2, leaf_cap, dt = _case(path)
    with _sim(ge, dims, theta, eps2, leaf_cap, dt, ge.PREC_EXACT) as s:
        s.upload(_inputs(g, dims))
        s.compute_morton_keys()
        s.sort_particles_by_morton_key()
        s.build_tree()
        s.count_interactions(True)
        s.calculate_force_from_grid()
        out = s.download()
        assert np.array_equal(out["ax"], g["walk_ax"])
        assert np.array_equal(out["ay"], g["walk_ay"])
        if dims == 3:
            assert np.array_equal(out["az"], g["walk_az"])
        assert s.stats().interactions == int(g["walk_inter"].astype(np.int64).sum())


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_forces_fast_mode_within_tolerance(ge, path):
    g, dims, theta, eps2, leaf_cap, dt = _case(path)
    with _sim(ge, dims, theta, eps2, leaf_cap, dt, ge.PREC_FAST) as s:
        s.upload(_inputs(g, dims))
        s.compute_morton_keys()
        s.sort_particles_by_morton_key()
        s.build_tree()
        s.calculate_force_from_grid()
        out = s.download()
        err = _rel_err(out["ax"], out["ay"], g["walk_ax"], g["walk_ay"],
                       out.get("az"), g.get("walk_az"))
        assert err.max() <= FAST_TOL, err.max()


@pytest.mark.parametrize("path", CASES, ids=IDS)
@pytest.mark.parametrize("precision", [0, 1], ids=["fast", "exact"])
def test_one_frame(ge, path, precision):
    g, dims, theta, eps2, leaf_cap, dt = _case(path)
    st = _inputs(g, dims)
    with _sim(ge, dims, theta, eps2, leaf_cap, dt, precision) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
    ref = {k[6:]: v for k, v in g.items() if k.startswith("frame_")}
    assert np.array_equal(out["id"], ref["id"])
    if precision == 1:
        for k in ref:
            assert np.array_equal(out[k], ref[k]), k
    else:
        err = _rel_err(out["ax"], out["ay"], ref["ax"], ref["ay"], out.get("az"), ref.get("az"))
        assert err.max() <= FAST_TOL, err.max()
        # positions/velocities only differ through the previous (zero) acceleration
        for k in ("x", "y", "m"):
            assert np.array_equal(out[k], ref[k]), k


def test_frame_host_drop_in(ge, O):
    """ge_frame_host: host arrays in, host arrays out, Morton order + ids."""
    g, dims, theta, eps2, leaf_cap, dt = _case(os.path.join(GOLDEN, "disk2d_n2048.npz"))
    st = {k: np.array(v, copy=True) for k, v in _inputs(g, dims).items()}
    st["ax"] = np.zeros_like(st["x"])
    st["ay"] = np.zeros_like(st["x"])
    with _sim(ge, dims, theta, eps2, leaf_cap, dt, ge.PREC_EXACT) as s:
        s.frame_host(st)
    for k in ("x", "y", "vx", "vy", "ax", "ay", "m", "id"):
        assert np.array_equal(st[k], g[f"frame_{k}"]), k


def _oracle_frames(O, params, st, steps, threads=None):
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if params.dims == 3 else ()):
        fr[k] = np.zeros(len(fr["x"]), np.float32)
    nt = threads or os.cpu_count() or 8
    for _ in range(steps):
        O.frame(params, fr, walk_kind=0, nthreads=nt)
    return fr


def test_disk_16k_hundred_steps(ge, ics, O):
    """N=16,384 disk, G=1, theta 0.7, softening 0.01, dt 1e-3, leaf capacity 1:
    1 and 100 steps against the oracle frame loop.  EXACT mode reproduces the
    oracle's trajectory bit for bit.  FAST mode rounds its force terms
    differently, so trajectories part slowly; its accelerations are checked
    against the oracle walk on the GPU's own final state, and its positions
    against the oracle trajectory."""
    st = ics.disk2d(16384, seed=0)
    eps2 = 0.01 ** 2
    prm = O.make_params(dims=2, theta=0.7, eps2=eps2, leaf_cap=1, dt=1e-3)
    for steps in (1, 100):
        ref = _oracle_frames(O, prm, st, steps)
        with _sim(ge, 2, 0.7, eps2, 1, 1e-3, ge.PREC_EXACT) as s:
            s.upload(st)
            s.step(steps)
            out = s.download()
        for k in ("x", "y", "vx", "vy", "ax", "ay", "id"):
            assert np.array_equal(out[k], ref[k]), (steps, k)
        with _sim(ge, 2, 0.7, eps2, 1, 1e-3, ge.PREC_FAST) as s:
            s.upload(st)
            s.step(steps)
            out = s.download()
            bb = s.bounding_box()
        # forces on the same state
        x, y, m = out["x"], out["y"], out["m"]
        h = O.build_tree(x, y, m, bb, leaf_cap=1, holder=True)
        ax, ay = O.walk(x, y, m, h, prm, nthreads=os.cpu_count() or 8)
        err = _rel_err(out["ax"], out["ay"], ax, ay)
        assert err.max() <= FAST_TOL, (steps, err.max())
        # trajectories stay close (compared by id)
        o_ref, o_out = np.argsort(ref["id"]), np.argsort(out["id"])
        dpos = np.hypot(out["x"][o_out] - ref["x"][o_ref], out["y"][o_out] - ref["y"][o_ref])
        assert dpos.max() < 1e-4 * float(bb[2]), (steps, dpos.max())


def test_two_disks_1m_one_step(ge, ics, O):
    """N=1,048,576 two-disk workload, theta 0.7, softening 0.005: tree
    bit-exact with the oracle's build of the same sorted state, and FAST
    accelerations within 1e-4 of the oracle walk for every particle."""
    st = ics.two_disks2d(1 << 20, seed=0)
    eps2 = 0.005 ** 2
    with _sim(ge, 2, 0.7, eps2, 4, 1e-3, ge.PREC_FAST) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
        t = s.export_tree()
        bb = s.bounding_box()
    assert np.array_equal(np.sort(out["id"]), np.arange(1 << 20, dtype=np.uint32))
    x, y, m = out["x"], out["y"], out["m"]
    k = O.morton_keys(x, y, bb)
    assert np.all(np.diff(k.astype(np.int64)) >= 0)
    h = O.build_tree(x, y, m, bb, leaf_cap=4, holder=True)
    tr = h.to_numpy()
    for a in TREE_KEYS:
        assert np.array_equal(t[a], getattr(tr, a)), a
    prm = O.make_params(dims=2, theta=0.7, eps2=eps2, leaf_cap=4, dt=1e-3)
    ax, ay = O.walk(x, y, m, h, prm, nthreads=os.cpu_count() or 8)
    err = _rel_err(out["ax"], out["ay"], ax, ay)
    assert err.max() <= FAST_TOL, err.max()


def test_plummer_3d_one_step(ge, ics, O):
    st = ics.plummer3d(1 << 16, seed=1)
    prm = O.make_params(dims=3, theta=0.5, eps2=0.01, leaf_cap=4, dt=5e-4)
    ref = _oracle_frames(O, prm, st, 1)
    for precision in (1, 0):
        with _sim(ge, 3, 0.5, 0.01, 4, 5e-4, precision) as s:
            s.upload(st)
            s.step(1)
            out = s.download()
        assert np.array_equal(out["id"], ref["id"])
        if precision == 1:
            for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
                assert np.array_equal(out[k], ref[k]), k
        else:
            err = _rel_err(out["ax"], out["ay"], ref["ax"], ref["ay"], out["az"], ref["az"])
            assert err.max() <= FAST_TOL, err.max()


@pytest.mark.parametrize("n", [1, 2, 3, 33])
def test_tiny_systems(ge, O, n):
    rng = np.random.default_rng(n)
    st = dict(x=rng.uniform(-1, 1, n).astype(np.float32), y=rng.uniform(-1, 1, n).astype(np.float32),
              vx=np.zeros(n, np.float32), vy=np.zeros(n, np.float32),
              m=np.full(n, 1.0 / n, np.float32), id=np.arange(n, dtype=np.uint32))
    prm = O.make_params(dims=2, theta=0.7, eps2=1e-4, leaf_cap=1, dt=1e-3)
    ref = _oracle_frames(O, prm, st, 3, threads=1)
    with _sim(ge, 2, 0.7, 1e-4, 1, 1e-3, ge.PREC_EXACT) as s:
        s.upload(st)
        s.step(3)
        out = s.download()
    for k in ("x", "y", "vx", "vy", "ax", "ay", "id"):
        assert np.array_equal(out[k], ref[k]), k


def test_pinned_particles_do_not_move(ge, ics):
    st = ics.disk2d(4096, seed=7)
    pinned = np.zeros(4096, np.uint8)
    pinned[::7] = 1
    with _sim(ge, 2, 0.7, 1e-4, 4, 1e-3, ge.PREC_FAST) as s:
        s.upload(st)
        s.upload_pinned(pinned)
        s.step(5)
        out = s.download()
    was = pinned[out["id"]] == 1
    assert np.array_equal(out["x"][was], st["x"][out["id"][was]])
    assert np.array_equal(out["vx"][was], st["vx"][out["id"][was]])
    assert not np.array_equal(out["x"][~was], st["x"][out["id"][~was]])
