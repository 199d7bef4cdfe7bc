"""GPU: the key-prefix tree build against the oracle's restatement of the
reference's recursive build (quadtree.cpp:5-292).

A step builds its tree from the sort's Morton keys and rebuilds exactly, with
the reference's partition-point cuts, only where the keys and the float
compares disagree (near cell midlines) or cannot decide (runs of equal keys
deeper than the keys' 18 / 21 levels).  These cases aim at each branch:
leaf capacities at and beyond the key path's limit (32), clumps of coincident
particles (rebuild roots of every size: one block, the grid's level loop,
warp subtrees), and particles placed a few ulps either side of many cell
midlines (suspect checks whose cuts differ from the key boundaries).  With
zero velocities and accelerations the first step builds on the given
positions, so the exported tree is compared node for node with the oracle's
build of the sorted state, and EXACT frames bit for bit.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TREE_KEYS = ["pos", "size", "com", "mass", "start", "end", "next", "child"]


def _state(x, y, z=None):
    n = len(x)
    st = dict(x=np.asarray(x, np.float32), y=np.asarray(y, np.float32),
              vx=np.zeros(n, np.float32), vy=np.zeros(n, np.float32),
              m=np.full(n, 1.0 / n, np.float32), id=np.arange(n, dtype=np.uint32))
    if z is not None:
        st["z"] = np.asarray(z, np.float32)
        st["vz"] = np.zeros(n, np.float32)
    return st


def _check(ge, O, st, dims, leaf_cap, eps2=1e-4, theta=0.7, steps=2):
    z = st.get("z")
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=leaf_cap, dt=1e-3,
                          precision=ge.PREC_EXACT)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)
        first = s.download()
        t = s.export_tree()
        bb = s.bounding_box()
        s.step(steps - 1)
        out = s.download()
    x, y, m = first["x"], first["y"], first["m"]
    zz = first.get("z")
    tr = O.build_tree(x, y, m, bb, z=zz, leaf_cap=leaf_cap)
    for a in TREE_KEYS:
        assert np.array_equal(t[a], getattr(tr, a)), a
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        fr[k] = np.zeros(len(fr["x"]), np.float32)
    prm = O.make_params(dims, G=1.0, theta=theta, eps2=eps2, dt=1e-3, leaf_cap=leaf_cap)
    for _ in range(steps):
        O.frame(prm, fr, walk_kind=0, nthreads=os.cpu_count() or 8)
    keys = ("x", "y", "vx", "vy", "ax", "ay", "id") + (("z", "vz", "az") if dims == 3 else ())
    for k in keys:
        assert np.array_equal(out[k], fr[k]), k


@pytest.mark.parametrize("leaf_cap", [1, 8, 32, 33])
def test_leaf_capacities(ge, ics, O, leaf_cap):
    """32 is the largest leaf capacity of the key path; 33 takes the
    top-down builder.  Both give the reference's tree."""
    st = ics.disk2d(20000, seed=leaf_cap)
    st = {k: np.array(v, copy=True) for k, v in st.items()}
    st["vx"][:] = 0.0
    st["vy"][:] = 0.0
    _check(ge, O, st, 2, leaf_cap)


@pytest.mark.parametrize("dims", [2, 3])
def test_clumps_of_coincident_particles(ge, O, dims):
    """Runs of equal keys that are not leaves: clumps of 2 to 3000 particles
    at one point (rebuilt exactly below the keys' last level, by a warp, a
    block or the grid's level loop) among a scattered background."""
    rng = np.random.default_rng(40 + dims)
    parts = [rng.uniform(-8, 8, (6000, dims))]
    for c in [2, 5, 33, 40, 300, 1000, 2100, 3000]:
        parts.append(np.repeat(rng.uniform(-8, 8, (1, dims)), c, axis=0))
    # near-coincident: a cluster finer than the keys' last cell
    parts.append(rng.uniform(0, 1e-6, (500, dims)) + 3.0)
    P = np.concatenate(parts).astype(np.float32)
    st = _state(P[:, 0], P[:, 1], P[:, 2] if dims == 3 else None)
    _check(ge, O, st, dims, 4, eps2=1e-2 if dims == 3 else 1e-4)


@pytest.mark.parametrize("dims", [2, 3])
def test_chains_that_end_in_splits(ge, O, dims):
    """Tight clusters (40 to 4000 particles spread over 1e-5 to 1e-3) in a
    wide box: each sits in one quadrant for many levels (a chain of
    single-child nodes, written in one go from the cluster's bounding box)
    and then splits; clusters inside clusters make chains below splits too.
    Rebuilt by the warp subtrees, a block and the grid's level loop."""
    rng = np.random.default_rng(70 + dims)
    parts = [rng.uniform(-50, 50, (3000, dims))]
    for c, w in [(40, 1e-5), (90, 3e-4), (700, 1e-3), (1500, 2e-5), (2600, 5e-4), (4000, 1e-4)]:
        ctr = rng.uniform(-40, 40, (1, dims))
        parts.append(ctr + rng.uniform(0.0, w, (c, dims)))
        parts.append(ctr + 0.37 * w + rng.uniform(0.0, w * 1e-3, (c // 3, dims)))
    P = np.concatenate(parts).astype(np.float32)
    st = _state(P[:, 0], P[:, 1], P[:, 2] if dims == 3 else None)
    _check(ge, O, st, dims, 4, eps2=1e-2 if dims == 3 else 1e-4)


@pytest.mark.parametrize("nbg", [4000, 60000])
@pytest.mark.parametrize("dims", [2, 3])
def test_particles_on_cell_midlines(ge, O, dims, nbg):
    """Particles within a few ulps of the midlines of cells of many levels,
    where the Morton digit and the float compare can disagree: every such
    node is checked with the reference's cuts and rebuilt where they differ.
    The root box is offset and not a power of two wide (the two-disk
    workload's), so the keys' grid and the halved cells round differently;
    with these seeds and 4000 background particles a pure key-prefix tree
    differs from the reference's in 91 (2D) / 338 (3D) nodes, all of which the
    exact check must repair.  With 60000, the differing nodes of the top
    levels hold more particles than one warp marks (the large-root list)."""
    rng = np.random.default_rng(17 + dims)
    lo, S = np.float32(-9.981265), np.float32(19.9565)
    bg = rng.uniform(0.0, 1.0, (nbg, dims)) * S + lo
    corners = np.array([[lo] * dims, [lo + S] * dims], np.float32)   # fixes the root box
    pts = []
    for L in range(1, 16):
        k = rng.integers(1, 2 ** L, 40)
        for a in range(dims):
            q = rng.uniform(0.0, 1.0, (40, dims)) * S + lo
            q[:, a] = lo + (2 * k - 1).astype(np.float64) / 2 ** (L + 1) * S
            pts.append(q)
    Q = np.concatenate(pts).astype(np.float32)
    # a few ulps either side of the midline
    ulps = rng.integers(-3, 4, Q.shape)
    Q = (Q.astype(np.float64) + ulps * np.spacing(Q).astype(np.float64)).astype(np.float32)
    P = np.clip(np.concatenate([corners, bg, Q]).astype(np.float32), lo, lo + S)
    st = _state(P[:, 0], P[:, 1], P[:, 2] if dims == 3 else None)
    _check(ge, O, st, dims, 4, eps2=1e-2 if dims == 3 else 1e-4, theta=0.5)
