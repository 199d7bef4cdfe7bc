"""CPU: pin the oracle (oracle/ge_oracle.c) against the golden fixtures and,
where it was compiled here, against the reference's own morton.cpp /
quadtree.cpp (oracle/_ref)."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

TREE_KEYS = ["pos", "size", "com", "mass", "start", "end", "next", "child"]
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def _load(path):
    return dict(np.load(path))


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_reproduces_golden(O, path):
    g = _load(path)
    dims, theta, eps2, leaf_cap, dt, _ = g["meta"]
    dims, leaf_cap = int(dims), int(leaf_cap)
    x, y, m = g["in_x"], g["in_y"], g["in_m"]
    z = g.get("in_z")
    bb = O.bbox(x, y, z)
    assert np.array_equal(bb, g["bbox"])
    keys = O.morton_keys(x, y, bb, z=z)
    assert np.array_equal(keys, g["keys"])
    perm = O.sort_perm(keys)
    assert np.array_equal(perm, g["perm"])
    xs, ys, ms = x[perm], y[perm], m[perm]
    zs = None if z is None else z[perm]
    for tag, lc, order in (("t4", 4, True), ("tc", leaf_cap, True), ("tu", 4, False)):
        if order:
            t = O.build_tree(xs, ys, ms, bb, z=zs, leaf_cap=lc)
        else:
            t = O.build_tree(x, y, m, bb, z=z, leaf_cap=lc)
        for a in TREE_KEYS:
            assert np.array_equal(getattr(t, a), g[f"{tag}_{a}"]), (tag, a)
    h = O.build_tree(xs, ys, ms, bb, z=zs, leaf_cap=leaf_cap, holder=True)
    prm = O.make_params(dims=dims, theta=float(theta), eps2=float(eps2), leaf_cap=leaf_cap,
                        dt=float(dt))
    acc = O.walk(xs, ys, ms, h, prm, z=zs, nthreads=2, want_counts=True)
    assert np.array_equal(acc[0], g["walk_ax"]) and np.array_equal(acc[1], g["walk_ay"])
    if dims == 3:
        assert np.array_equal(acc[2], g["walk_az"])
    assert np.array_equal(acc[-1], g["walk_inter"])
    fr = {k[3:]: np.array(v, copy=True) for k, v in g.items() if k.startswith("in_")}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        fr[k] = np.zeros(len(x), np.float32)
    O.frame(prm, fr, walk_kind=0, nthreads=2)
    for k, v in fr.items():
        assert np.array_equal(v, g[f"frame_{k}"]), k


def test_golden_fixtures_were_pinned_against_reference():
    # the fixtures were generated with the compiled reference sources present
    for path in CASES:
        assert _load(path)["meta"][5] == 1.0, path


def _ref_or_skip(O, fma=False):
    R = O.ref_lib(fma=fma)
    if R is None:
        pytest.skip("oracle/_ref not built (reference checkout absent when the oracle was built)")
    return R


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_reference_sources_random(O, ics, seed):
    """Keys and topology bit-exact with the reference's own code, on sorted
    and on unsorted particle orders (non-partitioned binary searches)."""
    R = _ref_or_skip(O)
    st = ics.disk2d(4000, seed=seed)
    x, y, m = st["x"], st["y"], st["m"]
    bb = O.bbox(x, y)
    k = O.morton_keys(x, y, bb)
    assert np.array_equal(k, O.ref_keys(R, x, y, bb))
    p = O.sort_perm(k)
    for xx, yy, mm in ((x[p], y[p], m[p]), (x, y, m)):
        t = O.build_tree(xx, yy, mm, bb)
        tr = O.ref_build_tree(R, xx, yy, mm, bb)
        for a in TREE_KEYS:
            assert np.array_equal(getattr(t, a), getattr(tr, a)), a
    st3 = ics.plummer3d(3000, seed=seed)
    x, y, z, m = st3["x"], st3["y"], st3["z"], st3["m"]
    bb = O.bbox(x, y, z)
    k = O.morton_keys(x, y, bb, z=z)
    assert np.array_equal(k, O.ref_keys(R, x, y, bb, z=z))
    p = O.sort_perm(k)
    t = O.build_tree(x[p], y[p], m[p], bb, z=z[p])
    tr = O.ref_build_tree(R, x[p], y[p], m[p], bb, z=z[p])
    for a in TREE_KEYS:
        assert np.array_equal(getattr(t, a), getattr(tr, a)), a


def test_reference_shipped_flags_change_only_com_rounding(O, ics):
    """The reference built with its shipped flags (gnu++20, -mfma, default
    FMA contraction) makes the same topology as the strict oracle; FMA
    contraction moves centres of mass by a few ulp at most."""
    R = _ref_or_skip(O, fma=True)
    st = ics.two_disks2d(20000, seed=4)
    x, y, m = st["x"], st["y"], st["m"]
    bb = O.bbox(x, y)
    k = O.morton_keys(x, y, bb)
    assert np.array_equal(k, O.ref_keys(R, x, y, bb))
    p = O.sort_perm(k)
    t = O.build_tree(x[p], y[p], m[p], bb)
    tr = O.ref_build_tree(R, x[p], y[p], m[p], bb)
    for a in ["pos", "size", "start", "end", "next", "child", "mass"]:
        assert np.array_equal(getattr(t, a), getattr(tr, a)), a
    # measured against the extent of the root box (components near 0 have no
    # meaningful relative error)
    assert (np.abs(t.com - tr.com) / bb[2]).max() < 1e-6


def test_reference_sort_is_a_key_sort(O, ics):
    """The reference's std::sort order differs from the canonical stable
    order only among equal keys."""
    R = _ref_or_skip(O)
    st = ics.disk2d(5000, seed=5)
    bb = O.bbox(st["x"], st["y"])
    k = O.morton_keys(st["x"], st["y"], bb)
    k[:50] = k[50:100]          # force ties
    order = np.zeros(len(k), np.uint32)
    R.ref_sort2d(len(k), k, order)
    assert np.array_equal(k[order], k[O.sort_perm(k)])


def test_fp64_direct_sum_matches_walk_at_theta_zero(O, ics):
    """theta = 0 opens every node: the walk is a direct sum, close to FP64."""
    st = ics.disk2d(1500, seed=6)
    x, y, m = st["x"], st["y"], st["m"]
    bb = O.bbox(x, y)
    p = O.sort_perm(O.morton_keys(x, y, bb))
    xs, ys, ms = x[p], y[p], m[p]
    h = O.build_tree(xs, ys, ms, bb, leaf_cap=1, holder=True)
    prm = O.make_params(theta=0.0, eps2=1e-4, leaf_cap=1)
    ax, ay = O.walk(xs, ys, ms, h, prm, nthreads=2)
    idx = np.arange(len(xs))
    dx, dy = O.direct_f64(xs, ys, ms, 1.0, 1e-4, idx, nthreads=2)
    err = np.hypot(ax - dx, ay - dy) / np.hypot(dx, dy)
    assert np.median(err) < 1e-6 and err.max() < 1e-3
