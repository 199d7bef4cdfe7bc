"""Generate the golden fixtures under tests/golden/ (run from the repo root).

    python tests/golden/make_golden.py

For each case the oracle (oracle/ge_oracle.c) computes bounding box, Morton
keys, the stable key order, the trees (leaf capacity 4 = the reference's
constant, and the case's own capacity), the scalar tree-walk accelerations and
one full frame.  Where the reference's own sources were compiled
(oracle/_ref/libgeref.so, built from the reference checkout by
``make -C oracle ref``), keys and trees are also computed by the reference
code and must match the oracle bit for bit; the fixture records whether that
pin was made (``pinned``).  The fixtures are small (a few thousand particles)
so the CPU suite can recompute them in seconds.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

ics = importlib.import_module("galaxy-engine_b200.ics")
OUT = os.path.dirname(os.path.abspath(__file__))
TREE_KEYS = ["pos", "size", "com", "mass", "start", "end", "next", "child"]


def edge_cases_2d():
    """Hand-placed 2D inputs: coincident particles, points on dyadic midlines,
    a particle pair closer than the key resolution, extreme corners."""
    rng = np.random.default_rng(11)
    pts = []
    pts += [(0.0, 0.0)] * 6                      # coincident (min-size leaf)
    g = np.linspace(-4.0, 4.0, 9)                # on midlines of the root box
    pts += [(a, b) for a in g for b in g]
    pts += [(1.0e-5, 2.0e-5), (1.0e-5 + 3e-7, 2.0e-5)]   # below key resolution
    pts += [(-4.0, -4.0), (4.0, 4.0), (4.0, -4.0)]
    pts += list(map(tuple, rng.uniform(-4, 4, size=(300, 2))))
    p = np.array(pts, np.float32)
    n = len(p)
    return dict(x=p[:, 0].copy(), y=p[:, 1].copy(),
                vx=rng.normal(0, 0.1, n).astype(np.float32), vy=rng.normal(0, 0.1, n).astype(np.float32),
                m=rng.uniform(0.5, 1.5, n).astype(np.float32) / n, id=np.arange(n, dtype=np.uint32))


def make_case(name, st, dims, theta, eps2, leaf_cap, dt, Rl):
    x, y, m = st["x"], st["y"], st["m"]
    z = st.get("z")
    out = {f"in_{k}": v for k, v in st.items()}
    bb = O.bbox(x, y, z)
    keys = O.morton_keys(x, y, bb, z=z)
    perm = O.sort_perm(keys)
    xs, ys, ms = x[perm], y[perm], m[perm]
    zs = None if z is None else z[perm]
    t4 = O.build_tree(xs, ys, ms, bb, z=zs, leaf_cap=4)
    tc = O.build_tree(xs, ys, ms, bb, z=zs, leaf_cap=leaf_cap)
    # the same builder over the unsorted input order (non-partitioned ranges)
    tu = O.build_tree(x, y, m, bb, z=z, leaf_cap=4)
    pinned = False
    if Rl is not None:
        assert np.array_equal(keys, O.ref_keys(Rl, x, y, bb, z=z)), name
        for tt, xx, yy, zz, mm in ((t4, xs, ys, zs, ms), (tu, x, y, z, m)):
            tr = O.ref_build_tree(Rl, xx, yy, mm, bb, z=zz)
            for a in TREE_KEYS:
                assert np.array_equal(getattr(tt, a), getattr(tr, a)), (name, a)
        pinned = True
    h = O.build_tree(xs, ys, ms, bb, z=zs, leaf_cap=leaf_cap, holder=True)
    prm = O.make_params(dims=dims, theta=theta, eps2=eps2, leaf_cap=leaf_cap, dt=dt)
    acc = O.walk(xs, ys, ms, h, prm, z=zs, nthreads=4, want_counts=True)
    out.update(bbox=bb, keys=keys, perm=perm, walk_ax=acc[0], walk_ay=acc[1],
               walk_inter=acc[-1])
    if dims == 3:
        out["walk_az"] = acc[2]
    for tag, tt in (("t4", t4), ("tc", tc), ("tu", tu)):
        for a in TREE_KEYS:
            out[f"{tag}_{a}"] = getattr(tt, a)
    # one full frame from the input order
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if dims == 3 else ()):
        fr[k] = np.zeros(len(x), np.float32)
    O.frame(prm, fr, walk_kind=0, nthreads=4)
    for k, v in fr.items():
        out[f"frame_{k}"] = v
    out["meta"] = np.array([dims, theta, eps2, leaf_cap, dt, 1.0 if pinned else 0.0], np.float64)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    print(f"{name}: n={len(x)} nodes(leaf {leaf_cap})={tc.count} pinned={pinned}")


def main():
    Rl = O.ref_lib()
    if Rl is None:
        print("warning: oracle/_ref not built; fixtures are not pinned against the reference")
    make_case("disk2d_n2048", ics.disk2d(2048, seed=0), 2, 0.7, 1e-4, 1, 1e-3, Rl)
    make_case("disk2d_n3000_leaf4", ics.disk2d(3000, seed=3), 2, 0.5, 0.005 ** 2, 4, 1e-3, Rl)
    make_case("plummer3d_n2048", ics.plummer3d(2048, seed=0), 3, 0.5, 0.01, 4, 5e-4, Rl)
    make_case("edge2d", edge_cases_2d(), 2, 0.7, 1e-4, 1, 1e-3, Rl)


if __name__ == "__main__":
    main()
