"""GPU parity beyond the golden fixtures: the FP64 accuracy reference against
the CPU FP64 oracle, the periodic tree walk, the theta sweep of the 1M
two-disk workload and the 3D Plummer walk at 1M particles.

Tolerances:
  * ge_direct_sum_f64 (the FP64 direct sum every accuracy figure is stated
    against) vs the oracle's FP64 direct sum: |a_gpu - a_cpu| <= 1e-12 of
    sum_j |G m_j d_ij / r_ij^3| (the sum's own scale; the relative error
    against |a| is reported too and is <= 1e-12 away from cancellation);
  * GE_PREC_EXACT: bit-exact against the strict oracle;
  * GE_PREC_FAST: per-particle relative error of the acceleration <= 1e-4
    against the strict oracle walk on the same state and tree.  Where a
    particle's force nearly cancels (cond = sum|F| / |sum F| large, e.g. a
    disk's central point mass) FAST's own rounding (rsqrt and FMA, about
    1e-7 per term) is amplified by cond, so the 1M sweep checks
    err <= max(1e-4, 5e-6 * cond) for every particle and the plain 1e-4 for
    at least 99.99 % of them.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-4
F64_TOL = 1e-12
NT = os.cpu_count() or 8


def _rel_err(out, ref, dims):
    num = sum((out[a] - ref[a]).astype(np.float64) ** 2 for a in range(dims))
    den = sum(ref[a].astype(np.float64) ** 2 for a in range(dims))
    return np.sqrt(num / np.maximum(den, 1e-300))


def _abs_term_sum(pos, m, tgt, G, eps2):
    """sum_j |G m_j d_ij| / (|d_ij|^2 + eps2)^(3/2), j != i, in FP64."""
    P = pos.astype(np.float64)
    M = m.astype(np.float64)
    out = np.zeros(len(tgt))
    for c0 in range(0, len(tgt), 64):
        t = tgt[c0:c0 + 64]
        d = P[None, :, :] - P[t][:, None, :]
        d2 = (d * d).sum(-1)
        r2 = d2 + eps2
        term = G * M[None, :] * np.sqrt(d2) / (r2 * np.sqrt(r2))
        term[np.arange(len(t)), t] = 0.0
        out[c0:c0 + 64] = term.sum(-1)
    return out


def _check_f64(gpu, cpu, scale, dims):
    diff = np.sqrt(sum((gpu[a] - cpu[a]) ** 2 for a in range(dims)))
    mag = np.sqrt(sum(cpu[a] ** 2 for a in range(dims)))
    assert np.all(diff <= F64_TOL * scale), (diff / scale).max()
    rel = diff / mag
    # away from cancellation (|a| at least 1 % of the terms' scale) the plain
    # relative error meets the same bound
    big = mag >= 0.01 * scale
    assert big.sum() > len(mag) // 2
    assert np.all(rel[big] <= F64_TOL), rel[big].max()


@pytest.mark.parametrize("dims", [2, 3])
def test_fp64_direct_sum_matches_cpu_fp64(ge, ics, O, dims):
    n = 65536
    st = ics.disk2d(n, seed=11) if dims == 2 else ics.plummer3d(n, seed=11)
    eps2 = 1e-4 if dims == 2 else 0.01
    p = ge.default_params(dims, G=1.0, theta=0.7, eps2=eps2, dt=1e-3)
    rng = np.random.default_rng(3)
    idx = np.sort(rng.choice(n, 1024, replace=False)).astype(np.uint32)
    with ge.Simulation(p) as s:
        s.upload(st)
        gpu = s.direct_sum_f64(idx)
    z = st.get("z")
    e2 = float(np.float32(eps2))   # the context holds eps2 as a float
    cpu = O.direct_f64(st["x"], st["y"], st["m"], 1.0, e2, idx.astype(np.int64), z=z,
                       nthreads=NT)
    pos = np.stack([st["x"], st["y"]] + ([z] if dims == 3 else []), axis=1)
    scale = _abs_term_sum(pos, st["m"], idx.astype(np.int64), 1.0, e2)
    _check_f64(gpu, cpu, scale, dims)


def test_fp64_direct_sum_in_a_batch_sums_each_sim_alone(ge, ics, O):
    """Targets of a batched context sum over their own simulation only."""
    sizes = [3000, 20000, 45000]
    sims = [ics.disk2d(n, seed=20 + k, center=(2.0 * k, -1.0 * k)) for k, n in enumerate(sizes)]
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3)
    rng = np.random.default_rng(4)
    with ge.Simulation(p) as b:
        handles = [b.add_sim(st) for st in sims]
        offs = [b.query(h)[1] for h in handles]
        idx = np.concatenate([off + np.sort(rng.choice(n, 400, replace=False))
                              for off, n in zip(offs, sizes)]).astype(np.uint32)
        gpu = b.direct_sum_f64(idx)
    k0 = 0
    for st, off, n in zip(sims, offs, sizes):
        loc = idx[k0:k0 + 400].astype(np.int64) - off
        e2 = float(np.float32(1e-4))   # the context holds eps2 as a float
        cpu = O.direct_f64(st["x"], st["y"], st["m"], 1.0, e2, loc, nthreads=NT)
        pos = np.stack([st["x"], st["y"]], axis=1)
        scale = _abs_term_sum(pos, st["m"], loc, 1.0, e2)
        _check_f64([g[k0:k0 + 400] for g in gpu], cpu, scale, 2)
        k0 += 400


def _periodic_case(ics, dims):
    """A system that straddles the domain's boundary, so the first drift
    wraps particles back in and the walk wraps the pairs farther apart than
    half the domain."""
    if dims == 2:
        # domain [0, 12) (physics.cpp:1104-1110): a disk of radius 5 centred at
        # x = 2, so its left part starts outside and is wrapped to the right
        st = ics.disk2d(6000, seed=12, center=(2.0, 6.0))
        return st, (12.0, 12.0, 0.0), 1e-4
    # domain [-3, 3)^3 (physics3D.cpp:785-802): a Plummer sphere cut to a
    # cube of half-side 2.9 and moved by +2 in x, so its far side is outside
    st = ics.plummer3d(12000, seed=12)
    keep = (np.abs(st["x"]) < 2.9) & (np.abs(st["y"]) < 2.9) & (np.abs(st["z"]) < 2.9)
    st = {k: np.ascontiguousarray(v[keep]) for k, v in st.items()}
    st["x"] = st["x"] + np.float32(2.0)
    st["id"] = np.arange(len(st["x"]), dtype=np.uint32)
    return st, (6.0, 6.0, 6.0), 0.01


def _oracle_frames(O, prm, st, steps):
    fr = {k: np.array(v, copy=True) for k, v in st.items()}
    for k in ("ax", "ay") + (("az",) if prm.dims == 3 else ()):
        fr[k] = np.zeros(len(fr["x"]), np.float32)
    for _ in range(steps):
        O.frame(prm, fr, walk_kind=0, nthreads=NT)
    return fr


@pytest.mark.parametrize("dims", [2, 3])
def test_periodic_tree_walk_matches_oracle(ge, ics, O, dims):
    """Periodic wrap in the walk (physics.cpp:118-121; physics3D.cpp's walk)
    and in the drift (physics.cpp:1104-1110; physics3D.cpp:785-802): three
    frames bit-exact in GE_PREC_EXACT; one frame within 1e-4 in FAST (the
    first frame's positions do not depend on the force arithmetic)."""
    st, domain, eps2 = _periodic_case(ics, dims)
    kw = dict(G=1.0, theta=0.7, eps2=eps2, leaf_cap=4, dt=2e-2, periodic=1, domain=domain)
    prm = O.make_params(dims=dims, G=1.0, theta=0.7, eps2=eps2, dt=2e-2, leaf_cap=4,
                        periodic=True, domain=domain)
    keys = ("x", "y", "vx", "vy", "ax", "ay", "id") + (("z", "vz", "az") if dims == 3 else ())
    ref3 = _oracle_frames(O, prm, st, 3)
    with ge.Simulation(ge.default_params(dims, precision=ge.PREC_EXACT, **kw)) as s:
        s.upload(st)
        s.count_interactions(True)
        s.step(3)
        out = s.download()
    for k in keys:
        assert np.array_equal(out[k], ref3[k]), k
    # the wrap was exercised: particles started outside the domain and are
    # inside it now, and some pairs are farther apart than half the domain
    lo = 0.0 if dims == 2 else -0.5 * domain[0]
    assert np.any(st["x"] < lo) or np.any(st["x"] >= lo + domain[0])
    assert np.all(out["x"] >= lo) and np.all(out["x"] < lo + domain[0])
    assert out["x"].max() - out["x"].min() > 0.5 * domain[0]
    ref1 = _oracle_frames(O, prm, st, 1)
    with ge.Simulation(ge.default_params(dims, precision=ge.PREC_FAST, **kw)) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
    assert np.array_equal(out["id"], ref1["id"])
    for k in ("x", "y") + (("z",) if dims == 3 else ()):
        assert np.array_equal(out[k], ref1[k]), k
    ax = ("ax", "ay", "az")[:dims]
    err = _rel_err([out[a] for a in ax], [ref1[a] for a in ax], dims)
    assert err.max() <= FAST_TOL, err.max()


@pytest.mark.parametrize("theta", [0.5, 1.0])
def test_two_disks_1m_theta_sweep(ge, ics, O, theta):
    """The 1M two-disk workload at the sweep's other opening angles (0.7 is in
    test_gpu_parity.py): tree bit-exact with the oracle's build of the same
    sorted state, FAST accelerations within 1e-4 of the oracle walk, and the
    same interaction count as the oracle."""
    st = ics.two_disks2d(1 << 20, seed=0)
    eps2 = 0.005 ** 2
    p = ge.default_params(2, G=1.0, theta=theta, eps2=eps2, leaf_cap=4, dt=1e-3,
                          precision=ge.PREC_FAST)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
        t = s.export_tree()
        bb = s.bounding_box()   # after the export: it reseeds the root nodes
        s.count_interactions(True)
        s.build_tree()
        s.calculate_force_from_grid()
        inter = s.stats().interactions
    x, y, m = out["x"], out["y"], out["m"]
    h = O.build_tree(x, y, m, bb, leaf_cap=4, holder=True)
    tr = h.to_numpy()
    for a in ("pos", "size", "com", "mass", "start", "end", "next", "child"):
        assert np.array_equal(t[a], getattr(tr, a)), a
    prm = O.make_params(dims=2, theta=theta, eps2=eps2, leaf_cap=4, dt=1e-3)
    ax, ay, cnt, cond = O.walk(x, y, m, h, prm, nthreads=NT, want_counts=True, want_cond=True)
    err = _rel_err([out["ax"], out["ay"]], [ax, ay], 2)
    bound = np.maximum(FAST_TOL, 5e-6 * cond.astype(np.float64))
    assert np.all(err <= bound), (err / bound).max()
    assert np.mean(err <= FAST_TOL) >= 0.9999, np.mean(err <= FAST_TOL)
    assert inter == int(cnt.astype(np.int64).sum())


def test_two_disks_1m_evolved_tree_and_walk(ge, ics, O):
    """The 1M two-disk workload after 1,000 steps (theta 0.7): particles flung
    out by the central masses make the box ~20x the disks, so long runs of
    equal keys, about 17,000 exact-rebuild roots, roots larger than one warp
    marks, chains of single-child nodes down to the minimum cell size and
    handed-over block rebuilds all occur.  The tree of the next step is
    bit-exact with the oracle's build of the same sorted state; FAST
    accelerations within the conditioning-aware tolerance of the oracle
    walk, with its interaction count."""
    st = ics.two_disks2d(1 << 20, seed=0)
    eps2 = 0.005 ** 2
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=eps2, leaf_cap=4, dt=1e-3,
                          precision=ge.PREC_FAST)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1000)
        s.count_interactions(True)
        s.step(1)
        inter = s.stats().interactions
        out = s.download()
        t = s.export_tree()
        bb = s.bounding_box()   # after the export: it reseeds the root nodes
    assert bb[2] > 100.0   # the evolved box (it starts near 20)
    x, y, m = out["x"], out["y"], out["m"]
    h = O.build_tree(x, y, m, bb, leaf_cap=4, holder=True)
    tr = h.to_numpy()
    for a in ("pos", "size", "com", "mass", "start", "end", "next", "child"):
        assert np.array_equal(t[a], getattr(tr, a)), a
    prm = O.make_params(dims=2, theta=0.7, eps2=eps2, leaf_cap=4, dt=1e-3)
    ax, ay, cnt, cond = O.walk(x, y, m, h, prm, nthreads=NT, want_counts=True, want_cond=True)
    err = _rel_err([out["ax"], out["ay"]], [ax, ay], 2)
    bound = np.maximum(FAST_TOL, 5e-6 * cond.astype(np.float64))
    assert np.all(err <= bound), (err / bound).max()
    assert np.mean(err <= FAST_TOL) >= 0.9999, np.mean(err <= FAST_TOL)
    assert inter == int(cnt.astype(np.int64).sum())


def test_plummer_3d_1m_fast(ge, ics, O):
    """3D Plummer sphere of 1,048,576 particles, theta 0.5, softening 0.01
    (added un-squared, physics3D.cpp:166): octree bit-exact with the
    oracle's, FAST accelerations within 1e-4 of the oracle's 3D walk."""
    n = 1 << 20
    st = ics.plummer3d(n, seed=1)
    p = ge.default_params(3, G=1.0, theta=0.5, eps2=0.01, leaf_cap=4, dt=5e-4,
                          precision=ge.PREC_FAST)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
        t = s.export_tree()
        bb = s.bounding_box()   # after the export: it reseeds the root nodes
    x, y, z, m = out["x"], out["y"], out["z"], out["m"]
    h = O.build_tree(x, y, m, bb, z=z, leaf_cap=4, holder=True)
    tr = h.to_numpy()
    for a in ("pos", "size", "com", "mass", "start", "end", "next", "child"):
        assert np.array_equal(t[a], getattr(tr, a)), a
    prm = O.make_params(dims=3, theta=0.5, eps2=0.01, leaf_cap=4, dt=5e-4)
    ax, ay, az = O.walk(x, y, m, h, prm, z=z, nthreads=NT)
    err = _rel_err([out["ax"], out["ay"], out["az"]], [ax, ay, az], 3)
    assert err.max() <= FAST_TOL, err.max()
