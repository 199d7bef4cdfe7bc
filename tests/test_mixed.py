"""GPU: the mixed-precision mode (GE_PREC_MIXED).

The mode keeps the reference's tree and walk order and changes what a node
contributes (FP64 moments, double-float centre of mass, offset-corrected
opening test, softened quadrupole, Kahan sums).  Checks:
  * the device walk -- particle by particle (group_size 0) and in groups of
    32, 64 or 128 -- against the oracle's statement of the same algorithm
    (oracle/ge_oracle_mixed.c, FP64) on the same tree: the opening decisions
    are made from the same FP32 values on both sides (the group walk's
    interaction counts agree exactly), so only the FP32 evaluation of the
    accepted terms differs;
  * the accuracy bound against the FP64 direct sum (median <= 1e-3: 2D at
    theta 0.6 particle by particle and at theta 0.7 in groups of 32, 3D at
    theta 0.5);
  * the Kahan-compensated leapfrog: a drift below half an ulp per step still
    moves the particle;
  * a simulation's result alone and inside a batch is the same.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIXED = 2


def _sorted_forces(ge, p, st):
    with ge.Simulation(p) as s:
        s.upload(st)
        s.compute_morton_keys()
        s.sort_particles_by_morton_key()
        s.build_tree()
        s.calculate_force_from_grid()
        return s.download()


def _rel(a, b):
    num = sum((a[k] - b[k]) ** 2 for k in range(len(a)))
    den = sum(b[k] ** 2 for k in range(len(b)))
    return np.sqrt(num / np.maximum(den, 1e-300))


@pytest.mark.parametrize("dims,n,theta,eps2", [(2, 16384, 0.6, 1e-4), (2, 30000, 0.7, 1e-4),
                                               (3, 16384, 0.5, 0.01)])
def test_mixed_walk_matches_oracle(ge, ics, O, dims, n, theta, eps2):
    st = ics.disk2d(n, seed=3) if dims == 2 else ics.plummer3d(n, seed=3)
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=4, dt=1e-3,
                          precision=MIXED, group_size=0)
    out = _sorted_forces(ge, p, st)
    z = out.get("z")
    bb = O.bbox(out["x"], out["y"], z)
    tree = O.build_tree(out["x"], out["y"], out["m"], bb, z=z, leaf_cap=4, holder=True)
    op = O.make_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=4)
    ref = O.walk_mixed(out["x"], out["y"], out["m"], tree, op, z=z)
    got = [out["ax"], out["ay"]] + ([out["az"]] if dims == 3 else [])
    e = _rel(got, ref)
    print(f"mixed vs oracle: median {np.median(e):.2e} p99 {np.percentile(e, 99):.2e} "
          f"max {e.max():.2e}")
    assert np.median(e) <= 1e-6
    assert np.percentile(e, 99) <= 5e-6
    assert e.max() <= 1e-4


@pytest.mark.parametrize("dims,n,theta,eps2,gs", [(2, 16384, 0.6, 1e-4, 32),
                                                  (2, 30000, 0.7, 1e-4, 64),
                                                  (2, 20000, 0.7, 1e-4, 128),
                                                  (3, 16384, 0.5, 0.01, 32),
                                                  (3, 12000, 0.7, 0.01, 64),
                                                  (2, 30000, 0.2, 1e-2, 64)])
def test_group_walk_matches_oracle(ge, ics, O, dims, n, theta, eps2, gs):
    """The group walk against the oracle's statement of it: the same groups,
    the same opening decisions (FP32 on both sides, so the interaction counts
    agree exactly), the accepted terms evaluated in FP32 on the device and in
    FP64 by the oracle.  At theta 0.2 the work stacks grow past their shared
    memory (about 420 entries, 256 in shared memory in 2D) and move to global
    memory mid-walk."""
    st = ics.disk2d(n, seed=4) if dims == 2 else ics.plummer3d(n, seed=4)
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=4, dt=1e-3,
                          precision=MIXED, group_size=gs)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.compute_morton_keys()
        s.sort_particles_by_morton_key()
        s.build_tree()
        s.count_interactions(True)
        s.calculate_force_from_grid()
        inter = s.stats().interactions
        out = s.download()
    z = out.get("z")
    bb = O.bbox(out["x"], out["y"], z)
    tree = O.build_tree(out["x"], out["y"], out["m"], bb, z=z, leaf_cap=4, holder=True)
    op = O.make_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=4)
    ref = O.walk_group(out["x"], out["y"], out["m"], tree, op, group_size=gs, z=z,
                       want_counts=True)
    got = [out["ax"], out["ay"]] + ([out["az"]] if dims == 3 else [])
    e = _rel(got, ref[:-1])
    print(f"group walk vs oracle: median {np.median(e):.2e} p99 {np.percentile(e, 99):.2e} "
          f"max {e.max():.2e}; interactions {inter} vs {int(ref[-1].sum())}")
    assert inter == int(ref[-1].sum())
    assert np.median(e) <= 1e-6
    assert np.percentile(e, 99) <= 5e-6
    assert e.max() <= 1e-4


@pytest.mark.parametrize("dims,n,theta,eps2,gs", [(2, 1 << 18, 0.6, 0.005 ** 2, 0),
                                                  (2, 1 << 18, 0.7, 0.005 ** 2, 64),
                                                  (3, 1 << 17, 0.5, 0.01, 0),
                                                  (3, 1 << 17, 0.5, 0.01, 32)])
def test_mixed_accuracy_vs_fp64(ge, ics, dims, n, theta, eps2, gs):
    st = ics.two_disks2d(n, seed=5) if dims == 2 else ics.plummer3d(n, seed=5)
    res = {}
    for prec in (0, MIXED):
        p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, leaf_cap=4, dt=1e-3,
                              precision=prec, group_size=gs)
        with ge.Simulation(p) as s:
            s.upload(st)
            s.step(1)
            out = s.download()
            idx = np.sort(np.random.default_rng(1).choice(n, 4096, replace=False)).astype(np.uint32)
            ref = s.direct_sum_f64(idx)
        got = [out["ax"][idx], out["ay"][idx]] + ([out["az"][idx]] if dims == 3 else [])
        res[prec] = np.median(_rel(got, ref))
    print(f"median error vs FP64: fast {res[0]:.2e} mixed {res[MIXED]:.2e}")
    assert res[MIXED] <= 1e-3
    assert res[MIXED] < 0.2 * res[0]


def test_group_walk_deep_stacks_3d(ge, ics):
    """3D at theta 0.3 over 1M particles: the work stacks grow past the 1024
    entries kept in shared memory (about 1400) and move to global memory
    mid-walk; the result keeps the mode's accuracy against the FP64 direct sum."""
    n = 1 << 20
    st = ics.plummer3d(n, seed=0)
    p = ge.default_params(3, G=1.0, theta=0.3, eps2=0.01, leaf_cap=16, dt=1e-3,
                          precision=MIXED, group_size=32)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)
        out = s.download()
        idx = np.sort(np.random.default_rng(2).choice(n, 4096, replace=False)).astype(np.uint32)
        ref = s.direct_sum_f64(idx)
    got = [out["ax"][idx], out["ay"][idx], out["az"][idx]]
    e = _rel(got, ref)
    print(f"3D theta 0.3 group walk vs FP64: median {np.median(e):.2e} max {e.max():.2e}")
    assert np.median(e) <= 3e-4
    assert e.max() <= 1e-2


@pytest.mark.parametrize("dims", [2, 3])
def test_mixed_kahan_leapfrog(ge, dims):
    """One particle (no force) drifting 1e-8 per step from x = 1: each step is
    below half an ulp of 1.0, so the plain update never moves it; the
    compensated update moves it by the full 1000 * 1e-8 after 1000 steps."""
    st = {"x": np.array([1.0], np.float32), "y": np.array([1.0], np.float32),
          "vx": np.array([1e-5], np.float32), "vy": np.array([0.0], np.float32),
          "m": np.array([1.0], np.float32)}
    if dims == 3:
        st["z"] = np.array([1.0], np.float32)
        st["vz"] = np.array([-1e-5], np.float32)
    res = {}
    for prec in (0, MIXED):
        p = ge.default_params(dims, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, precision=prec)
        with ge.Simulation(p) as s:
            s.upload(st)
            s.step(1000)
            res[prec] = s.download()
    assert res[0]["x"][0] == np.float32(1.0)
    assert abs(float(res[MIXED]["x"][0]) - (1.0 + 1e-5)) <= 2e-7
    if dims == 3:
        assert abs(float(res[MIXED]["z"][0]) - (1.0 - 1e-5)) <= 2e-7


def test_mixed_batch_equals_alone(ge, ics):
    p = ge.default_params(2, G=1.0, theta=0.6, softening=0.01, dt=1e-3, precision=MIXED)
    sizes = [3000, 1, 17000, 4097]
    sts = [ics.disk2d(n, seed=20 + k, center=(2.0 * k, 0.0)) for k, n in enumerate(sizes)]
    with ge.Simulation(p) as b:
        h = [b.add_sim(s) for s in sts]
        b.step(3)
        for k, s in enumerate(sts):
            got = b.download_sim(h[k])
            with ge.Simulation(p) as a:
                a.upload(s)
                a.step(3)
                ref = a.download()
            for key in ("x", "y", "vx", "vy", "ax", "ay", "id"):
                assert np.array_equal(got[key], ref[key]), key


def test_autotune_picks_a_configuration_and_keeps_state(ge, ics):
    """The autotuner times all 12 (group size, leaf capacity) pairs, keeps the
    fastest, leaves positions and velocities alone, and leaves the
    accelerations of the chosen configuration in the state."""
    st = ics.disk2d(65536, seed=8)
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, precision=MIXED)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(2)
        before = s.download()
        gs, leaf, table = s.autotune(reps=1)
        after = s.download()
        assert gs in (32, 64, 128) and leaf in (1, 4, 8, 16)
        assert len(table) == 12 and all(v > 0 for v in table.values())
        assert table[(gs, leaf)] == min(table.values())
        ob, oa = np.argsort(before["id"]), np.argsort(after["id"])
        for k in ("x", "y", "vx", "vy", "m"):
            assert np.array_equal(before[k][ob], after[k][oa]), k
        s.step(1)   # the chosen configuration steps on
    q = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, precision=MIXED,
                          group_size=gs, leaf_cap=leaf)
    with ge.Simulation(q) as r:
        r.upload({k: after[k] for k in ("x", "y", "vx", "vy", "m", "id")})
        r.compute_morton_keys()
        r.sort_particles_by_morton_key()
        r.build_tree()
        r.calculate_force_from_grid()
        ref = r.download()
    orr = np.argsort(ref["id"])
    e = _rel([after["ax"][oa], after["ay"][oa]], [ref["ax"][orr], ref["ay"][orr]])
    assert np.max(e) <= 1e-5


def test_autotune_refused_outside_mixed(ge, ics):
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3, precision=0)
    with ge.Simulation(p) as s:
        s.upload(ics.disk2d(4096, seed=1))
        with pytest.raises(ge.GeError) as ei:
            s.autotune()
        assert ei.value.code == 5


@pytest.mark.parametrize("dims,n,theta,eps2", [(2, 12000, 0.7, 1e-4), (3, 8192, 0.5, 0.01)])
def test_energy_pass_against_direct_sum(ge, ics, O, dims, n, theta, eps2):
    """Potential energy from the group walk's potential pass against the FP64
    direct sum; kinetic energy against the FP64 sums of the state."""
    st = ics.disk2d(n, seed=6) if dims == 2 else ics.plummer3d(n, seed=6)
    p = ge.default_params(dims, G=1.0, theta=theta, eps2=eps2, dt=1e-3, precision=MIXED)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(2)
        kin, pot, tot = s.energy_f64()
        sums = s.sums_f64()
        out = s.download()
    ref = O.potential_f64(out["x"], out["y"], out["m"], 1.0, eps2, z=out.get("z"))
    assert abs(pot - ref) <= 2e-4 * abs(ref)
    # FP64 atomic sums: equal up to the order of their additions
    assert abs(kin - sums[0]) <= 1e-12 * abs(sums[0]) and tot == kin + pot
