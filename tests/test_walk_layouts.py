"""GPU: the two 2D walk layouts give bit-identical results.

2D builds write packed walk entries (a node's level and subtree successor in
the entry's fourth word, size^2 recomputed from the root size) when every
level and successor fits and every size^2 stays a normal float; otherwise the
build writes the plain layout (size^2 in the entry, the successor in a link
array).  Both must give the walk and the trajectory preview exactly the
reference's numbers (physics.cpp:91-205; particlesSpawning.cpp:443-500):

  * min_size = 1e-20 (below the packed layout's 1e-18 floor) forces the plain
    layout without changing the tree of a disk, whose nodes never get near
    the 1e-6 default: every output equals the packed run's bit for bit;
  * a simulation whose root size is 1e19 or more forces the plain layout for
    the whole context (its size^2 is too close to the float range); a normal
    simulation batched with it gives the same result as alone (packed).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "vx", "vy", "ax", "ay", "m", "id")


def _params(ge, **kw):
    return ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, leaf_cap=4, dt=1e-3,
                             precision=ge.PREC_EXACT, **kw)


def test_plain_layout_equals_packed(ge, ics):
    st = ics.disk2d(20000, seed=13)
    rng = np.random.default_rng(5)
    pos = rng.uniform(-3.0, 3.0, (16, 2)).astype(np.float32)
    vel = rng.normal(0.0, 0.3, (16, 2)).astype(np.float32)
    mass = rng.uniform(1e-3, 1.0, 16).astype(np.float32)
    res = []
    for min_size in (1e-6, 1e-20):
        with ge.Simulation(_params(ge, min_size=min_size)) as s:
            s.upload(st)
            s.count_interactions(True)
            s.step(3)
            out = s.download()
            out["inter"] = s.stats().interactions
            out["path"] = s.predict_trajectory(pos, vel, mass, 60, 1e-4)
            out["tree"] = s.export_tree()
        res.append(out)
    packed, plain = res
    for k in KEYS + ("path",):
        assert np.array_equal(packed[k], plain[k]), k
    assert packed["inter"] == plain["inter"] > 0
    for a in packed["tree"]:
        assert np.array_equal(packed["tree"][a], plain["tree"][a]), a


def test_big_root_forces_plain_layout_without_changing_results(ge, ics):
    normal = ics.disk2d(5000, seed=14)
    big = ics.disk2d(3000, seed=15)
    scale = np.float32(4e18)   # disk radius 5: a root box of about 4e19
    for k in ("x", "y"):
        big[k] = (big[k] * scale).astype(np.float32)
    with ge.Simulation(_params(ge)) as s:
        s.upload(normal)
        s.step(2)
        alone = s.download()
    with ge.Simulation(_params(ge)) as b:
        h0 = b.add_sim(normal)
        h1 = b.add_sim(big)
        b.step(2)
        mixed = b.download_sim(h0)
        far = b.download_sim(h1)
    for k in KEYS:
        assert np.array_equal(alone[k], mixed[k]), k
    assert np.all(np.isfinite(far["x"])) and np.all(np.isfinite(far["ax"]))
