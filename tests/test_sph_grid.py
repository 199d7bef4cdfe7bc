"""The SPH neighbour grid (SPH::newGridGPU, GalaxyEngine/include/Physics/SPH.h:533-590).

The reference hashes every particle's cell, sorts the entries by key with a
bitonic network of GL compute dispatches and records each key's first entry.
The oracle restates those shaders, the network included.  The device sorts
with a stable radix sort: the sorted keys and the offsets must be identical
to the oracle's, and every key must hold the same entries (particle and
cell), in increasing particle order on the device.
"""
import numpy as np
import pytest


def _scatter(n, seed, spread=60.0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-spread, spread, n).astype(np.float32)
    y = rng.uniform(-spread, spread, n).astype(np.float32)
    # particles exactly on cell boundaries and coincident ones
    k = min(n, 64)
    x[:k] = (np.arange(k) - 32).astype(np.float32) * np.float32(3.0)
    y[:k] = np.float32(-6.0)
    if n > 100:
        x[70:80] = x[69]
        y[70:80] = y[69]
    return x, y


def _by_entry(g):
    order = np.lexsort((g["index"], g["keys"]))
    return {k: g[k][order] for k in ("keys", "index", "cell_x", "cell_y")}


def test_oracle_grid_is_sorted_and_complete(O):
    """CPU: the restated network sorts, keeps every entry, and its keys and
    cells are the shader's (checked against an independent numpy statement
    of the hash with wrapping 32-bit products)."""
    for n, table in ((1, 16384), (1000, 16384), (4097, 257), (3000, 1)):
        x, y = _scatter(n, seed=n)
        g = O.sph_grid(x, y, 3.0, table)
        assert np.all(np.diff(g["keys"].astype(np.int64)) >= 0)
        assert np.array_equal(np.sort(g["index"]), np.arange(n, dtype=np.uint32))
        cx = np.floor(x / np.float32(3.0)).astype(np.int64).astype(np.int32)
        cy = np.floor(y / np.float32(3.0)).astype(np.int64).astype(np.int32)
        h = ((cx.astype(np.uint32) * np.uint32(73856093)) ^
             (cy.astype(np.uint32) * np.uint32(19349663))) % np.uint32(table)
        i = g["index"]
        assert np.array_equal(g["keys"], h[i])
        assert np.array_equal(g["cell_x"], cx[i]) and np.array_equal(g["cell_y"], cy[i])
        ofs = g["offsets"]
        for key in np.unique(g["keys"]):
            first = int(np.argmax(g["keys"] == key))
            assert ofs[key] == first
        assert np.sum(ofs != 0xFFFFFFFF) == len(np.unique(g["keys"]))


@pytest.mark.gpu
@pytest.mark.parametrize("n,table,cell", [(1, 16384, 3.0), (5000, 16384, 3.0),
                                          (70001, 16384, 3.0), (20000, 256, 3.0),
                                          (20000, 257, 0.7), (100000, 1 << 20, 0.25),
                                          (4096, 1, 3.0)])
def test_sph_grid_matches_oracle(ge, O, n, table, cell):
    x, y = _scatter(n, seed=n + table)
    st = {"x": x, "y": y, "vx": np.zeros(n, np.float32), "vy": np.zeros(n, np.float32),
          "m": np.full(n, 1.0 / n, np.float32)}
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3)
    with ge.Simulation(p) as s:
        s.upload(st)
        s.step(1)                       # particles move into Morton order
        out = s.download()
        g = s.sph_grid(cell, table)
    ref = O.sph_grid(out["x"], out["y"], cell, table)
    assert np.array_equal(g["keys"], ref["keys"])
    assert np.array_equal(g["offsets"], ref["offsets"])
    a, b = _by_entry(g), _by_entry(ref)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # stable: a key's particles in increasing order
    same = g["keys"][1:] == g["keys"][:-1]
    assert np.all(g["index"][1:][same] > g["index"][:-1][same])


@pytest.mark.gpu
def test_sph_grid_of_one_simulation_in_a_batch(ge, O, ics):
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3)
    sts = [ics.disk2d(n, seed=50 + k, center=(7.0 * k, 0.0)) for k, n in
           enumerate([3000, 12000, 500])]
    with ge.Simulation(p) as b:
        hs = [b.add_sim(s) for s in sts]
        b.step(1)
        got = b.sph_grid(0.05, 16384, sim=hs[1])
        mine = b.download_sim(hs[1])
    ref = O.sph_grid(mine["x"], mine["y"], 0.05, 16384)
    assert np.array_equal(got["keys"], ref["keys"])
    assert np.array_equal(got["offsets"], ref["offsets"])
    a, b2 = _by_entry(got), _by_entry(ref)
    for k in a:
        assert np.array_equal(a[k], b2[k]), k


@pytest.mark.gpu
def test_sph_grid_refusals(ge, ics):
    p = ge.default_params(3, G=1.0, theta=0.7, softening=0.01, dt=1e-3)
    with ge.Simulation(p) as s:
        s.upload(ics.plummer3d(1000, seed=1))
        with pytest.raises(ge.GeError) as ei:
            s.sph_grid()
        assert ei.value.code == 8
    p = ge.default_params(2, G=1.0, theta=0.7, softening=0.01, dt=1e-3)
    with ge.Simulation(p) as s:
        s.upload(ics.disk2d(1000, seed=1))
        for cell, table in ((0.0, 16384), (3.0, 0), (3.0, (1 << 24) + 1)):
            with pytest.raises(ge.GeError) as ei:
                s.sph_grid(cell, table)
            assert ei.value.code == 1
