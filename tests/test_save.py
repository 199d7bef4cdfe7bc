"""Scene files: the reader of the reference's save format (ge_save_read).

The files are written here member by member in the order and with the types
of SaveSystem::saveSystem (src/UX/saveSystem.cpp:300-360 in 2D, :364-410 in
3D; member types from include/Particles/particle.h), every member filled
with distinct random bytes so a wrong offset shows.  The reader must return
the gravity step's members exactly.  The GPU test steps a loaded scene
(pin flags and temperatures included) and compares with the oracle frame.
"""
import os

import numpy as np
import pytest

SEP = b"\n---PARTICLE BINARY DATA---\n"


def record_dtype(dims):
    v = ("<f4", (dims,))
    return np.dtype([
        ("pos",) + v, ("predPos",) + v, ("vel",) + v, ("prevVel",) + v, ("predVel",) + v,
        ("acc",) + v, ("mass", "<f4"), ("press", "<f4"), ("pressTmp", "<f4"), ("pressF",) + v,
        ("dens", "<f4"), ("predDens", "<f4"), ("sphMass", "<f4"), ("restDens", "<f4"),
        ("stiff", "<f4"), ("visc", "<f4"), ("cohesion", "<f4"), ("temp", "<f4"), ("ke", "<f4"),
        ("prevKe", "<f4"), ("mortonKey", "<u8"), ("id", "<u4"), ("isHotPoint", "u1"),
        ("hasSolidified", "u1"), ("color", "u1", (4,)), ("pColor", "u1", (4,)),
        ("sColor", "u1", (4,)), ("sphColor", "u1", (4,)), ("size", "<f4"),
        ("uniqueColor", "u1"), ("isSolid", "u1"), ("canBeSubdivided", "u1"),
        ("canBeResized", "u1"), ("isDarkMatter", "u1"), ("isSPH", "u1"), ("isSelected", "u1"),
        ("isGrabbed", "u1"), ("previousSize", "<f4"), ("neighbors", "<i4"),
        ("totalRadius", "<f4"), ("lifeSpan", "<f4"), ("sphLabel", "<u4"), ("isPinned", "u1"),
        ("isBeingDrawn", "u1"), ("spawnCorrectIter", "<i4"), ("turbulence", "<f4"),
    ])


def write_save(path, rec, dims, version=190, yaml_extra=""):
    yaml = (f"G: 6.674e-11\nis3DMode: {'true' if dims == 3 else 'false'}\n"
            f"theta: 0.8\n{yaml_extra}")
    with open(path, "wb") as f:
        f.write(yaml.encode())
        f.write(SEP)
        f.write(np.array([version, 7, 3, 2, len(rec)], "<u4").tobytes())
        f.write(rec.tobytes())
        f.write(np.array([0], "<u4").tobytes())   # constraints follow; the reader stops before


def random_records(dims, n, seed):
    dt = record_dtype(dims)
    rng = np.random.default_rng(seed)
    raw = rng.integers(0, 256, n * dt.itemsize, dtype=np.uint8)
    rec = raw.view(dt).copy()
    rec["pos"] = rng.uniform(-5, 5, (n, dims))
    rec["vel"] = rng.normal(0, 0.3, (n, dims))
    rec["acc"] = rng.normal(0, 1.0, (n, dims))
    rec["mass"] = rng.uniform(1e-5, 1e-3, n)
    rec["temp"] = rng.uniform(100, 4000, n)
    rec["id"] = rng.permutation(n).astype(np.uint32) + 1000
    rec["isPinned"] = (rng.random(n) < 0.05).astype(np.uint8)
    return rec


def test_record_sizes():
    assert record_dtype(2).itemsize == 180
    assert record_dtype(3).itemsize == 208


@pytest.mark.parametrize("dims,version", [(2, 190), (3, 190), (2, 180), (3, 180)])
def test_reader_returns_the_members(ge, tmp_path, dims, version):
    rec = random_records(dims, 1234, seed=dims + version)
    path = str(tmp_path / "scene.bin")
    write_save(path, rec, dims, version)
    got = ge.load_save(path)
    assert got["dims"] == dims
    names = "xyz"
    for a in range(dims):
        assert np.array_equal(got[names[a]], rec["pos"][:, a])
        assert np.array_equal(got["v" + names[a]], rec["vel"][:, a])
        assert np.array_equal(got["a" + names[a]], rec["acc"][:, a])
    for k, src in (("m", "mass"), ("temp", "temp"), ("id", "id")):
        assert np.array_equal(got[k], rec[src]), k
    assert np.array_equal(got["pinned"], (rec["isPinned"] != 0).astype(np.uint8))


def test_reader_refuses_bad_files(ge, tmp_path):
    rec = random_records(2, 100, seed=1)
    p1 = str(tmp_path / "old.bin")
    write_save(p1, rec, 2, version=170)
    with pytest.raises(ge.GeError) as ei:
        ge.load_save(p1)
    assert ei.value.code == 8
    p2 = str(tmp_path / "cut.bin")
    write_save(p2, rec, 2)
    data = open(p2, "rb").read()
    open(p2, "wb").write(data[: len(data) - 500])
    with pytest.raises(ge.GeError) as ei:
        ge.load_save(p2)
    assert ei.value.code == 1
    p3 = str(tmp_path / "nosep.bin")
    open(p3, "wb").write(b"theta: 0.8\nno binary part\n")
    with pytest.raises(ge.GeError) as ei:
        ge.load_save(p3)
    assert ei.value.code == 1
    with pytest.raises(ge.GeError):
        ge.load_save(str(tmp_path / "missing.bin"))


@pytest.mark.gpu
def test_loaded_scene_steps_like_the_oracle(ge, ics, O, tmp_path):
    """A scene read from a file (pin flags and temperatures included) steps on
    the GPU exactly as the oracle frame steps the same arrays."""
    st = ics.disk2d(4000, seed=9)
    n = len(st["x"])
    rec = random_records(2, n, seed=4)
    rec["pos"] = np.stack([st["x"], st["y"]], 1)
    rec["vel"] = np.stack([st["vx"], st["vy"]], 1)
    rec["acc"] = 0.0
    rec["mass"] = st["m"]
    rec["id"] = np.arange(n, dtype=np.uint32)
    path = str(tmp_path / "disk.bin")
    write_save(path, rec, 2)
    sc = ge.load_save(path)
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, precision=ge.PREC_EXACT,
                          temp_enabled=1)
    with ge.Simulation(p) as s:
        s.upload({k: sc[k] for k in ("x", "y", "vx", "vy", "m", "id", "ax", "ay")})
        s.upload_pinned(sc["pinned"])
        s.upload_temp(sc["temp"])
        s.step(2)
        out = s.download()
        out["temp"] = s.download_temp()
    fr = {k: np.array(sc[k], copy=True) for k in ("x", "y", "vx", "vy", "ax", "ay", "m", "id",
                                                  "temp", "pinned")}
    op = O.make_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, leaf_cap=4, temp_enabled=True)
    for _ in range(2):
        O.frame(op, fr, walk_kind=0)
    assert np.any(sc["pinned"])
    for k in ("x", "y", "vx", "vy", "ax", "ay", "id", "temp"):
        assert np.array_equal(out[k], fr[k]), k


# --- fixtures written through the reference's own particle types ----------
# tests/golden/save{2d,3d}_ref.bin come from oracle/ref_save_fixture.cpp,
# compiled against the reference's include/Particles/particle.h (make -C
# oracle save-fixture REF=<checkout>/GalaxyEngine), 300 particles each, with
# the member values below.

def _ref_fixture_values(dims, n=300):
    i = np.arange(n)
    f = np.float32
    pos = [(i % 37) * f(0.25) - f(4), (i // 37) * f(0.5) - f(2), (i % 11) * f(0.125) - f(0.5)]
    vel = [(i % 5) * f(0.125) - f(0.25), (i % 7) * f(0.0625) - f(0.1875), (i % 3) * f(0.25) - f(0.25)]
    acc = [((i % 3) - f(1)) * f(0.5), ((i % 4) - f(2)) * f(0.5), ((i % 5) - f(2)) * f(0.5)]
    out = {}
    for a, c in enumerate("xyz"[:dims]):
        out[c] = pos[a].astype(np.float32)
        out["v" + c] = vel[a].astype(np.float32)
        out["a" + c] = acc[a].astype(np.float32)
    out["m"] = (1 + i % 9).astype(np.float32)
    out["temp"] = (100 + i).astype(np.float32)
    out["id"] = (1000 + i).astype(np.uint32)
    out["pinned"] = (i % 13 == 0).astype(np.uint8)
    return out


@pytest.mark.parametrize("dims", [2, 3])
def test_reader_on_files_written_with_the_reference_types(ge, dims):
    from conftest import GOLDEN
    path = os.path.join(GOLDEN, f"save{dims}d_ref.bin")
    got = ge.load_save(path)
    assert got["dims"] == dims
    want = _ref_fixture_values(dims)
    for k, v in want.items():
        assert np.array_equal(got[k], v), k


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [2, 3])
def test_reference_typed_scene_steps_like_the_oracle(ge, O, dims):
    """The reference-typed fixture, loaded and stepped three frames in
    GE_PREC_EXACT, equals the oracle frame loop on the same arrays."""
    from conftest import GOLDEN
    sc = ge.load_save(os.path.join(GOLDEN, f"save{dims}d_ref.bin"))
    keys = ["x", "y", "vx", "vy", "ax", "ay", "m", "id"] + (["z", "vz", "az"] if dims == 3 else [])
    eps2 = 0.01
    p = ge.default_params(dims, G=1e-3, theta=0.7, eps2=eps2, dt=1e-2, precision=ge.PREC_EXACT)
    with ge.Simulation(p) as s:
        s.upload({k: sc[k] for k in keys})
        s.upload_pinned(sc["pinned"])
        s.step(3)
        out = s.download()
    fr = {k: np.array(sc[k], copy=True) for k in keys + ["pinned"]}
    op = O.make_params(dims, G=1e-3, theta=0.7, eps2=eps2, dt=1e-2, leaf_cap=4)
    for _ in range(3):
        O.frame(op, fr, walk_kind=0)
    for k in keys:
        assert np.array_equal(out[k], fr[k]), k
