"""The reference's particle records in and out of the GPU step (ge_frame_aos).

The reference keeps ParticlePhysics / ParticleRendering records
(include/Particles/particle.h:5-277), flattens their gravity members before
the walk (physics.cpp:354-390), reads them back after (:542-565) and moves
both arrays into Morton order every frame (morton.cpp:40-63).
ge_frame_aos takes the records as they are:

  * CPU: ge_aos_layout_default equals the layout the compiler gives the
    reference's own headers (oracle/_ref/particle_layout.txt, written by
    `make -C oracle ref`);
  * GPU: one frame on the records gives bit for bit the same positions,
    velocities, accelerations and prevVel as the SoA path (ge_frame_host),
    written into each particle's own record; the records' other bytes are
    left as they were; `order` is the SoA path's Morton order, and moving
    the records by it each frame, as the reference does, keeps three frames
    bit-identical.
"""
import os

import numpy as np
import pytest

from conftest import ROOT

LAYOUT_TXT = os.path.join(ROOT, "oracle", "_ref", "particle_layout.txt")


def test_default_layout_matches_the_reference_headers(ge):
    if not os.path.exists(LAYOUT_TXT):
        pytest.skip("oracle/_ref/particle_layout.txt not built (no reference checkout)")
    rows = {int(r.split()[0]): [int(v) for v in r.split()[1:]]
            for r in open(LAYOUT_TXT).read().strip().splitlines()}
    for dims in (2, 3):
        L = ge.aos_layout(dims)
        got = [L.stride, L.off_pos, L.off_vel, L.off_acc, L.off_prev_vel, L.off_mass, L.off_id,
               L.off_temp, L.r_stride, L.r_off_pinned]
        assert got == rows[dims], (dims, got, rows[dims])


def record_dtypes(ge, dims):
    L = ge.aos_layout(dims)
    v = ("<f4", (dims,))
    phys = np.dtype({"names": ["pos", "vel", "acc", "prevVel", "mass", "temp", "id"],
                     "formats": [v, v, v, v, "<f4", "<f4", "<u4"],
                     "offsets": [L.off_pos, L.off_vel, L.off_acc, L.off_prev_vel, L.off_mass,
                                 L.off_temp, L.off_id],
                     "itemsize": L.stride})
    rend = np.dtype({"names": ["isPinned"], "formats": ["u1"], "offsets": [L.r_off_pinned],
                     "itemsize": L.r_stride})
    return phys, rend


def make_records(ge, st, dims, seed):
    pdt, rdt = record_dtypes(ge, dims)
    n = len(st["x"])
    rng = np.random.default_rng(seed)
    phys = rng.integers(0, 256, n * pdt.itemsize, dtype=np.uint8).view(pdt)
    rend = rng.integers(0, 256, n * rdt.itemsize, dtype=np.uint8).view(rdt)
    ax = "xyz"[:dims]
    phys["pos"] = np.stack([st[a] for a in ax], 1)
    phys["vel"] = np.stack([st["v" + a] for a in ax], 1)
    phys["acc"] = 0.0
    phys["mass"] = st["m"]
    phys["id"] = np.arange(n, dtype=np.uint32)
    rend["isPinned"] = (rng.random(n) < 0.03).astype(np.uint8)
    return phys, rend


def _take(rec, order):
    """rec[order] with every byte of each record (padding included)."""
    raw = rec.view(np.uint8).reshape(len(rec), -1)[order]
    return np.ascontiguousarray(raw).view(rec.dtype).reshape(len(rec))


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [2, 3])
def test_frame_aos_equals_the_soa_path(ge, ics, dims):
    st = ics.disk2d(6000, seed=8) if dims == 2 else ics.plummer3d(6000, seed=8)
    p = ge.default_params(dims, G=1.0, theta=0.7, eps2=1e-4 if dims == 2 else 0.01, dt=1e-3,
                          precision=ge.PREC_EXACT, track_prev_vel=1)
    phys, rend = make_records(ge, st, dims, seed=dims)
    ax = "xyz"[:dims]
    # the SoA path: the same frames through ge_frame_host, pin flags uploaded
    soa = {a: np.ascontiguousarray(phys["pos"][:, k]) for k, a in enumerate(ax)}
    soa.update({"v" + a: np.ascontiguousarray(phys["vel"][:, k]) for k, a in enumerate(ax)})
    soa.update({"a" + a: np.zeros(len(phys), np.float32) for a in ax})
    soa["m"] = phys["mass"].copy()
    soa["id"] = phys["id"].copy()
    pinned = rend["isPinned"].copy()
    with ge.Simulation(p) as a, ge.Simulation(p) as b:
        for frame in range(3):
            before = phys.view(np.uint8).copy()   # raw bytes: structured copies drop padding
            order = a.frame_aos(phys, rend)
            # the SoA path with the same input order and pin flags
            b.upload(soa)
            b.upload_pinned(pinned)
            b.step(1)
            out = b.download()
            pv = b.download_prev_vel()
            assert np.array_equal(phys["id"][order], out["id"]), frame
            for k, c in enumerate(ax):
                assert np.array_equal(phys["pos"][order, k], out[c]), (frame, c)
                assert np.array_equal(phys["vel"][order, k], out["v" + c]), (frame, c)
                assert np.array_equal(phys["acc"][order, k], out["a" + c]), (frame, c)
                assert np.array_equal(phys["prevVel"][order, k], pv[k]), (frame, c)
            # nothing else in the records moved (the bytes outside the members)
            raw_a = phys.view(np.uint8).reshape(len(phys), -1)
            raw_b = before.reshape(len(phys), -1)
            L = ge.aos_layout(dims)
            keep = np.ones(L.stride, bool)
            for off in (L.off_pos, L.off_vel, L.off_acc, L.off_prev_vel):
                keep[off:off + 4 * dims] = False
            diff = np.nonzero((raw_a != raw_b).any(0) & keep)[0]
            assert len(diff) == 0, (frame, diff[:16], int((raw_a != raw_b)[:, diff].sum()))
            # as the reference: both record arrays move into Morton order
            phys = _take(phys, order)
            rend = _take(rend, order)
            pinned = pinned[order].copy()
            soa = {c: out[c] for c in list(ax) + ["v" + c for c in ax] + ["a" + c for c in ax] + ["m", "id"]}


@pytest.mark.gpu
def test_frame_aos_rejects_bad_layouts(ge, ics):
    st = ics.disk2d(100, seed=1)
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3)
    phys, rend = make_records(ge, st, 2, seed=1)
    bad = ge.aos_layout(2)
    bad.off_mass = 126   # runs past the record
    with ge.Simulation(p) as s:
        with pytest.raises(ge.GeError) as ei:
            s.frame_aos(phys, rend, layout=bad)
        assert ei.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [2, 3])
def test_page_locked_records_give_the_same_frames(ge, ics, dims):
    """Records in page-locked memory (the copies are asynchronous DMA) give
    the same frames as pageable records, bit for bit."""
    import torch
    st = ics.disk2d(5000, seed=11) if dims == 2 else ics.plummer3d(5000, seed=11)
    p = ge.default_params(dims, G=1.0, theta=0.7, eps2=1e-4 if dims == 2 else 0.01, dt=1e-3,
                          precision=ge.PREC_EXACT)
    phys, rend = make_records(ge, st, dims, seed=7)
    pdt, rdt = phys.dtype, rend.dtype
    lphys = torch.zeros(phys.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    lrend = torch.zeros(rend.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    lphys[:] = phys.view(np.uint8).ravel()
    lrend[:] = rend.view(np.uint8).ravel()
    lphys, lrend = lphys.view(pdt), lrend.view(rdt)
    with ge.Simulation(p) as a, ge.Simulation(p) as b:
        for _ in range(2):
            oa = a.frame_aos(phys, rend)
            ob = b.frame_aos(lphys, lrend)
            assert np.array_equal(oa, ob)
            assert np.array_equal(phys.view(np.uint8), lphys.view(np.uint8))
