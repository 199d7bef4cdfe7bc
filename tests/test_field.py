"""GPU: the gravity field display (include/Physics/field.h) as CUDA.

The reference computes it with a GL compute shader and colours it with a
fragment shader; there is no graphics stack here, so the same arithmetic
runs as a CUDA kernel into a headless RGBA8 buffer.  Checked against the
oracle's C statement of both shaders: strengths bit for bit (one thread per
cell sums the particles in order, as the shader does), colours within one
level of 255 (logf may differ by an ulp between the device and the host).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("periodic,two_color", [(False, False), (True, True)])
def test_field_matches_oracle(ge, ics, O, periodic, two_color):
    st = ics.disk2d(6000, seed=12, center=(60.0, 40.0))
    for k in ("x", "y"):
        st[k] = (st[k] * 8.0).astype(np.float32)
    st["x"] += 300.0
    st["y"] += 200.0
    dom = (640.0, 360.0, 0.0)
    kw = dict(periodic=1) if periodic else {}
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-2, dt=1e-3, domain=dom, **kw)
    with ge.Simulation(p) as s:
        s.upload(st)
        strength, rgba = s.gravity_field(res=60, two_color=int(two_color), threshold=1e-4)
        out = s.download()
    ref_s, ref_c = O.gravity_field(out["x"], out["y"], out["m"], 1.0, dom, periodic=periodic,
                                   res=60, threshold=1e-4, two_color=two_color)
    assert strength.shape == ref_s.shape == (106, 60)
    assert np.array_equal(strength, ref_s)
    assert np.abs(rgba.astype(int) - ref_c.astype(int)).max() <= 1
    assert strength.max() > 0.0 and len(np.unique(rgba.reshape(-1, 4), axis=0)) > 10
