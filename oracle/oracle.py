"""ctypes binding of the CPU oracle (ge_oracle.c) and of the compiled reference
sources (oracle/_ref/libgeref.so).

TEST INFRASTRUCTURE ONLY.  The tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker; the product
library never imports it.  Every function documents the reference lines its
C implementation restates (see ge_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
U32_EMPTY = 0xFFFFFFFF

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class Params(C.Structure):
    """or_params (ge_oracle.h)."""
    _fields_ = [
        ("dims", C.c_int), ("G", C.c_float), ("theta", C.c_float), ("eps2", C.c_float),
        ("dt", C.c_float), ("leaf_cap", C.c_uint32), ("size_gate", C.c_float),
        ("min_size", C.c_float), ("periodic", C.c_int), ("domain", C.c_float * 3),
        ("temp_enabled", C.c_int), ("heat_cond", C.c_float), ("naive_soft", C.c_float),
        ("direct_below", C.c_int),
    ]


def make_params(dims=2, G=1.0, theta=0.7, eps2=1e-4, dt=1e-3, leaf_cap=4, size_gate=2.0,
                min_size=1e-6, periodic=False, domain=(0.0, 0.0, 0.0), temp_enabled=False,
                heat_cond=0.045, naive_soft=None, direct_below=0):
    p = Params()
    p.dims, p.G, p.theta, p.eps2, p.dt = dims, G, theta, eps2, dt
    p.leaf_cap, p.size_gate, p.min_size = leaf_cap, size_gate, min_size
    p.periodic = int(bool(periodic))
    for a in range(3):
        p.domain[a] = domain[a]
    p.temp_enabled, p.heat_cond = int(bool(temp_enabled)), heat_cond
    p.naive_soft = eps2 if naive_soft is None else naive_soft
    p.direct_below = int(direct_below)
    return p


class Tree(C.Structure):
    """or_tree (ge_oracle.h): pre-order node arrays."""
    _fields_ = [
        ("cap", C.c_int64), ("count", C.c_int64), ("dims", C.c_int), ("overflow", C.c_int),
        ("max_depth", C.c_int), ("pos", _vp), ("size", _vp), ("com", _vp), ("mass", _vp),
        ("temp", _vp), ("start", _vp), ("end", _vp), ("next", _vp), ("child", _vp),
    ]


def _build_if_needed(path, target):
    if not os.path.exists(path):
        subprocess.run(["make", "-C", HERE, target], check=True, capture_output=True)


def _load(strict=True):
    name = "liboracle.so" if strict else "liboracle_fma.so"
    path = os.path.join(HERE, name)
    _build_if_needed(path, name)
    lib = C.CDLL(path)
    lib.or_bbox2d.argtypes = [C.c_int64, _f32p, _f32p, _f32p]
    lib.or_bbox3d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p]
    lib.or_keys2d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _u64p]
    lib.or_keys3d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, _u64p]
    lib.or_sort_perm.argtypes = [C.c_int64, _u64p, _u32p]
    lib.or_tree_alloc.argtypes = [C.POINTER(Tree), C.c_int, C.c_int64]
    lib.or_tree_free.argtypes = [C.POINTER(Tree)]
    lib.or_build_quadtree.argtypes = [C.POINTER(Tree), C.c_int64, _f32p, _f32p, _f32p, _vp,
                                      _f32p, C.c_uint32, C.c_float, C.c_float]
    lib.or_build_octree.argtypes = [C.POINTER(Tree), C.c_int64, _f32p, _f32p, _f32p, _f32p,
                                    _vp, _f32p, C.c_uint32, C.c_float, C.c_float]
    lib.or_walk2d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _vp, C.POINTER(Tree),
                              C.POINTER(Params), _f32p, _f32p, _vp, _vp, C.c_int]
    lib.or_walk3d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, _vp, C.POINTER(Tree),
                              C.POINTER(Params), _f32p, _f32p, _f32p, _vp, _vp, C.c_int]
    lib.or_walk2d_avx2.argtypes = [C.c_int64, _f32p, _f32p, _f32p, C.POINTER(Tree),
                                   C.POINTER(Params), _f32p, _f32p, C.c_int]
    lib.or_walk3d_avx2.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, C.POINTER(Tree),
                                   C.POINTER(Params), _f32p, _f32p, _f32p, C.c_int]
    lib.or_naive2d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, C.POINTER(Params), _f32p,
                               _f32p, C.c_int]
    lib.or_naive3d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, C.POINTER(Params),
                               _f32p, _f32p, _f32p, C.c_int]
    lib.or_direct_f64.argtypes = [C.c_int, C.c_int64, _f32p, _f32p, _vp, _f32p, C.c_double,
                                  C.c_double, C.c_int64, _i64p, _f64p, _f64p, _vp, C.c_int]
    lib.or_predict_trajectory.argtypes = [C.POINTER(Tree), _f32p, _f32p, _vp, C.POINTER(Params),
                                          C.c_float, C.c_int64, _f32p, _f32p, _f32p, C.c_int32,
                                          _f32p, C.c_int]
    lib.or_gravity_field.argtypes = [C.c_int64, _f32p, _f32p, _f32p, C.c_float, C.c_float,
                                     C.c_float, C.c_int, C.c_int, C.c_float, C.c_float,
                                     C.c_float, C.c_float, C.c_int, _f32p, _f32p, _vp, _vp,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
    lib.or_sph_grid.argtypes = [C.c_int64, _f32p, _f32p, C.c_float, C.c_uint32] + [_vp] * 5
    lib.or_potential_f64.argtypes = [C.c_int, C.c_int64, _f32p, _f32p, _vp, _f32p, C.c_double,
                                     C.c_double, C.c_int]
    lib.or_potential_f64.restype = C.c_double
    lib.or_walk_mixed.argtypes = [C.c_int64, _f32p, _f32p, _vp, _f32p, C.POINTER(Tree),
                                  C.POINTER(Params), _f64p, _f64p, _vp, _vp, C.c_int]
    lib.or_walk_group.argtypes = [C.c_int64, _f32p, _f32p, _vp, _f32p, C.POINTER(Tree),
                                  C.POINTER(Params), C.c_int, _f64p, _f64p, _vp, _vp, C.c_int]
    lib.or_integrate_start.argtypes = [C.c_int, C.c_int64] + [_vp] * 12 + [_vp, C.POINTER(Params)]
    lib.or_integrate_end.argtypes = [C.c_int, C.c_int64] + [_vp] * 6 + [_vp, C.POINTER(Params)]
    lib.or_frame.argtypes = [C.POINTER(Params), C.c_int64] + [_vp] * 16 + [C.c_int, C.c_int,
                                                                           _vp, _vp, _vp]
    lib.or_frame.restype = C.c_int
    lib.or_build_quadtree.restype = C.c_int
    lib.or_build_octree.restype = C.c_int
    lib.or_scale_to_grid2d.argtypes = [C.c_float, C.c_float, C.c_float]
    lib.or_scale_to_grid2d.restype = C.c_uint64
    lib.or_scale_to_grid3d.argtypes = [C.c_float, C.c_float, C.c_float]
    lib.or_scale_to_grid3d.restype = C.c_uint64
    return lib


_LIBS = {}


def lib(strict=True):
    if strict not in _LIBS:
        _LIBS[strict] = _load(strict)
    return _LIBS[strict]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------------
def bbox(x, y, z=None, strict=True):
    """boundingBox / boundingBox3D (globalLogic.cpp:1083-1099, :1460-1477)."""
    x, y = _f32(x), _f32(y)
    if z is None:
        out = np.zeros(3, np.float32)
        lib(strict).or_bbox2d(len(x), x, y, out)
    else:
        out = np.zeros(4, np.float32)
        lib(strict).or_bbox3d(len(x), x, y, _f32(z), out)
    return out


def morton_keys(x, y, bb, z=None, strict=True):
    """computeMortonKeys / computeMortonKeys3D (morton.cpp:27-38, :92-112)."""
    x, y = _f32(x), _f32(y)
    keys = np.zeros(len(x), np.uint64)
    if z is None:
        lib(strict).or_keys2d(len(x), x, y, _f32(bb), keys)
    else:
        lib(strict).or_keys3d(len(x), x, y, _f32(z), _f32(bb), keys)
    return keys


def sort_perm(keys):
    """Stable (key, index) order: the canonical form of morton.cpp:40-63."""
    keys = np.ascontiguousarray(keys, np.uint64)
    perm = np.zeros(len(keys), np.uint32)
    lib().or_sort_perm(len(keys), keys, perm)
    return perm


class PreorderTree:
    """Reference `globalNodes` content, pre-order, as numpy arrays."""

    def __init__(self, dims, count, pos, size, com, mass, start, end, nxt, child, max_depth=0):
        self.dims, self.count = dims, count
        self.pos, self.size, self.com, self.mass = pos, size, com, mass
        self.start, self.end, self.next, self.child = start, end, nxt, child
        self.max_depth = max_depth

    def arrays(self):
        return dict(pos=self.pos, size=self.size, com=self.com, mass=self.mass,
                    start=self.start, end=self.end, next=self.next, child=self.child)


class _TreeHolder:
    def __init__(self, dims, cap, strict=True):
        self.t = Tree()
        self.lib = lib(strict)
        if self.lib.or_tree_alloc(C.byref(self.t), dims, int(cap)) != 0:
            raise MemoryError("or_tree_alloc")

    def __del__(self):
        try:
            self.lib.or_tree_free(C.byref(self.t))
        except Exception:
            pass

    def to_numpy(self):
        t, n, d = self.t, self.t.count, self.t.dims
        nq = 1 << d

        def arr(p, dt, k):
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(dt)), shape=(n * k,)).copy() if n else np.zeros(0)
        return PreorderTree(
            d, n,
            arr(t.pos, C.c_float, d).reshape(n, d), arr(t.size, C.c_float, 1),
            arr(t.com, C.c_float, d).reshape(n, d), arr(t.mass, C.c_float, 1),
            arr(t.start, C.c_uint32, 1), arr(t.end, C.c_uint32, 1), arr(t.next, C.c_uint32, 1),
            arr(t.child, C.c_uint32, nq).reshape(n, nq), t.max_depth)


def build_tree(x, y, m, bb, z=None, leaf_cap=4, size_gate=2.0, min_size=1e-6, strict=True,
               holder=False):
    """Quadtree / Octree build over sorted particles (quadtree.cpp:5-292)."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    dims = 2 if z is None else 3
    cap = (4 if dims == 2 else 8) * n + 64
    while True:
        h = _TreeHolder(dims, cap, strict)
        if dims == 2:
            rc = h.lib.or_build_quadtree(C.byref(h.t), n, x, y, m, None, _f32(bb), leaf_cap,
                                         size_gate, min_size)
        else:
            rc = h.lib.or_build_octree(C.byref(h.t), n, x, y, _f32(z), m, None, _f32(bb),
                                       leaf_cap, size_gate, min_size)
        if rc == 0:
            break
        cap *= 4
    return h if holder else h.to_numpy()


def walk(x, y, m, tree_holder, params, z=None, nthreads=8, want_counts=False, want_cond=False,
         strict=True, temp=None):
    """calculateForceFromGrid / calculateForceFromGrid3D (physics.cpp:91-205,
    physics3D.cpp:131-253): scalar walk; returns accelerations."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    ax, ay = np.zeros(n, np.float32), np.zeros(n, np.float32)
    inter = np.zeros(n, np.uint32) if want_counts else None
    cond = np.zeros(n, np.float32) if want_cond else None
    L = lib(strict)
    if z is None:
        L.or_walk2d(n, x, y, m, _ptr(temp), C.byref(tree_holder.t), C.byref(params), ax, ay,
                    _ptr(inter), _ptr(cond), nthreads)
        out = [ax, ay]
    else:
        az = np.zeros(n, np.float32)
        L.or_walk3d(n, x, y, _f32(z), m, _ptr(temp), C.byref(tree_holder.t), C.byref(params),
                    ax, ay, az, _ptr(inter), _ptr(cond), nthreads)
        out = [ax, ay, az]
    if want_counts:
        out.append(inter)
    if want_cond:
        out.append(cond)
    return out


def predict_trajectory(x, y, tree_holder, params, eps2, pos, vel, mass, steps, z=None,
                       nthreads=8):
    """predictTrajectory (particlesSpawning.cpp:443-500): probe paths against
    the fixed tree; returns [nprobes, steps, dims]."""
    x, y = _f32(x), _f32(y)
    pos, vel, mass = _f32(pos), _f32(vel), _f32(mass)
    dims = 2 if z is None else 3
    nprobes = len(mass)
    path = np.zeros(nprobes * steps * dims, np.float32)
    zz = None if z is None else _f32(z)
    lib().or_predict_trajectory(C.byref(tree_holder.t), x, y, _ptr(zz), C.byref(params), eps2,
                                nprobes, pos.ravel(), vel.ravel(), mass, int(steps), path,
                                nthreads)
    return path.reshape(nprobes, steps, dims)


def gravity_field(x, y, m, G, domain, periodic=False, res=150, softness=0.85, threshold=1000.0,
                  stretch=90.0, exposure=3.0, two_color=False, low=(0.0, 40 / 255, 68 / 255),
                  high=(155 / 255, 80 / 255, 40 / 255), nthreads=8):
    """The field view (field.h): strengths [ax, ay] and RGBA8 [ax, ay, 4]."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    dx, dy = float(domain[0]), float(domain[1])
    cell = np.float32(min(dx, dy)) / np.float32(res)
    ax, ay = int(np.float32(dx) / cell) + 2, int(np.float32(dy) / cell) + 2
    st = np.zeros(ax * ay, np.float32)
    px = np.zeros(ax * ay, np.uint32)
    oax, oay = C.c_int(0), C.c_int(0)
    lib().or_gravity_field(len(x), x, y, m, G, dx, dy, int(bool(periodic)), res, softness,
                           threshold, stretch, exposure, int(bool(two_color)),
                           np.array(low, np.float32), np.array(high, np.float32), _ptr(st),
                           _ptr(px), C.byref(oax), C.byref(oay), nthreads)
    n = oax.value * oay.value
    rgba = px[:n].view(np.uint8).reshape(oax.value, oay.value, 4)
    return st[:n].reshape(oax.value, oay.value), rgba


def potential_f64(x, y, m, G, eps2, z=None, nthreads=8):
    """FP64 direct-sum potential energy."""
    zz = None if z is None else _f32(z)
    return lib().or_potential_f64(2 if z is None else 3, len(x), _f32(x), _f32(y), _ptr(zz),
                                  _f32(m), G, eps2, nthreads)


def walk_mixed(x, y, m, tree_holder, params, z=None, nthreads=8, want_counts=False):
    """The mixed-precision walk (FP64 moments, offset-corrected opening test,
    softened quadrupole) on the reference tree; accelerations in FP64."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    out = [np.zeros(n, np.float64) for _ in range(2 if z is None else 3)]
    inter = np.zeros(n, np.uint32) if want_counts else None
    zz = None if z is None else _f32(z)
    lib().or_walk_mixed(n, x, y, _ptr(zz), m, C.byref(tree_holder.t), C.byref(params),
                        out[0], out[1], _ptr(out[2]) if z is not None else None,
                        _ptr(inter), nthreads)
    if want_counts:
        out.append(inter)
    return out


def walk_group(x, y, m, tree_holder, params, group_size=32, z=None, nthreads=8,
               want_counts=False):
    """The mixed-precision group walk (groups of group_size consecutive
    particles share one opening test); accelerations in FP64."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    out = [np.zeros(n, np.float64) for _ in range(2 if z is None else 3)]
    inter = np.zeros(n, np.uint32) if want_counts else None
    zz = None if z is None else _f32(z)
    lib().or_walk_group(n, x, y, _ptr(zz), m, C.byref(tree_holder.t), C.byref(params),
                        int(group_size), out[0], out[1],
                        _ptr(out[2]) if z is not None else None, _ptr(inter), nthreads)
    if want_counts:
        out.append(inter)
    return out


def walk_avx2(x, y, m, tree_holder, params, z=None, nthreads=8, strict=True):
    """calculateForceFromGridAVX2 / ...3DAVX2 (physics.cpp:207-352, physics3D.cpp:255-414)."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    ax, ay = np.zeros(n, np.float32), np.zeros(n, np.float32)
    if z is None:
        lib(strict).or_walk2d_avx2(n, x, y, m, C.byref(tree_holder.t), C.byref(params), ax, ay,
                                   nthreads)
        return [ax, ay]
    az = np.zeros(n, np.float32)
    lib(strict).or_walk3d_avx2(n, x, y, _f32(z), m, C.byref(tree_holder.t), C.byref(params),
                               ax, ay, az, nthreads)
    return [ax, ay, az]


def direct_f64(x, y, m, G, eps2, idx, z=None, nthreads=8):
    """FP64 direct sum for targets idx (j != i), the accuracy reference."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    idx = np.ascontiguousarray(idx, np.int64)
    nt = len(idx)
    ax, ay = np.zeros(nt), np.zeros(nt)
    az = np.zeros(nt) if z is not None else None
    lib().or_direct_f64(2 if z is None else 3, len(x), x, y, _ptr(_f32(z)) if z is not None else None,
                        m, float(G), float(eps2), nt, idx, ax, ay, _ptr(az), nthreads)
    return [ax, ay] if z is None else [ax, ay, az]


def frame(params, state, walk_kind=0, nthreads=8, strict=True):
    """One frame of globalLogic.cpp:1155-1370 (2D) / :1584-1719 (3D) on the
    dict of float32/uint32 arrays in ``state`` (modified in place, permuted
    into Morton order).  Returns (stage_ms[8], interactions, nodes)."""
    d3 = params.dims == 3
    g = state.get
    st = np.zeros(8, np.float64)
    inter = np.zeros(1, np.uint64)
    nodes = np.zeros(1, np.int64)
    n = len(state["x"])
    rc = lib(strict).or_frame(
        C.byref(params), n, _ptr(g("x")), _ptr(g("y")), _ptr(g("z")) if d3 else None,
        _ptr(g("vx")), _ptr(g("vy")), _ptr(g("vz")) if d3 else None,
        _ptr(g("ax")), _ptr(g("ay")), _ptr(g("az")) if d3 else None,
        _ptr(g("m")), _ptr(g("id")), _ptr(g("pvx")), _ptr(g("pvy")), _ptr(g("pvz")),
        _ptr(g("temp")), _ptr(g("pinned")), walk_kind, nthreads,
        _ptr(st), _ptr(inter), _ptr(nodes))
    if rc != 0:
        raise RuntimeError("or_frame failed")
    return st, int(inter[0]), int(nodes[0])


def sph_grid(x, y, cell=3.0, table=16384, strict=True):
    """SPH neighbour grid (SPH::newGridGPU) as the reference's shaders compute
    it, bitonic network included: dict of keys, index, cell_x, cell_y
    (network order) and offsets."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n = len(x)
    out = {k: np.empty(n, np.uint32) for k in ("keys", "index")}
    out.update({k: np.empty(n, np.int32) for k in ("cell_x", "cell_y")})
    out["offsets"] = np.empty(int(table), np.uint32)
    lib(strict).or_sph_grid(n, x, y, float(cell), int(table),
                            *(_ptr(out[k]) for k in ("keys", "index", "cell_x", "cell_y",
                                                      "offsets")))
    return out


# --------------------------------------------------------------------------
# compiled reference sources (oracle/_ref); present only where the reference
# checkout was available when the oracle was built.
def ref_lib(fma=False):
    path = os.path.join(HERE, "_ref", "libgeref_fma.so" if fma else "libgeref.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.ref_keys2d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _u64p]
    L.ref_keys3d.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, _u64p]
    L.ref_sort2d.argtypes = [C.c_int64, _u64p, _u32p]
    L.ref_build_quadtree.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, C.c_int64,
                                     _f32p, _f32p, _f32p, _f32p, _u32p, _u32p, _u32p, _u32p]
    L.ref_build_quadtree.restype = C.c_int64
    L.ref_build_octree.argtypes = [C.c_int64, _f32p, _f32p, _f32p, _f32p, _f32p, C.c_int64,
                                   _f32p, _f32p, _f32p, _f32p, _u32p, _u32p, _u32p, _u32p]
    L.ref_build_octree.restype = C.c_int64
    return L


def ref_build_tree(L, x, y, m, bb, z=None):
    """Run the reference's own Quadtree / Octree constructor."""
    x, y, m = _f32(x), _f32(y), _f32(m)
    n = len(x)
    dims = 2 if z is None else 3
    nq = 1 << dims
    cap = nq * n + 64
    pos = np.zeros(cap * dims, np.float32); com = np.zeros(cap * dims, np.float32)
    size = np.zeros(cap, np.float32); mass = np.zeros(cap, np.float32)
    start = np.zeros(cap, np.uint32); end = np.zeros(cap, np.uint32)
    nxt = np.zeros(cap, np.uint32); child = np.zeros(cap * nq, np.uint32)
    if dims == 2:
        cnt = L.ref_build_quadtree(n, x, y, m, _f32(bb), cap, pos, size, com, mass, start, end,
                                   nxt, child)
    else:
        cnt = L.ref_build_octree(n, x, y, _f32(z), m, _f32(bb), cap, pos, size, com, mass,
                                 start, end, nxt, child)
    cnt = int(cnt)
    return PreorderTree(dims, cnt, pos[:cnt * dims].reshape(cnt, dims), size[:cnt],
                        com[:cnt * dims].reshape(cnt, dims), mass[:cnt], start[:cnt], end[:cnt],
                        nxt[:cnt], child[:cnt * nq].reshape(cnt, nq))


def ref_keys(L, x, y, bb, z=None):
    x, y = _f32(x), _f32(y)
    keys = np.zeros(len(x), np.uint64)
    if z is None:
        L.ref_keys2d(len(x), x, y, _f32(bb), keys)
    else:
        L.ref_keys3d(len(x), x, y, _f32(z), _f32(bb), keys)
    return keys
