"""galaxy-engine_b200 -- B200 Barnes-Hut gravity step for Galaxy Engine.

Python binding of the C ABI in ``include/ge_bh.h`` (libgebh.so, built in-tree
by ``build.py``).  The names mirror the reference's gravity call surface
(NarcisCalin/Galaxy-Engine):

=============================  ==============================================
this module                    reference
=============================  ==============================================
``Simulation.upload``          ``Physics::flattenParticles`` (physics.cpp:354-390)
``Simulation.download``        ``Physics::readFlattenBack`` (physics.cpp:542-565)
``integrate_start``            ``Physics::integrateStart`` (physics.cpp:1069-1112)
``bounding_box``               ``boundingBox`` (globalLogic.cpp:1083-1099)
``compute_morton_keys``        ``Morton::computeMortonKeys`` (morton.cpp:27-38)
``sort_particles_by_morton_key``  ``Morton::sortParticlesByMortonKey`` (morton.cpp:40-63)
``build_tree``                 ``Quadtree`` / ``Octree`` (quadtree.cpp:5-292)
``calculate_force_from_grid``  ``Physics::calculateForceFromGrid`` (physics.cpp:91-205)
``integrate_end``              ``Physics::integrateEnd`` (physics.cpp:1114-1125)
``step``                       the gravity block of ``updateScene`` (globalLogic.cpp:1155-1370)
=============================  ==============================================

There is no CPU fallback: constructing a Simulation without a B200-class GPU
or without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgebh.so")

PREC_FAST, PREC_EXACT, PREC_MIXED = 0, 1, 2
STATUS = {0: "GE_OK", 1: "GE_ERR_ARG", 2: "GE_ERR_NO_DEVICE", 3: "GE_ERR_CUDA",
          4: "GE_ERR_CAPACITY", 5: "GE_ERR_STATE", 6: "GE_ERR_TIMEOUT", 7: "GE_ERR_OOM",
          8: "GE_ERR_UNSUPPORTED"}
EMPTY = 0xFFFFFFFF


class GeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


STATE_KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "id", "kx", "ky", "kz",
              "kvx", "kvy", "kvz", "pvx", "pvy", "pvz", "temp", "pinned")


class Params(C.Structure):
    """ge_params (include/ge_bh.h)."""
    _fields_ = [
        ("dims", C.c_int32), ("precision", C.c_int32), ("G", C.c_float), ("theta", C.c_float),
        ("eps2", C.c_float), ("dt", C.c_float), ("leaf_cap", C.c_uint32),
        ("size_gate", C.c_float), ("min_size", C.c_float), ("node_cap_factor", C.c_float),
        ("periodic", C.c_int32), ("domain", C.c_float * 3), ("track_prev_vel", C.c_int32),
        ("group_size", C.c_int32), ("temp_enabled", C.c_int32), ("heat_cond", C.c_float),
        ("direct_below", C.c_int32), ("direct_eps2", C.c_float), ("no_graph", C.c_int32),
        ("walk_kind", C.c_int32),
    ]


class Stats(C.Structure):
    """ge_stats (include/ge_bh.h)."""
    _fields_ = [
        ("n", C.c_int64), ("nodes", C.c_int64), ("depth", C.c_int32), ("steps", C.c_int32),
        ("interactions", C.c_uint64), ("bbox", C.c_float * 4), ("ms_last_step", C.c_float),
        ("stage_ms", C.c_float * 8),
    ]


class StateArrays(C.Structure):
    """ge_state_arrays (include/ge_bh.h): host arrays of a checkpoint."""
    _fields_ = [(k, C.c_void_p) for k in STATE_KEYS]


class AosLayout(C.Structure):
    """ge_aos_layout (include/ge_bh.h): byte offsets of the record members."""
    _fields_ = [(k, C.c_int32) for k in ("stride", "off_pos", "off_vel", "off_acc",
                                          "off_prev_vel", "off_mass", "off_id", "off_temp",
                                          "r_stride", "r_off_pinned")]


class ServerConfig(C.Structure):
    """ge_server_config (include/ge_bh.h)."""
    _fields_ = [
        ("hbm_budget_bytes", C.c_int64), ("frac_2d", C.c_double), ("max_sims", C.c_int32),
        ("reserved", C.c_int32 * 7), ("params", Params * 2),
    ]


class ServerStats(C.Structure):
    """ge_server_stats (include/ge_bh.h)."""
    _fields_ = [
        ("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
        ("queued", C.c_int64), ("running", C.c_int64), ("iterations", C.c_int64),
        ("particle_steps", C.c_int64), ("busy_s", C.c_double), ("step_ms_p50", C.c_double),
        ("step_ms_p99", C.c_double), ("latency_s_p50", C.c_double),
        ("latency_s_p99", C.c_double), ("pool_bytes", C.c_int64 * 2),
        ("pool_capacity", C.c_int64 * 2), ("pool_iterations", C.c_int64 * 2),
        ("pool_step_ms_p50", C.c_double * 2), ("pool_step_ms_p99", C.c_double * 2),
        ("pool_busy_s", C.c_double * 2), ("pool_admit_s", C.c_double * 2),
        ("pool_retire_s", C.c_double * 2), ("pool_particle_steps", C.c_int64 * 2),
        ("queue_wait_s_p50", C.c_double), ("queue_wait_s_p99", C.c_double),
    ]


class TuneResult(C.Structure):
    """ge_tune_result (include/ge_bh.h)."""
    _fields_ = [("group_size", C.c_int32), ("leaf_cap", C.c_int32), ("tried", C.c_int32),
                ("reserved", C.c_int32), ("ms", C.c_float * 12)]


class FieldParams(C.Structure):
    """ge_field_params (include/ge_bh.h)."""
    _fields_ = [("res", C.c_int32), ("softness", C.c_float), ("threshold", C.c_float),
                ("stretch", C.c_float), ("exposure", C.c_float), ("two_color", C.c_int32),
                ("color_low", C.c_float * 3), ("color_high", C.c_float * 3),
                ("reserved", C.c_int32 * 4)]


class SaveInfo(C.Structure):
    """ge_save_info (include/ge_bh.h)."""
    _fields_ = [("version", C.c_uint32), ("dims", C.c_int32), ("n", C.c_int64),
                ("global_id", C.c_uint32), ("global_shape_id", C.c_uint32),
                ("global_wall_id", C.c_uint32), ("record_bytes", C.c_int32)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

_vp = C.c_void_p
_LIB = None

# Every symbol include/ge_bh.h declares, with its ctypes signature.
SIGNATURES = {
    "ge_abi_version": ([], C.c_int),
    "ge_params_default": ([C.POINTER(Params), C.c_int], None),
    "ge_create": ([C.POINTER(Params), C.POINTER(_vp)], C.c_int),
    "ge_destroy": ([_vp], C.c_int),
    "ge_last_error": ([_vp], C.c_char_p),
    "ge_set_params": ([_vp, C.POINTER(Params)], C.c_int),
    "ge_set_stream": ([_vp, _vp], C.c_int),
    "ge_sync": ([_vp], C.c_int),
    "ge_get_stats": ([_vp, C.POINTER(Stats)], C.c_int),
    "ge_upload": ([_vp, C.c_int64] + [_vp] * 11, C.c_int),
    "ge_download": ([_vp] + [_vp] * 11, C.c_int),
    "ge_upload_pinned": ([_vp, _vp], C.c_int),
    "ge_download_prev_vel": ([_vp, _vp, _vp, _vp], C.c_int),
    "ge_upload_temp": ([_vp, _vp], C.c_int),
    "ge_save_read_info": ([C.c_char_p, C.POINTER(SaveInfo)], C.c_int),
    "ge_field_params_default": ([C.POINTER(FieldParams)], None),
    "ge_gravity_field": ([_vp, C.c_int32, C.POINTER(FieldParams), C.c_int64, _vp, _vp,
                          C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "ge_save_read": ([C.c_char_p, C.c_int64] + [_vp] * 13, C.c_int),
    "ge_sph_grid": ([_vp, C.c_int32, C.c_float, C.c_uint32, C.c_int64] + [_vp] * 5, C.c_int),
    "ge_predict_trajectory": ([_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_float, C.c_int32,
                               _vp], C.c_int),
    "ge_download_temp": ([_vp, _vp], C.c_int),
    "ge_step": ([_vp, C.c_int32], C.c_int),
    "ge_download_state": ([_vp, C.POINTER(StateArrays)], C.c_int),
    "ge_aos_layout_default": ([C.POINTER(AosLayout), C.c_int], None),
    "ge_frame_aos": ([_vp, C.c_int64, _vp, _vp, C.POINTER(AosLayout), _vp], C.c_int),
    "ge_upload_state": ([_vp, C.c_int64, C.POINTER(StateArrays)], C.c_int),
    "ge_set_sort_wait_test": ([_vp, C.c_uint32, C.c_int32], C.c_int),
    "ge_profile_step": ([_vp], C.c_int),
    "ge_frame_host": ([_vp, C.c_int64] + [_vp] * 11, C.c_int),
    "ge_integrate_start": ([_vp], C.c_int),
    "ge_bounding_box": ([_vp, _vp], C.c_int),
    "ge_compute_morton_keys": ([_vp, _vp], C.c_int),
    "ge_sort_by_morton_key": ([_vp, _vp], C.c_int),
    "ge_build_tree": ([_vp], C.c_int),
    "ge_compute_forces": ([_vp], C.c_int),
    "ge_integrate_end": ([_vp], C.c_int),
    "ge_set_count_interactions": ([_vp, C.c_int32], C.c_int),
    "ge_export_tree": ([_vp, C.c_int64, _vp] + [_vp] * 8, C.c_int),
    "ge_direct_sum_f64": ([_vp, C.c_int64, _vp, _vp, _vp, _vp], C.c_int),
    "ge_sums_f64": ([_vp, _vp], C.c_int),
    "ge_energy_f64": ([_vp, _vp], C.c_int),
    "ge_build_timeline": ([_vp, C.c_int32, _vp, _vp], C.c_int),
    "ge_morton_sort_2d_noalloc": ([C.c_int64, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "ge_batch_create": ([C.POINTER(Params), C.POINTER(_vp)], C.c_int),
    "ge_batch_step": ([_vp, C.c_int32], C.c_int),
    "ge_batch_add_sim": ([_vp, C.c_int64] + [_vp] * 8 + [C.POINTER(C.c_int32)], C.c_int),
    "ge_batch_remove_sim": ([_vp, C.c_int32], C.c_int),
    "ge_batch_list": ([_vp, C.c_int32, _vp, C.POINTER(C.c_int32)], C.c_int),
    "ge_batch_query": ([_vp, C.c_int32, _vp, _vp, _vp], C.c_int),
    "ge_batch_download_sim": ([_vp, C.c_int32] + [_vp] * 11, C.c_int),
    "ge_batch_remove_sims": ([_vp, C.c_int32, _vp], C.c_int),
    "ge_step_async": ([_vp, C.c_int32], C.c_int),
    "ge_autotune": ([_vp, C.c_int32, C.POINTER(TuneResult)], C.c_int),
    "ge_step_wait": ([_vp], C.c_int),
    "ge_reserve": ([_vp, C.c_int64, C.c_int64], C.c_int),
    "ge_memory_bytes": ([_vp, C.POINTER(C.c_int64)], C.c_int),
    "ge_estimate_bytes": ([C.POINTER(Params), C.c_int64, C.c_int64, C.POINTER(C.c_int64)],
                          C.c_int),
    "ge_server_create": ([C.POINTER(ServerConfig), C.POINTER(_vp)], C.c_int),
    "ge_server_destroy": ([_vp], C.c_int),
    "ge_server_last_error": ([_vp], C.c_char_p),
    "ge_server_submit": ([_vp, C.c_int32, C.c_int64] + [_vp] * 7 + [C.c_int32,
                         C.POINTER(C.c_int64)], C.c_int),
    "ge_server_start": ([_vp], C.c_int),
    "ge_server_stop": ([_vp], C.c_int),
    "ge_server_poll": ([_vp, C.POINTER(C.c_int32)], C.c_int),
    "ge_server_wait": ([_vp, C.c_int64, C.c_double], C.c_int),
    "ge_server_status": ([_vp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                          C.POINTER(C.c_double)], C.c_int),
    "ge_server_take": ([_vp, C.c_int64] + [_vp] * 11, C.c_int),
    "ge_server_get_stats": ([_vp, C.POINTER(ServerStats)], C.c_int),
}
NOALLOC_MAX_N = 262144   # GE_NOALLOC_MAX_N


def lib():
    """Load libgebh.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run galaxy-engine_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


def default_params(dims=2, **kw):
    """ge_params_default, then keyword overrides (softening= sets eps2 the
    way the reference walk uses it: squared in 2D, as-is in 3D; and
    direct_eps2 the way its direct sum does: as-is in both)."""
    p = Params()
    lib().ge_params_default(C.byref(p), dims)
    soft = kw.pop("softening", None)
    if soft is not None:
        p.eps2 = soft * soft if dims == 2 else soft
        p.direct_eps2 = soft
    for k, v in kw.items():
        if k == "domain":
            for a in range(3):
                p.domain[a] = v[a]
        else:
            setattr(p, k, v)
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


class Simulation:
    """One resident simulation on the GPU (a ge_ctx)."""

    def __init__(self, params=None, **kw):
        L = lib()
        if params is None:
            params = default_params(**kw)
        self.params = params
        h = _vp()
        rc = L.ge_create(C.byref(params), C.byref(h))
        if rc != 0:
            raise GeError(rc, "ge_create failed (a B200-class CUDA device is required)")
        self._h = h
        self.dims = params.dims
        self.n = 0

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            msg = lib().ge_last_error(self._h)
            raise GeError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            lib().ge_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_params(self, params):
        self._check(lib().ge_set_params(self._h, C.byref(params)))
        self.params = params

    def set_stream(self, cuda_stream_handle):
        self._check(lib().ge_set_stream(self._h, _vp(cuda_stream_handle) if cuda_stream_handle else None))

    def stats(self):
        s = Stats()
        self._check(lib().ge_get_stats(self._h, C.byref(s)))
        return s

    def sync(self):
        self._check(lib().ge_sync(self._h))

    # -- state ------------------------------------------------------------
    def upload(self, state):
        """state: dict with x, y, (z,) vx, vy, (vz,) m and optional id, ax, ay, az."""
        g = state.get
        arrs = {k: _f32(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "ax", "ay", "az")}
        ids = None if g("id") is None else np.ascontiguousarray(g("id"), np.uint32)
        n = len(arrs["x"])
        self._keep = (arrs, ids)
        self._check(lib().ge_upload(self._h, n, _ptr(arrs["x"]), _ptr(arrs["y"]), _ptr(arrs["z"]),
                                    _ptr(arrs["vx"]), _ptr(arrs["vy"]), _ptr(arrs["vz"]),
                                    _ptr(arrs["m"]), _ptr(ids), _ptr(arrs["ax"]),
                                    _ptr(arrs["ay"]), _ptr(arrs["az"])))
        self.n = n

    def frame_aos(self, phys, rend=None, layout=None, order=True):
        """One frame on the reference's particle records (ge_frame_aos):
        phys / rend are numpy byte-record arrays (updated in place, in their
        own order); returns the Morton order (slot -> record) when asked."""
        if layout is None:
            layout = aos_layout(self.dims)
        phys = np.ascontiguousarray(phys)
        n = len(phys)
        out = np.zeros(n, np.uint32) if order else None
        self._check(lib().ge_frame_aos(self._h, n, _ptr(phys), _ptr(rend), C.byref(layout),
                                       _ptr(out)))
        self.n = n
        return out

    def download_state(self):
        """Checkpoint: every term the next step reads (ge_download_state), as
        a dict of host arrays in the current particle order."""
        n = self.n
        out = {}
        for k in STATE_KEYS:
            if k in ("z", "vz", "az", "kz", "kvz", "pvz") and self.dims == 2:
                continue
            out[k] = np.zeros(n, np.uint32 if k == "id" else np.uint8 if k == "pinned" else np.float32)
        arr = StateArrays(*[_ptr(out.get(k)) for k in STATE_KEYS])
        self._check(lib().ge_download_state(self._h, C.byref(arr)))
        return out

    def upload_state(self, state):
        """Resume from download_state()'s dict (ge_upload_state); keys that
        are missing are left out."""
        conv = {k: (np.ascontiguousarray(v, np.uint32) if k == "id" else
                    np.ascontiguousarray(v, np.uint8) if k == "pinned" else _f32(v))
                for k, v in state.items() if k in STATE_KEYS and v is not None}
        n = len(conv["x"])
        if self.params.precision != PREC_MIXED:
            for k in ("kx", "ky", "kz", "kvx", "kvy", "kvz"):
                conv.pop(k, None)
        self._keep = conv
        arr = StateArrays(*[_ptr(conv.get(k)) for k in STATE_KEYS])
        self._check(lib().ge_upload_state(self._h, n, C.byref(arr)))
        self.n = n

    def upload_pinned(self, pinned):
        p = None if pinned is None else np.ascontiguousarray(pinned, np.uint8)
        self._check(lib().ge_upload_pinned(self._h, _ptr(p)))

    def _host_state(self, n):
        out = {k: np.empty(n, np.float32) for k in ("x", "y", "vx", "vy", "ax", "ay", "m")}
        if self.dims == 3:
            for k in ("z", "vz", "az"):
                out[k] = np.empty(n, np.float32)
        out["id"] = np.empty(n, np.uint32)
        g = out.get
        ptrs = [_ptr(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "id")]
        return out, ptrs

    def download(self):
        out, ptrs = self._host_state(self.n)
        self._check(lib().ge_download(self._h, *ptrs))
        return out

    # -- batched simulations ------------------------------------------------
    def add_sim(self, state):
        """Append an independent simulation (same dict as upload, no ax/ay/az);
        returns its handle.  Every later step advances all simulations."""
        g = state.get
        arrs = {k: _f32(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        ids = None if g("id") is None else np.ascontiguousarray(g("id"), np.uint32)
        h = C.c_int32(0)
        self._check(lib().ge_batch_add_sim(self._h, len(arrs["x"]), _ptr(arrs["x"]),
                                           _ptr(arrs["y"]), _ptr(arrs["z"]), _ptr(arrs["vx"]),
                                           _ptr(arrs["vy"]), _ptr(arrs["vz"]), _ptr(arrs["m"]),
                                           _ptr(ids), C.byref(h)))
        self.n = int(self.stats().n)
        return h.value

    def remove_sim(self, sim):
        self._check(lib().ge_batch_remove_sim(self._h, int(sim)))
        self.n = int(self.stats().n)

    def remove_sims(self, sims):
        h = np.ascontiguousarray(sims, np.int32)
        self._check(lib().ge_batch_remove_sims(self._h, len(h), _ptr(h)))
        self.n = int(self.stats().n)

    def autotune(self, reps=2):
        """Mixed mode: pick group_size and leaf_cap by timing the force pass
        on the resident state; returns (group_size, leaf_cap, {(g, l): ms})."""
        r = TuneResult()
        self._check(lib().ge_autotune(self._h, int(reps), C.byref(r)))
        self.params.group_size = r.group_size
        self.params.leaf_cap = r.leaf_cap
        table = {(g, l): float(r.ms[4 * a + b]) for a, g in enumerate((32, 64, 128))
                 for b, l in enumerate((1, 4, 8, 16))}
        return r.group_size, r.leaf_cap, table

    def step_async(self, nsteps=1):
        self._check(lib().ge_step_async(self._h, int(nsteps)))

    def step_wait(self):
        self._check(lib().ge_step_wait(self._h))

    def reserve(self, n, sims=1):
        self._check(lib().ge_reserve(self._h, int(n), int(sims)))

    def memory_bytes(self):
        b = C.c_int64(0)
        self._check(lib().ge_memory_bytes(self._h, C.byref(b)))
        return b.value

    def sims(self):
        """Handles of the simulations, in slot order."""
        cnt = C.c_int32(0)
        self._check(lib().ge_batch_list(self._h, 0, None, C.byref(cnt)))
        out = np.zeros(max(cnt.value, 1), np.int32)
        self._check(lib().ge_batch_list(self._h, len(out), _ptr(out), C.byref(cnt)))
        return [int(v) for v in out[: cnt.value]]

    def query(self, sim):
        """(particles, first slot, steps since added) of a simulation."""
        n, off, steps = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        self._check(lib().ge_batch_query(self._h, int(sim), C.byref(n), C.byref(off),
                                         C.byref(steps)))
        return n.value, off.value, steps.value

    def download_sim(self, sim):
        n = self.query(sim)[0]
        out, ptrs = self._host_state(n)
        self._check(lib().ge_batch_download_sim(self._h, int(sim), *ptrs))
        return out

    def predict_trajectory(self, pos, vel, mass, steps, eps2, sim=0):
        """predictTrajectory (particlesSpawning.cpp:443-500): probe paths on the
        tree of the last step; returns [nprobes, steps, dims]."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, self.dims)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, self.dims)
        mass = np.ascontiguousarray(mass, np.float32).ravel()
        path = np.zeros((len(mass), int(steps), self.dims), np.float32)
        self._check(lib().ge_predict_trajectory(self._h, int(sim), len(mass), _ptr(pos),
                                                _ptr(vel), _ptr(mass), float(eps2), int(steps),
                                                _ptr(path)))
        return path

    def gravity_field(self, sim=0, colors=True, **kw):
        """The field view (field.h): cell strengths [amount_x, amount_y] and,
        with colors, RGBA8 pixels [amount_x, amount_y, 4]."""
        fp = FieldParams()
        lib().ge_field_params_default(C.byref(fp))
        for k, v in kw.items():
            if k in ("color_low", "color_high"):
                for a in range(3):
                    getattr(fp, k)[a] = v[a]
            else:
                setattr(fp, k, v)
        ax, ay = C.c_int32(0), C.c_int32(0)
        rc = lib().ge_gravity_field(self._h, int(sim), C.byref(fp), 0, None, None, C.byref(ax),
                                    C.byref(ay))
        if rc not in (0, 4):
            self._check(rc)
        n = ax.value * ay.value
        st = np.zeros(n, np.float32)
        px = np.zeros(n * 4, np.uint8) if colors else None
        self._check(lib().ge_gravity_field(self._h, int(sim), C.byref(fp), n, _ptr(st), _ptr(px),
                                           C.byref(ax), C.byref(ay)))
        st = st.reshape(ax.value, ay.value)
        return (st, px.reshape(ax.value, ay.value, 4)) if colors else st

    def sph_grid(self, cell_size=3.0, table_size=16384, sim=0):
        """SPH neighbour grid (SPH::newGridGPU): entries sorted by hashed
        cell key (keys, index, cell_x, cell_y, one per particle of the
        simulation) and offsets[table_size] (first entry of each key,
        0xFFFFFFFF for none)."""
        n = self.query(sim)[0] if sim else self._first_n()
        out = {k: np.empty(n, np.uint32) for k in ("keys", "index")}
        out.update({k: np.empty(n, np.int32) for k in ("cell_x", "cell_y")})
        out["offsets"] = np.empty(int(table_size), np.uint32)
        self._check(lib().ge_sph_grid(self._h, int(sim), float(cell_size), int(table_size), n,
                                      *(_ptr(out[k]) for k in ("keys", "index", "cell_x",
                                                                "cell_y", "offsets"))))
        return out

    def _first_n(self):
        hs = self.sims()
        return self.query(hs[0])[0] if hs else self.n

    def upload_temp(self, temp):
        t = np.ascontiguousarray(temp, np.float32)
        self._check(lib().ge_upload_temp(self._h, _ptr(t)))

    def download_temp(self):
        t = np.empty(self.n, np.float32)
        self._check(lib().ge_download_temp(self._h, _ptr(t)))
        return t

    def download_prev_vel(self):
        n = self.n
        pv = [np.empty(n, np.float32) for _ in range(self.dims)]
        self._check(lib().ge_download_prev_vel(self._h, _ptr(pv[0]), _ptr(pv[1]),
                                               _ptr(pv[2]) if self.dims == 3 else None))
        return pv

    # -- the step ---------------------------------------------------------
    def step(self, nsteps=1):
        self._check(lib().ge_step(self._h, int(nsteps)))

    def profile_step(self):
        self._check(lib().ge_profile_step(self._h))
        return list(self.stats().stage_ms)

    def frame_host(self, state):
        """One frame on host arrays (modified in place; Morton order on return)."""
        g = state.get
        for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m"):
            if g(k) is not None:
                assert state[k].dtype == np.float32 and state[k].flags.c_contiguous
        n = len(state["x"])
        self._check(lib().ge_frame_host(self._h, n, _ptr(g("x")), _ptr(g("y")), _ptr(g("z")),
                                        _ptr(g("vx")), _ptr(g("vy")), _ptr(g("vz")),
                                        _ptr(g("ax")), _ptr(g("ay")), _ptr(g("az")),
                                        _ptr(g("m")), _ptr(g("id"))))
        self.n = n

    # -- stage calls mirroring the reference surface ------------------------
    def integrate_start(self):
        self._check(lib().ge_integrate_start(self._h))

    def bounding_box(self):
        out = np.zeros(4, np.float32)
        self._check(lib().ge_bounding_box(self._h, _ptr(out)))
        return out[: (3 if self.dims == 2 else 4)]

    def compute_morton_keys(self):
        keys = np.zeros(self.n, np.uint64)
        self._check(lib().ge_compute_morton_keys(self._h, _ptr(keys)))
        return keys

    def sort_particles_by_morton_key(self):
        perm = np.zeros(self.n, np.uint32)
        self._check(lib().ge_sort_by_morton_key(self._h, _ptr(perm)))
        return perm

    def build_tree(self):
        self._check(lib().ge_build_tree(self._h))

    def calculate_force_from_grid(self):
        self._check(lib().ge_compute_forces(self._h))

    def integrate_end(self):
        self._check(lib().ge_integrate_end(self._h))

    def count_interactions(self, enable=True):
        self._check(lib().ge_set_count_interactions(self._h, 1 if enable else 0))

    def set_sort_wait_test(self, spin_limit=0, withhold=False):
        """Test hook of the bounded waits (ge_set_sort_wait_test): cap the
        sort's look-back polls, and make the first tile withhold its counts
        so that the waits run out (the next sort returns GE_ERR_TIMEOUT)."""
        self._check(lib().ge_set_sort_wait_test(self._h, int(spin_limit), 1 if withhold else 0))

    def direct_sum_f64(self, idx):
        """FP64 direct-sum accelerations of the particles at indices idx of the
        current order (the accuracy reference)."""
        idx = np.ascontiguousarray(idx, np.uint32)
        out = [np.zeros(len(idx), np.float64) for _ in range(self.dims)]
        self._check(lib().ge_direct_sum_f64(self._h, len(idx), _ptr(idx), _ptr(out[0]),
                                            _ptr(out[1]), _ptr(out[2]) if self.dims == 3 else None))
        return out

    def build_timeline(self):
        """Device time (ns) at each grid barrier of the last tree build."""
        ns = np.zeros(256, np.uint64)
        cnt = C.c_int32(0)
        self._check(lib().ge_build_timeline(self._h, 256, _ptr(ns), C.byref(cnt)))
        return ns[: cnt.value].copy()

    def energy_f64(self):
        """(kinetic, potential, total) in FP64 (mixed mode, group walk)."""
        out = np.zeros(3, np.float64)
        self._check(lib().ge_energy_f64(self._h, _ptr(out)))
        return tuple(float(v) for v in out)

    def sums_f64(self):
        """{kinetic energy, p_x, p_y, p_z, total mass} in FP64."""
        out = np.zeros(5, np.float64)
        self._check(lib().ge_sums_f64(self._h, _ptr(out)))
        return out

    def export_tree(self):
        """The tree as the reference's globalNodes: pre-order numpy arrays."""
        cnt = C.c_int64(0)
        st = self.stats()
        cap = int(st.nodes) + 1
        d, q = self.dims, 1 << self.dims
        out = dict(pos=np.zeros((cap, d), np.float32), size=np.zeros(cap, np.float32),
                   com=np.zeros((cap, d), np.float32), mass=np.zeros(cap, np.float32),
                   start=np.zeros(cap, np.uint32), end=np.zeros(cap, np.uint32),
                   next=np.zeros(cap, np.uint32), child=np.zeros((cap, q), np.uint32))
        self._check(lib().ge_export_tree(self._h, cap, C.byref(cnt), _ptr(out["pos"]),
                                         _ptr(out["size"]), _ptr(out["com"]), _ptr(out["mass"]),
                                         _ptr(out["start"]), _ptr(out["end"]), _ptr(out["next"]),
                                         _ptr(out["child"])))
        k = cnt.value
        return {a: v[:k] for a, v in out.items()}


def aos_layout(dims):
    """The reference's record layout (ge_aos_layout_default)."""
    L = AosLayout()
    lib().ge_aos_layout_default(C.byref(L), dims)
    return L


def estimate_bytes(params, n, sims=1):
    """Device bytes of a context with these parameters after reserve(n, sims)."""
    b = C.c_int64(0)
    rc = lib().ge_estimate_bytes(C.byref(params), int(n), int(sims), C.byref(b))
    if rc != 0:
        raise GeError(rc, "ge_estimate_bytes failed")
    return b.value


class Server:
    """Continuous-batching server (ge_server): requests are simulations with a
    step count, run in a 2D and a 3D pool sized from an HBM budget."""

    def __init__(self, hbm_budget_bytes, params2d=None, params3d=None, frac_2d=0.5,
                 max_sims=1024):
        cfg = ServerConfig()
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.frac_2d = float(frac_2d)
        cfg.max_sims = int(max_sims)
        cfg.params[0] = params2d if params2d is not None else default_params(2)
        cfg.params[1] = params3d if params3d is not None else default_params(3)
        h = _vp()
        rc = lib().ge_server_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise GeError(rc, "ge_server_create failed")
        self._h = h
        self._keep = {}

    def _check(self, rc):
        if rc != 0:
            msg = lib().ge_server_last_error(self._h)
            raise GeError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            lib().ge_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, state, steps):
        """Queue a simulation (dict as Simulation.upload; 3D when it has z)."""
        g = state.get
        dims = 3 if g("z") is not None else 2
        a = {k: _f32(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        rid = C.c_int64(0)
        self._check(lib().ge_server_submit(self._h, dims, len(a["x"]), _ptr(a["x"]), _ptr(a["y"]),
                                           _ptr(a["z"]), _ptr(a["vx"]), _ptr(a["vy"]),
                                           _ptr(a["vz"]), _ptr(a["m"]), int(steps), C.byref(rid)))
        self._keep[rid.value] = (dims, len(a["x"]))
        return rid.value

    def start(self):
        self._check(lib().ge_server_start(self._h))

    def stop(self):
        self._check(lib().ge_server_stop(self._h))

    def poll(self):
        st = C.c_int32(0)
        self._check(lib().ge_server_poll(self._h, C.byref(st)))
        return bool(st.value)

    def wait(self, rid, timeout_s=600.0):
        self._check(lib().ge_server_wait(self._h, int(rid), float(timeout_s)))

    def status(self, rid):
        st, done, lat = C.c_int32(0), C.c_int32(0), C.c_double(0)
        self._check(lib().ge_server_status(self._h, int(rid), C.byref(st), C.byref(done),
                                           C.byref(lat)))
        return st.value, done.value, lat.value

    def take(self, rid):
        dims, n = self._keep.pop(rid)
        out = {k: np.empty(n, np.float32) for k in ("x", "y", "vx", "vy", "ax", "ay", "m")}
        if dims == 3:
            for k in ("z", "vz", "az"):
                out[k] = np.empty(n, np.float32)
        out["id"] = np.empty(n, np.uint32)
        g = out.get
        self._check(lib().ge_server_take(
            self._h, int(rid), *[_ptr(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay",
                                                       "az", "m", "id")]))
        return out

    def stats(self):
        s = ServerStats()
        self._check(lib().ge_server_get_stats(self._h, C.byref(s)))
        return s


def load_save(path):
    """A Galaxy Engine scene file (SaveSystem, versions 190 / 180) as a dict of
    arrays for Simulation.upload (+ "temp", "pinned"), plus "dims"."""
    info = SaveInfo()
    p = os.fsencode(path)
    rc = lib().ge_save_read_info(p, C.byref(info))
    if rc != 0:
        raise GeError(rc, f"cannot read scene file {path}")
    n, d = int(info.n), int(info.dims)
    keys = ["x", "y", "vx", "vy", "ax", "ay", "m", "temp"] + (["z", "vz", "az"] if d == 3 else [])
    out = {k: np.zeros(n, np.float32) for k in keys}
    out["id"] = np.zeros(n, np.uint32)
    out["pinned"] = np.zeros(n, np.uint8)
    g = out.get
    rc = lib().ge_save_read(p, n, *[_ptr(g(k)) for k in ("x", "y", "z", "vx", "vy", "vz", "ax",
                                                          "ay", "az", "m", "temp", "id",
                                                          "pinned")])
    if rc != 0:
        raise GeError(rc, f"cannot read scene file {path}")
    out["dims"] = d
    return out
