"""GPU: the allocation-free 2D Morton sort (ge_morton_sort_2d_noalloc).

Callers that cannot allocate device memory (a fixed device-memory arena, a
frame loop that must not call cudaMalloc) pass their own device buffers and
the sort uses a fixed array inside the library.  Its result must equal the
context path's (ge_compute_morton_keys + ge_sort_by_morton_key) bit for bit,
also on a second call in a row, which finds the array holding the first
call's leftovers.  This file is collected last on purpose.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _context_result(ge, st):
    p = ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, leaf_cap=4, dt=1e-3)
    with ge.Simulation(p) as s:
        s.upload(st)
        keys = s.compute_morton_keys()
        perm = s.sort_particles_by_morton_key()
    return perm, keys[perm]


def _oracle_result(st):
    """The oracle's statement of the reference's box, keys and sort
    (globalLogic.cpp:1083-1099, morton.cpp:27-63), stable on equal keys."""
    import oracle as O
    bb = O.bbox(st["x"], st["y"])
    keys = O.morton_keys(st["x"], st["y"], bb)
    perm = O.sort_perm(keys)
    return perm, keys[perm]


def test_noalloc_sort_matches_context_path_twice_in_a_row(ge):
    import torch
    ics = importlib.import_module("galaxy-engine_b200.ics")
    L = ge.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # two different inputs, the larger at the size limit, one after the other
    for n, seed in ((ge.NOALLOC_MAX_N, 3), (100003, 4)):
        st = ics.two_disks2d(n, seed=seed)
        perm_ref, keys_ref = _context_result(ge, st)
        perm_or, keys_or = _oracle_result(st)
        assert np.array_equal(perm_ref, perm_or) and np.array_equal(keys_ref, keys_or), n
        x = torch.from_numpy(st["x"]).cuda()
        y = torch.from_numpy(st["y"]).cuda()
        perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        keys = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        for call in range(2):
            perm.fill_(-1)
            keys.fill_(-1)
            torch.cuda.synchronize()
            rc = L.ge_morton_sort_2d_noalloc(n, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                             C.c_void_p(perm.data_ptr()), C.c_void_p(keys.data_ptr()),
                                             C.c_void_p(stream))
            assert rc == 0, (n, call, rc)
            torch.cuda.synchronize()
            assert np.array_equal(perm.cpu().numpy().view(np.uint32), perm_ref), (n, call)
            assert np.array_equal(keys.cpu().numpy().view(np.uint64), keys_ref), (n, call)


def test_noalloc_sort_without_keys_output(ge):
    """d_keys is optional: a NULL keys pointer gives the same permutation."""
    import torch
    ics = importlib.import_module("galaxy-engine_b200.ics")
    n = 5000
    st = ics.disk2d(n, seed=9)
    perm_ref, _ = _context_result(ge, st)
    x = torch.from_numpy(st["x"]).cuda()
    y = torch.from_numpy(st["y"]).cuda()
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = ge.lib().ge_morton_sort_2d_noalloc(n, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                            C.c_void_p(perm.data_ptr()), None, C.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), perm_ref)


def test_noalloc_sort_rejects_sizes_beyond_the_limit(ge):
    import torch
    n = ge.NOALLOC_MAX_N + 1
    x = torch.zeros(n, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = ge.lib().ge_morton_sort_2d_noalloc(n, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                                            C.c_void_p(perm.data_ptr()), None, None)
    assert rc == 4   # GE_ERR_CAPACITY
