"""CPU: the C-ABI library loads, exports every symbol include/ge_bh.h declares,
and refuses to run without a GPU (there is no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "ge_bh.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ge_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for need in ("ge_create", "ge_destroy", "ge_step", "ge_upload", "ge_download",
                 "ge_bounding_box", "ge_compute_morton_keys", "ge_sort_by_morton_key",
                 "ge_build_tree", "ge_compute_forces", "ge_integrate_start",
                 "ge_integrate_end", "ge_export_tree", "ge_frame_host"):
        assert need in names


def test_library_exports_every_declared_symbol(ge):
    L = ge.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert sorted(ge.SIGNATURES) == declared_functions()


def test_abi_version_and_defaults(ge):
    assert ge.lib().ge_abi_version() == 1
    p = ge.default_params(2)
    assert p.dims == 2 and abs(p.theta - 0.8) < 1e-7 and abs(p.eps2 - 2.25) < 1e-6
    assert p.leaf_cap == 4 and p.size_gate == 2.0 and abs(p.dt - 0.045) < 1e-7
    p3 = ge.default_params(3)
    assert abs(p3.eps2 - 1.5) < 1e-6 and p3.node_cap_factor == 8.0
    assert p3.direct_below == 0 and abs(p3.direct_eps2 - 1.5) < 1e-6
    p = ge.default_params(2, softening=0.01, theta=0.7)
    assert abs(p.eps2 - 1e-4) < 1e-10 and abs(p.theta - 0.7) < 1e-7
    assert abs(p.direct_eps2 - 0.01) < 1e-9   # the direct sum adds softening un-squared


def test_struct_layouts_match_header(ge):
    # ge_params: 11 scalars + domain[3] + track_prev_vel, group_size, temp_enabled,
    # heat_cond, direct_below, direct_eps2 + reserved[2]
    assert C.sizeof(ge.Params) == 4 * (11 + 3 + 1 + 1 + 2 + 2 + 2)
    # ge_stats: 84 bytes of fields, padded to the 8-byte alignment of its int64 members
    assert C.sizeof(ge.Stats) == 88


def test_struct_layouts_match_c_compiler(ge, tmp_path):
    """sizeof / offsetof of every ABI struct as the C compiler lays it out
    against the ctypes mirrors."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    structs = {"ge_params": ge.Params, "ge_stats": ge.Stats,
               "ge_server_config": ge.ServerConfig, "ge_server_stats": ge.ServerStats,
               "ge_tune_result": ge.TuneResult, "ge_save_info": ge.SaveInfo,
               "ge_field_params": ge.FieldParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ge_bh.h"', 'int main(void) {']
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-I", inc, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU refusal")
def test_no_cpu_fallback_without_gpu(ge):
    with pytest.raises(ge.GeError) as ei:
        ge.Simulation(ge.default_params(2))
    assert ei.value.code == 2    # GE_ERR_NO_DEVICE


def test_invalid_params_rejected(ge):
    L = ge.lib()
    p = ge.default_params(2)
    p.dims = 4
    h = C.c_void_p()
    assert L.ge_create(C.byref(p), C.byref(h)) == 1
    p = ge.default_params(2)
    p.leaf_cap = 0
    assert L.ge_create(C.byref(p), C.byref(h)) == 1
