"""CPU tests of the C ABI boundary: the library loads, exports every entry point
include/smokesim.h declares, rejects bad arguments with status codes (no GPU
is touched on those paths) and reports the reference's defaults."""
import ctypes as C
import os
import re
import subprocess

import pytest

from smokesim_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "smokesim.h")


@pytest.fixture(scope="module")
def L():
    return abi.lib()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ss_[a-z0-9_]+)\s*\(", src)))


def test_header_and_exports(L):
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), f"libsmokesim.so does not export {n}"
    assert set(abi.EXPORTED) <= set(names)


def test_abi_version_and_strerror(L):
    assert L.ss_abi_version() == 1
    assert L.ss_strerror(abi.SS_E_INVALID) == b"invalid argument"
    assert L.ss_strerror(abi.SS_E_NOT_CONVERGED).startswith(b"pressure solve")
    assert L.ss_strerror(12345) == b"unknown status"


def test_struct_layouts_match_header(tmp_path):
    """Compile the header with the system C compiler and compare sizeof/offsetof
    of every ABI struct with the ctypes mirror."""
    structs = {"ss_desc": abi.Desc, "ss_emitter": abi.Emitter, "ss_obstacle": abi.Obstacle, "ss_box": abi.Box,
               "ss_mg_schedule": abi.MGSchedule, "ss_params": abi.Params, "ss_stats": abi.Stats,
               "ss_render_desc": abi.RenderDesc}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True, env=env)
    out = subprocess.run([str(exe)], check=True, stdout=subprocess.PIPE, text=True).stdout.split("\n")
    got = dict(l.split() for l in out if l.strip())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_default_params_are_reference_defaults(L):
    p = abi.Params()
    L.ss_default_params(C.byref(p))
    # common/physics/physics.c:7-20 and grid.c:179-180
    assert abs(p.time_step - 1 / 120) < 1e-9
    assert p.density == 1.0 and p.t_ambient == 293.0
    assert abs(p.t_weight_coeff - 0.07) < 1e-7 and p.t_temp_coeff == 1.0 and p.vorticity_confinement == 1.0
    assert (p.mg.n_pre, p.mg.n_post, p.mg.n_coarse, p.mg.n_vcycles) == (16, 16, 80, 1)
    assert p.mg.ref_quirks == 1 and p.stage_mask == abi.STAGE_ALL


@pytest.mark.parametrize("bad", [
    dict(dim=4, n=(8, 8, 8)),
    dict(dim=3, n=(2, 8, 8)),
    dict(dim=2, n=(8, 8, 4)),
    dict(dim=3, n=(8, 8, 8), cell_size=0.0),
    dict(dim=3, n=(8, 8, 8), density_channels=2),
    dict(dim=3, n=(2048, 2048, 1024)),
])
def test_create_rejects_bad_desc(L, bad):
    d = abi.Desc()
    d.dim = bad["dim"]
    n = bad["n"]
    d.n[0], d.n[1], d.n[2] = n
    d.cell_size = bad.get("cell_size", 1.0)
    d.density_channels = bad.get("density_channels", 1)
    d.enclosed = 1
    d.min_coarse = 4
    h = C.c_void_p()
    rc = L.ss_create(C.byref(d), None, C.byref(h))
    assert rc == abi.SS_E_INVALID
    assert not h.value
    assert L.ss_last_error_message()


def test_nonfinite_desc(L):
    d = abi.make_desc(3, (8, 8, 8), t_ambient=float("nan"))
    h = C.c_void_p()
    assert L.ss_create(C.byref(d), None, C.byref(h)) == abi.SS_E_NONFINITE


def test_null_handles(L):
    assert L.ss_destroy(None) == abi.SS_E_INVALID
    p = abi.make_params()
    assert L.ss_run_physics_step(None, C.byref(p), 1, None) == abi.SS_E_INVALID
    assert L.ss_create(None, None, None) == abi.SS_E_INVALID
    s = abi.Stats()
    assert L.ss_get_stats(None, C.byref(s)) == abi.SS_E_INVALID
