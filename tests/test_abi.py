"""The C ABI, checked without a GPU: the library loads, exports every function include/sdot_b200.h declares,
and the ctypes mirrors of its structs have the header's sizes and offsets (gcc compiles the header here)."""
import ctypes
import os
import re
import subprocess

import pytest

from sdot import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sdot_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sdot_[a-z_0-9]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 18
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert L.sdot_abi_version() == 1


STRUCTS = {
    "sdot_status": (_lib.Status, ["code", "kind", "id", "value", "needed", "message"]),
    "sdot_density": (_lib.Density, ["kind", "value", "shape", "origin", "step", "values", "count", "centres", "sigmas", "masses"]),
    "sdot_diagram_desc": (_lib.DiagramDesc, ["dim", "n", "positions", "weights", "box_lo", "box_hi", "density", "memory"]),
    "sdot_cells_out": (_lib.CellsOut, ["masses", "barycentres", "costs", "cap", "nb_count", "nb_ids", "nb_coef", "nb_measure", "precision"]),
    "sdot_solve_desc": (_lib.SolveDesc, ["diagram", "nu", "options"]),
    "sdot_solve_out": (_lib.SolveOut, ["weights", "masses", "barycentres", "cost", "stats", "history", "cap_history", "nb_history"]),
    "sdot_server_config": (_lib.ServerConfig, ["device", "memory_budget", "max_active"]),
}


def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append('printf("SDOT_NB_OPTIONS %d\\n", (int)SDOT_NB_OPTIONS);')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        parts = line.split()
        if len(parts) == 3:
            got[(parts[0], parts[1])] = int(parts[2])
        elif len(parts) == 2:
            got[parts[0]] = int(parts[1])
    assert got["SDOT_NB_OPTIONS"] == _lib.NB_OPTIONS
    for cname, (cls, fields) in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in fields:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)


def test_options_enum_order_matches_the_header():
    src = open(HEADER).read()
    body = src[src.index("enum sdot_option {"): src.index("SDOT_NB_OPTIONS\n")]
    names = [m.lower() for m in re.findall(r"SDOT_OPT_([A-Z_0-9]+)", body)]
    assert names == _lib.OPTIONS


def test_calls_fail_loudly_without_a_device():
    """no CPU fallback: without a CUDA device the context cannot be made and the error says why"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = _lib.load()
    h = ctypes.c_void_p()
    st = _lib.Status()
    code = L.sdot_context_create(0, 0, ctypes.byref(h), ctypes.byref(st))
    assert code == _lib.SDOT_ERR_CUDA
    assert st.message


def test_the_counters_and_the_moments_adjoint_refuse_null_arguments():
    """argument checks that come before any device work: a null context, a missing output, a dimension other than 2 or 3,
    an adjoint with neither cotangent"""
    L = _lib.load()
    counts = (ctypes.c_uint64 * 5)()
    assert L.sdot_context_set_counters(None, 1) == _lib.SDOT_ERR_ARGS
    assert L.sdot_context_gather_counters(None, 2, counts, 0) == _lib.SDOT_ERR_ARGS
    st = _lib.Status()
    desc = _lib.DiagramDesc()
    assert L.sdot_cells_vjp_moments(None, ctypes.byref(desc), None, None, None, None, ctypes.byref(st)) == _lib.SDOT_ERR_ARGS
    assert st.code == _lib.SDOT_ERR_ARGS and st.message


def _build_c_caller(tmp_path):
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "c_caller"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_caller.c"), "-o", str(exe), "-L", libdir, "-lsdot_b200",
                    f"-Wl,-rpath,{libdir}", "-lm"], check=True)
    return exe


def test_a_c_program_binds_the_library(tmp_path):
    """tests/c_caller.c, a plain C caller of the header (no Python in its process), compiles with gcc -std=c11
    -Wall -Werror and links against the library; without a device it reports the context's CUDA error and stops"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the solve itself is test_a_c_program_solves_on_the_device's")
    out = subprocess.run([str(_build_c_caller(tmp_path))], check=True, capture_output=True, text=True).stdout.split()
    assert out[0] == "context" and int(out[1]) == _lib.SDOT_ERR_CUDA, out


@pytest.mark.gpu
def test_a_c_program_solves_on_the_device(tmp_path):
    """the same plain C program on a GPU: its 2D solve of 2000 seeds through sdot_solve (host buffers) converges to the
    relative mass tolerance 1e-8, with the library's own kernels launched"""
    out = subprocess.run([str(_build_c_caller(tmp_path))], check=True, capture_output=True, text=True).stdout.split()
    assert out[0] == "solve", out
    code, status, worst, launches = int(out[1]), int(out[2]), float(out[3]), int(out[4])
    assert code == _lib.SDOT_OK and status == 1, out          # status 1: converged
    assert worst <= 1e-8, worst
    assert launches > 0, out
