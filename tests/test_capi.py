"""The C ABI library loads and exports every function include/cg2d.h declares; struct layouts agree (no GPU)."""

import ctypes
import re
from pathlib import Path

import pytest

from mit_jax_b200 import capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "cg2d.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]*?\b(cg2d_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_bound_functions():
    decl = declared_functions()
    assert set(capi.EXPORTED) <= set(decl), set(capi.EXPORTED) - set(decl)


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts():
    assert ctypes.sizeof(capi.Params) == 56
    assert capi.Params.stages.offset == 52
    assert capi.Params.unit_deal.offset == 48
    assert ctypes.sizeof(capi.Diag) == 48
    assert ctypes.sizeof(capi.Group) == 8 + 4 + 4 + 6 * 8 + 8 + 8 + 5 * 16 + 16 + 8


def test_default_params_and_status_strings():
    p = capi.default_params()
    assert (p.precision, p.sum_order, p.rows_per_block, p.replace_every) == (0, 0, 8, 25)
    assert p.replace_above == 100.0 and p.timeout_s == 10.0
    lib = capi.lib()
    assert lib.cg2d_status_string(capi.CG2D_BARRIER_TIMEOUT).startswith(b"grid-wide wait")


def test_bad_arguments_are_rejected_without_a_gpu():
    lib = capi.lib()
    out = ctypes.c_void_p()
    assert lib.cg2d_topology_create(0, 8, 1, 1, 13, None, None, ctypes.byref(out)) == capi.CG2D_BAD_ARG
    g = (capi.Group * 1)()
    assert lib.cg2d_workspace_size(g, 1, None) == 0          # no topology
    assert lib.cg2d_solve_groups(g, 0, None, None, 0, None) == capi.CG2D_BAD_ARG


def test_newer_entry_points_reject_bad_arguments_without_a_gpu():
    """Null topologies, empty batches and missing outputs are refused before any device work."""
    lib = capi.lib()
    fs = capi.FreeSurf()
    fs.Nr = 5
    p15 = [None] * 15
    assert lib.cg2d_update_operator(None, 1, ctypes.byref(fs), 1.0, None, 0.51, *p15, None) == capi.CG2D_BAD_ARG
    assert lib.cg2d_pressure_rhs(None, 1, ctypes.byref(fs), *p15, None) == capi.CG2D_BAD_ARG
    assert lib.cg2d_pressure_post(None, 1, None, None, None, None, None) == capi.CG2D_BAD_ARG
    assert lib.cg2d_solve_exact_workspace_size(None, 1, 300, 8, 30) == 0
    assert lib.cg2d_solve_exact(None, 1, 1.0, None, *([None] * 8), 1e-12, 300, None, 8, 30, *([None] * 9), None, 0,
                                None) == capi.CG2D_BAD_ARG
    assert lib.cg2d_adjoint_ecco_workspace_size(None, 1, 300, None) == 0
    assert lib.cg2d_adjoint_ecco(None, 1, 1.0, None, *([None] * 8), 1e-13, 2000, 1, *([None] * 5), None, None, 0,
                                 None) == capi.CG2D_BAD_ARG
    assert lib.cg2d_adjoint_exact_workspace_size(None, 1, 300, 30) == 0


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """sizeof and every field offset of cg2d_params_t and cg2d_diag_t as gcc lays out include/cg2d.h."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    root = Path(__file__).resolve().parents[1]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cg2d.h"', 'int main(void) {']
    for cname, st in (("cg2d_params_t", capi.Params), ("cg2d_diag_t", capi.Diag)):
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in st._fields_:
            lines.append(f'  printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                         text=True).stdout.splitlines())
    for cname, st in (("cg2d_params_t", capi.Params), ("cg2d_diag_t", capi.Diag)):
        assert int(got[cname]) == ctypes.sizeof(st), cname
        for f, _ in st._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(st, f).offset, (cname, f)
