"""CPU-side checks of the C ABI boundary: the library loads and exports every declared entry point, and the
host-side structures match the header.  No compute call is made (no GPU here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from comech_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "feb200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"FEB_API\s+[\w\s\*]+?\b(feb_\w+)\s*\(", txt)))


def test_header_declares_the_binding_list():
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name), name


def test_default_options_and_errors():
    o = _lib.default_options()
    assert o.precision == 0 and o.maxiter == 800 and abs(o.tol - 1e-6) < 1e-18
    assert o.min_dofs == 6000 and o.max_levels == 6 and o.cheb_degree == 3
    lib = _lib.load()
    # argument validation runs on the host and must not touch a device
    h = C.c_void_p()
    assert lib.feb_create(None, None, None, None, C.byref(h)) == -1
    assert b"null" in lib.feb_last_error()
    assert lib.feb_solve(None, None, None, None, None) == -1
    assert lib.feb_destroy(None) == 0
    with pytest.raises(_lib.FebError):
        _lib.check(-1)


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """ctypes field offsets == offsetof() of the header compiled by the C compiler."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    from comech_b200 import labels
    structs = [_lib.FebGrid, _lib.FebOperator, _lib.FebOptions, _lib.FebInfo, _lib.FebNetGrid, _lib.FebConv,
               _lib.FebWgrad, labels.FebLabelFacet, labels.FebLabelGrown, labels.FebLabelParams]
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for st in structs:
        lines.append(f'printf("{st.__name__} %zu\\n", sizeof({st.__name__}));')
        for f in st._fields_:
            lines.append(f'printf("{st.__name__}.{f[0]} %zu\\n", offsetof({st.__name__}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if l)
    for st in structs:
        assert int(got[st.__name__]) == C.sizeof(st), st.__name__
        for f in st._fields_:
            assert int(got[f"{st.__name__}.{f[0]}"]) == getattr(st, f[0]).offset, (st.__name__, f[0])


def test_engine_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from comech_b200 import engine
    g = type("G", (), dict(xe=np.arange(3.0), ye=np.arange(3.0), ze=np.arange(3.0), nx=2, ny=2, nz=2))()
    with pytest.raises(RuntimeError, match="CUDA"):
        engine.solve_cn(g, np.ones(8), np.ones(8), np.ones(8, bool), np.zeros((8, 8), np.int64), np.arange(27),
                        (np.zeros(0, np.int64), np.zeros(0)), [])


def test_every_export_has_argtypes():
    """Integer arguments past the sixth travel on the stack: without argtypes ctypes would pass a 32-bit int
    into a 64-bit slot.  Every binding declares its argument types."""
    lib = _lib.load()
    for name in _lib.EXPORTS:
        assert getattr(lib, name).argtypes is not None, name
    assert len(lib.feb_sample_cells.argtypes) == 24
