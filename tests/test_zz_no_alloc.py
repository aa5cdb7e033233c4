"""feb_cell_stress_noalloc: the stress entry point for callers that cannot allocate device memory when they
call it (fixed memory arenas, plugin enqueue callbacks, latency-critical loops).  Its scratch lives in a
static device array, so it must give the same results as feb_cell_stress, call after call, even though
every call reuses (and overwrites) the same scratch.

This file is collected last on purpose: a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

from comech_b200 import _lib
from comech_b200.engine import _grid_struct
from comech_b200.grid import Grid

pytestmark = pytest.mark.gpu


def _stress_both(g, mat_mode, mat, U, cells, cn, nan_to_zero):
    import torch
    lib = _lib.load()
    n = len(cells)
    dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
    matd, Ud, cd = dev(mat, np.float64), dev(U.ravel(), np.float64), dev(cells, np.int64)
    cnd = dev(cn, np.int64) if cn is not None else None
    gs = _grid_struct(g)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = []
    for fn in (lib.feb_cell_stress, lib.feb_cell_stress_noalloc):
        sig = torch.full((n, 6), np.nan, dtype=torch.float64, device="cuda")
        vm = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        eps = torch.full((n, 6), np.nan, dtype=torch.float64, device="cuda")
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)
        _lib.check(fn(C.byref(gs), mat_mode, p(matd), p(Ud), n, p(cd), p(cnd), nan_to_zero, p(sig), p(vm), p(eps),
                      stream))
        torch.cuda.synchronize()
        out.append((sig.cpu().numpy(), vm.cpu().numpy(), eps.cpu().numpy()))
    return out


def _close(a, b):
    tol = 1e-12 * max(np.abs(b).max(), 1e-300)
    np.testing.assert_allclose(a, b, rtol=0, atol=tol)


def test_noalloc_stress_matches_allocating_entry_point_twice(golden):
    # first call: split-node hindfoot (SRI isotropic material, split connectivity, NaN on unused nodes)
    z = golden("hindfoot_small")
    g = Grid(z["xe"], z["ye"], z["ze"])
    cells = np.flatnonzero(z["active"])
    ref, got = _stress_both(g, _lib.MAT_ISO_SRI, np.concatenate([z["lam"], z["mu"]]), z["U"], cells, z["cn"], 1)
    for a, b in zip(got, ref):
        _close(a, b)
    _close(got[1], z["vm"])
    # second call right after, on a different grid and material model, overwriting the shared scratch
    zb = golden("block_small")
    gb = Grid(zb["xe"], zb["ye"], zb["ze"])
    cb = np.arange(gb.ncell)
    ref, got = _stress_both(gb, _lib.MAT_ORTHO, zb["coeffs"], zb["U_pen"], cb, None, 0)
    for a, b in zip(got, ref):
        _close(a, b)
    _close(got[1], zb["vm_pen"])


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = _lib.load()
    e = np.linspace(0.0, 1.0, 4098)
    small = np.linspace(0.0, 1.0, 3)
    gs = _lib.FebGrid(4097, 2, 2, e.ctypes.data, small.ctypes.data, small.ctypes.data)
    dummy = C.c_void_p(8)   # never dereferenced: the size check comes first
    code = lib.feb_cell_stress_noalloc(C.byref(gs), 0, dummy, dummy, 1, dummy, None, 0, dummy, dummy, None, None)
    assert code == _lib.FEB_OK - 1
    assert b"4096" in lib.feb_last_error()
