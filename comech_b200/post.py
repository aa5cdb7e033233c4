"""Post-processing of a solve on the device, with the reference's entry points and results.

* ``region_forces_cn`` / ``forces_on`` -- the forces on a bone from each neighbouring region, rb/rbfe.py:194-213
* ``ground_fz``                        -- the vertical ground reaction split heel / mid / fore, rb/rbfe.py:214-219
* ``rigid_fit``                        -- rb/rbsim.py:99-107
* ``relative_displacement``            -- the displacement relative to a rigid fit, rb/rbsim.py:183-186
* ``sample_fe``                        -- rb/rbsim.py:110-138 (also sets ``sample_fe.sig`` like the reference)
* ``sample_nodes`` / ``nearest_active`` -- rb/rbsim.py:141-161 (nearest active cell by an exact Euclidean
                                        feature transform on the device)

Inputs are NumPy arrays (or CUDA tensors); the work runs in libfeb200.so.  No CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _lib
from .engine import _dev, _grid_struct, _host, _ptr, _stream, _torch


def region_forces_cn(g, lam, mu, U, cn, active, part, lab, nlab, target):
    """Minus the nodal forces that every active cell outside part ``target`` exerts on the nodes of the active
    cells of that part, summed per cell label ``lab`` (0..nlab-1).  Returns (forces (nlab, 3), present (nlab,)):
    ``present[i]`` is True when some contributing cell has label i (the reference lists only those)."""
    torch = _torch()
    ncell = g.nx * g.ny * g.nz
    mat = _dev(np.concatenate([np.asarray(lam, np.float64).ravel(), np.asarray(mu, np.float64).ravel()]), np.float64)
    Ud = _dev(np.asarray(U, np.float64).reshape(-1), np.float64)
    cnd = _dev(np.asarray(cn, np.int64), np.int64) if cn is not None else None
    act = _dev(np.asarray(active, bool).view(np.uint8), np.uint8)
    pt = _dev(np.asarray(part), np.int32)
    lb = _dev(np.asarray(lab), np.int32)
    if pt.numel() != ncell or lb.numel() != ncell:
        raise ValueError("part and lab need one entry per cell")
    out = torch.empty(3 * int(nlab), dtype=torch.float64, device="cuda")
    present = torch.empty(int(nlab), dtype=torch.int32, device="cuda")
    gs = _grid_struct(g)
    nnode_total = Ud.numel() // 3
    _lib.check(_lib.load().feb_region_forces(C.byref(gs), _ptr(mat), _ptr(Ud), _ptr(cnd), _ptr(act), _ptr(pt), _ptr(lb),
                                             int(nlab), int(target), nnode_total, _ptr(out), _ptr(present), _stream()))
    F, p = _host(out.view(int(nlab), 3), present)
    return F, p.astype(bool)


def forces_on(g, lam, mu, U, cn, active, part, lab, names, target):
    """The engine's ``res[f"F_on_{bone}"]`` (rb/rbfe.py:211-213): {region name: [Fx, Fy, Fz]} rounded to 0.01,
    for the regions that touch the bone."""
    F, present = region_forces_cn(g, lam, mu, U, cn, active, part, lab, len(names), target)
    return {nm: [round(float(x), 2) for x in F[i]] for i, nm in enumerate(names) if present[i]}


def ground_fz(R, x, x_heel, x_fore):
    """Vertical ground reaction by region of the node x coordinate (rb/rbfe.py:214-219)."""
    R = np.asarray(R)
    x = np.asarray(x)
    return {"heel": round(float(R[x < x_heel, 2].sum()), 2),
            "mid": round(float(R[(x >= x_heel) & (x < x_fore), 2].sum()), 2),
            "fore": round(float(R[x >= x_fore, 2].sum()), 2)}


def rigid_fit(X, U):
    """Least-squares rigid motion of points X with displacements U: U ~ t + w x (X - c) (rb/rbsim.py:99-107).
    Returns (t, w, c)."""
    torch = _torch()
    Xd = _dev(np.asarray(X, np.float64).reshape(-1, 3), np.float64)
    Ud = _dev(np.asarray(U, np.float64).reshape(-1, 3), np.float64)
    n = Xd.shape[0]
    if Ud.shape[0] != n or n < 1:
        raise ValueError("X and U need the same number of points (>= 1)")
    fit = np.zeros(9)
    _lib.check(_lib.load().feb_rigid_fit(_ptr(Xd), _ptr(Ud), n, fit.ctypes.data_as(C.c_void_p), _stream()))
    torch.cuda.current_stream().synchronize()
    return fit[:3].copy(), fit[3:6].copy(), fit[6:9].copy()


def relative_displacement(g, orig, U, t, w, c):
    """nan_to_num(U) - (t + w x (X - c)) at every node id, X the node coordinates (copies at their grid node)."""
    Ud = _dev(np.asarray(U, np.float64).reshape(-1), np.float64)
    nnode_total = Ud.numel() // 3
    origd = _dev(np.asarray(orig, np.int64), np.int64) if orig is not None else None
    out = _torch().empty_like(Ud)
    fit = np.ascontiguousarray(np.concatenate([t, w, c]).astype(np.float64))
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_relative_displacement(C.byref(gs), _ptr(origd), nnode_total, _ptr(Ud),
                                                     fit.ctypes.data_as(C.c_void_p), _ptr(out), _stream()))
    return _host(out.view(nnode_total, 3))


def _axis_samples(fe_edges, ml_edges, sub):
    # per analysis-grid axis: sample points, the FE cell holding each, local coordinate, inside flag
    # (rb/rbsim.py:112-119; host arithmetic on a few hundred points, the same float operations)
    oo = (np.arange(sub) + 0.5) / sub
    X = (ml_edges[:-1, None] + np.diff(ml_edges)[:, None] * oo).ravel()
    n = len(fe_edges) - 1
    i = np.clip(np.searchsorted(fe_edges, X) - 1, 0, n - 1)
    t = np.clip((X - fe_edges[i]) / np.diff(fe_edges)[i], 0, 1)
    inside = (X >= fe_edges[0]) & (X <= fe_edges[-1])
    return i.astype(np.int32), t.astype(np.float64), inside.astype(np.uint8)


def sample_fe(o, grid_ml, Urel, sub=2):
    """Mean von Mises stress and relative displacement of every analysis cell over its sub^3 points that fall in
    active FE cells, and the fraction of such points (rb/rbsim.py:110-138).  ``o``: g, cn, active, VM, SIG.
    Returns (vm, u, frac) as float32 like the reference and sets ``sample_fe.sig`` (mean stress)."""
    torch = _torch()
    g = o["g"]
    axes = [_axis_samples(np.asarray(e, np.float64), np.asarray(m, np.float64), sub)
            for e, m in zip((g.xe, g.ye, g.ze), (grid_ml.xe, grid_ml.ye, grid_ml.ze))]
    dev_axes = []
    for i, t, ins in axes:
        dev_axes += [_dev(i, np.int32), _dev(t, np.float64), _dev(ins, np.uint8)]
    mx, my, mz = (len(e) - 1 for e in (grid_ml.xe, grid_ml.ye, grid_ml.ze))
    ncm = mx * my * mz
    cn = _dev(np.asarray(o["cn"], np.int64), np.int64) if o.get("cn") is not None else None
    act = _dev(np.asarray(o["active"], bool).view(np.uint8), np.uint8)
    Ud = _dev(np.asarray(Urel, np.float64).reshape(-1), np.float64)
    VM = _dev(np.asarray(o["VM"], np.float32), np.float32)
    SIG = _dev(np.asarray(o["SIG"], np.float32).reshape(-1), np.float32)
    vm = torch.empty(ncm, dtype=torch.float32, device="cuda")
    u = torch.empty(3 * ncm, dtype=torch.float32, device="cuda")
    frac = torch.empty(ncm, dtype=torch.float32, device="cuda")
    sig = torch.empty(6 * ncm, dtype=torch.float32, device="cuda")
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_sample_cells(C.byref(gs), mx, my, mz, int(sub), *[_ptr(a) for a in dev_axes], _ptr(cn),
                                            _ptr(act), _ptr(Ud), _ptr(VM), _ptr(SIG), _ptr(vm), _ptr(u), _ptr(frac),
                                            _ptr(sig), _stream()))
    vm_h, u_h, frac_h, sig_h = _host(vm, u.view(ncm, 3), frac, sig.view(ncm, 6))
    sample_fe.sig = sig_h
    return vm_h, u_h, frac_h


def nearest_active(g, active):
    """Cell id of the nearest active cell of every cell (exact Euclidean feature transform over cell indices,
    ties as scipy.ndimage.distance_transform_edt; -1 when no cell is active), as a device int32 tensor."""
    torch = _torch()
    act = _dev(np.asarray(active, bool).view(np.uint8).ravel(), np.uint8)
    ft = torch.empty(g.nx * g.ny * g.nz, dtype=torch.int32, device="cuda")
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_nearest_active(C.byref(gs), _ptr(act), _ptr(ft), _stream()))
    return ft


def sample_nodes(o, grid_ml, Urel):
    """Relative displacement at the nodes of the analysis grid: trilinear in the FE cell that holds the node,
    or in the nearest active FE cell with clamped local coordinates (rb/rbsim.py:141-161).  float32, node order
    x fastest."""
    torch = _torch()
    g = o["g"]
    axes = []
    for fe, ml, n in ((g.xe, grid_ml.xe, g.nx), (g.ye, grid_ml.ye, g.ny), (g.ze, grid_ml.ze, g.nz)):
        P = np.asarray(ml, np.float64)
        i = np.clip(np.searchsorted(np.asarray(fe, np.float64), P) - 1, 0, n - 1).astype(np.int32)
        axes += [_dev(i, np.int32), _dev(P, np.float64)]
    m1 = [len(e) for e in (grid_ml.xe, grid_ml.ye, grid_ml.ze)]
    ft = nearest_active(g, o["active"])
    cn = _dev(np.asarray(o["cn"], np.int64), np.int64) if o.get("cn") is not None else None
    Ud = _dev(np.asarray(Urel, np.float64).reshape(-1), np.float64)
    out = torch.empty(3 * m1[0] * m1[1] * m1[2], dtype=torch.float32, device="cuda")
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_sample_nodes(C.byref(gs), *m1, *[_ptr(a) for a in axes], _ptr(ft), _ptr(cn), _ptr(Ud),
                                            _ptr(out), _stream()))
    return _host(out.view(-1, 3))
