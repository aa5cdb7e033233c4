"""Host layer over libfeb200: the reference's solve entry points with their signatures and results.

* ``solve_cn``        -- rb/splitfe.py:123  (split-node engine solve; the engine's hot path)
* ``solve``           -- fe/solver.py:202   (single-connectivity solve: springs, loads, rank-1 penalties,
                                            orthotropic coefficients, rigid groups, warm start)
* ``cell_stress_cn``  -- rb/splitfe.py:161,  ``cell_stress`` -- fe/solver.py:257
* ``element_forces_cn`` -- rb/splitfe.py:178

Inputs arrive as NumPy arrays (the reference's types); they are copied to the current CUDA device with
torch (used only as the carrier of device memory and streams), the operator and the multigrid hierarchy
are built and solved by the C ABI of libfeb200.so, and the results come back as NumPy arrays.  There
is no CPU fallback: without a CUDA device or the library every call raises.

Extra keyword-only arguments (not in the reference): ``precision`` ('fp64', 'mixed', 'refine'),
``x0`` (warm start, full node layout), ``options`` (dict of FebOptions fields) and ``keep_device``
(return device tensors in ``info['device']`` for a following stress call without a round trip).
"""
import ctypes as C
import time

import numpy as np

from . import _lib
from .grid import CORNERS

K_GROUND = 1e6      # ground penalty per unit area of rb/splitfe.py:143


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("comech_b200 needs a CUDA device (no CPU fallback)")
    return torch


_TDT = {np.float64: "float64", np.int64: "int64", np.uint8: "uint8", np.float32: "float32", np.int32: "int32"}


def _dev(a, dtype):
    """Device tensor of ``a`` (CUDA tensors of the right dtype pass through untouched)."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        want = getattr(torch, _TDT[dtype])
        if a.is_cuda and a.dtype == want and a.is_contiguous():
            return a
        return a.to(device="cuda", dtype=want).contiguous()
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=dtype))
    return t.to("cuda", non_blocking=False)


def _dev_cat(arrays, dtype):
    """One device tensor of the arrays' concatenation, uploaded piece by piece (no host-side concatenation);
    the copies are asynchronous from page-locked sources, which the caller keeps until its stream is synchronised."""
    torch = _torch()
    parts = [a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a, dtype=dtype).ravel())
             for a in arrays]
    out = torch.empty(sum(int(p.numel()) for p in parts), dtype=getattr(torch, _TDT[dtype]), device="cuda")
    at = 0
    for p in parts:
        out[at:at + p.numel()].copy_(p.reshape(-1), non_blocking=True)
        at += p.numel()
    return out


def _host(*ts):
    """NumPy copies of device tensors through page-locked buffers (torch's caching host allocator reuses them
    once the arrays are released), one stream synchronisation for all of them."""
    torch = _torch()
    outs = []
    for t in ts:
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        outs.append(h)
    torch.cuda.current_stream().synchronize()
    return [h.numpy() for h in outs] if len(outs) > 1 else outs[0].numpy()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _grid_struct(g):
    xe, ye, ze = (np.ascontiguousarray(e, dtype=np.float64) for e in (g.xe, g.ye, g.ze))
    s = _lib.FebGrid(len(xe) - 1, len(ye) - 1, len(ze) - 1, xe.ctypes.data, ye.ctypes.data, ze.ctypes.data)
    s._keep = (xe, ye, ze)
    return s


def _options(precision, tol, maxiter, options):
    o = _lib.default_options()
    o.precision = _lib.PREC[precision]
    o.tol = float(tol)
    o.maxiter = int(maxiter)
    for k, v in (options or {}).items():
        setattr(o, k, v)
    return o


class Problem:
    """A level-0 operator on the device with its multigrid hierarchy (one FebHandle)."""

    def __init__(self, g, mat_mode, mat, active, cn=None, orig=None, pen_node=None, pen_k=None, extra_coo=None,
                 precision="fp64", tol=1e-6, maxiter=800, options=None, mark_used=None):
        _lib.load()
        torch = _torch()
        self.g = g
        self.grid = _grid_struct(g)
        self.ncell = g.nx * g.ny * g.nz
        self.nnode = (g.nx + 1) * (g.ny + 1) * (g.nz + 1)
        self.ntotal = len(orig) if orig is not None else self.nnode
        self.mat_mode = mat_mode
        self.mat = _dev(mat, np.float64)
        if isinstance(active, torch.Tensor):
            self.active = _dev(active, np.uint8)
        else:
            self.active = _dev(np.asarray(active, dtype=bool).view(np.uint8), np.uint8)
        self.cn = _dev(cn, np.int64) if cn is not None else None
        self.orig = _dev(orig, np.int64) if (orig is not None and self.ntotal > self.nnode) else None
        pen_node = np.ascontiguousarray(pen_node if pen_node is not None else np.zeros(0), dtype=np.int64)
        pen_k = np.ascontiguousarray(pen_k if pen_k is not None else np.zeros((0, 3)), dtype=np.float64)
        if extra_coo is None:
            er = ec = np.zeros(0, np.int64); ev = np.zeros(0)
        else:
            er, ec, ev = (np.ascontiguousarray(a, dtype=t) for a, t in zip(extra_coo, (np.int64, np.int64, np.float64)))
        mu = np.ascontiguousarray(mark_used if mark_used is not None else np.zeros(0), dtype=np.int64)
        op = _lib.FebOperator(mat_mode, self.mat.data_ptr(), self.active.data_ptr(),
                              self.cn.data_ptr() if self.cn is not None else None, self.ntotal,
                              self.orig.data_ptr() if self.orig is not None else None, len(pen_node),
                              pen_node.ctypes.data, pen_k.ctypes.data, len(ev), er.ctypes.data, ec.ctypes.data,
                              ev.ctypes.data, len(mu), mu.ctypes.data)
        self.opt = _options(precision, tol, maxiter, options)
        h = C.c_void_p()
        _lib.check(_lib.load().feb_create(C.byref(self.grid), C.byref(op), C.byref(self.opt), _stream(), C.byref(h)))
        self.h = h
        self.torch = torch

    def close(self):
        if getattr(self, "h", None):
            _lib.load().feb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_rigid_groups(self, node_groups, offsets=None):
        """node_groups: list of node-id arrays, or (with ``offsets``) one concatenated array / device tensor."""
        if node_groups is None or (offsets is None and len(node_groups) == 0):
            return
        if offsets is None:
            groups = [np.asarray(gr, dtype=np.int64) for gr in node_groups]
            off = np.zeros(len(groups) + 1, np.int64)
            off[1:] = np.cumsum([len(gr) for gr in groups])
            nodes = _dev(np.concatenate(groups), np.int64)
        else:
            off = np.ascontiguousarray(offsets, dtype=np.int64)
            groups = [None] * (len(off) - 1)
            nodes = _dev(node_groups, np.int64)
        _lib.check(_lib.load().feb_set_rigid_groups(self.h, len(groups), off.ctypes.data, _ptr(nodes)))

    def rhs(self, loads):
        """Nodal load vector (full layout) from (nodes, area, traction) lists (rb/splitfe.py:144-147), or from
        (nodes, values (n, 3)) pairs already on the device."""
        f = self.torch.zeros(3 * self.ntotal, dtype=self.torch.float64, device="cuda")
        for item in loads:
            if len(item) == 2:
                nd, vd = _dev(item[0], np.int64), _dev(item[1], np.float64)
                nodes = nd
            else:
                nodes, area, t = item
                nodes = np.asarray(nodes, dtype=np.int64)
                vals = np.asarray(area, dtype=np.float64)[:, None] * np.asarray(t, dtype=np.float64)[None, :]
                nd, vd = _dev(nodes, np.int64), _dev(vals, np.float64)
            _lib.check(_lib.load().feb_accumulate_nodal(len(nodes), _ptr(nd), _ptr(vd), _ptr(f), _stream()))
        return f

    def solve(self, f, x0=None):
        x = self.torch.empty_like(f)
        info = _lib.FebInfo()
        _lib.check(_lib.load().feb_solve(self.h, _ptr(f), _ptr(x0), _ptr(x), C.byref(info)))
        return x, info

    def precondition(self, r):
        """z = M r (one V-cycle plus the rigid-mode correction; FP64 full-layout device vectors)."""
        z = self.torch.empty_like(r)
        _lib.check(_lib.load().feb_precondition(self.h, _ptr(r), _ptr(z)))
        return z

    def apply(self, u):
        y = self.torch.empty_like(u)
        prec = 0 if u.dtype == self.torch.float64 else 1
        _lib.check(_lib.load().feb_apply(self.h, prec, _ptr(u), _ptr(y)))
        return y

    def export(self, x):
        U = self.torch.empty_like(x)
        _lib.check(_lib.load().feb_export_solution(self.h, _ptr(x), _ptr(U)))
        return U

    def used_mask(self):
        m = self.torch.empty(self.ntotal, dtype=self.torch.uint8, device="cuda")
        n = C.c_int64()
        _lib.check(_lib.load().feb_used_nodes(self.h, C.byref(n), _ptr(m)))
        return m, int(n.value)


def _info_dict(info, t0, extra=None):
    d = dict(iters=int(info.iters), flag=int(info.flag), relres=float(info.relres), levels=int(info.levels),
             ndof=int(info.ndof), sweeps=int(info.sweeps), t_setup=round(info.t_setup_ms / 1e3, 4),
             t_gpu=round(info.t_solve_ms / 1e3, 4), coarse="dense-inverse", coarse_n=int(info.coarse_n),
             level_dofs=[int(info.level_dofs[i]) for i in range(int(info.levels))],
             lmax=[float(info.lmax[i]) for i in range(max(int(info.levels) - 1, 0))],
             kernel_launches=int(info.kernel_launches), ku_shape=list(info.ku_shape), ku_kind=int(info.ku_kind),
             t_stage_ms=[round(float(v), 3) for v in info.t_stage_ms], device=f"cuda:{_torch().cuda.current_device()}",
             x0_used=bool(info.x0_used), x0_scale=float(info.x0_scale), t_wall=round(time.perf_counter() - t0, 4),
             # the reference GPU path's keys (rb/gpusolve.py:285): hierarchy set-up seconds and the attempt that
             # succeeded (the device path makes one attempt: a failure raises, there is no CPU retry)
             t_hier=round(info.t_setup_ms / 1e3, 2), gpu_attempt=0)
    if extra:
        d.update(extra)
    return d


def _extra_entries(extra, used_nodes_fn, ntotal):
    """Full-layout COO of the reference's ``extra(nmap, n)`` hook; objects exposing ``node_coo()`` skip the
    compact numbering (no device->host round trip of the used-node map)."""
    if extra is None:
        return None
    if hasattr(extra, "node_coo"):
        nr, cr, nc, cc, v = extra.node_coo()
        return 3 * np.asarray(nr, np.int64) + cr, 3 * np.asarray(nc, np.int64) + cc, np.asarray(v, np.float64)
    nused = used_nodes_fn()
    nmap = -np.ones(ntotal, np.int64)
    nmap[nused] = np.arange(len(nused))
    M = extra(nmap, 3 * len(nused)).tocoo()
    return 3 * nused[M.row // 3] + M.row % 3, 3 * nused[M.col // 3] + M.col % 3, M.data


def solve_cn(g, lam, mu, active, cn, orig, fixed, loads, extra=None, node_groups=None, tol=1e-6, maxiter=800,
             aniso=None, *, precision="fp64", x0=None, options=None, keep_device=False, warm_start=None):
    """Split-node solve on the GPU (rb/splitfe.py:123-158): returns (U (nnew, 3) with NaN on unused nodes,
    info, reactions R).  ``warm_start``: True (the packaged network) or a ``warmnet.WarmNet`` predicts the initial
    guess when no ``x0`` is given; the solve falls back to a zero start if the guess's residual is not below
    ||f|| (info["x0_used"])."""
    ctx = prepare_cn(g, lam, mu, active, cn, orig, fixed, loads, extra, node_groups, tol, maxiter, aniso,
                     precision=precision, x0=x0, options=options, warm_start=warm_start)
    try:
        x, info = ctx["P"].solve(ctx["f"], ctx["x0"])
        ctx["stamps"].append(("solve", time.perf_counter()))
        return finish_cn(ctx, x, info, keep_device=keep_device)
    finally:
        if not keep_device:
            ctx["P"].close()


def prepare_cn(g, lam, mu, active, cn, orig, fixed, loads, extra=None, node_groups=None, tol=1e-6, maxiter=800,
               aniso=None, *, precision="fp64", x0=None, options=None, warm_start=None):
    """The part of solve_cn before the solve: the operator and its hierarchy (a Problem), the rigid groups, the
    right-hand side and the start.  Returns a context for finish_cn; the caller closes ctx["P"]."""
    if aniso is not None:
        raise NotImplementedError("laminate (aniso) joint cells are not supported by the device solver")
    t0 = time.perf_counter()
    stamps = [("start", t0)]
    orig = np.asarray(orig)
    ntotal = len(orig)
    fn, fa = fixed
    fn = np.asarray(fn, np.int64)
    fa = np.asarray(fa, np.float64)
    pen_k = np.repeat((fa * K_GROUND)[:, None], 3, axis=1)
    active = np.asarray(active, bool)

    def used_nodes():
        return np.unique(np.asarray(cn)[np.flatnonzero(active)])

    coo = _extra_entries(extra, used_nodes, ntotal)
    mat = _dev_cat((lam, mu), np.float64)
    stamps.append(("host_inputs", time.perf_counter()))
    P = Problem(g, _lib.MAT_ISO_SRI, mat, active, cn=cn, orig=orig, pen_node=fn, pen_k=pen_k, extra_coo=coo,
                precision=precision, tol=tol, maxiter=maxiter, options=options)
    stamps.append(("create", time.perf_counter()))
    try:
        P.set_rigid_groups(node_groups)
        stamps.append(("rigid", time.perf_counter()))
        f = P.rhs(loads)
        if x0 is not None:
            x0d = _dev(np.nan_to_num(np.asarray(x0, np.float64)).ravel(), np.float64)
        elif warm_start is not None and warm_start is not False:
            from . import warmnet
            net = warmnet.default_net() if warm_start is True else warm_start
            ln, lz = warmnet.load_z(loads)
            nc = g.nx * g.ny * g.nz       # the operator's device copies of lam, mu and active serve the network too
            x0d = net.predict_x0(g, P.mat[:nc], P.mat[nc:], P.active, orig, fn, ln, lz, ntotal, orig_dev=P.orig)
            stamps.append(("warm_start", time.perf_counter()))
        else:
            x0d = None
    except BaseException:
        P.close()
        raise
    return dict(P=P, f=f, x0=x0d, fn=fn, fa=fa, ntotal=ntotal, stamps=stamps, t0=t0)


def finish_cn(ctx, x, info, keep_device=False):
    """The part of solve_cn after the solve: U (NaN on unused nodes), reactions of the ground springs, info."""
    P, fn, fa, ntotal, stamps = ctx["P"], ctx["fn"], ctx["fa"], ctx["ntotal"], ctx["stamps"]
    Ud = P.export(x)
    U = _host(Ud.view(ntotal, 3))
    stamps.append(("download", time.perf_counter()))
    R = np.zeros((ntotal, 3))
    np.add.at(R, fn, -(fa[:, None] * K_GROUND) * U[fn])
    stamps.append(("reactions", time.perf_counter()))
    d = _info_dict(info, ctx["t0"], dict(t_host={b[0]: round(b[1] - a[1], 4) for a, b in zip(stamps, stamps[1:])}))
    if keep_device:
        d["device"] = dict(U=Ud, mat=P.mat, cn=P.cn, problem=P)
    return U, d, R


def solve_batch_device(problems, fs, x0s=None):
    """One feb_solve_batch call: problems (Problem), right-hand sides and optional starts (device tensors, full
    layout).  Returns [(x, FebInfo)] in order."""
    torch = _torch()
    n = len(problems)
    xs = [torch.empty_like(f) for f in fs]
    infos = (_lib.FebInfo * n)()
    hs = (C.c_void_p * n)(*[P.h.value for P in problems])
    fp = (C.c_void_p * n)(*[f.data_ptr() for f in fs])
    xp = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
    x0p = None
    if x0s is not None:
        x0p = (C.c_void_p * n)(*[(x.data_ptr() if x is not None else 0) for x in x0s])
    _lib.check(_lib.load().feb_solve_batch(hs, n, fp, x0p, xp, infos))
    return [(xs[i], infos[i]) for i in range(n)]


def _used_from_grid(g, active):
    nx1, ny1 = g.nx + 1, g.ny + 1
    cells = np.flatnonzero(active)
    k = cells % g.nz; j = (cells // g.nz) % g.ny; i = cells // (g.nz * g.ny)
    used = np.zeros((g.nx + 1) * (g.ny + 1) * (g.nz + 1), bool)
    for a, b, c in CORNERS:
        used[(i + a) + nx1 * ((j + b) + ny1 * (k + c))] = True
    return used


def solve(grid, lam, mu, active, springs, loads, method="cg", tol=1e-8, x0=None, maxiter=20000, penalties=(),
          coeffs=None, node_groups=None, U0=None, *, precision="fp64", options=None):
    """Single-connectivity solve on the GPU (fe/solver.py:202-254).  Every method ('gmg', 'direct', 'cg')
    runs the device GMG-PCG; 'direct' tightens the tolerance to 1e-12.  Returns (U (nnode, 3) with NaN on
    unused nodes, info)."""
    t0 = time.perf_counter()
    g = grid
    active = np.asarray(active, bool)
    used = _used_from_grid(g, active)
    nnode = len(used)
    if method == "direct":
        tol = min(tol, 1e-12)
    # diagonal springs on used nodes (fe/solver.py:212-215)
    pn, pk = [], []
    for nodes, area, kvec in springs:
        nodes = np.asarray(nodes, np.int64); ok = used[nodes]
        pn.append(nodes[ok]); pk.append(np.asarray(area, np.float64)[ok][:, None] * np.asarray(kvec, np.float64)[None])
    pen_node = np.concatenate(pn) if pn else np.zeros(0, np.int64)
    pen_k = np.concatenate(pk) if pk else np.zeros((0, 3))
    # rank-1 penalties k w w^T, w normalised to unit sum over used nodes (fe/solver.py:224-232)
    er, ec, ev = [], [], []
    for nodes, weights, comp, k in penalties:
        nodes = np.asarray(nodes, np.int64); ok = used[nodes]
        dof = 3 * nodes[ok] + int(comp)
        w = np.asarray(weights, np.float64)[ok]
        ud, inv = np.unique(dof, return_inverse=True)
        wv = np.bincount(inv, weights=w)
        wv /= wv.sum()
        er.append(np.repeat(ud, len(ud))); ec.append(np.tile(ud, len(ud))); ev.append(k * np.outer(wv, wv).ravel())
    coo = (np.concatenate(er), np.concatenate(ec), np.concatenate(ev)) if er else None
    if coeffs is not None:
        mode, mat = _lib.MAT_ORTHO, np.asarray(coeffs, np.float64).reshape(-1, 6)
    else:
        mode, mat = _lib.MAT_ISO_FULL, np.concatenate([np.asarray(lam, np.float64), np.asarray(mu, np.float64)])
    P = Problem(g, mode, mat, active, pen_node=pen_node, pen_k=pen_k, extra_coo=coo, precision=precision, tol=tol,
                maxiter=maxiter, options=options)
    try:
        P.set_rigid_groups(node_groups)
        lo = []
        for nodes, area, t in loads:
            nodes = np.asarray(nodes, np.int64); ok = used[nodes]
            lo.append((nodes[ok], np.asarray(area, np.float64)[ok], t))
        f = P.rhs(lo)
        if U0 is not None:
            x0 = np.where(used[:, None], np.nan_to_num(np.asarray(U0, np.float64)), 0.0)
        elif x0 is not None:
            full = np.zeros((nnode, 3)); full[used] = np.asarray(x0, np.float64).reshape(-1, 3)
            x0 = full
        x0d = _dev(np.asarray(x0).ravel(), np.float64) if x0 is not None else None
        x, info = P.solve(f, x0d)
        U = _host(P.export(x).view(nnode, 3))
        usedn = np.flatnonzero(used)
        fh = _host(f.view(nnode, 3))[usedn].ravel()
        return U, _info_dict(info, t0, dict(K=None, f=fh, used=usedn))
    finally:
        P.close()


def _stress(g, mode, mat, U, cells, cn, nan_to_zero, to_host=True):
    torch = _torch()
    n = len(cells)
    Ud = U if isinstance(U, torch.Tensor) else _dev(np.asarray(U, np.float64).ravel(), np.float64)
    matd = mat if isinstance(mat, torch.Tensor) else _dev(mat, np.float64)
    cnd = cn if (cn is None or isinstance(cn, torch.Tensor)) else _dev(cn, np.int64)
    cd = _dev(cells, np.int64)
    sig = torch.empty(6 * n, dtype=torch.float64, device="cuda")
    vm = torch.empty(n, dtype=torch.float64, device="cuda")
    eps = torch.empty(6 * n, dtype=torch.float64, device="cuda")
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_cell_stress(C.byref(gs), mode, _ptr(matd), _ptr(Ud), n, _ptr(cd), _ptr(cnd),
                                           int(nan_to_zero), _ptr(sig), _ptr(vm), _ptr(eps), _stream()))
    if not to_host:
        return sig.view(n, 6), vm, eps.view(n, 6)
    return tuple(_host(sig.view(n, 6), vm, eps.view(n, 6)))


def cell_stress_cn(g, lam, mu, U, cells, cn, aniso=None, *, device=None):
    """Centre-point strain, stress, von Mises of the split-node model (rb/splitfe.py:161-175); NaN
    displacements count as 0.  ``device``: the ``info['device']`` of a ``solve_cn(..., keep_device=True)``
    call with the same lam, mu, cn and U, to skip their upload."""
    if aniso is not None:
        raise NotImplementedError("laminate (aniso) joint cells are not supported by the device solver")
    if device is not None:
        return _stress(g, _lib.MAT_ISO_SRI, device["mat"], device["U"], cells, device["cn"], True)
    mat = np.concatenate([np.asarray(lam, np.float64), np.asarray(mu, np.float64)])
    return _stress(g, _lib.MAT_ISO_SRI, mat, U, cells, cn, True)


def cell_stress(grid, lam, mu, U, cells, coeffs=None):
    """Centre-point strain, stress, von Mises (fe/solver.py:257-272); NaN displacements propagate."""
    if coeffs is not None:
        return _stress(grid, _lib.MAT_ORTHO, np.asarray(coeffs, np.float64).reshape(-1, 6), U, cells, None, False)
    mat = np.concatenate([np.asarray(lam, np.float64), np.asarray(mu, np.float64)])
    return _stress(grid, _lib.MAT_ISO_SRI, mat, U, cells, None, False)


def element_forces_cn(g, lam, mu, U, cells, cn, aniso=None):
    """Internal nodal forces K_e u_e (SRI lambda term) of listed cells (rb/splitfe.py:178-193)."""
    if aniso is not None:
        raise NotImplementedError("laminate (aniso) joint cells are not supported by the device solver")
    torch = _torch()
    cells = np.asarray(cells, np.int64)
    n = len(cells)
    mat = _dev(np.concatenate([np.asarray(lam, np.float64), np.asarray(mu, np.float64)]), np.float64)
    Ud = _dev(np.asarray(U, np.float64).ravel(), np.float64)
    cd, cnd = _dev(cells, np.int64), _dev(cn, np.int64)
    out = torch.empty(24 * n, dtype=torch.float64, device="cuda")
    gs = _grid_struct(g)
    _lib.check(_lib.load().feb_element_forces(C.byref(gs), _ptr(mat), _ptr(Ud), n, _ptr(cd), _ptr(cnd), _ptr(out),
                                              _stream()))
    return _host(out.view(n, 8, 3))


def _rigid_groups_from_Z(Z, n):
    """Node groups of a Z built like fe/solver.py:177-199 (6 columns per group: 3 unit translations, then 3
    rotations); returns the compact node indices of every group, or raises if Z has another structure."""
    import scipy.sparse as sp
    Zc = sp.csc_matrix(Z)
    if Zc.shape[1] % 6:
        raise NotImplementedError("Z must hold 6 rigid-body columns per node group")
    groups = []
    for g in range(Zc.shape[1] // 6):
        col = Zc[:, 6 * g].tocoo()
        dofs = col.row[col.data != 0]
        if len(dofs) == 0 or np.any(dofs % 3) or not np.allclose(col.data[col.data != 0], 1.0):
            raise NotImplementedError("Z columns are not translations of node groups")
        groups.append(dofs // 3)
    return groups


def pcg_gmg(A, b, used_nodes, grid_edges, tol=1e-7, maxiter=500, x0=None, A_op=None, Z=None, *, precision="fp64",
            options=None):
    """GMG-preconditioned CG for an assembled matrix on compact dofs (fe/gmg.py:120-137, the plugin point
    that rb/rbfe.py:21-27 swaps).  Compatibility path: the fine level applies A as a sparse matrix on the
    device and the coarse levels are its Galerkin products on the structured grid; node ``i`` of A sits at
    grid node ``used_nodes[i]`` (split copies share their grid node, rb/splitfe.py:153).  A Z made of the
    per-group rigid-body modes of fe/solver.py:177-199 runs on the device with the rest of the solve; with any
    other Z, or with a separate Krylov operator A_op, the V-cycle still runs on the device (feb_precondition) and
    SciPy's cg drives the iteration on the host (_pcg_host_operator).  Returns (x, info)."""
    import scipy.sparse as sp
    from .grid import Grid
    t0 = time.perf_counter()
    xe, ye, ze = grid_edges
    g = Grid(xe, ye, ze)
    used_nodes = np.asarray(used_nodes, np.int64)
    n_c = len(used_nodes)
    # full layout: the first compact node at a grid position takes the grid id, later ones become copies
    order = np.argsort(used_nodes, kind="stable")
    first = np.ones(n_c, bool)
    first[order[1:]] = used_nodes[order[1:]] != used_nodes[order[:-1]]
    node_of = np.empty(n_c, np.int64)
    node_of[first] = used_nodes[first]
    dup = np.flatnonzero(~first)
    node_of[dup] = g.nnode + np.arange(len(dup))
    orig = np.concatenate([np.arange(g.nnode), used_nodes[dup]])
    M = sp.coo_matrix(A)
    coo = (3 * node_of[M.row // 3] + M.row % 3, 3 * node_of[M.col // 3] + M.col % 3, M.data)
    ncell = g.nx * g.ny * g.nz
    # no cells: the whole operator is the sparse part; the used nodes are the ones A is given on
    P = Problem(g, _lib.MAT_ISO_SRI, np.zeros(2 * ncell), np.zeros(ncell, bool), cn=None, orig=orig, extra_coo=coo,
                precision=precision, tol=tol, maxiter=maxiter, options=options, mark_used=node_of)
    try:
        groups = None
        if Z is not None and A_op is None:
            try:
                groups = _rigid_groups_from_Z(Z, n_c)
            except NotImplementedError:
                groups = None
        if A_op is not None or (Z is not None and groups is None):
            # a separate Krylov operator, or a Z other than per-group rigid modes: host Krylov loop
            return _pcg_host_operator(P, A, A if A_op is None else A_op, b, x0, Z, tol, maxiter, node_of, len(orig),
                                      t0)
        if groups is not None:
            P.set_rigid_groups([node_of[gr] for gr in groups])
        bf = np.zeros((len(orig), 3)); bf[node_of] = np.asarray(b, np.float64).reshape(-1, 3)
        f = _dev(bf.ravel(), np.float64)
        x0d = None
        if x0 is not None:
            xf = np.zeros((len(orig), 3)); xf[node_of] = np.asarray(x0, np.float64).reshape(-1, 3)
            x0d = _dev(xf.ravel(), np.float64)
        x, info = P.solve(f, x0d)
        xh = _host(x.view(-1, 3))[node_of].ravel()
        return xh, _info_dict(info, t0)
    finally:
        P.close()


def _pcg_host_operator(P, A, A_op, b, x0, Z, tol, maxiter, node_of, ntot, t0):
    """pcg_gmg with a separate Krylov operator A_op (fe/gmg.py:127-136): the preconditioner is still built from A
    (the device V-cycle, plus the rigid-mode correction whose coarse matrix Z^T A_op Z is formed with A_op as the
    reference forms it), and SciPy's cg runs the iteration with A_op, a host operator, so each iteration moves r to
    the device and M r back.  Returns (x, info) like the device path."""
    import scipy.sparse.linalg as spla
    torch = _torch()
    n = A.shape[0]
    dofs = (3 * node_of[:, None] + np.arange(3)[None, :]).ravel()

    def vcycle(r):
        rf = np.zeros(3 * ntot); rf[dofs] = np.asarray(r, np.float64).ravel()
        return _host(P.precondition(_dev(rf, np.float64)))[dofs]

    if Z is not None:
        # P carries no rigid groups here: the correction is applied on the host with A_op, as fe/gmg.py:127-135
        Zd = Z.toarray() if hasattr(Z, "toarray") else np.asarray(Z)
        AZ = np.column_stack([A_op @ Zd[:, i] for i in range(Zd.shape[1])])
        Ec = Zd.T @ AZ
        Einv = np.linalg.pinv(0.5 * (Ec + Ec.T))
        M = spla.LinearOperator((n, n), matvec=lambda r: vcycle(r) + Zd @ (Einv @ (Zd.T @ r)))
    else:
        M = spla.LinearOperator((n, n), matvec=vcycle)
    it = [0]
    x, flag = spla.cg(A_op, np.asarray(b, np.float64), x0=x0, rtol=tol, maxiter=maxiter, M=M,
                      callback=lambda xk: it.__setitem__(0, it[0] + 1))
    torch.cuda.synchronize()
    r = np.asarray(b, np.float64) - A_op @ x
    bn = np.linalg.norm(b)
    return x, dict(iters=it[0], flag=int(flag), relres=float(np.linalg.norm(r) / (bn if bn > 0 else 1.0)),
                   levels=None, krylov="host (A_op)", t_wall=round(time.perf_counter() - t0, 4), t_hier=None,
                   gpu_attempt=0)
