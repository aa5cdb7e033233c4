"""Voxel labelling of a foot lattice on the GPU (rb/rbgeom.py:493-524 label_lattice, :358-464 label_points).

A virtual foot and a surgical action are applied to the engine's label template by the inverse map of each
lattice point into the template frame (isotropic scale about the ground point c0, osteotomy fragment shift,
hindfoot alignment shear, smooth local warps of the sustentaculum and the posterior facet dome, undone by a
fixed-point iteration), a raster lookup there, and the subtalar edits near the joint (facet sizes, anterior facet
mode, coalition bars, resection defects, interposition, fusion).  ``label_lattice`` returns the same labels as
the reference's ``label_points`` at every lattice point: the device kernel (csrc/labels.cu, ``feb_label_lattice``)
runs the whole per-point rule for every point, in FP64 with the reference's operation order.

The template is a ``Template`` (this module): the label raster, the distance maps of the subtalar region, the three
facet frames and footprints, and the scalars of the warps.  The reference's own template (``rb_template.npz``,
built from the CT atlas) is not distributed; ``synth.synthetic_template`` builds seeded stand-ins with the same
fields.  The foot and the action are any objects with the fields of rb/rbgeom.py:55-99 ``Foot`` and ``Action``
(``Foot`` and ``Action`` below carry the same fields and defaults).
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

# label ids of the engine (rb/rbgeom.py:35-42): new bodies of the edits, soft tissue, the facets' cartilage
COAL, FIB, INTERP, FUSE, GAP = 101, 102, 103, 104, 105
SOFT = 63
FACETS = {"post": 12, "mid": 8, "ant": 10}
NOMINAL = {"post": (12.0, 9.5), "mid": (6.5, 4.5), "ant": (4.5, 4.0)}
FACET_PAR = {"post": ("post_a", "post_b"), "mid": ("mid_a", "mid_b"), "ant": ("ant_a", "ant_b")}
# template frame box in which every subtalar edit happens (rb/rbgeom.py:490)
JOINT_BOX = ((-82.0, -12.0), (-32.0, 32.0), (36.0, 92.0))
CTYPES = {"none": 0, "I": 1, "II": 2, "III": 3, "IV": 4}
RTYPES = {"none": 0, "R1": 1, "R2": 2, "R3": 3, "R4": 4}


@dataclass
class Foot:
    """Virtual foot parameters (fields and defaults of rb/rbgeom.py:55-73)."""
    scale: float = 1.0
    post_a: float = 12.0
    post_b: float = 9.5
    mid_a: float = 6.5
    mid_b: float = 4.5
    ant_a: float = 4.5
    ant_b: float = 4.0
    ant_mode: int = 0
    sust_y: float = 11.0
    post_dome: float = 1.5
    cart_t: float = 2.0
    align: float = 0.0
    ctype: str = "none"
    rtype: str = "none"
    cov_mid: float = 0.0
    cov_post: float = 0.0
    seed_ang: float = 0.0
    fib_frac: float = 0.0


@dataclass
class Action:
    """Surgical action parameters (fields and defaults of rb/rbgeom.py:86-93)."""
    resect: int = 0
    d_mid: float = 0.0
    d_post: float = 0.0
    osteo: float = 0.0
    interp: int = 0
    fusion: int = 0
    load: float = 1.0


class Template:
    """Label template: raster ``lab`` (int8, origin ``o``, spacing ``h``), subtalar distance maps ``dt``/``dc``
    (float32, origin ``so``, spacing ``h``), facet frames ``facets[name]`` (c, n, e1, e2, footprint raster F0
    with its origin ua/va and resolution res, a0, b0, uc, vc, wmax, gap, xyz_lo, xyz_hi), the scale centre c0,
    the shear scalars (z_ref, x_w0, x_w1), the osteotomy plane (x_cut0, z_cut0, cut_slope, z_frag_top) and the
    bodies that never move with the fragment (static_bodies) -- the fields of rb/rbgeom.py:183-218."""

    def __init__(self, lab, o, h, dt, dc, so, facets, static_bodies, z_frag_top=76.0, x_w0=-30.0, x_w1=10.0):
        self.lab = np.ascontiguousarray(lab, np.int8)
        self.o = np.asarray(o, np.float64)
        self.h = float(h)
        self.dt = np.ascontiguousarray(dt, np.float32)
        self.dc = np.ascontiguousarray(dc, np.float32)
        self.so = np.asarray(so, np.float64)
        self.facets = facets
        fp, fm = facets["post"], facets["mid"]
        cxy = 0.5 * (fp["c"][:2] + fm["c"][:2])
        self.c0 = np.array([cxy[0], cxy[1], 0.0])
        self.z_ref = float(min(fp["c"][2], fm["c"][2]) - 8.0)
        self.x_w0, self.x_w1 = float(x_w0), float(x_w1)
        self.x_cut0, self.z_cut0, self.cut_slope = float(fp["c"][0] - 15.0), float(fp["c"][2]), -0.5
        self.z_frag_top = float(z_frag_top)
        self.static_bodies = np.asarray(sorted(static_bodies), np.int64)

    def lookup(self, P):
        idx = np.floor((P - self.o) / self.h).astype(np.int64)
        ok = np.all((idx >= 0) & (idx < np.array(self.lab.shape)), 1)
        out = np.zeros(len(P), np.int16)
        i = idx[ok]
        out[ok] = self.lab[i[:, 0], i[:, 1], i[:, 2]]
        return out

    def sub_lookup(self, arr, P, fill=99.0):
        idx = np.floor((P - self.so) / self.h).astype(np.int64)
        ok = np.all((idx >= 0) & (idx < np.array(arr.shape)), 1)
        out = np.full(len(P), fill, np.float32)
        i = idx[ok]
        out[ok] = arr[i[:, 0], i[:, 1], i[:, 2]]
        return out

    def x_cut(self, z):
        return self.x_cut0 + self.cut_slope * (z - self.z_cut0)


def facet_factors(foot):
    return {k: (getattr(foot, a) / NOMINAL[k][0], getattr(foot, b) / NOMINAL[k][1]) for k, (a, b) in FACET_PAR.items()}


def coalition_dirs(foot):
    rot = np.deg2rad(foot.seed_ang)
    R = np.array([[np.cos(rot), -np.sin(rot)], [np.sin(rot), np.cos(rot)]])
    return R @ np.array([1.0, -0.35]), R @ np.array([0.25, -1.0])


def grown_threshold(F, fa, fb, d, frac):
    """(direction, threshold) of the front that covers ``frac`` of the scaled facet from its edge
    (rb/rbgeom.py:332-342): a point is inside when (u - uc) d0 + (v - vc) d1 <= threshold; None when frac <= 0."""
    if frac <= 0:
        return None
    d = np.asarray(d, float)
    d = d / np.linalg.norm(d)
    if frac >= 1:
        return d, np.inf
    iu, iv = np.nonzero(F["F0"])
    u = F["ua"] + (iu + 0.5) * F["res"]
    v = F["va"] + (iv + 0.5) * F["res"]
    us, vs = F["uc"] + fa * (u - F["uc"]), F["vc"] + fb * (v - F["vc"])
    proj = (us - F["uc"]) * d[0] + (vs - F["vc"]) * d[1]
    return d, float(np.quantile(proj, min(frac, 1.0)))


# ------------------------------------------------------------------------------------------------ device
class FebLabelFacet(C.Structure):
    _fields_ = [("c", C.c_double * 3), ("n", C.c_double * 3), ("e1", C.c_double * 3), ("e2", C.c_double * 3),
                ("ua", C.c_double), ("va", C.c_double), ("res", C.c_double), ("a0", C.c_double), ("b0", C.c_double),
                ("uc", C.c_double), ("vc", C.c_double), ("wmax", C.c_double), ("gap", C.c_double),
                ("xyz_lo", C.c_double * 3), ("xyz_hi", C.c_double * 3),
                ("F0", C.c_void_p), ("nu", C.c_int32), ("nv", C.c_int32)]


class FebLabelGrown(C.Structure):
    _fields_ = [("on", C.c_int32), ("pad", C.c_int32), ("d", C.c_double * 2), ("thr", C.c_double)]


class FebLabelParams(C.Structure):
    _fields_ = [("lab", C.c_void_p), ("lnx", C.c_int32), ("lny", C.c_int32), ("lnz", C.c_int32), ("pad0", C.c_int32),
                ("o", C.c_double * 3), ("h", C.c_double),
                ("dt", C.c_void_p), ("dc", C.c_void_p), ("snx", C.c_int32), ("sny", C.c_int32), ("snz", C.c_int32),
                ("pad1", C.c_int32), ("so", C.c_double * 3),
                ("facet", FebLabelFacet * 3),                      # post, mid, ant
                ("c0", C.c_double * 3), ("z_ref", C.c_double), ("x_w0", C.c_double), ("x_w1", C.c_double),
                ("x_cut0", C.c_double), ("z_cut0", C.c_double), ("cut_slope", C.c_double),
                ("z_frag_top", C.c_double), ("static_mask", C.c_uint32 * 4),
                ("scale", C.c_double), ("fa", C.c_double * 3), ("fb", C.c_double * 3), ("ant_mode", C.c_int32),
                ("ctype", C.c_int32), ("sust_y", C.c_double), ("post_dome", C.c_double), ("tan_align", C.c_double),
                ("align_on", C.c_int32), ("rtype", C.c_int32), ("cov_mid", C.c_double), ("fib_frac", C.c_double),
                ("g_cov_mid", FebLabelGrown), ("g_cov_post", FebLabelGrown), ("g_d_mid", FebLabelGrown), ("g_d_post", FebLabelGrown),
                ("resect", C.c_int32), ("interp", C.c_int32), ("fusion", C.c_int32), ("void_fill", C.c_int32),
                ("osteo", C.c_double)]


def _grown_struct(t):
    g = FebLabelGrown()
    if t is None:
        g.on = 0
    else:
        g.on = 1
        g.d[0], g.d[1] = float(t[0][0]), float(t[0][1])
        g.thr = t[1]
    return g


class DeviceTemplate:
    """A Template's arrays on the device (uploaded once; reused for every foot and action)."""

    def __init__(self, T):
        from .engine import _dev
        self.T = T
        self.lab = _dev(T.lab.view(np.uint8), np.uint8)
        self.dt = _dev(T.dt, np.float32)
        self.dc = _dev(T.dc, np.float32)
        self.F0 = {k: _dev(np.ascontiguousarray(T.facets[k]["F0"], dtype=bool).view(np.uint8), np.uint8)
                   for k in FACETS}

    def params(self, foot, act, defect_fill="soft"):
        T = self.T
        p = FebLabelParams()
        p.lab = self.lab.data_ptr()
        p.lnx, p.lny, p.lnz = T.lab.shape
        p.o[:] = list(T.o); p.h = T.h
        p.dt, p.dc = self.dt.data_ptr(), self.dc.data_ptr()
        p.snx, p.sny, p.snz = T.dt.shape
        p.so[:] = list(T.so)
        for q, k in enumerate(("post", "mid", "ant")):
            F, f = T.facets[k], p.facet[q]
            for name in ("c", "n", "e1", "e2", "xyz_lo", "xyz_hi"):
                getattr(f, name)[:] = [float(x) for x in F[name]]
            for name in ("ua", "va", "res", "a0", "b0", "uc", "vc", "wmax", "gap"):
                setattr(f, name, float(F[name]))
            f.F0 = self.F0[k].data_ptr()
            f.nu, f.nv = F["F0"].shape
        p.c0[:] = list(T.c0)
        p.z_ref, p.x_w0, p.x_w1 = T.z_ref, T.x_w0, T.x_w1
        p.x_cut0, p.z_cut0, p.cut_slope, p.z_frag_top = T.x_cut0, T.z_cut0, T.cut_slope, T.z_frag_top
        mask = [0, 0, 0, 0]
        for b in T.static_bodies:
            if 0 <= b < 128:
                mask[b // 32] |= 1 << (b % 32)
        p.static_mask[:] = mask
        fac = facet_factors(foot)
        p.scale = float(foot.scale)
        for q, k in enumerate(("post", "mid", "ant")):
            p.fa[q], p.fb[q] = fac[k]
        p.ant_mode = int(foot.ant_mode)
        p.ctype = CTYPES[foot.ctype]
        p.rtype = RTYPES.get(foot.rtype, 0)
        p.sust_y, p.post_dome = float(foot.sust_y), float(foot.post_dome)
        p.align_on = int(foot.align != 0.0)
        p.tan_align = float(np.tan(np.deg2rad(foot.align)))
        p.cov_mid, p.fib_frac = float(foot.cov_mid), float(foot.fib_frac)
        d_mid, d_post = coalition_dirs(foot)
        Fm, Fp = T.facets["mid"], T.facets["post"]
        p.g_cov_mid = _grown_struct(grown_threshold(Fm, *fac["mid"], d_mid, foot.cov_mid))
        p.g_cov_post = _grown_struct(grown_threshold(Fp, *fac["post"], d_post, foot.cov_post))
        p.g_d_mid = _grown_struct(grown_threshold(Fm, *fac["mid"], d_mid, act.d_mid))
        p.g_d_post = _grown_struct(grown_threshold(Fp, *fac["post"], d_post, act.d_post))
        p.resect, p.interp, p.fusion = int(act.resect), int(act.interp), int(act.fusion)
        p.void_fill = int(defect_fill == "void")
        p.osteo = float(act.osteo)
        return p


def label_lattice(sx, sy, sz, foot, act=None, T=None, defect_fill="soft", device_template=None, to_host=True):
    """Labels (int16, shape len(sx) x len(sy) x len(sz)) of the lattice sx x sy x sz (world frame) for the foot
    and action on template T: equal to label_points at every lattice point (rb/rbgeom.py:493-524)."""
    from .engine import _dev, _ptr, _stream, _host, _torch
    torch = _torch()
    act = act if act is not None else Action()
    D = device_template if device_template is not None else DeviceTemplate(T)
    p = D.params(foot, act, defect_fill)
    X, Y, Z = (_dev(np.ascontiguousarray(a, np.float64), np.float64) for a in (sx, sy, sz))
    out = torch.empty((len(sx), len(sy), len(sz)), dtype=torch.int16, device="cuda")
    _lib.check(_lib.load().feb_label_lattice(C.byref(p), _ptr(X), len(sx), _ptr(Y), len(sy), _ptr(Z), len(sz),
                                             _ptr(out), _stream()))
    return _host(out) if to_host else out
