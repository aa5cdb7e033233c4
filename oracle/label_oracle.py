"""CPU oracle of the voxel labelling (test infrastructure: imported only by tests/ and bench.py's CPU legs).

A NumPy restatement of rb/rbgeom.py's per-point labelling of a foot lattice:
  inverse map (scale, osteotomy fragment, alignment shear, local warps)   rb/rbgeom.py:243-305
  raster / sub-raster lookups                                             rb/rbgeom.py:221-236
  facet frames, footprints and grown fronts                               rb/rbgeom.py:308-355
  label_points (fragment relabelling, subtalar edits, actions)            rb/rbgeom.py:358-464
  label_lattice (separable lookup plus the points edits can reach)        rb/rbgeom.py:493-524
on a template object with the fields of comech_b200.labels.Template.  Pinned against the reference's own
label_lattice on seeded synthetic templates (tests/golden/labels.npz, tests/golden/make_golden.py).
"""
import numpy as np

from comech_b200.labels import (COAL, FIB, INTERP, FUSE, GAP, SOFT, FACETS, JOINT_BOX, facet_factors,
                                coalition_dirs, grown_threshold)


def _warp(T, foot, P):
    """Local displacement template -> foot of the sustentaculum and the posterior dome (rb/rbgeom.py:243-256)."""
    d = np.zeros_like(P)
    fm, fp = T.facets["mid"], T.facets["post"]
    if foot.sust_y != 11.0:
        r2 = ((P - fm["c"]) ** 2).sum(1)
        d[:, 1] += (foot.sust_y - 11.0) * np.exp(-r2 / (2 * 8.0 ** 2))
    if foot.post_dome != 1.5:
        q = P - fp["c"]
        u = (q @ fp["e1"] - fp["uc"]) / (fp["a0"] + 2.0)
        v = (q @ fp["e2"] - fp["vc"]) / (fp["b0"] + 2.0)
        w = q @ fp["n"]
        amp = (foot.post_dome - 1.5) * np.clip(1 - u ** 2 - v ** 2, 0, None) * np.exp(-w ** 2 / (2 * 6.0 ** 2))
        d += amp[:, None] * fp["n"][None, :]
    return d


def _lateral_shift(T, foot, P):
    """Alignment shear of the hindfoot below the joint (rb/rbgeom.py:259-264)."""
    if foot.align == 0.0:
        return np.zeros(len(P))
    w = np.clip((T.x_w1 - P[:, 0]) / (T.x_w1 - T.x_w0), 0, 1)
    return -np.tan(np.deg2rad(foot.align)) * np.clip(T.z_ref - P[:, 2], 0, None) * w


def to_template(T, foot, act, P):
    """World -> template points: (static point, fragment point or None, in-fragment mask) (rb/rbgeom.py:284-305)."""
    p3 = T.c0 + (np.asarray(P, float) - T.c0) / foot.scale
    frag = np.zeros(len(p3), bool)
    cands = [p3]
    if act is not None and act.osteo != 0.0:
        frag = (p3[:, 0] < T.x_cut(p3[:, 2])) & (p3[:, 2] < T.z_frag_top)
        pm = p3.copy()
        pm[:, 1] -= act.osteo
        cands.append(pm)
    res = []
    for p2 in cands:
        p1 = p2.copy()
        p1[:, 1] -= _lateral_shift(T, foot, p2)
        if foot.sust_y != 11.0 or foot.post_dome != 1.5:
            p = p1 - _warp(T, foot, p1)
            for _ in range(3):
                p = p1 - _warp(T, foot, p)
        else:
            p = p1
        res.append(p)
    return res[0], (res[1] if len(res) > 1 else None), frag


def _uvw(F, P):
    q = P - F["c"]
    return q @ F["e1"], q @ F["e2"], q @ F["n"]


def _footprint(F, u, v):
    iu = np.floor((u - F["ua"]) / F["res"]).astype(np.int64)
    iv = np.floor((v - F["va"]) / F["res"]).astype(np.int64)
    ok = (iu >= 0) & (iu < F["F0"].shape[0]) & (iv >= 0) & (iv < F["F0"].shape[1])
    out = np.zeros(len(u), bool)
    out[ok] = F["F0"][iu[ok], iv[ok]]
    return out


def _inside_scaled(F, u, v, fa, fb):
    return _footprint(F, F["uc"] + (u - F["uc"]) / fa, F["vc"] + (v - F["vc"]) / fb)


def _front(F, g, u, v):
    if g is None:
        return np.zeros(len(u), bool)
    d, thr = g
    return (u - F["uc"]) * d[0] + (v - F["vc"]) * d[1] <= thr


def label_points(P, foot, act, T, defect_fill="soft"):
    """Body label of every world point P (N, 3) (rb/rbgeom.py:358-464)."""
    ps, pm, frag = to_template(T, foot, act, P)
    L = T.lookup(ps)
    if pm is not None and frag.any():
        Lm, Ls = T.lookup(pm[frag]), L[frag]
        ms, mm = ~np.isin(Ls, T.static_bodies), ~np.isin(Lm, T.static_bodies)
        L[frag] = np.where(ms, np.where(mm, Lm, SOFT), Ls)
    ext = np.array(T.dt.shape) * T.h
    idx = np.nonzero(np.all((ps >= T.so) & (ps < T.so + ext), 1) & ~frag)[0]
    if not len(idx):
        return L
    q, Lq = ps[idx], L[idx].copy()
    dt, dc = T.sub_lookup(T.dt, q), T.sub_lookup(T.dc, q)
    gapw = dt + dc
    fac = facet_factors(foot)
    uvw = {k: _uvw(T.facets[k], q) for k in FACETS}
    soft_or_empty = lambda: np.isin(Lq, [SOFT, 0])
    for k, b in FACETS.items():       # facet size (post, mid, ant in this order)
        F, (fa, fb), (u, v, w) = T.facets[k], fac[k], uvw[k]
        ins = (np.abs(w) <= F["wmax"] + 1.0) & (np.abs(u - F["uc"]) <= 1.7 * F["a0"] * max(fa, 1)) & \
              (np.abs(v - F["vc"]) <= 1.7 * F["b0"] * max(fb, 1))
        ins &= _inside_scaled(F, u, v, fa, fb)
        if fa != 1.0 or fb != 1.0:
            Lq[ins & (gapw <= 1.6 * F["gap"]) & soft_or_empty()] = b
            Lq[(Lq == b) & ~ins] = SOFT
    Fm, Fa, Fp = T.facets["mid"], T.facets["ant"], T.facets["post"]
    if foot.ant_mode == 1:            # anterior facet confluent with the middle one
        seg = Fa["c"] - Fm["c"]
        t = ((q - Fm["c"]) @ seg) / (seg @ seg)
        dist = np.linalg.norm(q - Fm["c"] - t[:, None] * seg[None, :], axis=1)
        conf = (t > 0) & (t < 1) & (dist < 0.75 * min(Fm["b0"] * fac["mid"][1], Fa["b0"] * fac["ant"][1])) & \
               (gapw <= 1.6 * max(Fm["gap"], Fa["gap"])) & soft_or_empty()
        Lq[conf] = FACETS["ant"]
    elif foot.ant_mode == 2:
        Lq[Lq == FACETS["ant"]] = SOFT
    d_mid, d_post = coalition_dirs(foot)
    mid_c, post_c = Lq == FACETS["mid"], Lq == FACETS["post"]
    um, vm, wm = uvw["mid"]
    up, vp, _ = uvw["post"]
    br = np.zeros(len(q), bool)
    fib = np.zeros(len(q), bool)
    kk = 2.0 / np.sqrt(np.pi)
    if foot.ctype != "none":
        gap_bar = (dt <= 4.0) & (dc <= 4.0) & soft_or_empty()
        if foot.ctype in ("I", "IV"):
            if foot.rtype in ("R1", "R2", "R3"):
                bb = Fm["b0"] * fac["mid"][1]
                band = mid_c & (vm >= Fm["vc"] + bb * (1 - 2 * foot.cov_mid))
                br |= band
                if foot.rtype == "R2":
                    xe = Fm["c"][0] - (Fm["c"][0] - Fm["xyz_lo"][0]) * fac["mid"][0]
                    br |= gap_bar & (((q[:, 0] - (xe - 2.5)) / (3.5 * kk)) ** 2 +
                                     ((q[:, 1] - (Fm["c"][1] + 1.5)) / (2.0 * kk)) ** 2 <= 1) & (np.abs(wm) < 6.0)
                if foot.rtype == "R3":
                    aa = Fm["a0"] * fac["mid"][0]
                    fib = band & (um < Fm["uc"] - aa + 2 * aa * foot.fib_frac)
                    br &= ~fib
            else:
                br |= mid_c & _front(Fm, grown_threshold(Fm, *fac["mid"], d_mid, foot.cov_mid), um, vm)
        if foot.ctype in ("II", "IV"):
            br |= post_c & _front(Fp, grown_threshold(Fp, *fac["post"], d_post, foot.cov_post), up, vp)
        if foot.ctype in ("III", "IV"):
            x_lo = Fp["c"][0] + 2.0
            x_hi = Fm["c"][0] - (Fm["c"][0] - Fm["xyz_lo"][0]) * fac["mid"][0] + 1.0
            y_lo = Fp["c"][1] + (Fp["xyz_hi"][1] - Fp["c"][1]) * fac["post"][1] - 3.0
            y_hi = Fm["c"][1] + 3.0
            ex, ey = 0.5 * (x_hi - x_lo) * kk, 0.5 * (y_hi - y_lo) * kk
            br |= gap_bar & (((q[:, 0] - 0.5 * (x_lo + x_hi)) / ex) ** 2 + ((q[:, 1] - 0.5 * (y_lo + y_hi)) / ey) ** 2 <= 1)
    dm = mid_c & _front(Fm, grown_threshold(Fm, *fac["mid"], d_mid, act.d_mid), um, vm)
    dp = post_c & _front(Fp, grown_threshold(Fp, *fac["post"], d_post, act.d_post), up, vp)
    if act.fusion:
        fz = np.isin(Lq, list(FACETS.values())) | br | fib | ((gapw <= 4.0) & (dt <= 4.0) & (dc <= 4.0) & soft_or_empty())
        Lq[fz] = FUSE
    elif act.resect:
        hole = br | fib | dm | dp
        if act.interp:
            Lq[hole] = INTERP
        elif defect_fill == "void":
            Lq[hole] = GAP
        else:
            on_facet = hole & (mid_c | post_c)
            Lq[hole & ~on_facet] = GAP
            Lq[on_facet] = SOFT
    else:
        Lq[br] = COAL
        Lq[fib] = FIB
        Lq[(dm | dp) & ~br & ~fib] = GAP if defect_fill == "void" else SOFT
    L[idx] = Lq
    return L


def label_lattice(sx, sy, sz, foot, act, T, defect_fill="soft"):
    """Labels of the lattice sx x sy x sz (rb/rbgeom.py:493-524): raster lookup with separable indices, then
    label_points on every point an edit can reach."""
    s, c0 = foot.scale, T.c0
    t = [c0[a] + (np.asarray(v, float) - c0[a]) / s for a, v in enumerate((sx, sy, sz))]
    ind = []
    for a in range(3):
        i = np.floor((t[a] - T.o[a]) / T.h).astype(np.int64)
        ok = (i >= 0) & (i < T.lab.shape[a])
        ind.append((np.where(ok, i, 0), ok))
    (ix, okx), (iy, oky), (iz, okz) = ind
    L = T.lab[np.ix_(ix, iy, iz)].astype(np.int16)
    L[~okx] = 0
    L[:, ~oky] = 0
    L[:, :, ~okz] = 0
    tx, ty, tz = t
    box = lambda v, lo, hi: (v >= lo) & (v <= hi)
    (jx0, jx1), (jy0, jy1), (jz0, jz1) = JOINT_BOX
    need = box(tx, jx0, jx1)[:, None, None] & box(ty, jy0, jy1)[None, :, None] & box(tz, jz0, jz1)[None, None, :]
    if foot.align != 0.0:
        need = need | ((tx < T.x_w1 + 1.0)[:, None, None] & (tz < T.z_ref + 1.0)[None, None, :])
    if act.osteo != 0.0:
        need = need | ((tx[:, None] < T.x_cut(tz)[None, :] + 1.0) & (tz < T.z_frag_top + 1.0)[None, :])[:, None, :]
    if foot.sust_y != 11.0:
        c = T.facets["mid"]["c"]
        r = 4 * 8.0 + abs(foot.sust_y - 11.0) + 1.0
        need = need | ((np.abs(tx - c[0]) < r)[:, None, None] & (np.abs(ty - c[1]) < r)[None, :, None] &
                       (np.abs(tz - c[2]) < r)[None, None, :])
    if foot.post_dome != 1.5:
        c = T.facets["post"]["c"]
        r = 40.0
        need = need | ((np.abs(tx - c[0]) < r)[:, None, None] & (np.abs(ty - c[1]) < r)[None, :, None] &
                       (np.abs(tz - c[2]) < r)[None, None, :])
    I, J, K = np.nonzero(need)
    if len(I):
        P = np.column_stack([np.asarray(sx, float)[I], np.asarray(sy, float)[J], np.asarray(sz, float)[K]])
        L[I, J, K] = label_points(P, foot, act, T, defect_fill)
    return L
