"""Seeded synthetic voxel FE problems (no dataset is involved: every input is generated from a seed).

* ``block_problem``     -- two-material block: cortical matrix with seeded cancellous ellipsoid
                           inclusions, z=0 face on penalty springs, -z traction on the top face.
                           Inputs of ``fe/solver.py:202 solve`` (springs, loads).
* ``hindfoot_problem``  -- three seeded super-ellipsoid bones (talus, calcaneus, navicular) with a
                           cortical shell and cancellous core inside a soft-tissue envelope, patchy
                           cartilage between bones, a talocalcaneal coalition bridge, split nodes with
                           interface springs, plantar ground springs, 40 node-pair ligaments and a
                           load on the talar dome.  Inputs of ``rb/splitfe.py:123 solve_cn``.

The hindfoot follows the conventions of the reference engine's model builder (rb/rbfe.py:137-182):
``part`` is the bone filling at least half of a cell (0 for joint / soft cells), split nodes come from
``split_connectivity`` (rb/splitfe.py:261-305), ground springs are ``fixed = (nodes, area)`` with the
reference's k = 1e6 per unit area, loads are ``(nodes, area, traction)`` and springs between bones go
through the ``extra(nmap, n)`` hook (rb/splitfe.py:149-150).
"""
from dataclasses import dataclass, field
import numpy as np
import scipy.sparse as sp

from .grid import Grid, lame, face_node_areas
from .split import split_connectivity

E_CORTICAL, E_CANCELLOUS, NU_BONE = 1.0e4, 5.0e2, 0.3       # MPa
E_BRIDGE, NU_BRIDGE = 2.0e3, 0.3
E_CART, NU_CART = 10.0, 0.4
E_SOFT, NU_SOFT = 1.15, 0.45
K_GROUND = 1.0e2                                              # N/mm per plantar node (interior node)
K_INTERFACE = 1.0e3                                           # N/mm, split copy <-> grid node
BONES = ("talus", "calcaneus", "navicular")
ACTIONS = ("none", "resection", "osteotomy", "interposition", "fusion", "load")


def uniform_edges(n, h):
    return np.arange(n + 1) * float(h)


# ------------------------------------------------------------------------------------------ block (C1)
def block_problem(nx=48, ny=32, nz=24, h=1.0, seed=0, frac_cancellous=0.3, total_load=300.0, clamp_k=1e9):
    """Two-material block for ``solve``: E = 10 GPa with seeded 0.5 GPa ellipsoid inclusions (centres
    uniform in the grid, semi-axes U(3, 8) voxels) until ``frac_cancellous`` of the cells are cancellous,
    nu = 0.3; z=0 face nodes on springs ``clamp_k`` per unit area (all three directions); uniform -z
    traction on the top face summing to ``total_load`` N."""
    rng = np.random.default_rng(seed)
    g = Grid(uniform_edges(nx, h), uniform_edges(ny, h), uniform_edges(nz, h))
    ci, cj, ck = g.cI + 0.5, g.cJ + 0.5, g.cK + 0.5
    canc = np.zeros(g.ncell, bool)
    while canc.mean() < frac_cancellous:
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        a = rng.uniform(3, 8, 3)
        canc |= ((ci - c[0]) / a[0]) ** 2 + ((cj - c[1]) / a[1]) ** 2 + ((ck - c[2]) / a[2]) ** 2 <= 1.0
    E = np.where(canc, E_CANCELLOUS, E_CORTICAL)
    nu = np.full(g.ncell, NU_BONE)
    lam, mu = lame(E, nu)
    active = np.ones(g.ncell, bool)
    cells = np.arange(g.ncell)
    nb, ab = face_node_areas(g, g.cell_nodes, cells[g.cK == 0], "z-")
    nt, at = face_node_areas(g, g.cell_nodes, cells[g.cK == nz - 1], "z+")
    t = -total_load / at.sum()
    return dict(grid=g, E=E, nu=nu, lam=lam, mu=mu, active=active,
                springs=[(nb, ab, np.array([clamp_k] * 3))], loads=[(nt, at, np.array([0.0, 0.0, t]))],
                name=f"block {nx}x{ny}x{nz} h={h}")


# ------------------------------------------------------------------------------------------ springs
@dataclass
class SpringSet:
    """Springs between nodes, usable as the reference's ``extra(nmap, n)`` hook (a callable returning the
    sparse matrix on compact dofs).  Two kinds:

    * interface springs: isotropic 3x3 diagonal springs k between node pairs (split copy, grid node);
    * line springs (ligaments): k (d.(u_a - u_b))^2 with unit direction d, i.e. K += k w w^T with
      w = +d on node a, -d on node b (the rank-1 form of rb/replica3.py:68-86 with one node per end).
    """
    pair_a: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    pair_b: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    pair_k: np.ndarray = field(default_factory=lambda: np.zeros(0))
    line_a: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    line_b: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    line_d: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    line_k: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def node_coo(self):
        """(node_r, comp_r, node_c, comp_c, value) entries of the spring matrix on node ids."""
        nr, cr, nc, cc, v = [], [], [], [], []
        c3 = np.arange(3)
        if len(self.pair_a):
            a = np.repeat(self.pair_a, 3); b = np.repeat(self.pair_b, 3)
            k = np.repeat(self.pair_k, 3); c = np.tile(c3, len(self.pair_a))
            for (x, y, s) in ((a, a, 1.0), (b, b, 1.0), (a, b, -1.0), (b, a, -1.0)):
                nr.append(x); cr.append(c); nc.append(y); cc.append(c); v.append(s * k)
        if len(self.line_a):
            ends = np.stack([self.line_a, self.line_b], 1)                 # (m, 2)
            wv = np.stack([self.line_d, -self.line_d], 1)                   # (m, 2, 3)
            m = len(self.line_a)
            node = np.repeat(ends, 3, axis=1)                              # (m, 6)
            comp = np.tile(c3, (m, 2))
            w = wv.reshape(m, 6)
            nr.append(np.repeat(node, 6, 1).ravel()); cr.append(np.repeat(comp, 6, 1).ravel())
            nc.append(np.tile(node, (1, 6)).ravel()); cc.append(np.tile(comp, (1, 6)).ravel())
            v.append((self.line_k[:, None, None] * w[:, :, None] * w[:, None, :]).ravel())
        if not nr:
            z = np.zeros(0, np.int64)
            return z, z, z, z, np.zeros(0)
        return (np.concatenate(nr), np.concatenate(cr), np.concatenate(nc), np.concatenate(cc), np.concatenate(v))

    def __call__(self, nmap, n):
        nr, cr, nc, cc, v = self.node_coo()
        return sp.csr_matrix((v, (3 * nmap[nr] + cr, 3 * nmap[nc] + cc)), shape=(n, n))


# ------------------------------------------------------------------------------------------ hindfoot
def _superellipsoid(x, y, z, c, a, p):
    return (np.abs((x - c[0]) / a[0]) ** p + np.abs((y - c[1]) / a[1]) ** p + np.abs((z - c[2]) / a[2]) ** p)


def _bone_layout(rng, L, W, H):
    """Centres, semi-axes and exponents of talus, calcaneus, navicular in a box L x W x H (mm)."""
    p = rng.uniform(2.0, 4.0, 3)
    s = min(L / 80.0, W / 56.0, H / 48.0)
    ca = np.array([rng.uniform(24, 30), rng.uniform(13, 16), rng.uniform(12, 14)]) * s      # calcaneus
    ta = np.array([rng.uniform(15, 19), rng.uniform(12, 15), rng.uniform(12, 13)]) * s      # talus
    na = np.array([rng.uniform(12, 13), rng.uniform(12, 15), rng.uniform(12, 13)]) * s      # navicular
    cc = np.array([4.0 * s + ca[0], W / 2, 3.0 * s + ca[2]])
    tc = np.array([cc[0] + 0.45 * ca[0], W / 2 + rng.uniform(-2, 2) * s, cc[2] + 0.75 * ca[2] + 0.7 * ta[2]])
    nc = np.array([tc[0] + 0.9 * ta[0] + 0.45 * na[0], W / 2 + rng.uniform(-2, 2) * s, tc[2] - 0.2 * ta[2]])
    tc[2] = min(tc[2], H - 2.0 * s - ta[2] * 0.85)
    nc[0] = min(nc[0], L - 2.0 * s - na[0] * 0.8)
    return [(tc, ta, p[0]), (cc, ca, p[1]), (nc, na, p[2])]


def hindfoot_problem(nx=160, ny=112, nz=96, h=0.5, seed=0, action="none", n_ligaments=40, total_load=450.0):
    """Synthetic hindfoot for ``solve_cn``; ``action`` in ACTIONS applies a seeded surgical edit:
    resection (bridge cells inactive), osteotomy (calcaneal fragment behind a plane shifted 3-8 mm along
    x), interposition (bridge E = 5 MPa), fusion (no split between talus and calcaneus: both become one
    part), load (load x U(0.5, 2)).  ``h`` is the voxel edge (mm), or (hx, hy, hz) for box-shaped voxels."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = (float(h),) * 3 if np.isscalar(h) else (float(v) for v in h)
    g = Grid(uniform_edges(nx, hx), uniform_edges(ny, hy), uniform_edges(nz, hz))
    L, W, H = nx * hx, ny * hy, nz * hz
    bones = _bone_layout(rng, L, W, H)
    arng = np.random.default_rng(seed + 7919)
    shift = 0.0
    if action == "osteotomy":
        shift = arng.uniform(3.0, 8.0)
    cut_x = bones[1][0][0] - 0.35 * bones[1][1][0]
    load_scale = arng.uniform(0.5, 2.0) if action == "load" else 1.0

    # 2x2x2 sub-samples per cell: bone label by depth (smallest super-ellipsoid value) where bones overlap
    ns = 2
    off = (np.arange(ns) + 0.5) / ns
    xs = (g.xe[:-1, None] + off[None] * g.dx[:, None]).ravel()
    ys = (g.ye[:-1, None] + off[None] * g.dy[:, None]).ravel()
    zs = (g.ze[:-1, None] + off[None] * g.dz[:, None]).ravel()
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")                 # (nx ns, ny ns, nz ns)
    best = np.full(X.shape, np.inf, np.float32)
    lab = np.zeros(X.shape, np.int8)
    depth = np.full(X.shape, np.inf, np.float32)
    for k, (c, a, p) in enumerate(bones, start=1):
        Xk = X
        if k == 2 and shift:
            Xk = np.where(X < cut_x, X + shift, X)                        # posterior fragment moved back
        v = _superellipsoid(Xk, Y, Z, c, a, p).astype(np.float32)
        inside = (v <= 1.0) & (v < best)
        lab[inside] = k; best[inside] = v[inside]
        depth = np.where(inside, (1.0 - v ** (1.0 / p)) * a.min(), depth)
    if shift:
        gap = (X >= cut_x - 0.5 * hx) & (X < cut_x + shift) & (lab == 2)
        lab[gap] = 0
    sub = lab.reshape(nx, ns, ny, ns, nz, ns).transpose(0, 2, 4, 1, 3, 5).reshape(nx, ny, nz, ns ** 3)
    share = np.stack([(sub == k).mean(-1) for k in range(len(bones) + 1)], -1).reshape(g.ncell, len(bones) + 1)
    dsub = depth.reshape(nx, ns, ny, ns, nz, ns).transpose(0, 2, 4, 1, 3, 5).reshape(g.ncell, ns ** 3)
    dmin = np.where(np.isfinite(dsub), dsub, np.inf).min(1)

    xc, yc, zc = g.cell_xyz.T
    # soft-tissue envelope (rounded box) and part / material per cell
    env = _superellipsoid(xc, yc, zc, (L / 2, W / 2, H / 2), (0.5 * L, 0.5 * W, 0.53 * H), 8.0) <= 1.0
    bone_frac = share[:, 1:].sum(1)
    part = np.where(share[:, 1:].max(1) >= 0.5, share[:, 1:].argmax(1) + 1, 0)
    # patchy cartilage: bone cells next to another bone become joint cells where a seeded field says so
    pg = part.reshape(nx, ny, nz)
    other = np.zeros_like(pg, bool)
    for d in range(3):
        for sgn in (1, -1):
            nb = np.roll(pg, sgn, axis=d)
            edge = [slice(None)] * 3; edge[d] = 0 if sgn == 1 else -1
            nb[tuple(edge)] = 0
            other |= (nb > 0) & (nb != pg) & (pg > 0)
    patch_c = rng.uniform([0, 0, 0], [L, W, H], (24, 3)); patch_r = rng.uniform(2.0, 5.0, 24)
    d2 = ((g.cell_xyz[:, None, :] - patch_c[None]) ** 2).sum(-1)
    in_patch = (d2 <= patch_r[None] ** 2).any(1)
    cart = other.ravel() & (part != 1) & in_patch
    # talocalcaneal coalition bridge: a slab between talus and calcaneus on the medial side
    (tcen, tax, _), (ccen, cax, _) = bones[0], bones[1]
    z_lo = ccen[2] + 0.55 * cax[2]; thick = rng.uniform(2.0, 4.0)
    bridge = (np.abs(xc - 0.5 * (tcen[0] + ccen[0])) < 0.35 * tax[0]) & (yc < W / 2 - 0.35 * tax[1]) & \
             (yc > W / 2 - 0.9 * tax[1]) & (zc > z_lo) & (zc < z_lo + thick) & (bone_frac < 0.5)
    part = np.where(cart, 0, part)
    if action == "fusion":
        part = np.where(part == 2, 1, part)                            # calcaneus joins the talus part
    shell = dmin < 1.5
    E = np.full(g.ncell, E_SOFT); nu = np.full(g.ncell, NU_SOFT)
    isbone = part > 0
    E[isbone & shell] = E_CORTICAL; E[isbone & ~shell] = E_CANCELLOUS; nu[isbone] = NU_BONE
    E[cart] = E_CART; nu[cart] = NU_CART
    if action == "interposition":
        E[bridge] = 5.0; nu[bridge] = NU_CART
    else:
        E[bridge] = E_BRIDGE; nu[bridge] = NU_BRIDGE
    active = env | isbone | bridge
    if action == "resection":
        active &= ~bridge
    lam, mu = lame(E, nu)
    cn, orig, nsplit = split_connectivity(g, active, part, share)

    cells = np.arange(g.ncell)
    xyz = g.node_xyz[orig]
    # plantar ground springs: z- faces of the active cells of the lowest layer, K_GROUND per interior node
    bottom = cells[(g.cK == 0) & active]
    fn, fa = face_node_areas(g, cn, bottom, "z-")
    fa = fa * (K_GROUND / (1e6 * hx * hy))
    # load on the talar dome: z+ faces of talus cells with no talus above, upper half of the talus
    tal = (part == 1) & active
    above = np.zeros(g.ncell, bool)
    kk = g.cK < nz - 1
    above[kk] = tal[cells[kk] + 1]
    dome = tal & ~above & (zc > tcen[2] + 0.3 * tax[2])
    ln, la = face_node_areas(g, cn, cells[dome], "z+")
    t = -total_load * load_scale / la.sum()
    loads = [(ln, la, np.array([0.0, 0.0, t]))]
    # interface springs: every split copy to the node that kept the grid id
    copies = np.arange(g.nnode, len(orig))
    springs = SpringSet(pair_a=copies, pair_b=orig[copies], pair_k=np.full(len(copies), K_INTERFACE))
    # ligaments: node pairs on different bones, 3 - 12 mm apart
    bone_nodes = {k: np.unique(cn[cells[(part == k) & active]].ravel()) for k in (1, 2, 3)}
    la_, lb_, ld_, lk_ = [], [], [], []
    pairs = [(1, 2), (1, 3), (2, 3)]
    tries = 0
    while len(la_) < n_ligaments and tries < 100 * n_ligaments:
        tries += 1
        ka, kb = pairs[rng.integers(len(pairs))]
        if not len(bone_nodes[ka]) or not len(bone_nodes[kb]):
            break
        a = bone_nodes[ka][rng.integers(len(bone_nodes[ka]))]
        bset = bone_nodes[kb]
        dist = np.linalg.norm(xyz[bset] - xyz[a], axis=1)
        ok = np.flatnonzero((dist > 3.0) & (dist < 12.0))
        if not len(ok):
            continue
        b = bset[ok[rng.integers(len(ok))]]
        d = xyz[b] - xyz[a]
        la_.append(a); lb_.append(b); ld_.append(d / np.linalg.norm(d)); lk_.append(rng.uniform(50.0, 200.0))
    springs.line_a = np.array(la_, np.int64); springs.line_b = np.array(lb_, np.int64)
    springs.line_d = np.array(ld_).reshape(-1, 3); springs.line_k = np.array(lk_)
    groups = [bone_nodes[k] for k in (1, 2, 3) if ((part == k) & active).sum() > 3]
    return dict(grid=g, E=E, nu=nu, lam=lam, mu=mu, active=active, part=part, bone_share=share, cn=cn, orig=orig,
                nsplit=nsplit, fixed=(fn, fa), loads=loads, extra=springs, node_groups=groups,
                contact=np.isin(cells, bottom), bridge=bridge, action=action,
                name=f"hindfoot {nx}x{ny}x{nz} h={h} seed={seed} action={action}")


def synthetic_template(seed=0, h=1.0):
    """A seeded stand-in for the engine's label template (rb/rbgeom.py:127-181 builds the real one from the CT
    atlas, which is not distributed): calcaneus below and talus above the subtalar joint, each a cortical shell
    around cancellous bone, three cartilage facets (posterior, middle, anterior) in the joint, tibia above the
    talus, a navicular in front, soft tissue around, in the template frame of the real one (joint inside
    labels.JOINT_BOX).  Distance maps of the subtalar region, facet frames and footprints are derived from the
    raster the way the real template derives them.  Returns a labels.Template."""
    from scipy import ndimage
    from .labels import Template, FACETS, SOFT
    rng = np.random.default_rng(seed)
    o = np.array([-112.0, -40.0, 0.0])
    shape = (int(round(136 / h)), int(round(80 / h)), int(round(110 / h)))
    x = o[0] + (np.arange(shape[0]) + 0.5) * h
    y = o[1] + (np.arange(shape[1]) + 0.5) * h
    z = o[2] + (np.arange(shape[2]) + 0.5) * h
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    lab = np.zeros(shape, np.int8)

    def ell(c, r, p=2.0):
        return (np.abs((X - c[0]) / r[0]) ** p + np.abs((Y - c[1]) / r[1]) ** p + np.abs((Z - c[2]) / r[2]) ** p) <= 1.0

    j = lambda s: s * (1.0 + 0.06 * rng.uniform(-1, 1))
    lab[ell((-50.0, 0.0, 52.0), (62.0, 32.0, 52.0))] = SOFT
    # the subtalar joint: a tilted surface z_j(x, y) with a gap of 2 g between the bones
    g = 1.2
    zj = 56.0 + j(0.12) * (X + 45.0) - 0.05 * Y
    cal = ell((-58.0, 0.0, 40.0), (j(42.0), j(17.0), j(22.0)), 2.4) & (Z < zj - g)
    tal = ell((-44.0, 2.0, 66.0), (j(22.0), j(15.0), j(14.0)), 2.2) & (Z > zj + g)
    for mask, cort, canc in ((cal, 1, 53), (tal, 2, 52)):
        inner = ndimage.binary_erosion(mask, iterations=max(1, int(round(1.5 / h))))
        lab[mask] = cort
        lab[inner] = canc
    tib = ell((-40.0, 0.0, 102.0), (j(12.0), j(12.0), j(20.0))) & ~tal
    lab[tib] = 4
    lab[ell((-40.0, 0.0, 104.0), (7.0, 7.0, 20.0)) & tib] = 13
    nav = ell((-8.0, 4.0, 58.0), (j(8.0), j(12.0), j(10.0))) & ~tal & ~cal
    lab[nav] = 40
    lab[ell((-44.0, 2.0, 86.5), (16.0, 11.0, 2.0)) & ~tal & ~tib] = 5          # ankle cartilage
    # facets: cartilage in the joint gap, elliptical patches centred where talus and calcaneus come closest
    gap = ~cal & ~tal & (lab == SOFT) & (np.abs(Z - zj) <= g)
    for name, cxy, ab in (("post", (-56.0, -3.0), (j(11.0), j(8.5))), ("mid", (-37.0, 8.0), (j(6.0), j(4.2))),
                          ("ant", (-28.0, 9.0), (j(4.2), j(3.6)))):
        patch = gap & (((X - cxy[0]) / ab[0]) ** 2 + ((Y - cxy[1]) / ab[1]) ** 2 <= 1.0)
        lab[patch] = FACETS[name]
    # subtalar region and distance maps (rb/rbgeom.py:140-150)
    sub_box = ((-100.0, 10.0), (-30.0, 38.0), (10.0, 100.0))
    i0, i1 = (int(round((b - o[0]) / h)) for b in sub_box[0])
    j0, j1 = (int(round((b - o[1]) / h)) for b in sub_box[1])
    k0, k1 = (int(round((b - o[2]) / h)) for b in sub_box[2])
    S = lab[i0:i1, j0:j1, k0:k1].astype(np.int16)
    talS = np.isin(S, (2, 52)); calS = np.isin(S, (1, 53))
    dt = (ndimage.distance_transform_edt(~talS) * h).astype(np.float16).astype(np.float32)
    dc = (ndimage.distance_transform_edt(~calS) * h).astype(np.float16).astype(np.float32)
    so = np.array([o[0] + i0 * h, o[1] + j0 * h, o[2] + k0 * h])
    grad = np.stack(np.gradient(dc - dt), -1)
    facets = {}
    for name, b in FACETS.items():
        P = (np.argwhere(S == b) + 0.5) * h + so
        c = P.mean(0)
        gv = grad[S == b]
        gv = gv / (np.linalg.norm(gv, axis=1, keepdims=True) + 1e-9)
        n = gv.mean(0); n /= np.linalg.norm(n)
        e1 = np.array([1.0, 0, 0]) - n[0] * n; e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)
        if e2[1] < 0:
            e2 = -e2
        u = (P - c) @ e1; v = (P - c) @ e2; w = (P - c) @ n
        res = 0.25
        ua, va = np.floor(u.min()) - 2, np.floor(v.min()) - 2
        nu_, nv_ = int((np.ceil(u.max()) + 2 - ua) / res), int((np.ceil(v.max()) + 2 - va) / res)
        F0 = np.zeros((nu_, nv_), bool)
        for du in np.arange(-h / 2 + res / 2, h / 2, res):
            for dv in np.arange(-h / 2 + res / 2, h / 2, res):
                iu = np.clip(((u + du - ua) / res).astype(int), 0, nu_ - 1)
                iv = np.clip(((v + dv - va) / res).astype(int), 0, nv_ - 1)
                F0[iu, iv] = True
        F0 = ndimage.binary_fill_holes(ndimage.binary_closing(F0, np.ones((5, 5)), iterations=2))
        gw = (dt.astype(float) + dc.astype(float))[S == b]
        facets[name] = dict(c=c, n=n, e1=e1, e2=e2, ua=float(ua), va=float(va), res=res, F0=F0,
                            a0=float(u.max() - u.min()) / 2, b0=float(v.max() - v.min()) / 2,
                            uc=float((u.max() + u.min()) / 2), vc=float((v.max() + v.min()) / 2),
                            wmax=float(np.abs(w).max()), gap=float(np.median(gw)),
                            xyz_lo=P.min(0) - h / 2, xyz_hi=P.max(0) + h / 2)
    static = {2, 52, 4, 13, 3, 54, 5, 6, 7}
    return Template(lab, o, h, dt, dc, so, facets, static)
