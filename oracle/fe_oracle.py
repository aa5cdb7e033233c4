"""CPU oracle for the voxel linear-elastic FE hot path of CoMech.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``comech_b200``) imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg do, and only as the
checker (or, for ``bench.py --impl reference``, as the timed CPU implementation of the reference
algorithm).

It is a NumPy/SciPy restatement, written for this project, of the reference algorithm:

* element matrices, grid indexing, Lame constants      -- fe/solver.py:11-134
* assembly, penalties, rank-1 penalties, solve          -- fe/solver.py:137-254
* stress / von Mises recovery                           -- fe/solver.py:257-272, rb/splitfe.py:161-175
* split-node connectivity                               -- rb/splitfe.py:261-305 (== :17-55)
* SRI lambda matrices, split assembly, solve_cn         -- rb/splitfe.py:58-158
* element forces                                        -- rb/splitfe.py:178-193
* geometric multigrid + PCG                             -- fe/gmg.py:7-137
* forces between regions, rigid fit, relative displacement, resampling on an analysis grid
                                                        -- rb/rbfe.py:194-219, rb/rbsim.py:99-161
* CG stopping rule                                      -- SciPy 1.18.1 ``scipy.sparse.linalg.cg``
  (installed dependency of the reference, not vendored): ``||r|| < rtol*||b||`` tested before
  every iteration, ``info = maxiter`` when the loop is exhausted.

Parity of this restatement is pinned against golden vectors produced by running the reference
itself (``tests/golden/make_golden.py``, committed fixtures in ``tests/golden/``).
"""
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# corner l of a hex8 cell sits at offset (l & 1, (l >> 1) & 1, (l >> 2) & 1)   (fe/solver.py:11-12)
CORNERS = np.array([(l & 1, (l >> 1) & 1, (l >> 2) & 1) for l in range(8)], dtype=np.int64)
GAUSS = 1.0 / np.sqrt(3.0)


def shape_gradients(pt, dims):
    """d N_l / d x_ax at natural point pt in [-1,1]^3 for a box of edge lengths dims (fe/solver.py:15-23)."""
    s = 2.0 * CORNERS - 1.0
    g = np.empty((8, 3))
    for ax in range(3):
        o1, o2 = [a for a in range(3) if a != ax]
        g[:, ax] = s[:, ax] * (1.0 + s[:, o1] * pt[o1]) * (1.0 + s[:, o2] * pt[o2]) / (4.0 * dims[ax])
    return g


def strain_matrix(g):
    """6x24 strain-displacement matrix, Voigt order xx yy zz xy yz xz, engineering shear (fe/solver.py:26-36)."""
    B = np.zeros((6, 8, 3))
    B[0, :, 0] = g[:, 0]
    B[1, :, 1] = g[:, 1]
    B[2, :, 2] = g[:, 2]
    B[3, :, 0] = g[:, 1]; B[3, :, 1] = g[:, 0]
    B[4, :, 1] = g[:, 2]; B[4, :, 2] = g[:, 1]
    B[5, :, 0] = g[:, 2]; B[5, :, 2] = g[:, 0]
    return B.reshape(6, 24)


D_LAMBDA = np.zeros((6, 6)); D_LAMBDA[:3, :3] = 1.0
D_MU = np.diag([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])
# orthotropic (z-normal) constitutive patterns, D = sum_k c_k P_k (fe/solver.py:43-52)
ORTHO_P = np.zeros((6, 6, 6))
ORTHO_P[0, 0, 0] = ORTHO_P[0, 1, 1] = 1
ORTHO_P[1, 0, 1] = ORTHO_P[1, 1, 0] = 1
ORTHO_P[2, 0, 2] = ORTHO_P[2, 2, 0] = ORTHO_P[2, 1, 2] = ORTHO_P[2, 2, 1] = 1
ORTHO_P[3, 2, 2] = 1
ORTHO_P[4, 3, 3] = 1
ORTHO_P[5, 4, 4] = ORTHO_P[5, 5, 5] = 1


def _gauss_points():
    return [np.array([x, y, z]) for x in (-GAUSS, GAUSS) for y in (-GAUSS, GAUSS) for z in (-GAUSS, GAUSS)]


def hex8_matrices(dims):
    """(K_lambda, K_mu, B_centre) of a box cell, 2x2x2 Gauss (fe/solver.py:77-90)."""
    dims = np.asarray(dims, float)
    w = dims.prod() / 8.0
    KL = np.zeros((24, 24)); KM = np.zeros((24, 24))
    for pt in _gauss_points():
        B = strain_matrix(shape_gradients(pt, dims))
        KL += w * (B.T @ D_LAMBDA @ B)
        KM += w * (B.T @ D_MU @ B)
    return KL, KM, strain_matrix(shape_gradients(np.zeros(3), dims))


def hex8_ortho_basis(dims):
    """(6, 24, 24) element matrices of the six orthotropic patterns (fe/solver.py:63-74)."""
    dims = np.asarray(dims, float)
    w = dims.prod() / 8.0
    K = np.zeros((6, 24, 24))
    for pt in _gauss_points():
        B = strain_matrix(shape_gradients(pt, dims))
        K += w * np.einsum("ai,kab,bj->kij", B, ORTHO_P, B)
    return K


def ortho_coeffs(lam, mu, shear_factor=None):
    """Isotropic (lam, mu) as orthotropic pattern coefficients (fe/solver.py:55-60)."""
    c = np.stack([lam + 2 * mu, lam, lam, lam + 2 * mu, mu, mu], 1)
    if shear_factor is not None:
        c[:, 5] *= shear_factor
    return c


def lame(E, nu):
    """Lame constants (fe/solver.py:131-134)."""
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


class OGrid:
    """Rectilinear voxel grid (fe/solver.py:93-128).

    node id = i + (nx+1) (j + (ny+1) k)  (x fastest); cell id = (i ny + j) nz + k  (z fastest)."""

    def __init__(self, xe, ye, ze):
        self.xe, self.ye, self.ze = (np.asarray(e, float) for e in (xe, ye, ze))
        self.nx, self.ny, self.nz = len(self.xe) - 1, len(self.ye) - 1, len(self.ze) - 1
        self.shape = (self.nx, self.ny, self.nz)
        self.ncell = self.nx * self.ny * self.nz
        self.nnode = (self.nx + 1) * (self.ny + 1) * (self.nz + 1)
        self.dx, self.dy, self.dz = np.diff(self.xe), np.diff(self.ye), np.diff(self.ze)
        ci = np.arange(self.ncell)
        self.cK = ci % self.nz
        self.cJ = (ci // self.nz) % self.ny
        self.cI = ci // (self.nz * self.ny)
        nx1, ny1 = self.nx + 1, self.ny + 1
        self.cell_nodes = np.stack([(self.cI + a) + nx1 * ((self.cJ + b) + ny1 * (self.cK + c))
                                    for a, b, c in CORNERS], axis=1)
        dims = np.stack([self.dx[self.cI], self.dy[self.cJ], self.dz[self.cK]], 1)
        ud, inv = np.unique(np.round(dims, 6), axis=0, return_inverse=True)
        self.dim_id = inv.ravel()
        self.udims = ud
        mats = [hex8_matrices(d) for d in ud]
        self.KL = np.stack([m[0] for m in mats])
        self.KM = np.stack([m[1] for m in mats])
        self.Bc = np.stack([m[2] for m in mats])
        self._KB = None
        self.cell_vol = dims.prod(1)
        nid = np.arange(self.nnode)
        self.node_xyz = np.stack([self.xe[nid % nx1], self.ye[(nid // nx1) % ny1], self.ze[nid // (nx1 * ny1)]], 1)
        self.cell_xyz = np.stack([(self.xe[:-1] + self.xe[1:])[self.cI] / 2, (self.ye[:-1] + self.ye[1:])[self.cJ] / 2,
                                  (self.ze[:-1] + self.ze[1:])[self.cK] / 2], 1)

    @property
    def KB(self):
        if self._KB is None:
            self._KB = np.stack([hex8_ortho_basis(d) for d in self.udims])
        return self._KB

    def cid(self, i, j, k):
        return (i * self.ny + j) * self.nz + k


def kl_sri(g):
    """One-point (cell-centre) lambda matrices per dim family (rb/splitfe.py:58-69)."""
    vol = g.udims.prod(1)
    return np.stack([vol[d] * (g.Bc[d].T @ D_LAMBDA @ g.Bc[d]) for d in range(len(g.udims))])


def face_node_areas(g, cn, cells, face):
    """Tributary area (1/4 of the face) of the 4 face nodes of each cell (fe/solver.py:165-174,
    rb/splitfe.py:94-102); cn is g.cell_nodes or a split connectivity."""
    ax = "xyz".index(face[0]); side = 1 if face[1] == "+" else 0
    sel = CORNERS[:, ax] == side
    nodes = cn[cells][:, sel]
    d = [g.dx[g.cI[cells]], g.dy[g.cJ[cells]], g.dz[g.cK[cells]]]
    o = [d[i] for i in range(3) if i != ax]
    return nodes.ravel(), np.repeat(o[0] * o[1] / 4.0, 4)


# ----------------------------------------------------------------------------------------- split nodes
def split_connectivity(g, active, part, bone_share):
    """Split nodes shared by cells of >=2 bones into one copy per bone (rb/splitfe.py:261-305).

    The lowest bone keeps the grid id; every other (node, bone) pair of a split node gets id nnode+k in
    ascending (node, bone) order.  A part-0 cell at a split node takes the copy of the bone with the
    largest share in the cell (first maximum in ascending bone order), or, when it holds none of them,
    the bone with the most bone cells at the node.  Returns cn (ncell, 8), orig (nnew,), nsplit."""
    cells = np.flatnonzero(active)
    corner_nodes = g.cell_nodes[cells]
    pc = np.asarray(part)[cells].astype(np.int64)
    nb = bone_share.shape[1]
    bone_rows = pc > 0
    pair_key = corner_nodes[bone_rows].astype(np.int64) * nb + pc[bone_rows, None]
    keys, counts = np.unique(pair_key.ravel(), return_counts=True)
    knode, kbone = keys // nb, keys % nb
    nbones_at = np.bincount(knode, minlength=g.nnode)
    is_split = nbones_at >= 2
    first_of_node = np.r_[True, knode[1:] != knode[:-1]]
    gets_copy = is_split[knode] & ~first_of_node
    copy_id = np.full(len(keys), -1, np.int64)
    copy_id[gets_copy] = g.nnode + np.arange(int(gets_copy.sum()))
    orig = np.concatenate([np.arange(g.nnode), knode[gets_copy]])
    start = np.searchsorted(knode, np.arange(g.nnode))
    cn = g.cell_nodes.copy()
    r, l = np.nonzero(is_split[corner_nodes])
    if len(r):
        n = corner_nodes[r, l]
        c = cells[r]
        b = pc[r].copy()
        soft = np.flatnonzero(b == 0)
        if len(soft):
            ns, cs = n[soft], c[soft]
            best_share = np.full(len(soft), -1.0); best_share_bone = np.zeros(len(soft), np.int64)
            best_cnt = np.full(len(soft), -1, np.int64); best_cnt_bone = np.zeros(len(soft), np.int64)
            for j in range(int(nbones_at[ns].max())):
                has = j < nbones_at[ns]
                idx = np.flatnonzero(has)
                p = start[ns[idx]] + j
                bb = kbone[p]
                sh = bone_share[cs[idx], bb]
                better = sh > best_share[idx]
                best_share[idx[better]] = sh[better]; best_share_bone[idx[better]] = bb[better]
                more = counts[p] > best_cnt[idx]
                best_cnt[idx[more]] = counts[p][more]; best_cnt_bone[idx[more]] = bb[more]
            b[soft] = np.where(best_share > 0, best_share_bone, best_cnt_bone)
        cid = copy_id[np.searchsorted(keys, n * nb + b)]
        take = cid >= 0
        cn[c[take], l[take]] = cid[take]
    return cn, orig, int(is_split.sum())


# ----------------------------------------------------------------------------------------- assembly
def assemble(g, lam, mu, cells, cn, lam_mats, coeffs=None):
    """Global stiffness on compact dofs: dof = 3 nmap[node] + comp, nmap over the used nodes in ascending
    id order (fe/solver.py:137-162, rb/splitfe.py:72-91).  lam_mats: per-family lambda matrices
    (full 2x2x2 or SRI); coeffs: orthotropic pattern coefficients (ncell, 6) instead of (lam, mu)."""
    nused = np.unique(cn[cells])
    nmap = -np.ones(int(cn.max()) + 1, np.int64)
    nmap[nused] = np.arange(len(nused))
    dofs = (3 * nmap[cn[cells]][:, :, None] + np.arange(3)).reshape(len(cells), 24)
    did = g.dim_id[cells]
    Ke = np.empty((len(cells), 24, 24))
    for d in np.unique(did):
        m = np.flatnonzero(did == d)
        if coeffs is None:
            Ke[m] = lam[cells[m], None, None] * lam_mats[d] + mu[cells[m], None, None] * g.KM[d]
        else:
            Ke[m] = np.einsum("nk,kij->nij", coeffs[cells[m]], g.KB[d])
    n = 3 * len(nused)
    rows = np.broadcast_to(dofs[:, :, None], Ke.shape).ravel()
    cols = np.broadcast_to(dofs[:, None, :], Ke.shape).ravel()
    K = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(n, n)).tocsr()
    return K, nmap, nused


def rigid_modes(xyz, nmap, n, node_groups):
    """Per group 3 translations + 3 rotations (about x, y, z) with r = (X - mean X) / 20
    (fe/solver.py:177-199, rb/splitfe.py:105-120); groups with <4 used nodes are skipped."""
    rows, cols, vals = [], [], []
    col = 0
    for nodes in node_groups:
        nodes = np.asarray(nodes)
        ln = nmap[nodes]
        ok = ln >= 0
        nodes, ln = nodes[ok], ln[ok]
        if len(nodes) < 4:
            continue
        X = xyz[nodes]
        r = (X - X.mean(0)) / 20.0
        for d in range(3):
            rows.append(3 * ln + d); cols.append(np.full(len(ln), col)); vals.append(np.ones(len(ln)))
            col += 1
        for pairs in (((1, -r[:, 2]), (2, r[:, 1])), ((0, r[:, 2]), (2, -r[:, 0])), ((0, -r[:, 1]), (1, r[:, 0]))):
            for d, v in pairs:
                rows.append(3 * ln + d); cols.append(np.full(len(ln), col)); vals.append(v)
            col += 1
    if not rows:
        return sp.csr_matrix((n, 0))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, col))


# ----------------------------------------------------------------------------------------- multigrid
def p1d(coords):
    """1-D linear prolongation from every other node plus the last one (fe/gmg.py:7-26)."""
    coords = np.asarray(coords, float)
    n = len(coords)
    cidx = np.arange(0, n, 2)
    if cidx[-1] != n - 1:
        cidx = np.r_[cidx, n - 1]
    fine = np.setdiff1d(np.arange(n), cidx)
    right = np.searchsorted(cidx, fine)
    left = right - 1
    w = (coords[fine] - coords[cidx[left]]) / (coords[cidx[right]] - coords[cidx[left]])
    rows = np.r_[cidx, fine, fine]
    cols = np.r_[np.arange(len(cidx)), left, right]
    vals = np.r_[np.ones(len(cidx)), 1 - w, w]
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, len(cidx))), coords[cidx]


def block_diag_inverse(A):
    """Inverses of the 3x3 diagonal blocks; blocks with |det| < 1e-30 become I (fe/gmg.py:29-44)."""
    A = A.tocoo()
    same = (A.row // 3) == (A.col // 3)
    D = np.zeros((A.shape[0] // 3, 3, 3))
    np.add.at(D, (A.row[same] // 3, A.row[same] % 3, A.col[same] % 3), A.data[same])
    D[np.abs(np.linalg.det(D)) < 1e-30] = np.eye(3)
    return np.linalg.inv(D)


class ChebyshevLevel:
    """Block-Jacobi preconditioned Chebyshev smoother; lambda_max of M^-1 A from 12 power steps from
    a standard-normal vector of rng seed 0; lmax = 1.1 lambda, lmin = lmax / 30 (fe/gmg.py:47-76)."""

    def __init__(self, A, start=None):
        self.A = A.tocsr()
        self.Dinv = block_diag_inverse(self.A)
        x = np.random.default_rng(0).standard_normal(A.shape[0]) if start is None else np.array(start, float)
        lam = 1.0
        for _ in range(12):
            y = self.M(self.A @ x)
            lam = np.linalg.norm(y) / np.linalg.norm(x)
            x = y / np.linalg.norm(y)
        self.lam = lam
        self.lmax = 1.1 * lam
        self.lmin = self.lmax / 30.0

    def M(self, r):
        return np.einsum("nij,nj->ni", self.Dinv, r.reshape(-1, 3)).ravel()

    def smooth(self, x, b, deg=3):
        theta = (self.lmax + self.lmin) / 2
        delta = (self.lmax - self.lmin) / 2
        sigma = theta / delta
        rho = 1.0 / sigma
        r = b - self.A @ x
        d = self.M(r) / theta
        for k in range(deg):
            x = x + d
            if k == deg - 1:
                break
            r = r - self.A @ d
            rho_next = 1.0 / (2.0 * sigma - rho)
            d = rho_next * rho * d + (2.0 * rho_next / delta) * self.M(r)
            rho = rho_next
        return x


class Multigrid:
    """Galerkin geometric multigrid (fe/gmg.py:79-113): P = kron(Pz, Py, Px) (x) I3 restricted to the
    active dofs, coarse dofs = nonzero columns, A_c = P^T A P, at most 6 levels, stop at <= 6000 dofs,
    coarsest level solved directly."""

    def __init__(self, A, used_nodes, xe, ye, ze, min_dofs=6000, max_levels=6):
        self.levels, self.P = [], []
        act = (3 * np.asarray(used_nodes)[:, None] + np.arange(3)).ravel()
        coords = (np.asarray(xe, float), np.asarray(ye, float), np.asarray(ze, float))
        Acur = A.tocsr()
        for _ in range(max_levels):
            self.levels.append(ChebyshevLevel(Acur))
            if Acur.shape[0] <= min_dofs:
                break
            (Px, cx), (Py, cy), (Pz, cz) = (p1d(c) for c in coords)
            Pd = sp.kron(sp.kron(Pz, sp.kron(Py, Px)), sp.identity(3)).tocsr()[act]
            keep = np.flatnonzero(np.asarray(abs(Pd).sum(0)).ravel() > 0)
            Pd = Pd[:, keep].tocsr()
            Acur = (Pd.T @ Acur @ Pd).tocsr()
            self.P.append(Pd)
            act = keep
            coords = (cx, cy, cz)
        self.coarse = spla.splu(Acur.tocsc(), permc_spec="MMD_AT_PLUS_A")

    def vcycle(self, b, l=0):
        if l == len(self.levels) - 1:
            return self.coarse.solve(b)
        L = self.levels[l]
        x = L.smooth(np.zeros_like(b), b)
        ec = self.vcycle(self.P[l].T @ (b - L.A @ x), l + 1)
        return L.smooth(x + self.P[l] @ ec, b)


def pcg(A, b, precond, tol, maxiter, x0=None):
    """Preconditioned CG with SciPy's stopping rule: before each iteration stop when ||r|| < tol ||b||;
    flag = maxiter when the loop runs out (scipy.sparse.linalg.cg, SciPy 1.18.1)."""
    bn = np.linalg.norm(b)
    if bn == 0:
        return b.copy(), 0, 0
    thr = tol * bn
    x = np.zeros_like(b) if x0 is None else np.array(x0, float)
    r = b - A @ x if x.any() else b.copy()
    p = None; rz_prev = None
    for it in range(maxiter):
        if np.linalg.norm(r) < thr:
            return x, 0, it
        z = precond(r)
        rz = r @ z
        p = z.copy() if it == 0 else z + (rz / rz_prev) * p
        q = A @ p
        alpha = rz / (p @ q)
        x = x + alpha * p
        r = r - alpha * q
        rz_prev = rz
    return x, maxiter, maxiter


def pcg_gmg(A, b, used_nodes, grid_edges, tol=1e-7, maxiter=500, x0=None, Z=None):
    """GMG-preconditioned CG with an optional additive correction Z pinv(Z^T A Z) Z^T (fe/gmg.py:120-137)."""
    t0 = time.perf_counter()
    mg = Multigrid(A, used_nodes, *grid_edges)
    prec = mg.vcycle
    if Z is not None and Z.shape[1] > 0:
        Zd = Z.toarray() if sp.issparse(Z) else np.asarray(Z)
        Ec = Zd.T @ (A @ Zd)
        Einv = np.linalg.pinv(0.5 * (Ec + Ec.T))
        prec = lambda r: mg.vcycle(r) + Zd @ (Einv @ (Zd.T @ r))
    t1 = time.perf_counter()
    x, flag, iters = pcg(A, b, prec, tol, maxiter, x0)
    t2 = time.perf_counter()
    return x, dict(iters=iters, flag=flag, levels=len(mg.levels), t_setup=t1 - t0, t_pcg=t2 - t1)


def spring_matrix_cn(xyz, springs, bone_nodes):
    """Ligament hook for solve_cn's ``extra`` (rb/replica3.py:68-86): spring s pulls along d = (b - a)/|b - a|;
    each end is the mean over the used nodes of its bone within max(4 mm, distance of the 8th-nearest), so
    w = +d/n_A on the A-end nodes and -d/n_B on the B-end nodes, and K += k w w^T."""
    def build(nmap, n):
        rows, cols, vals = [], [], []
        for s in springs:
            a, b = np.asarray(s["a"], float), np.asarray(s["b"], float)
            d = (b - a) / np.linalg.norm(b - a)
            w = np.zeros(n)
            for pt, sign, key in ((a, 1.0, "A"), (b, -1.0, "B")):
                cand = np.asarray(bone_nodes[s[key]])
                cand = cand[nmap[cand] >= 0]
                dist = np.linalg.norm(xyz[cand] - pt, axis=1)
                radius = max(4.0, np.sort(dist)[min(7, len(dist) - 1)])
                ln = nmap[cand[dist <= radius]]
                for c in range(3):
                    np.add.at(w, 3 * ln + c, sign * d[c] / len(ln))
            nz = np.flatnonzero(w)
            rows.append(np.repeat(nz, len(nz)))
            cols.append(np.tile(nz, len(nz)))
            vals.append(s["k"] * np.outer(w[nz], w[nz]).ravel())
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return build


# ----------------------------------------------------------------------------------------- solves
def solve_cn(g, lam, mu, active, cn, orig, fixed, loads, extra=None, node_groups=None, tol=1e-6, maxiter=800):
    """Split-node solve (rb/splitfe.py:123-158): ground penalty k = 1e6 per unit area on all three
    components of the fixed nodes, nodal loads area * t, K += diag(kd) + extra(nmap, n), per-bone rigid
    modes, GMG-PCG.  Returns U (nnew, 3) with NaN on unused nodes, info, reactions R."""
    t0 = time.perf_counter()
    cells = np.flatnonzero(active)
    K, nmap, nused = assemble(g, lam, mu, cells, cn, kl_sri(g))
    n = K.shape[0]
    f = np.zeros(n); kd = np.zeros(n)
    fn, fa = fixed
    for c in range(3):
        np.add.at(kd, 3 * nmap[fn] + c, fa * 1e6)
    for nodes, area, t in loads:
        for c in range(3):
            np.add.at(f, 3 * nmap[nodes] + c, area * t[c])
    K = K + sp.diags(kd)
    if extra is not None:
        K = K + extra(nmap, n)
    Z = rigid_modes(g.node_xyz[orig], nmap, n, node_groups) if node_groups else None
    t_asm = time.perf_counter() - t0
    u, info = pcg_gmg(K, f, orig[nused], (g.xe, g.ye, g.ze), tol=tol, Z=Z, maxiter=maxiter)
    info["t_assemble"] = t_asm
    U = np.full((len(orig), 3), np.nan)
    U[nused] = u.reshape(-1, 3)
    R = np.zeros((len(orig), 3))
    np.add.at(R, fn, -(fa[:, None] * 1e6) * U[fn])
    info["ndof"] = n
    return U, info, R


def solve(g, lam, mu, active, springs, loads, method="cg", tol=1e-8, x0=None, maxiter=20000, penalties=(),
          coeffs=None, node_groups=None, U0=None):
    """Single-connectivity solve (fe/solver.py:202-254): per-direction area springs, nodal loads, rank-1
    penalties k w w^T with w normalised to unit sum; method gmg / direct / cg (Jacobi PCG)."""
    cells = np.flatnonzero(active)
    K, nmap, used = assemble(g, lam, mu, cells, g.cell_nodes, g.KL, coeffs)
    n = K.shape[0]
    if U0 is not None:
        x0 = np.nan_to_num(U0[used]).ravel()
    f = np.zeros(n); kd = np.zeros(n)
    for nodes, area, kvec in springs:
        ln = nmap[nodes]; ok = ln >= 0
        for c in range(3):
            np.add.at(kd, 3 * ln[ok] + c, area[ok] * kvec[c])
    for nodes, area, t in loads:
        ln = nmap[nodes]; ok = ln >= 0
        for c in range(3):
            np.add.at(f, 3 * ln[ok] + c, area[ok] * t[c])
    K = K + sp.diags(kd)
    for nodes, weights, comp, k in penalties:
        ln = nmap[nodes]; ok = ln >= 0
        w = np.zeros(n)
        np.add.at(w, 3 * ln[ok] + comp, weights[ok])
        w /= w.sum()
        nz = np.flatnonzero(w)
        K = K + sp.csr_matrix((k * np.outer(w[nz], w[nz]).ravel(), (np.repeat(nz, len(nz)), np.tile(nz, len(nz)))),
                              shape=K.shape)
    info = {}
    if method == "gmg":
        Z = rigid_modes(g.node_xyz, nmap, n, node_groups) if node_groups else None
        u, inf = pcg_gmg(K, f, used, (g.xe, g.ye, g.ze), tol=tol, x0=x0, Z=Z)
        info.update(inf)
    elif method == "direct":
        u = spla.spsolve(K.tocsc(), f, permc_spec="MMD_AT_PLUS_A")
        info["iters"] = 0
    else:
        dinv = 1.0 / K.diagonal()
        u, flag, iters = pcg(K, f, lambda r: dinv * r, tol, maxiter, x0)
        info["iters"] = iters; info["flag"] = flag
    U = np.full((g.nnode, 3), np.nan)
    U[used] = u.reshape(-1, 3)
    info.update(ndof=n, K=K, f=f, used=used)
    return U, info


def von_mises(sig):
    sx, sy, sz, txy, tyz, txz = sig.T
    return np.sqrt(0.5 * ((sx - sy) ** 2 + (sy - sz) ** 2 + (sz - sx) ** 2) + 3 * (txy ** 2 + tyz ** 2 + txz ** 2))


def cell_stress(g, lam, mu, U, cells, cn=None, coeffs=None, nan_to_zero=False):
    """Centre-point strain, Cauchy stress and von Mises (fe/solver.py:257-272; the split version
    rb/splitfe.py:161-175 passes its connectivity and zeroes NaNs first)."""
    cn = g.cell_nodes if cn is None else cn
    ue = U[cn[cells]].reshape(len(cells), 24)
    if nan_to_zero:
        ue = np.nan_to_num(ue)
    eps = np.einsum("nij,nj->ni", g.Bc[g.dim_id[cells]], ue)
    if coeffs is None:
        tr = eps[:, :3].sum(1)
        sig = np.empty_like(eps)
        sig[:, :3] = lam[cells, None] * tr[:, None] + 2 * mu[cells, None] * eps[:, :3]
        sig[:, 3:] = mu[cells, None] * eps[:, 3:]
    else:
        sig = np.einsum("nij,nj->ni", np.einsum("nk,kij->nij", coeffs[cells], ORTHO_P), eps)
    return sig, von_mises(sig), eps


def element_forces(g, lam, mu, U, cells, cn):
    """Internal nodal forces K_e u_e of selected cells with SRI lambda matrices (rb/splitfe.py:178-193)."""
    ue = np.nan_to_num(U[cn[cells]].reshape(len(cells), 24))
    KLs = kl_sri(g)
    did = g.dim_id[cells]
    out = np.zeros((len(cells), 24))
    for d in np.unique(did):
        m = did == d
        out[m] = lam[cells[m], None] * (ue[m] @ KLs[d].T) + mu[cells[m], None] * (ue[m] @ g.KM[d].T)
    return out.reshape(len(cells), 8, 3)


# ------------------------------------------------------------------------------------------ post-processing
def region_forces(g, lam, mu, U, cn, active, part, lab, nlab, target):
    """Forces on the nodes of the active cells of part ``target`` from every other active cell touching them,
    summed per cell label (the sums of rb/rbfe.py:199-213).  Returns (nlab x 3, present flags)."""
    cells = np.arange(g.ncell)
    tgt = (part == target) & active
    tn = np.zeros(len(U), bool)
    tn[cn[cells[tgt]].ravel()] = True
    oc = cells[active & ~tgt]
    oc = oc[tn[cn[oc]].any(1)]
    fsum = -(element_forces(g, lam, mu, U, oc, cn) * tn[cn[oc]][:, :, None]).sum(1)
    out = np.zeros((nlab, 3))
    present = np.zeros(nlab, bool)
    for i in range(nlab):
        m = lab[oc] == i
        if m.any():
            out[i] = fsum[m].sum(0)
            present[i] = True
    return out, present


def rigid_fit(X, U):
    """Least-squares rigid motion U ~ t + w x (X - c) (rb/rbsim.py:99-107); minimum-norm lstsq."""
    c = X.mean(0)
    r = X - c
    A = np.zeros((3 * len(X), 6))
    A[0::3, 0] = A[1::3, 1] = A[2::3, 2] = 1.0
    A[0::3, 4], A[0::3, 5] = r[:, 2], -r[:, 1]
    A[1::3, 3], A[1::3, 5] = -r[:, 2], r[:, 0]
    A[2::3, 3], A[2::3, 4] = r[:, 1], -r[:, 0]
    sol = np.linalg.lstsq(A, U.ravel(), rcond=None)[0]
    return sol[:3], sol[3:], c


def relative_displacement(xyz, U, t, w, c):
    """nan_to_num(U) minus the rigid motion (rb/rbsim.py:184)."""
    return np.nan_to_num(U) - (t[None, :] + np.cross(w[None, :], xyz - c[None, :]))


def _axis_samples(fe_edges, ml_edges, sub):
    """Per analysis-grid axis: the sub points per cell, the FE cell holding each, the local coordinate in it
    and whether the point lies inside the FE grid (rb/rbsim.py:112-119)."""
    oo = (np.arange(sub) + 0.5) / sub
    X = (ml_edges[:-1, None] + np.diff(ml_edges)[:, None] * oo).ravel()
    n = len(fe_edges) - 1
    i = np.clip(np.searchsorted(fe_edges, X) - 1, 0, n - 1)
    t = np.clip((X - fe_edges[i]) / np.diff(fe_edges)[i], 0, 1)
    inside = (X >= fe_edges[0]) & (X <= fe_edges[-1])
    return i, t, inside


def sample_fe(g, cn, active, VM, SIG, Urel, ml_edges, sub=2):
    """Mean von Mises, relative displacement and stress over the sub^3 points of every analysis cell that
    fall in active FE cells, and the fraction of such points (rb/rbsim.py:110-138).  Returns
    (vm, u, frac, sig), float32."""
    (i, tx, ix), (j, ty, iy), (k, tz, iz) = (_axis_samples(e, m, sub) for e, m in zip((g.xe, g.ye, g.ze), ml_edges))
    I, J, K = np.meshgrid(i, j, k, indexing="ij")
    c = ((I * g.ny + J) * g.nz + K).ravel()
    ok = (ix[:, None, None] & iy[None, :, None] & iz[None, None, :]).ravel() & active[c]
    TX, TY, TZ = (a.ravel() for a in np.meshgrid(tx, ty, tz, indexing="ij"))
    u = np.zeros((len(c), 3))
    for l in range(8):
        a, b, d = CORNERS[l]
        w = np.where(a, TX, 1 - TX) * np.where(b, TY, 1 - TY) * np.where(d, TZ, 1 - TZ)
        u += w[:, None] * np.nan_to_num(Urel[cn[c, l]])
    vm = np.where(ok, VM[c], 0.0)
    sg = np.where(ok[:, None], SIG[c], 0.0)
    mx, my, mz = (len(m) - 1 for m in ml_edges)

    def cellsum(a):
        a = a.reshape(mx, sub, my, sub, mz, sub, *a.shape[1:]).transpose(0, 2, 4, 1, 3, 5, *range(6, a.ndim + 5))
        return a.reshape(mx * my * mz, sub ** 3, *a.shape[6:]).sum(1)
    okc = cellsum(ok.astype(np.float32))
    den = np.maximum(okc, 1)
    return ((cellsum(vm) / den).astype(np.float32), (cellsum(u * ok[:, None]) / den[:, None]).astype(np.float32),
            okc / sub ** 3, (cellsum(sg) / den[:, None]).astype(np.float32))


def sample_nodes(g, cn, active, Urel, ml_node_xyz):
    """Relative displacement at analysis-grid nodes: trilinear in the FE cell that holds the node, or in the
    nearest active FE cell (exact Euclidean feature transform over cell indices, clamped local coordinates)
    for nodes in empty cells (rb/rbsim.py:141-161)."""
    from scipy import ndimage
    P = ml_node_xyz
    i = np.clip(np.searchsorted(g.xe, P[:, 0]) - 1, 0, g.nx - 1)
    j = np.clip(np.searchsorted(g.ye, P[:, 1]) - 1, 0, g.ny - 1)
    k = np.clip(np.searchsorted(g.ze, P[:, 2]) - 1, 0, g.nz - 1)
    _, ind = ndimage.distance_transform_edt(~active.reshape(g.nx, g.ny, g.nz), return_indices=True)
    ci, cj, ck = ind[0, i, j, k], ind[1, i, j, k], ind[2, i, j, k]
    c = (ci * g.ny + cj) * g.nz + ck
    dx, dy, dz = np.diff(g.xe), np.diff(g.ye), np.diff(g.ze)
    tx = np.clip((P[:, 0] - g.xe[ci]) / dx[ci], 0, 1)
    ty = np.clip((P[:, 1] - g.ye[cj]) / dy[cj], 0, 1)
    tz = np.clip((P[:, 2] - g.ze[ck]) / dz[ck], 0, 1)
    u = np.zeros((len(P), 3))
    for l in range(8):
        a, b, d = CORNERS[l]
        w = np.where(a, tx, 1 - tx) * np.where(b, ty, 1 - ty) * np.where(d, tz, 1 - tz)
        u += w[:, None] * np.nan_to_num(Urel[cn[c, l]])
    return u.astype(np.float32)


# ------------------------------------------------------------------------------------------ material mixing
MIX_CLASSES = ["void", "cortical", "cancellous", "cartilage", "fascia", "soft", "plate", "fibrous", "fat", "gap"]
MIX_MAT = {"cortical": (7300.0, 0.3), "cancellous": (100.0, 0.3), "cartilage": (10.0, 0.4), "fascia": (350.0, 0.4),
           "soft": (1.15, 0.49), "plate": (17000.0, 0.1), "fibrous": (60.0, 0.4), "fat": (1.15, 0.45),
           "gap": (0.01, 0.3)}


def mix_materials(cls, L, shape, groups, cart_E=10.0, nu_soft=0.49):
    """Class fractions and constrained-modulus mixing of the engine (rb/rbfe.py:75-134).  cls: body -> class,
    L: ncell x ns^3 body labels, groups: bone body -> group id.  Returns (E, nu, active, F, ser)."""
    from scipy import ndimage
    nb = max(max(cls), int(L.max()))
    lut = np.zeros(nb + 1, np.int16)
    for b, c in cls.items():
        lut[b] = c
    C = lut[L]
    F = np.stack([(C == k).mean(1) for k in range(len(MIX_CLASSES))], 1).astype(np.float64)
    mat = dict(MIX_MAT)
    mat["cartilage"] = (cart_E, 0.4)
    mat["soft"] = (1.15, nu_soft)
    E_ = np.array([1.0] + [mat[c][0] for c in MIX_CLASSES[1:]])
    nu_ = np.array([0.3] + [mat[c][1] for c in MIX_CLASSES[1:]])
    lam_i = E_ * nu_ / ((1 + nu_) * (1 - 2 * nu_))
    mu_i = E_ / (2 * (1 + nu_))
    H, LAY, SOFTC, GAPC = [1, 2, 4], [3, 7], [5, 8], [9]
    PH = H + LAY + SOFTC
    occ = F[:, PH].sum(1)
    hard, lay, fgap = F[:, H].sum(1), F[:, LAY].sum(1), F[:, GAPC].sum(1)
    with np.errstate(divide="ignore", invalid="ignore"):
        lamV = (F[:, PH] * lam_i[PH]).sum(1) / occ
        muV = (F[:, PH] * mu_i[PH]).sum(1) / occ
        lam_h = (F[:, H] * lam_i[H]).sum(1) / hard
        mu_h = (F[:, H] * mu_i[H]).sum(1) / hard
        M_h, G_h = lam_h + 2 * mu_h, mu_h
        hM = np.where(hard > 0, hard / M_h, 0.0)
        hG = np.where(hard > 0, hard / G_h, 0.0)
        Mi = lam_i + 2 * mu_i
        gapM = (F[:, GAPC] / Mi[GAPC]).sum(1)
        gapG = (F[:, GAPC] / mu_i[GAPC]).sum(1)
        layM = (F[:, LAY] / Mi[LAY]).sum(1) + gapM
        layG = (F[:, LAY] / mu_i[LAY]).sum(1) + gapG
        fch = lay + hard + fgap
        occ_g = occ + fgap
        M_ch, G_ch = fch / (layM + hM), fch / (layG + hG)
        lam_soft = (F[:, SOFTC] * lam_i[SOFTC]).sum(1)
        mu_soft = (F[:, SOFTC] * mu_i[SOFTC]).sum(1)
        lam_c = (fch * (M_ch - 2 * G_ch) + lam_soft) / occ_g
        mu_c = (fch * G_ch + mu_soft) / occ_g
        softM = (F[:, SOFTC] / Mi[SOFTC]).sum(1)
        softG = (F[:, SOFTC] / mu_i[SOFTC]).sum(1)
        M_s = occ_g / (softM + hM + gapM)
        G_s = occ_g / (softG + hG + gapG)
        lam_s, mu_s = M_s - 2 * G_s, G_s
    lutg = np.zeros(nb + 1, np.int16)
    for b, k in groups.items():
        lutg[b] = k
    Gb = lutg[L]
    count = np.zeros(len(L), np.int16)
    for k in np.unique(Gb[Gb > 0]):
        count += ndimage.binary_dilation((Gb == k).any(1).reshape(shape), np.ones((3, 3, 3), bool)).ravel()
    cart = lay > 0
    ser = cart | (count >= 2)
    lamX = np.where(cart, lam_c, np.where(ser, lam_s, lamV))
    muX = np.where(cart, mu_c, np.where(ser, mu_s, muV))
    with np.errstate(divide="ignore", invalid="ignore"):
        E = muX * (3 * lamX + 2 * muX) / (lamX + muX)
        nu = lamX / (2 * (lamX + muX))
    active = np.where(ser, occ > 0.15, occ >= 0.5)
    E = np.where(active, E, 1.0)
    nu = np.where(active, np.clip(nu, 0.0, 0.4995), 0.3)
    return np.nan_to_num(E, nan=1.0), np.nan_to_num(nu, nan=0.3), active, F, ser
