"""Rectilinear voxel grid, Lame constants, face areas and host-side element matrices.

Mirrors the reference's ``fe/solver.py`` grid API (``Grid`` fe/solver.py:93-128, ``lame`` :131-134,
``face_node_areas`` :165-174, ``element_matrices`` :77-90, ``element_basis`` :63-74) with the same
index conventions:

* node id  = i + (nx+1) (j + (ny+1) k)        (x fastest)
* cell id  = (i ny + j) nz + k                 (z fastest, the reference's per-cell array order)
* corner l of a cell = (l & 1, l >> 1 & 1, l >> 2 & 1)

Heavy per-cell arrays (``cell_nodes``, ``cI``...) are built lazily: the solver itself only needs the
edge arrays, the device computes every index on the fly.
"""
import numpy as np

CORNERS = np.array([(l & 1, (l >> 1) & 1, (l >> 2) & 1) for l in range(8)], dtype=np.int64)
_G = 1.0 / np.sqrt(3.0)


def lame(E, nu):
    """(lambda, mu) from Young's modulus and Poisson's ratio (fe/solver.py:131-134)."""
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def _grad(pt, dims):
    s = 2.0 * CORNERS - 1.0
    out = np.empty((8, 3))
    for ax in range(3):
        o = [a for a in range(3) if a != ax]
        out[:, ax] = s[:, ax] * (1 + s[:, o[0]] * pt[o[0]]) * (1 + s[:, o[1]] * pt[o[1]]) / (4.0 * dims[ax])
    return out


def _bmat(gr):
    B = np.zeros((6, 8, 3))
    B[0, :, 0], B[1, :, 1], B[2, :, 2] = gr[:, 0], gr[:, 1], gr[:, 2]
    B[3, :, 0], B[3, :, 1] = gr[:, 1], gr[:, 0]
    B[4, :, 1], B[4, :, 2] = gr[:, 2], gr[:, 1]
    B[5, :, 0], B[5, :, 2] = gr[:, 2], gr[:, 0]
    return B.reshape(6, 24)


ORTHO_PATTERNS = np.zeros((6, 6, 6))
for _k, _ij in enumerate([[(0, 0), (1, 1)], [(0, 1), (1, 0)], [(0, 2), (2, 0), (1, 2), (2, 1)], [(2, 2)], [(3, 3)],
                          [(4, 4), (5, 5)]]):
    for _i, _j in _ij:
        ORTHO_PATTERNS[_k, _i, _j] = 1.0
D_LAM = np.zeros((6, 6)); D_LAM[:3, :3] = 1.0
D_MU = np.diag([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])


def element_matrices(dims):
    """(K_lambda 2x2x2, K_mu, B_centre) of a box cell with edges dims."""
    dims = np.asarray(dims, float)
    w = dims.prod() / 8.0
    KL = np.zeros((24, 24)); KM = np.zeros((24, 24))
    for x in (-_G, _G):
        for y in (-_G, _G):
            for z in (-_G, _G):
                B = _bmat(_grad((x, y, z), dims))
                KL += w * B.T @ D_LAM @ B
                KM += w * B.T @ D_MU @ B
    return KL, KM, _bmat(_grad((0.0, 0.0, 0.0), dims))


def element_lambda_sri(dims):
    """One-point (cell-centre) lambda matrix: B_c^T D_lam B_c vol (rb/splitfe.py:58-69)."""
    dims = np.asarray(dims, float)
    Bc = _bmat(_grad((0.0, 0.0, 0.0), dims))
    return dims.prod() * Bc.T @ D_LAM @ Bc


def element_basis(dims):
    """(6, 24, 24) element matrices of the six orthotropic patterns (fe/solver.py:63-74)."""
    dims = np.asarray(dims, float)
    w = dims.prod() / 8.0
    K = np.zeros((6, 24, 24))
    for x in (-_G, _G):
        for y in (-_G, _G):
            for z in (-_G, _G):
                B = _bmat(_grad((x, y, z), dims))
                K += w * np.einsum("ai,kab,bj->kij", B, ORTHO_PATTERNS, B)
    return K


def ortho_coeffs(lam, mu, shear_factor=None):
    """Isotropic (lam, mu) as orthotropic pattern coefficients (fe/solver.py:55-60)."""
    c = np.stack([lam + 2 * mu, lam, lam, lam + 2 * mu, mu, mu], 1)
    if shear_factor is not None:
        c[:, 5] *= shear_factor
    return c


class Grid:
    """Rectilinear grid with the attribute names of the reference ``Grid``; per-cell arrays are lazy."""

    def __init__(self, xe, ye, ze):
        self.xe, self.ye, self.ze = (np.ascontiguousarray(e, dtype=np.float64) for e in (xe, ye, ze))
        self.nx, self.ny, self.nz = len(self.xe) - 1, len(self.ye) - 1, len(self.ze) - 1
        self.shape = (self.nx, self.ny, self.nz)
        self.ncell = self.nx * self.ny * self.nz
        self.nnode = (self.nx + 1) * (self.ny + 1) * (self.nz + 1)
        self.dx, self.dy, self.dz = np.diff(self.xe), np.diff(self.ye), np.diff(self.ze)
        self.xc = (self.xe[:-1] + self.xe[1:]) / 2
        self.yc = (self.ye[:-1] + self.ye[1:]) / 2
        self.zc = (self.ze[:-1] + self.ze[1:]) / 2
        self._cache = {}

    def _get(self, key, fn):
        if key not in self._cache:
            self._cache[key] = fn()
        return self._cache[key]

    @property
    def cI(self):
        return self._get("cI", lambda: np.arange(self.ncell) // (self.ny * self.nz))

    @property
    def cJ(self):
        return self._get("cJ", lambda: (np.arange(self.ncell) // self.nz) % self.ny)

    @property
    def cK(self):
        return self._get("cK", lambda: np.arange(self.ncell) % self.nz)

    @property
    def cell_nodes(self):
        def build():
            nx1, ny1 = self.nx + 1, self.ny + 1
            base = self.cI + nx1 * (self.cJ + ny1 * self.cK)
            offs = CORNERS[:, 0] + nx1 * (CORNERS[:, 1] + ny1 * CORNERS[:, 2])
            return base[:, None] + offs[None, :]
        return self._get("cell_nodes", build)

    def _families(self):
        dims = np.stack([self.dx[self.cI], self.dy[self.cJ], self.dz[self.cK]], 1)
        ud, inv = np.unique(np.round(dims, 6), axis=0, return_inverse=True)
        return ud, inv.ravel()

    @property
    def udims(self):
        return self._get("fam", self._families)[0]

    @property
    def dim_id(self):
        return self._get("fam", self._families)[1]

    @property
    def KL(self):
        return self._get("KL", lambda: np.stack([element_matrices(d)[0] for d in self.udims]))

    @property
    def KM(self):
        return self._get("KM", lambda: np.stack([element_matrices(d)[1] for d in self.udims]))

    @property
    def Bc(self):
        return self._get("Bc", lambda: np.stack([element_matrices(d)[2] for d in self.udims]))

    @property
    def KB(self):
        return self._get("KB", lambda: np.stack([element_basis(d) for d in self.udims]))

    @property
    def cell_vol(self):
        return self._get("vol", lambda: self.dx[self.cI] * self.dy[self.cJ] * self.dz[self.cK])

    @property
    def node_xyz(self):
        def build():
            nid = np.arange(self.nnode)
            nx1, ny1 = self.nx + 1, self.ny + 1
            return np.stack([self.xe[nid % nx1], self.ye[(nid // nx1) % ny1], self.ze[nid // (nx1 * ny1)]], 1)
        return self._get("node_xyz", build)

    @property
    def cell_xyz(self):
        return self._get("cell_xyz", lambda: np.stack([self.xc[self.cI], self.yc[self.cJ], self.zc[self.cK]], 1))

    def cid(self, i, j, k):
        return (i * self.ny + j) * self.nz + k


def face_node_areas(g, cn, cells, face):
    """Tributary area (a quarter of the face) of the 4 nodes of face ``face`` ('x-' ... 'z+') of each cell,
    for the grid's own connectivity or a split one (fe/solver.py:165-174, rb/splitfe.py:94-102)."""
    ax = "xyz".index(face[0])
    side = 1 if face[1] == "+" else 0
    sel = CORNERS[:, ax] == side
    cells = np.asarray(cells)
    nodes = cn[cells][:, sel]
    I = cells // (g.ny * g.nz); J = (cells // g.nz) % g.ny; K = cells % g.nz
    d = [g.dx[I], g.dy[J], g.dz[K]]
    o = [d[i] for i in range(3) if i != ax]
    return nodes.ravel(), np.repeat(o[0] * o[1] / 4.0, 4)
