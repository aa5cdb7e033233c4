"""CPU oracle of the learned warm start's network (float64 NumPy).

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``comech_b200``) imports this module; only ``tests/`` use it,
as the checker of the device layers (forward values and every gradient) and of the device network as a whole.

The reference has no network on this path (its PCG starts from zero or from a caller's x0, fe/gmg.py:120-137);
this is the restatement of the project's own architecture, with the same tap order and weight layouts as the
device kernels, so that the two can be compared tensor for tensor:

* ``conv3``  -- 3x3x3 convolution, stride 1, zero padding: out[v] = b + sum_t W[t] @ X[v + d(t)],
                tap t = 9 (dx+1) + 3 (dy+1) + (dz+1); W is [27][co][ci]
* ``down``   -- 2x2x2 convolution, stride 2: out[V] = b + sum_t W[t] @ X[2V + e(t)], t = 4 ex + 2 ey + ez
* ``up``     -- transposed 2x2x2 stride-2 convolution: out[2V + e(t)] = b + W[t] @ X[V]
* ``head``   -- 1x1 convolution to 3 channels and the weighted mean squared error
* ``Net``    -- the 4-level encoder-decoder (skip connections by concatenation, ReLU after every convolution
                but the head), forward and backward by the chain rule, plus ``numeric_grad`` for finite
                differences.

Arrays are [nx, ny, nz, C] over the cells (z fastest, like the FE cell id).
"""
import numpy as np

TAPS3 = [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)]
TAPS2 = [(t >> 2, (t >> 1) & 1, t & 1) for t in range(8)]


def _shift(Xp, d, shape):
    nx, ny, nz = shape
    return Xp[1 + d[0]:1 + d[0] + nx, 1 + d[1]:1 + d[1] + ny, 1 + d[2]:1 + d[2] + nz]


def _pad(X):
    return np.pad(X, ((1, 1), (1, 1), (1, 1), (0, 0)))


def conv3(X, W, b=None):
    shape = X.shape[:3]
    Xp = _pad(X)
    out = np.zeros(shape + (W.shape[1],))
    for t, d in enumerate(TAPS3):
        out += _shift(Xp, d, shape) @ W[t].T
    return out + b if b is not None else out


def conv3_back(X, W, G):
    """Gradients of conv3 for the output gradient G (pre-activation): (dX, dW, db)."""
    shape = X.shape[:3]
    Xp, Gp = _pad(X), _pad(G)
    dW = np.zeros_like(W)
    dX = np.zeros_like(X)
    for t, d in enumerate(TAPS3):
        dW[t] = np.einsum("xyzo,xyzi->oi", G, _shift(Xp, d, shape))
        dX += _shift(Gp, tuple(-c for c in d), shape) @ W[t]
    return dX, dW, G.sum((0, 1, 2))


def _sub(X, e):
    return X[e[0]::2, e[1]::2, e[2]::2]


def down(X, W, b=None):
    out = sum(_sub(X, e) @ W[t].T for t, e in enumerate(TAPS2))
    return out + b if b is not None else out


def down_back(X, W, G):
    dX = np.zeros_like(X)
    dW = np.zeros_like(W)
    for t, e in enumerate(TAPS2):
        dW[t] = np.einsum("xyzo,xyzi->oi", G, _sub(X, e))
        dX[e[0]::2, e[1]::2, e[2]::2] = G @ W[t]
    return dX, dW, G.sum((0, 1, 2))


def up(X, W, b=None):
    nx, ny, nz, _ = X.shape
    out = np.zeros((2 * nx, 2 * ny, 2 * nz, W.shape[1]))
    for t, e in enumerate(TAPS2):
        out[e[0]::2, e[1]::2, e[2]::2] = X @ W[t].T
    return out + b if b is not None else out


def up_back(X, W, G):
    dW = np.zeros_like(W)
    dX = np.zeros_like(X)
    for t, e in enumerate(TAPS2):
        Gs = _sub(G, e)
        dW[t] = np.einsum("xyzo,xyzi->oi", Gs, X)
        dX += Gs @ W[t]
    return dX, dW, G.sum((0, 1, 2))


def head(X, W, b):
    return X @ W.T + b


def head_loss(X, W, b, target, wgt):
    """Weighted mean squared error of the head's output and its gradients (loss, dX (before the ReLU mask), dW,
    db); the mean is over the weight sum."""
    pred = head(X, W, b)
    inv_n = 1.0 / max(wgt.sum(), 1.0)
    e = (pred - target) * wgt[..., None]
    loss = float((e * (pred - target)).sum() * inv_n)
    d = 2.0 * inv_n * e
    return loss, pred, d @ W, np.einsum("xyzc,xyzk->ck", d, X), d.sum((0, 1, 2))


def relu(x):
    return np.maximum(x, 0.0)


# layer name, kind, input channels, output channels (c = the level widths c0..c3)
def layers(c, cin=32):
    c0, c1, c2, c3 = c
    return [("e0a", "conv3", cin, c0), ("e0b", "conv3", c0, c0), ("d0", "down", c0, c1), ("e1", "conv3", c1, c1),
            ("d1", "down", c1, c2), ("e2", "conv3", c2, c2), ("d2", "down", c2, c3), ("bt", "conv3", c3, c3),
            ("u2", "up", c3, c2), ("f2", "conv3", 2 * c2, c2), ("u1", "up", c2, c1), ("f1", "conv3", 2 * c1, c1),
            ("u0", "up", c1, c0), ("f0a", "conv3", 2 * c0, c0), ("f0b", "conv3", c0, c0)]


TAPS_OF = {"conv3": 27, "down": 8, "up": 8}
FWD = {"conv3": conv3, "down": down, "up": up}
BACK = {"conv3": conv3_back, "down": down_back, "up": up_back}


class Net:
    """The encoder-decoder with parameters P = {name: (W, b)} and P["head"] = (W [3][c0], b [3]).

    ``rnd`` (identity by default) is applied wherever the device stores a tensor in BF16: every layer output,
    and every activation gradient after its ReLU mask (skip gradients after the sum of both paths); a checker
    passes BF16 rounding to compare with the device tensor for tensor."""

    def __init__(self, P, c, rnd=None):
        self.P, self.c, self.L = P, c, layers(c, P["e0a"][0].shape[2])
        self.rnd = rnd or (lambda a: a)

    def _layer(self, name, X):
        kind = dict((n, k) for n, k, _, _ in self.L)[name]
        W, b = self.P[name]
        return self.rnd(relu(FWD[kind](X, W, b)))

    def forward(self, x):
        A = {"x": x}
        f = self._layer
        A["e0a"] = f("e0a", x)
        A["e0b"] = f("e0b", A["e0a"])
        A["d0"] = f("d0", A["e0b"])
        A["e1"] = f("e1", A["d0"])
        A["d1"] = f("d1", A["e1"])
        A["e2"] = f("e2", A["d1"])
        A["d2"] = f("d2", A["e2"])
        A["bt"] = f("bt", A["d2"])
        A["u2"] = f("u2", A["bt"])
        A["cat2"] = np.concatenate([A["e2"], A["u2"]], -1)
        A["f2"] = f("f2", A["cat2"])
        A["u1"] = f("u1", A["f2"])
        A["cat1"] = np.concatenate([A["e1"], A["u1"]], -1)
        A["f1"] = f("f1", A["cat1"])
        A["u0"] = f("u0", A["f1"])
        A["cat0"] = np.concatenate([A["e0b"], A["u0"]], -1)
        A["f0a"] = f("f0a", A["cat0"])
        A["f0b"] = f("f0b", A["f0a"])
        A["pred"] = head(A["f0b"], *self.P["head"])
        self.A = A
        return A["pred"]

    def loss_and_grads(self, x, target, wgt):
        self.forward(x)
        A, P, r = self.A, self.P, self.rnd
        loss, _, dX, dWh, dbh = head_loss(A["f0b"], *P["head"], target, wgt)
        g = {"head": (dWh, dbh)}
        kinds = dict((n, k) for n, k, _, _ in self.L)
        inputs = {"e0a": "x", "e0b": "e0a", "d0": "e0b", "e1": "d0", "d1": "e1", "e2": "d1", "d2": "e2", "bt": "d2",
                  "u2": "bt", "f2": "cat2", "u1": "f2", "f1": "cat1", "u0": "f1", "f0a": "cat0", "f0b": "f0a"}

        def back(name, G):
            """G: gradient of the layer's pre-activation output (already through its ReLU)."""
            dIn, dW, db = BACK[kinds[name]](A[inputs[name]], P[name][0], G)
            g[name] = (dW, db)
            return dIn

        def mask(d, name):
            return d * (A[name] > 0)

        c0, c1, c2, _ = self.c
        G = r(mask(dX, "f0b"))
        G = r(mask(back("f0b", G), "f0a"))
        gcat0 = r(mask(back("f0a", G), "cat0"))
        G = r(mask(back("u0", gcat0[..., c0:]), "f1"))
        gcat1 = r(mask(back("f1", G), "cat1"))
        G = r(mask(back("u1", gcat1[..., c1:]), "f2"))
        gcat2 = r(mask(back("f2", G), "cat2"))
        G = r(mask(back("u2", gcat2[..., c2:]), "bt"))
        G = r(mask(back("bt", G), "d2"))
        G = r(gcat2[..., :c2] + mask(back("d2", G), "e2"))
        G = r(mask(back("e2", G), "d1"))
        G = r(gcat1[..., :c1] + mask(back("d1", G), "e1"))
        G = r(mask(back("e1", G), "d0"))
        G = r(gcat0[..., :c0] + mask(back("d0", G), "e0b"))
        G = r(mask(back("e0b", G), "e0a"))
        back("e0a", G)
        return loss, g

    def numeric_grad(self, x, target, wgt, name, which, index, eps=1e-6):
        """Central difference of the loss in one parameter entry."""
        arr = self.P[name][which]
        old = arr[index]
        arr[index] = old + eps
        lp = head_loss(self._fwd_f0b(x), *self.P["head"], target, wgt)[0]
        arr[index] = old - eps
        lm = head_loss(self._fwd_f0b(x), *self.P["head"], target, wgt)[0]
        arr[index] = old
        return (lp - lm) / (2 * eps)

    def _fwd_f0b(self, x):
        self.forward(x)
        return self.A["f0b"]


def init_params(c, cin=32, cin_used=6, seed=0):
    """He-normal weights (fan-in of the used input channels), zero biases, a small head."""
    rng = np.random.default_rng(seed)
    P = {}
    for name, kind, ci, co in layers(c, cin):
        taps = TAPS_OF[kind]
        fan = (1 if kind == "up" else taps) * (cin_used if name == "e0a" else ci)
        W = rng.normal(0.0, np.sqrt(2.0 / fan), (taps, co, ci))
        if name == "e0a":
            W[:, :, cin_used:] = 0.0
        P[name] = (W, np.zeros(co))
    P["head"] = (rng.normal(0.0, 1e-2, (3, c[0])), np.zeros(3))
    return P


def edge_loss(xin, pred, target, wgt, e_ref_inv, mse_scale, h1_scale):
    """Training loss of the warm start with its stiffness-weighted edge term, and its gradient in the prediction.

    mse_scale sum_v wgt |e|^2 + h1_scale sum over edges (v, v + unit step along x, y or z; both with wgt > 0) of
    w(v) |e(v + step) - e(v)|^2, e = pred - target, w(v) = 10^(4 xin[v][0]) e_ref_inv for active cells
    (xin[v][2] > 0), else 0.  Arrays over the cells [nx, ny, nz, ...].  Returns (loss, dpred)."""
    e = np.where((wgt > 0)[..., None], pred - target, 0.0)
    valid = wgt > 0
    loss = mse_scale * float((e * e).sum())
    g = 2.0 * mse_scale * e
    w = np.where(xin[..., 2] > 0, 10.0 ** (4.0 * xin[..., 0]) * e_ref_inv, 0.0) * valid
    for a in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[a] = slice(0, -1)
        hi[a] = slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        m = w[lo] * valid[hi]
        d = (pred[hi] - target[hi]) - (pred[lo] - target[lo])
        loss += h1_scale * float((m[..., None] * d * d).sum())
        gd = 2.0 * h1_scale * m[..., None] * d
        g[hi] += gd
        g[lo] -= gd
    return loss, g


def energy_loss(xin, pred, target, wgt, h, scale):
    """Strain energy of the prediction's error, and its gradient: scale * sum over cells (x < nx-1, y < ny-1,
    z < nz-1) that are active (xin[..., 2] > 0) and whose 8 corner nodes have wgt > 0 of e_c^T K_e e_c, e = pred -
    target at the corners (corner l at offset (l & 1, (l >> 1) & 1, l >> 2), dof 3 l + c), K_e = lambda K_lambda(one
    point) + mu K_mu(2x2x2) of a cell of edges h (the hex8 matrices of oracle/fe_oracle.py), E = 10^(4 xin[0]),
    nu = xin[1] / 4 + 0.3.  Arrays over the network nodes [nx, ny, nz, ...].  Returns (loss, dpred)."""
    from oracle import fe_oracle as F
    KL, KM, Bc = F.hex8_matrices(h)
    KLs = np.prod(h) * (Bc.T @ F.D_LAMBDA @ Bc)
    nx, ny, nz = wgt.shape
    e = pred - target
    g = np.zeros_like(pred)
    loss = 0.0
    for x in range(nx - 1):
        for y in range(ny - 1):
            for z in range(nz - 1):
                if xin[x, y, z, 2] <= 0:
                    continue
                corners = [(x + (l & 1), y + ((l >> 1) & 1), z + (l >> 2)) for l in range(8)]
                if not all(wgt[c] > 0 for c in corners):
                    continue
                E = 10.0 ** (4.0 * xin[x, y, z, 0])
                nu = xin[x, y, z, 1] / 4.0 + 0.3
                lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
                ue = np.concatenate([e[c] for c in corners])
                f = (lam * KLs + mu * KM) @ ue
                loss += scale * float(ue @ f)
                for l, c in enumerate(corners):
                    g[c] += 2.0 * scale * f[3 * l:3 * l + 3]
    return loss, g
