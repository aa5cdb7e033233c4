"""Learned warm start of the PCG: a 3D convolutional encoder-decoder that predicts the displacement field of a
solve from the solve's own inputs, used as the initial guess x0 (the reference starts from zero or from a
caller's x0, fe/gmg.py:120-137, rb/gpusolve.py:265).

Network (4 levels, widths 32-64-128-256, BF16 activations and weights, FP32 accumulation and master weights):

    e0a, e0b: 3x3x3 conv      (32 input channels, 6 used)       level 0   (the network grid, e.g. 96 x 64 x 48)
    d0 -> e1, d1 -> e2, d2 -> bt: 2x2x2 stride-2 conv, 3x3x3 conv levels 1-3
    u2 -> f2, u1 -> f1, u0 -> f0a, f0b: transposed 2x2x2 stride-2 conv, skip concatenation, 3x3x3 conv
    head: 1x1 conv to the 3 displacement components (no activation)

with ReLU after every convolution but the head.  Every layer runs in libfeb200.so (tensor-core implicit GEMMs
for the forward and data-gradient passes, warp-MMA weight gradients, fused bias / ReLU / mask epilogues); this
module only lays out buffers and sequences the calls.

Inputs (6 channels per network cell, ``feb_net_inputs``): log10 E / 4 and (nu - 0.3) * 4 of the FE cell at the
network cell's centre, the active flag, and marks of the FE nodes in the cell: split nodes, ground-spring
(contact) nodes and the z load (as a fraction of the total load x 100).  A surgical action enters through the
fields it edits (inactive bridge cells, a moved fragment, a soft bridge, merged split nodes, a scaled load).
Output: displacement / (u_unit * total load / 450 N) at the lower-corner node of every network cell; the
initial guess is its trilinear interpolation at the FE nodes (``feb_net_to_nodes``), so a network trained on one
voxel size serves any FE grid over the same box.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from .engine import _dev, _grid_struct, _ptr, _stream, _torch

WIDTHS = (32, 64, 128, 256)
CIN = 32
TAPS = {"conv3": 27, "down": 8, "up": 8}
REF_LOAD = 450.0
E_REF_INV = 1e-4          # 1 / E of cortical bone (MPa): stiffness weights of the edge term of the training loss
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warm_hindfoot_96x64x48.npz")


def layer_table(c=WIDTHS, cin=CIN):
    """(name, kind, input channels, output channels) of every convolution, in forward order."""
    c0, c1, c2, c3 = c
    return [("e0a", "conv3", cin, c0), ("e0b", "conv3", c0, c0), ("d0", "down", c0, c1), ("e1", "conv3", c1, c1),
            ("d1", "down", c1, c2), ("e2", "conv3", c2, c2), ("d2", "down", c2, c3), ("bt", "conv3", c3, c3),
            ("u2", "up", c3, c2), ("f2", "conv3", 2 * c2, c2), ("u1", "up", c2, c1), ("f1", "conv3", 2 * c1, c1),
            ("u0", "up", c1, c0), ("f0a", "conv3", 2 * c0, c0), ("f0b", "conv3", c0, c0)]


def _rows(d):
    return (d[0] + 2) * (d[1] + 2) * (d[2] + 2)


class WarmNet:
    """The network's parameters (one flat FP32 buffer with Adam moments), BF16 weight tables, and per-grid
    activation / gradient buffers."""

    def __init__(self, widths=WIDTHS, seed=0, theta=None, u_unit=1.0, grid=(96, 64, 48)):
        torch = _torch()
        self.torch = torch
        self.c = tuple(int(v) for v in widths)
        if any(v % 32 for v in self.c) or self.c[0] != 32:
            raise ValueError("layer widths must be multiples of 32, the first one 32 (the head's input)")
        self.L = layer_table(self.c)
        self.u_unit = float(u_unit)
        self.grid = tuple(int(v) for v in grid)
        # parameter layout: per layer W [taps][co][ci] then b [co]; head W [3][c0], b [3]
        self.off = {}
        n = 0
        for name, kind, ci, co in self.L:
            t = TAPS[kind]
            self.off[name] = (n, t, co, ci)
            n += t * co * ci + co
        self.off["head"] = (n, 1, 3, self.c[0])
        n += 3 * self.c[0] + 3
        self.nparam = n
        if theta is None:
            theta = self._init(seed)
        self.theta = torch.as_tensor(np.asarray(theta, np.float32)).cuda().contiguous()
        if self.theta.numel() != n:
            raise ValueError(f"parameter count {self.theta.numel()} != {n} of widths {self.c}")
        self.grad = torch.zeros_like(self.theta)
        self.m = torch.zeros_like(self.theta)
        self.v = torch.zeros_like(self.theta)
        self.step_no = 0
        self.fwd, self.bwd = {}, {}
        for name, kind, ci, co in self.L:
            t = TAPS[kind]
            self.fwd[name] = torch.empty(t * co * ci, dtype=torch.bfloat16, device="cuda")
            self.bwd[name] = torch.empty(t * co * ci, dtype=torch.bfloat16, device="cuda")
        self.status = torch.zeros(1, dtype=torch.int32, device="cuda")
        self._bufs = {}
        self.tables()

    # ------------------------------------------------------------------------------------------ parameters
    def _init(self, seed):
        """He-normal convolution weights (fan-in of the used input channels), zero biases, a small head."""
        rng = np.random.default_rng(seed)
        th = np.zeros(self.nparam, np.float32)
        for name, kind, ci, co in self.L:
            o, t, _, _ = self.off[name]
            used = 6 if name == "e0a" else ci
            fan = (1 if kind == "up" else t) * used
            W = rng.normal(0.0, np.sqrt(2.0 / fan), (t, co, ci))
            if name == "e0a":
                W[:, :, used:] = 0.0
            th[o:o + t * co * ci] = W.ravel()
        o = self.off["head"][0]
        th[o:o + 3 * self.c[0]] = rng.normal(0.0, 1e-2, 3 * self.c[0])
        return th

    def W(self, name):
        o, t, co, ci = self.off[name]
        return self.theta[o:o + t * co * ci]

    def b(self, name):
        o, t, co, ci = self.off[name]
        return self.theta[o + t * co * ci:o + t * co * ci + co]

    def gW(self, name):
        o, t, co, ci = self.off[name]
        return self.grad[o:o + t * co * ci]

    def gb(self, name):
        o, t, co, ci = self.off[name]
        return self.grad[o + t * co * ci:o + t * co * ci + co]

    def params_numpy(self):
        """{name: (W [taps][co][ci], b [co])} and the head, as float64 arrays."""
        th = self.theta.double().cpu().numpy()
        out = {}
        for name in [n for n, _, _, _ in self.L] + ["head"]:
            o, t, co, ci = self.off[name]
            W = th[o:o + t * co * ci]
            b = th[o + t * co * ci:o + t * co * ci + co]
            out[name] = (W.reshape(co, ci) if name == "head" else W.reshape(t, co, ci), b)
        return out

    def tables(self):
        """BF16 forward and data-gradient weight tables from the FP32 master weights."""
        lib, s = _lib.load(), _stream()
        for name, kind, ci, co in self.L:
            t = TAPS[kind]
            _lib.check(lib.feb_net_weights(_ptr(self.W(name)), t, co, ci, _ptr(self.fwd[name]), _ptr(self.bwd[name]),
                                           1 if kind == "conv3" else 0, s))

    def save(self, path, **meta):
        np.savez_compressed(path, theta=self.theta.cpu().numpy().astype(np.float16), widths=np.array(self.c),
                            u_unit=self.u_unit, grid=np.array(self.grid), **meta)

    @classmethod
    def load(cls, path=WEIGHTS):
        z = np.load(path)
        return cls(widths=tuple(z["widths"]), theta=z["theta"].astype(np.float32), u_unit=float(z["u_unit"]),
                   grid=tuple(int(v) for v in z["grid"]))

    # ------------------------------------------------------------------------------------------ buffers
    def buffers(self, dims):
        dims = tuple(int(v) for v in dims)
        if dims in self._bufs:
            return self._bufs[dims]
        if any(v % 8 for v in dims):
            raise ValueError("network grid dimensions must be multiples of 8")
        torch = self.torch
        c0, c1, c2, c3 = self.c
        G = [tuple(v >> l for v in dims) for l in range(4)]
        R = [_rows(g) for g in G]

        def z(l, ch, dt=torch.bfloat16):
            return torch.zeros(R[l], ch, dtype=dt, device="cuda")

        B = dict(G=G, R=R,
                 a0=z(0, c0), cat0=z(0, 2 * c0), D1=z(1, c1), cat1=z(1, 2 * c1), D2=z(2, c2), cat2=z(2, 2 * c2),
                 D3=z(3, c3), B3=z(3, c3), F2=z(2, c2), F1=z(1, c1), F0a=z(0, c0), F0b=z(0, c0),
                 pred=z(0, 3, torch.float32), dpred=z(0, 3, torch.float32),
                 gA0=z(0, c0), gB0=z(0, c0), gcat0=z(0, 2 * c0), gcat1=z(1, 2 * c1), gcat2=z(2, 2 * c2),
                 gA1=z(1, c1), gB1=z(1, c1), gA2=z(2, c2), gB2=z(2, c2), gA3=z(3, c3), gB3=z(3, c3),
                 loss=torch.zeros(1, dtype=torch.float64, device="cuda"))
        self._bufs[dims] = B
        return B

    # ------------------------------------------------------------------------------------------ layer calls
    def _conv(self, gather, G, fine, src, src_c0, kc, wt, n, out, out_c0, relu=1, bias=None, mask=None, mask_c0=0,
              accumulate=0, scatter_c=0):
        c = _lib.FebConv()
        c.gather, c.scatter = gather, 1 if scatter_c else 0
        c.grid = _lib.FebNetGrid(*G)
        if fine is not None:
            c.fine = _lib.FebNetGrid(*fine)
        setattr(c, "in", src.data_ptr())
        c.in_ld, c.in_c0, c.kc, c.n = src.shape[1], src_c0, kc, n
        c.wt = wt.data_ptr()
        c.out, c.out_ld, c.out_c0 = out.data_ptr(), out.shape[1], out_c0
        c.scatter_c, c.relu = scatter_c, relu
        c.bias = bias.data_ptr() if bias is not None else None
        if mask is not None:
            c.mask, c.mask_ld, c.mask_c0 = mask.data_ptr(), mask.shape[1], mask_c0
        c.accumulate = accumulate
        c.status = self.status.data_ptr()
        _lib.check(_lib.load().feb_net_conv(C.byref(c), _stream()))

    def _wgrad(self, mode, G, fine, P, p_c0, na, Q, q_c0, nb, dw):
        w = _lib.FebWgrad()
        w.mode = mode
        w.grid = _lib.FebNetGrid(*G)
        if fine is not None:
            w.fine = _lib.FebNetGrid(*fine)
        w.p, w.p_ld, w.p_c0, w.na = P.data_ptr(), P.shape[1], p_c0, na
        w.q, w.q_ld, w.q_c0, w.nb = Q.data_ptr(), Q.shape[1], q_c0, nb
        w.dw = dw.data_ptr()
        _lib.check(_lib.load().feb_net_wgrad(C.byref(w), _stream()))

    def _colsum(self, g, c0, nc, out):
        _lib.check(_lib.load().feb_net_colsum(_ptr(g), g.shape[0], g.shape[1], c0, nc, _ptr(out), _stream()))

    # ------------------------------------------------------------------------------------------ passes
    def forward(self, x, dims):
        """Prediction [rows][3] (FP32) of the input x [rows][32] (BF16) on a grid of `dims` cells."""
        B = self.buffers(dims)
        G = B["G"]
        c0, c1, c2, c3 = self.c
        S, D, O = _lib.GATHER_SHIFT, _lib.GATHER_DOWN, _lib.GATHER_ONE
        f, bb = self.fwd, self.b
        self._conv(S, G[0], None, x, 0, CIN, f["e0a"], c0, B["a0"], 0, bias=bb("e0a"))
        self._conv(S, G[0], None, B["a0"], 0, c0, f["e0b"], c0, B["cat0"], 0, bias=bb("e0b"))
        self._conv(D, G[1], G[0], B["cat0"], 0, c0, f["d0"], c1, B["D1"], 0, bias=bb("d0"))
        self._conv(S, G[1], None, B["D1"], 0, c1, f["e1"], c1, B["cat1"], 0, bias=bb("e1"))
        self._conv(D, G[2], G[1], B["cat1"], 0, c1, f["d1"], c2, B["D2"], 0, bias=bb("d1"))
        self._conv(S, G[2], None, B["D2"], 0, c2, f["e2"], c2, B["cat2"], 0, bias=bb("e2"))
        self._conv(D, G[3], G[2], B["cat2"], 0, c2, f["d2"], c3, B["D3"], 0, bias=bb("d2"))
        self._conv(S, G[3], None, B["D3"], 0, c3, f["bt"], c3, B["B3"], 0, bias=bb("bt"))
        self._conv(O, G[3], G[2], B["B3"], 0, c3, f["u2"], 8 * c2, B["cat2"], c2, bias=bb("u2"), scatter_c=c2)
        self._conv(S, G[2], None, B["cat2"], 0, 2 * c2, f["f2"], c2, B["F2"], 0, bias=bb("f2"))
        self._conv(O, G[2], G[1], B["F2"], 0, c2, f["u1"], 8 * c1, B["cat1"], c1, bias=bb("u1"), scatter_c=c1)
        self._conv(S, G[1], None, B["cat1"], 0, 2 * c1, f["f1"], c1, B["F1"], 0, bias=bb("f1"))
        self._conv(O, G[1], G[0], B["F1"], 0, c1, f["u0"], 8 * c0, B["cat0"], c0, bias=bb("u0"), scatter_c=c0)
        self._conv(S, G[0], None, B["cat0"], 0, 2 * c0, f["f0a"], c0, B["F0a"], 0, bias=bb("f0a"))
        self._conv(S, G[0], None, B["F0a"], 0, c0, f["f0b"], c0, B["F0b"], 0, bias=bb("f0b"))
        Wh = self.W("head")
        _lib.check(_lib.load().feb_net_head(_ptr(B["F0b"]), c0, B["R"][0], _ptr(Wh), _ptr(self.b("head")),
                                            _ptr(B["pred"]), None, None, C.c_float(0.0), None, None, 0, None, None,
                                            _stream()))
        return B["pred"]

    def backward(self, x, dims, target, wgt, inv_n, h1=None, energy=None):
        """Loss (device scalar, accumulated in the buffers' `loss`) and parameter gradients (accumulated in
        `grad`) of the last forward pass: the weighted mean squared error (scaled by inv_n), or with ``h1`` =
        (mse_scale, h1_scale) that error times mse_scale plus the stiffness-weighted squared error of the
        prediction's differences along the grid edges times h1_scale (``feb_net_loss``); ``energy`` = (scale,
        spacing (3,)) adds scale times the strain energy of the prediction's error (``feb_net_energy_loss``)."""
        B = self.buffers(dims)
        G = B["G"]
        c0, c1, c2, c3 = self.c
        S, D, O = _lib.GATHER_SHIFT, _lib.GATHER_DOWN, _lib.GATHER_ONE
        U = _lib.GATHER_UP
        k = self.bwd
        lib, s = _lib.load(), _stream()
        if h1 is None and energy is not None:
            h1 = (0.0, 0.0)
        if h1 is None:
            _lib.check(lib.feb_net_head(_ptr(B["F0b"]), c0, B["R"][0], _ptr(self.W("head")), _ptr(self.b("head")),
                                        None, _ptr(target), _ptr(wgt), C.c_float(inv_n), _ptr(B["loss"]),
                                        _ptr(B["gA0"]), c0, _ptr(self.gW("head")), _ptr(self.gb("head")), s))
        else:
            B["dpred"].zero_()
            _lib.check(lib.feb_net_loss(_lib.FebNetGrid(*dims), _ptr(x), _ptr(B["pred"]), _ptr(target), _ptr(wgt),
                                        E_REF_INV, float(h1[0]), float(h1[1]), _ptr(B["loss"]), _ptr(B["dpred"]), s))
            if energy is not None:
                hsp = np.ascontiguousarray(energy[1], np.float64)
                _lib.check(lib.feb_net_energy_loss(_lib.FebNetGrid(*dims), hsp.ctypes.data_as(C.c_void_p), _ptr(x),
                                                   _ptr(B["pred"]), _ptr(target), _ptr(wgt), float(energy[0]),
                                                   _ptr(B["loss"]), _ptr(B["dpred"]), s))
            _lib.check(lib.feb_net_head_grad(_ptr(B["F0b"]), c0, B["R"][0], _ptr(self.W("head")), _ptr(B["dpred"]),
                                             _ptr(B["gA0"]), c0, _ptr(self.gW("head")), _ptr(self.gb("head")), s))

        def conv_back(name, G_, Pbuf, p_c0, na, Qbuf, q_c0, nb):
            self._wgrad(S, G_, None, Pbuf, p_c0, na, Qbuf, q_c0, nb, self.gW(name))
            self._colsum(Pbuf, p_c0, na, self.gb(name))

        # level 0 decoder
        conv_back("f0b", G[0], B["gA0"], 0, c0, B["F0a"], 0, c0)
        self._conv(S, G[0], None, B["gA0"], 0, c0, k["f0b"], c0, B["gB0"], 0, relu=0, mask=B["F0a"])
        conv_back("f0a", G[0], B["gB0"], 0, c0, B["cat0"], 0, 2 * c0)
        self._conv(S, G[0], None, B["gB0"], 0, c0, k["f0a"], 2 * c0, B["gcat0"], 0, relu=0, mask=B["cat0"])
        # u0 (level 1 -> 0)
        self._wgrad(U, G[1], G[0], B["gcat0"], c0, c0, B["F1"], 0, c1, self.gW("u0"))
        self._colsum(B["gcat0"], c0, c0, self.gb("u0"))
        self._conv(D, G[1], G[0], B["gcat0"], c0, c0, k["u0"], c1, B["gA1"], 0, relu=0, mask=B["F1"])
        # level 1 decoder
        conv_back("f1", G[1], B["gA1"], 0, c1, B["cat1"], 0, 2 * c1)
        self._conv(S, G[1], None, B["gA1"], 0, c1, k["f1"], 2 * c1, B["gcat1"], 0, relu=0, mask=B["cat1"])
        self._wgrad(U, G[2], G[1], B["gcat1"], c1, c1, B["F2"], 0, c2, self.gW("u1"))
        self._colsum(B["gcat1"], c1, c1, self.gb("u1"))
        self._conv(D, G[2], G[1], B["gcat1"], c1, c1, k["u1"], c2, B["gA2"], 0, relu=0, mask=B["F2"])
        # level 2 decoder
        conv_back("f2", G[2], B["gA2"], 0, c2, B["cat2"], 0, 2 * c2)
        self._conv(S, G[2], None, B["gA2"], 0, c2, k["f2"], 2 * c2, B["gcat2"], 0, relu=0, mask=B["cat2"])
        self._wgrad(U, G[3], G[2], B["gcat2"], c2, c2, B["B3"], 0, c3, self.gW("u2"))
        self._colsum(B["gcat2"], c2, c2, self.gb("u2"))
        self._conv(D, G[3], G[2], B["gcat2"], c2, c2, k["u2"], c3, B["gA3"], 0, relu=0, mask=B["B3"])
        # bottleneck
        conv_back("bt", G[3], B["gA3"], 0, c3, B["D3"], 0, c3)
        self._conv(S, G[3], None, B["gA3"], 0, c3, k["bt"], c3, B["gB3"], 0, relu=0, mask=B["D3"])
        # d2: gradient into the level-2 skip half (accumulated), then e2
        self._wgrad(D, G[3], G[2], B["gB3"], 0, c3, B["cat2"], 0, c2, self.gW("d2"))
        self._colsum(B["gB3"], 0, c3, self.gb("d2"))
        self._conv(O, G[3], G[2], B["gB3"], 0, c3, k["d2"], 8 * c2, B["gcat2"], 0, relu=0, mask=B["cat2"],
                   accumulate=1, scatter_c=c2)
        conv_back("e2", G[2], B["gcat2"], 0, c2, B["D2"], 0, c2)
        self._conv(S, G[2], None, B["gcat2"], 0, c2, k["e2"], c2, B["gB2"], 0, relu=0, mask=B["D2"])
        self._wgrad(D, G[2], G[1], B["gB2"], 0, c2, B["cat1"], 0, c1, self.gW("d1"))
        self._colsum(B["gB2"], 0, c2, self.gb("d1"))
        self._conv(O, G[2], G[1], B["gB2"], 0, c2, k["d1"], 8 * c1, B["gcat1"], 0, relu=0, mask=B["cat1"],
                   accumulate=1, scatter_c=c1)
        conv_back("e1", G[1], B["gcat1"], 0, c1, B["D1"], 0, c1)
        self._conv(S, G[1], None, B["gcat1"], 0, c1, k["e1"], c1, B["gB1"], 0, relu=0, mask=B["D1"])
        self._wgrad(D, G[1], G[0], B["gB1"], 0, c1, B["cat0"], 0, c0, self.gW("d0"))
        self._colsum(B["gB1"], 0, c1, self.gb("d0"))
        self._conv(O, G[1], G[0], B["gB1"], 0, c1, k["d0"], 8 * c0, B["gcat0"], 0, relu=0, mask=B["cat0"],
                   accumulate=1, scatter_c=c0)
        conv_back("e0b", G[0], B["gcat0"], 0, c0, B["a0"], 0, c0)
        self._conv(S, G[0], None, B["gcat0"], 0, c0, k["e0b"], c0, B["gA0"], 0, relu=0, mask=B["a0"])
        conv_back("e0a", G[0], B["gA0"], 0, c0, x, 0, CIN)
        return B["loss"]

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, clip=None):
        """One Adam step on the accumulated gradients (zeroed afterwards); refreshes the BF16 tables."""
        self.step_no += 1
        gscale = 1.0
        if clip is not None:
            ss = self.torch.zeros(1, dtype=self.torch.float64, device="cuda")
            _lib.check(_lib.load().feb_net_sumsq(_ptr(self.grad), self.nparam, _ptr(ss), _stream()))
            norm = float(ss.sqrt().item())
            if norm > clip:
                gscale = clip / norm
        _lib.check(_lib.load().feb_net_adam(_ptr(self.theta), _ptr(self.grad), _ptr(self.m), _ptr(self.v),
                                            self.nparam, lr, beta1, beta2, eps, self.step_no, gscale, _stream()))
        self.tables()

    def check_status(self):
        """Raise if a bounded tensor-core wait of any network pass ran out (its results are then invalid)."""
        if int(self.status.item()):
            raise _lib.FebError(-6, "a tensor-core wait of the network ran out")

    # ------------------------------------------------------------------------------------------ coupling
    def inputs(self, g, lam, mu, active, orig, fixed_nodes, load_nodes, load_z, dims=None, out=None):
        """Network input [rows][32] on the network grid (default: this network's grid) over the FE grid's box."""
        torch = self.torch
        dims = tuple(dims or self.grid)
        h = _uniform_spacing(g)
        box = (h[0] * g.nx, h[1] * g.ny, h[2] * g.nz)
        hn = np.array([box[d] / dims[d] for d in range(3)], np.float64)
        nnode = (g.nx + 1) * (g.ny + 1) * (g.nz + 1)
        orig_h = np.asarray(orig, np.int64) if orig is not None else np.arange(nnode)
        split = np.unique(orig_h[nnode:]) if len(orig_h) > nnode else np.zeros(0, np.int64)
        contact = np.unique(orig_h[np.asarray(fixed_nodes, np.int64)])
        ln = orig_h[np.asarray(load_nodes, np.int64)]
        lz = np.asarray(load_z, np.float64)
        total = float(np.abs(lz).sum()) or 1.0
        mat = _dev(np.concatenate([np.asarray(lam, np.float64).ravel(), np.asarray(mu, np.float64).ravel()])
                   if not isinstance(lam, torch.Tensor) else torch.cat([lam, mu]), np.float64)
        act = _dev(np.asarray(active, bool).view(np.uint8) if not isinstance(active, torch.Tensor) else active,
                   np.uint8)
        sd, cd, ld_, lzd = (_dev(a, t) for a, t in ((split, np.int64), (contact, np.int64), (ln, np.int64),
                                                    (lz, np.float64)))
        rows = _rows(dims)
        if out is None:
            out = torch.empty(rows, CIN, dtype=torch.bfloat16, device="cuda")
        scratch = torch.empty(dims[0] * dims[1] * dims[2] * 3, dtype=torch.float32, device="cuda")
        gs = _grid_struct(g)
        lib = _lib.load()
        _lib.check(lib.feb_net_inputs(_lib.FebNetGrid(*dims), hn.ctypes.data_as(C.c_void_p), C.byref(gs),
                                      np.asarray(h, np.float64).ctypes.data_as(C.c_void_p), _ptr(mat), _ptr(act),
                                      len(split), _ptr(sd), len(contact), _ptr(cd), len(ln), _ptr(ld_), _ptr(lzd),
                                      100.0 / total, _ptr(scratch), _ptr(out), _stream()))
        return out, dict(hn=hn, h=np.asarray(h, np.float64), total_load=total, dims=dims)

    def predict_x0(self, g, lam, mu, active, orig, fixed_nodes, load_nodes, load_z, nnode_total, orig_dev=None):
        """Initial guess (full layout, FP64, device) for the solve of these inputs (orig: host node map; orig_dev:
        the same map already on the device, if any)."""
        x, meta = self.inputs(g, lam, mu, active, orig, fixed_nodes, load_nodes, load_z)
        self.status.zero_()
        pred = self.forward(x, meta["dims"])
        self.check_status()                  # a network pass whose tensor-core wait ran out gives no start value
        scale = self.u_unit * meta["total_load"] / REF_LOAD
        x0 = self.torch.empty(3 * nnode_total, dtype=self.torch.float64, device="cuda")
        nnode = (g.nx + 1) * (g.ny + 1) * (g.nz + 1)
        if orig_dev is not None:
            origd = orig_dev
        else:
            origd = _dev(np.asarray(orig, np.int64), np.int64) if orig is not None and nnode_total > nnode else None
        gs = _grid_struct(g)
        _lib.check(_lib.load().feb_net_to_nodes(_lib.FebNetGrid(*meta["dims"]), meta["hn"].ctypes.data_as(C.c_void_p),
                                                _ptr(pred), scale, C.byref(gs),
                                                meta["h"].ctypes.data_as(C.c_void_p), _ptr(origd), nnode_total,
                                                _ptr(x0), _stream()))
        return x0


def _uniform_spacing(g):
    h = []
    for e in (g.xe, g.ye, g.ze):
        d = np.diff(np.asarray(e, np.float64))
        if not np.allclose(d, d[0], rtol=1e-9, atol=0):
            raise ValueError("the warm start needs a grid of uniform spacing per axis")
        h.append(float(d[0]))
    return h


def load_z(loads):
    """(nodes, z load per node) of the solve's load list [(nodes, area, traction)] or [(nodes, values (n, 3))]."""
    ln, lz = [], []
    for item in loads:
        if len(item) == 2:
            nodes, vals = item
            vals = vals.cpu().numpy() if hasattr(vals, "cpu") else np.asarray(vals)
            nodes = nodes.cpu().numpy() if hasattr(nodes, "cpu") else np.asarray(nodes)
            ln.append(np.asarray(nodes, np.int64)); lz.append(np.asarray(vals, np.float64).reshape(-1, 3)[:, 2])
        else:
            nodes, area, t = item
            ln.append(np.asarray(nodes, np.int64)); lz.append(np.asarray(area, np.float64) * float(np.asarray(t)[2]))
    if not ln:
        return np.zeros(0, np.int64), np.zeros(0)
    return np.concatenate(ln), np.concatenate(lz)


def h1_norm(x, net_dims, target, wgt):
    """The stiffness-weighted edge-difference norm of a target (the normaliser of that loss term); a host float."""
    torch = _torch()
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().feb_net_loss(_lib.FebNetGrid(*net_dims), _ptr(x), None, _ptr(target), _ptr(wgt), E_REF_INV,
                                        0.0, 1.0, _ptr(acc), None, _stream()))
    return float(acc.item())


def energy_norm(x, net_dims, spacing, target, wgt):
    """The strain energy of a target field on the network grid (the normaliser of the energy loss); a host float."""
    torch = _torch()
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    hsp = np.ascontiguousarray(spacing, np.float64)
    _lib.check(_lib.load().feb_net_energy_loss(_lib.FebNetGrid(*net_dims), hsp.ctypes.data_as(C.c_void_p), _ptr(x), None,
                                               _ptr(target), _ptr(wgt), 1.0, _ptr(acc), None, _stream()))
    return float(acc.item())


def load_targets(net_dims, U, scale):
    """Training target and weights on a network grid equal to the FE grid (U: device full-layout FP64)."""
    torch = _torch()
    rows = _rows(net_dims)
    T = torch.empty(rows, 3, dtype=torch.float32, device="cuda")
    w = torch.empty(rows, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().feb_net_targets(_lib.FebNetGrid(*net_dims), _ptr(U), float(scale), _ptr(T), _ptr(w),
                                           _stream()))
    return T, w


_default = None


def default_net():
    """The trained network shipped with the package (loaded once)."""
    global _default
    if _default is None:
        if not os.path.exists(WEIGHTS):
            raise RuntimeError(f"{WEIGHTS} is missing: train it with `python -m comech_b200.warm_train`")
        _default = WarmNet.load(WEIGHTS)
    return _default
