"""The learned warm start on the device against the float64 CPU oracle of the network (oracle/net_oracle.py):
every layer kind forward and backward through the C ABI, the whole network's prediction and parameter gradients,
the head and its loss, the Adam step, the coupling to the solve (inputs, targets, initial guess), and a training
run that lowers the loss.

Tolerances: activations, weights and gradients are stored in BF16 (8 significant bits) and accumulated in FP32, so
layer outputs and gradients are compared by relative L2 error, 1.5e-2 per layer.  Through the whole 16-layer
network BF16 storage alone moves deep gradients by up to ~20 % from the exact float64 values (measured by the oracle
rounding at the same storage points), so there the device must stay within 1.5 x that distance + 1e-2.  FP32-only
steps (head, Adam, the initial guess) to 1e-5."""
import ctypes as C

import numpy as np
import pytest

from comech_b200 import _lib, warmnet
from comech_b200.engine import _ptr, _stream
from oracle import net_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def bf16(a):
    import torch
    return torch.as_tensor(np.asarray(a, np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def to_rows(A):
    nx, ny, nz, c = A.shape
    P = np.zeros((nx + 2, ny + 2, nz + 2, c))
    P[1:-1, 1:-1, 1:-1] = A
    return P.reshape(-1, c)


def from_rows(R, dims, c0=0, c=None):
    nx, ny, nz = dims
    A = np.asarray(R, np.float64).reshape(nx + 2, ny + 2, nz + 2, -1)[1:-1, 1:-1, 1:-1]
    return A[..., c0:c0 + c] if c is not None else A[..., c0:]


def dev_rows(A, width=None):
    import torch
    R = to_rows(A)
    if width is not None and width > R.shape[1]:
        R = np.concatenate([R, np.zeros((R.shape[0], width - R.shape[1]))], 1)
    return torch.as_tensor(R.astype(np.float32)).to(torch.bfloat16).cuda().contiguous()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.float().cpu().numpy().astype(np.float64)


def conv(gather, grid, fine, src, kc, wt, n, out, relu=1, bias=None, mask=None, accumulate=0, scatter_c=0,
         src_c0=0, out_c0=0, mask_c0=0):
    import torch
    c = _lib.FebConv()
    c.gather, c.scatter, c.grid = gather, 1 if scatter_c else 0, _lib.FebNetGrid(*grid)
    if fine is not None:
        c.fine = _lib.FebNetGrid(*fine)
    setattr(c, "in", src.data_ptr())
    c.in_ld, c.in_c0, c.kc, c.n = src.shape[1], src_c0, kc, n
    c.wt, c.out, c.out_ld, c.out_c0 = wt.data_ptr(), out.data_ptr(), out.shape[1], out_c0
    c.scatter_c, c.relu, c.accumulate = scatter_c, relu, accumulate
    c.bias = bias.data_ptr() if bias is not None else None
    if mask is not None:
        c.mask, c.mask_ld, c.mask_c0 = mask.data_ptr(), mask.shape[1], mask_c0
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    c.status = st.data_ptr()
    _lib.check(_lib.load().feb_net_conv(C.byref(c), _stream()))
    assert int(st.item()) == 0


def wgrad(mode, grid, fine, P, na, Q, nb, taps, p_c0=0, q_c0=0):
    import torch
    dw = torch.zeros(taps * na * nb, dtype=torch.float32, device="cuda")
    w = _lib.FebWgrad()
    w.mode, w.grid = mode, _lib.FebNetGrid(*grid)
    if fine is not None:
        w.fine = _lib.FebNetGrid(*fine)
    w.p, w.p_ld, w.p_c0, w.na = P.data_ptr(), P.shape[1], p_c0, na
    w.q, w.q_ld, w.q_c0, w.nb = Q.data_ptr(), Q.shape[1], q_c0, nb
    w.dw = dw.data_ptr()
    _lib.check(_lib.load().feb_net_wgrad(C.byref(w), _stream()))
    return host(dw).reshape(taps, na, nb)


def tables(W, flip):
    import torch
    t, co, ci = W.shape
    Wd = torch.as_tensor(W.astype(np.float32)).cuda().contiguous()
    f = torch.empty(t * co * ci, dtype=torch.bfloat16, device="cuda")
    b = torch.empty_like(f)
    _lib.check(_lib.load().feb_net_weights(_ptr(Wd), t, co, ci, _ptr(f), _ptr(b), flip, _stream()))
    return f, b


def empty_rows(dims, c):
    import torch
    return torch.zeros((dims[0] + 2) * (dims[1] + 2) * (dims[2] + 2), c, dtype=torch.bfloat16, device="cuda")


@pytest.mark.parametrize("ci,co,dims", [(32, 32, (8, 6, 10)), (64, 128, (6, 4, 4)), (96, 64, (5, 7, 3))])
def test_conv3_forward_and_gradients(ci, co, dims):
    import torch
    rng = np.random.default_rng(ci + co)
    X = bf16(np.maximum(rng.normal(size=dims + (ci,)), 0))
    W = bf16(rng.normal(0, np.sqrt(2 / (27 * ci)), (27, co, ci)))
    b = rng.normal(0, 0.1, co)
    f, bw = tables(W, flip=1)
    Xd = dev_rows(X)
    out = empty_rows(dims, co)
    bd = torch.as_tensor(b.astype(np.float32)).cuda()
    conv(_lib.GATHER_SHIFT, dims, None, Xd, ci, f, co, out, bias=bd)
    ref = O.relu(O.conv3(X, W, b))
    assert rel(from_rows(host(out), dims), ref) < 1.5e-2
    assert np.abs(host(out).reshape(dims[0] + 2, dims[1] + 2, dims[2] + 2, co)[0]).max() == 0   # zero shell
    # data gradient with the ReLU mask of the layer input, weight gradient, bias gradient
    G = bf16(rng.normal(size=dims + (co,)))
    Gd = dev_rows(G)
    dX = empty_rows(dims, ci)
    conv(_lib.GATHER_SHIFT, dims, None, Gd, co, bw, ci, dX, relu=0, mask=Xd)
    rX, rW, rb = O.conv3_back(X, W, G)
    assert rel(from_rows(host(dX), dims), rX * (X > 0)) < 1.5e-2
    dW = wgrad(_lib.GATHER_SHIFT, dims, None, Gd, co, Xd, ci, 27)
    assert rel(dW, rW) < 1.5e-2
    db = torch.zeros(co, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().feb_net_colsum(_ptr(Gd), Gd.shape[0], co, 0, co, _ptr(db), _stream()))
    assert rel(host(db), rb) < 1e-2


@pytest.mark.parametrize("ci,co,coarse", [(32, 64, (4, 3, 5)), (64, 32, (2, 2, 3))])
def test_down_and_up_forward_and_gradients(ci, co, coarse):
    import torch
    rng = np.random.default_rng(7 * ci + co)
    fine = tuple(2 * v for v in coarse)
    # down: fine ci -> coarse co
    X = bf16(np.maximum(rng.normal(size=fine + (ci,)), 0))
    W = bf16(rng.normal(0, np.sqrt(2 / (8 * ci)), (8, co, ci)))
    b = rng.normal(0, 0.1, co)
    f, bw = tables(W, flip=0)
    Xd = dev_rows(X)
    out = empty_rows(coarse, co)
    conv(_lib.GATHER_DOWN, coarse, fine, Xd, ci, f, co, out, bias=torch.as_tensor(b.astype(np.float32)).cuda())
    assert rel(from_rows(host(out), coarse), O.relu(O.down(X, W, b))) < 1.5e-2
    G = bf16(rng.normal(size=coarse + (co,)))
    Gd = dev_rows(G)
    rX, rW, _ = O.down_back(X, W, G)
    # scatter data gradient, accumulated onto an existing gradient and masked by the input
    base = bf16(rng.normal(size=fine + (ci,)))
    dX = dev_rows(base)
    conv(_lib.GATHER_ONE, coarse, fine, Gd, co, bw, 8 * ci, dX, relu=0, mask=Xd, accumulate=1, scatter_c=ci)
    assert rel(from_rows(host(dX), fine), (rX + base) * (X > 0)) < 1.5e-2
    assert rel(wgrad(_lib.GATHER_DOWN, coarse, fine, Gd, co, Xd, ci, 8), rW) < 1.5e-2
    # up (transposed): coarse ci -> fine co, written into channels [co, 2 co) of a concatenation buffer
    Xc = bf16(np.maximum(rng.normal(size=coarse + (ci,)), 0))
    Wu = bf16(rng.normal(0, np.sqrt(2 / ci), (8, co, ci)))
    bu = rng.normal(0, 0.1, co)
    fu, bwu = tables(Wu, flip=0)
    Xcd = dev_rows(Xc)
    cat = empty_rows(fine, 2 * co)
    conv(_lib.GATHER_ONE, coarse, fine, Xcd, ci, fu, 8 * co, cat, bias=torch.as_tensor(bu.astype(np.float32)).cuda(),
         scatter_c=co, out_c0=co)
    got = host(cat)
    assert rel(from_rows(got, fine, co, co), O.relu(O.up(Xc, Wu, bu))) < 1.5e-2
    assert np.abs(from_rows(got, fine, 0, co)).max() == 0          # the other half untouched
    Gf = bf16(rng.normal(size=fine + (co,)))
    Gcat = dev_rows(np.concatenate([np.zeros(fine + (co,)), Gf], -1))
    rXc, rWu, rbu = O.up_back(Xc, Wu, Gf)
    dXc = empty_rows(coarse, ci)
    conv(_lib.GATHER_DOWN, coarse, fine, Gcat, co, bwu, ci, dXc, relu=0, mask=Xcd, src_c0=co)
    assert rel(from_rows(host(dXc), coarse), rXc * (Xc > 0)) < 1.5e-2
    assert rel(wgrad(_lib.GATHER_UP, coarse, fine, Gcat, co, Xcd, ci, 8, p_c0=co), rWu) < 1.5e-2


def test_head_loss_and_gradients():
    import torch
    rng = np.random.default_rng(3)
    dims = (6, 5, 4)
    X = bf16(np.maximum(rng.normal(size=dims + (32,)), 0))
    W, b = rng.normal(0, 0.2, (3, 32)), rng.normal(0, 0.1, 3)
    T = rng.normal(size=dims + (3,))
    w = (rng.random(dims) < 0.6).astype(np.float64)
    loss, pred, dXr, dWr, dbr = O.head_loss(X, W, b, T, w)
    Xd = dev_rows(X)
    R = Xd.shape[0]
    f32 = lambda a: torch.as_tensor(np.asarray(a, np.float32)).cuda().contiguous()
    Wd, bd, Td, wd = f32(W), f32(b), f32(to_rows(T)), f32(to_rows(w[..., None])[:, 0])
    pr = torch.empty(R, 3, dtype=torch.float32, device="cuda")
    ls = torch.zeros(1, dtype=torch.float64, device="cuda")
    dX = empty_rows(dims, 32)
    dW = torch.zeros(3 * 32, dtype=torch.float32, device="cuda")
    db = torch.zeros(3, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().feb_net_head(_ptr(Xd), 32, R, _ptr(Wd), _ptr(bd), _ptr(pr), _ptr(Td), _ptr(wd),
                                        C.c_float(1.0 / w.sum()), _ptr(ls), _ptr(dX), 32, _ptr(dW), _ptr(db),
                                        _stream()))
    assert rel(from_rows(host(pr), dims), pred) < 1e-5
    assert abs(float(ls.item()) - loss) < 1e-5 * loss
    assert rel(from_rows(host(dX), dims), dXr * (X > 0)) < 1e-2
    assert rel(host(dW).reshape(3, 32), dWr) < 1e-5
    assert rel(host(db), dbr) < 1e-5


def test_adam_step_matches_formula():
    import torch
    rng = np.random.default_rng(4)
    n = 1000
    w0, g, m0, v0 = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n) * 0.1, rng.random(n) * 0.1
    f32 = lambda a: torch.as_tensor(np.asarray(a, np.float32)).cuda().contiguous()
    wd, gd, md, vd = f32(w0), f32(g), f32(m0), f32(v0)
    lr, b1, b2, eps, step, gs = 1e-3, 0.9, 0.999, 1e-8, 7, 0.5
    _lib.check(_lib.load().feb_net_adam(_ptr(wd), _ptr(gd), _ptr(md), _ptr(vd), n, lr, b1, b2, eps, step, gs,
                                        _stream()))
    ge = g * gs
    m = b1 * m0 + (1 - b1) * ge
    v = b2 * v0 + (1 - b2) * ge * ge
    lr_t = lr * np.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    assert rel(host(wd), w0 - lr_t * m / (np.sqrt(v) + eps)) < 1e-6
    assert np.abs(host(gd)).max() == 0


def test_whole_network_matches_oracle():
    """Prediction and every parameter gradient of the 16-layer network against the float64 oracle.  The device
    stores activations and gradients in BF16; the oracle run with BF16 rounding at the same storage points shows
    how far that storage alone moves each tensor from the exact float64 result, and the device's distance from the
    exact result must stay within that (x 1.5, + 1e-2 for the FP32 summation order)."""
    rng = np.random.default_rng(5)
    dims = (16, 8, 8)
    net = warmnet.WarmNet(seed=3)
    P = net.params_numpy()
    # the device keeps BF16 weight tables: give the oracle the same rounded weights
    P = {k: (bf16(W) if k != "head" else W, b) for k, (W, b) in P.items()}
    x = np.zeros(dims + (32,))
    x[..., :6] = bf16(rng.normal(size=dims + (6,)))
    T = rng.normal(size=dims + (3,))
    w = (rng.random(dims) < 0.8).astype(np.float64)
    exact = O.Net(P, net.c)
    loss, g = exact.loss_and_grads(x, T, w)
    stored = O.Net(P, net.c, rnd=bf16)
    loss_b, gb16 = stored.loss_and_grads(x, T, w)
    import torch
    xd = dev_rows(x)
    pred = host(net.forward(xd, dims))
    floor = rel(stored.A["pred"], exact.A["pred"])
    assert rel(from_rows(pred, dims), exact.A["pred"]) <= 1.5 * floor + 1e-3
    Td = torch.as_tensor(to_rows(T).astype(np.float32)).cuda()
    wd = torch.as_tensor(to_rows(w[..., None])[:, 0].astype(np.float32)).cuda()
    lossd = net.backward(xd, dims, Td, wd, 1.0 / w.sum())
    net.check_status()
    assert abs(float(lossd.item()) - loss) < 1e-2 * loss
    bad = {}
    for name in [n for n, _, _, _ in net.L] + ["head"]:
        for which, got in ((0, host(net.gW(name)).reshape(g[name][0].shape)), (1, host(net.gb(name)))):
            e_dev, e_b16 = rel(got, g[name][which]), rel(gb16[name][which], g[name][which])
            if e_dev > 1.5 * e_b16 + 1e-2:
                bad[(name, which)] = (round(e_dev, 4), round(e_b16, 4))
    assert not bad, bad


def test_training_lowers_the_loss():
    import torch
    rng = np.random.default_rng(6)
    dims = (16, 16, 8)
    net = warmnet.WarmNet(seed=1)
    x = np.zeros(dims + (32,))
    x[..., :6] = bf16(rng.normal(size=dims + (6,)))
    xi = np.arange(dims[0])[:, None, None] / dims[0]
    T = np.stack([np.sin(3 * xi) + 0 * x[..., 0], x[..., 0] * 0.5, np.cos(2 * xi) + 0 * x[..., 0]], -1)
    w = np.ones(dims)
    xd = dev_rows(x)
    Td = torch.as_tensor(to_rows(T).astype(np.float32)).cuda()
    wd = torch.as_tensor(to_rows(w[..., None])[:, 0].astype(np.float32)).cuda()
    losses = []
    for it in range(60):
        net.forward(xd, dims)
        net.buffers(dims)["loss"].zero_()
        losses.append(float(net.backward(xd, dims, Td, wd, 1.0 / w.sum()).item()))
        net.adam(1e-3)
    net.check_status()
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])


def test_initial_guess_interpolates_the_prediction():
    """feb_net_to_nodes: exact on a network grid equal to the FE grid; exact for a linear field on a finer FE grid
    over the same box (trilinear interpolation), clamped at the far faces."""
    import torch
    from comech_b200.grid import Grid
    from comech_b200.engine import _grid_struct
    dims = (8, 8, 8)
    hn = np.array([1.0, 1.5, 2.0])
    R = (dims[0] + 2) * (dims[1] + 2) * (dims[2] + 2)
    ii, jj, kk = np.meshgrid(*(np.arange(d + 2) - 1 for d in dims), indexing="ij")
    lin = lambda x, y, z: np.stack([x + 2 * y, 3 * z - y, x * 0 + 1.5], -1)
    pred = lin(ii * hn[0], jj * hn[1], kk * hn[2]).reshape(R, 3)
    pd = torch.as_tensor(pred.astype(np.float32)).cuda()
    for fine in (1, 2):
        fd = tuple(d * fine for d in dims)
        h = hn / fine
        g = Grid(*(np.arange(n + 1) * hh for n, hh in zip(fd, h)))
        nn = (fd[0] + 1) * (fd[1] + 1) * (fd[2] + 1)
        x0 = torch.empty(3 * nn, dtype=torch.float64, device="cuda")
        gs = _grid_struct(g)
        _lib.check(_lib.load().feb_net_to_nodes(_lib.FebNetGrid(*dims), hn.ctypes.data_as(C.c_void_p), _ptr(pd), 2.0,
                                                C.byref(gs), h.ctypes.data_as(C.c_void_p), None, nn, _ptr(x0),
                                                _stream()))
        got = host(x0).reshape(-1, 3)
        node = np.arange(nn)
        i, j, k = node % (fd[0] + 1), (node // (fd[0] + 1)) % (fd[1] + 1), node // ((fd[0] + 1) * (fd[1] + 1))
        # nodes on the far faces take the last network cell's value (clamped)
        ci = np.minimum(i * h[0], (dims[0] - 1) * hn[0]); cj = np.minimum(j * h[1], (dims[1] - 1) * hn[1])
        ck = np.minimum(k * h[2], (dims[2] - 1) * hn[2])
        np.testing.assert_allclose(got, 2.0 * lin(ci, cj, ck), rtol=1e-6, atol=1e-6)


def test_inputs_and_targets_of_a_hindfoot():
    """Input channels from the solve's inputs and the target from a displacement field, on the FE grid."""
    import torch
    from comech_b200 import synth
    from comech_b200.engine import _grid_struct
    P = synth.hindfoot_problem(32, 24, 16, h=2.5, seed=4)
    g = P["grid"]
    net = warmnet.WarmNet(seed=0)
    (ln, la, lt), = P["loads"]
    x, meta = net.inputs(g, P["lam"], P["mu"], P["active"], P["orig"], P["fixed"][0], ln, la * lt[2],
                         dims=(32, 24, 16))
    X = from_rows(host(x), (32, 24, 16))
    act = P["active"].reshape(32, 24, 16)
    np.testing.assert_array_equal(X[..., 2], act)
    E = P["E"].reshape(32, 24, 16)
    np.testing.assert_allclose(X[..., 0][act], bf16(np.log10(E[act]) / 4), rtol=1e-2)
    nnode = 33 * 25 * 17
    gid = P["orig"][P["fixed"][0]]
    cell = lambda n: (np.minimum(n % 33, 31), np.minimum((n // 33) % 25, 23), np.minimum(n // (33 * 25), 15))
    contact = np.zeros((32, 24, 16), bool)
    contact[cell(gid)] = True
    np.testing.assert_array_equal(X[..., 4] > 0, contact)
    split = np.zeros((32, 24, 16), bool)
    split[cell(np.unique(P["orig"][nnode:]))] = True
    np.testing.assert_array_equal(X[..., 3] > 0, split)
    assert abs(X[..., 5].sum() + 100.0) < 1.0            # the load marks sum to -100 (z load / total load x 100)
    U = np.random.default_rng(0).normal(size=(len(P["orig"]), 3))
    U[np.random.default_rng(1).random(len(P["orig"])) < 0.1] = np.nan
    T, w = warmnet.load_targets((32, 24, 16), torch.as_tensor(U.ravel()).cuda(), 2.0)
    Tg, wg = from_rows(host(T), (32, 24, 16)), from_rows(host(w)[:, None], (32, 24, 16))[..., 0]
    node = lambda i, j, k: i + 33 * (j + 25 * k)
    ii, jj, kk = np.meshgrid(np.arange(32), np.arange(24), np.arange(16), indexing="ij")
    Ug = U[node(ii, jj, kk)]
    fin = np.isfinite(Ug).all(-1)
    np.testing.assert_array_equal(wg > 0, fin)
    np.testing.assert_allclose(Tg[fin], (Ug[fin] / 2.0).astype(np.float32), rtol=1e-6)


def test_packaged_network_on_held_out_instances():
    """The network shipped in comech_b200/weights (trained on seeds 1000-2999 of the 96x64x48 generator against the
    strain energy of its error plus 0.2 x the relative squared error) on six instances it never saw, one per
    action.  Three starts of the same mixed-precision solve are compared: zero; the network's prediction; and the
    same preparation from x0 = 0, i.e. one preconditioner application to the load scaled to its energy-optimal
    multiple (a start that needs no network).  The preparation (a K product, a V-cycle, a K product and two dot
    products) costs about one CG iteration.

    Measured on 20 held-out instances (seeds 5000-5019): mean iterations in the mixed precision 73.45 from zero,
    72.15 from the learned start, 72.90 from the preconditioned load; in FP64 (no run-to-run rounding noise)
    69.35 from zero, 69.00 from the learned start, 68.35 from the preconditioned load.  So the learned start
    saves at most about one iteration, which its preparation costs again, and a start that needs no network does
    as well: no net gain on this hindfoot family.  The count is set by the slow inter-bone modes (bones held
    only by soft tissue, cartilage and springs) that the Krylov space finds within a few iterations whatever
    the start; a start shortens the solve only by the log of its energy-norm error reduction over the
    per-iteration rate (about 0.75).

    Bars: the prediction is within 90 % relative L2 of the FP64 solution; every solve converges; per instance the
    learned start takes at most 8 more iterations than the zero start; and on average over the six it takes no
    more than one iteration more than the zero start (it does not slow the solve down)."""
    import os
    import torch
    from comech_b200 import warm_train as W
    assert os.path.exists(warmnet.WEIGHTS), "packaged network missing"
    net = warmnet.default_net()
    counts = []
    for seed in range(5000, 5006):
        _, P = W.make_instance(seed)
        ln, lz = W.load_parts(P)
        U64, _ = W.solve(P, "fp64")
        _, i0 = W.solve(P, "mixed")
        x0 = net.predict_x0(P["grid"], P["lam"], P["mu"], P["active"], P["orig"], P["fixed"][0], ln, lz,
                            len(P["orig"]))
        _, i1 = W.solve(P, "mixed", x0)
        _, i2 = W.solve(P, "mixed", torch.zeros_like(x0))
        Ur = host(U64).reshape(-1, 3)
        ok = np.isfinite(Ur).all(1)
        pr = host(x0).reshape(-1, 3)
        assert np.linalg.norm(pr[ok] - Ur[ok]) < 0.9 * np.linalg.norm(Ur[ok])
        assert i0.flag == 0 and i1.flag == 0 and i2.flag == 0 and i1.relres < 1e-8
        assert i1.x0_used == 1 and i1.x0_scale > 0
        assert i1.iters <= i0.iters + 8, (seed, i0.iters, i1.iters)
        counts.append((i0.iters, i1.iters, i2.iters))
    c = np.array(counts, float)
    assert c[:, 1].mean() <= c[:, 0].mean() + 1.0, counts


def test_edge_loss_and_head_gradient():
    """feb_net_loss (squared error plus the stiffness-weighted edge term) and feb_net_head_grad against the oracle."""
    import torch
    rng = np.random.default_rng(8)
    dims = (7, 5, 6)
    x = np.zeros(dims + (32,))
    x[..., 0] = bf16(np.log10(rng.choice([1.15, 10.0, 500.0, 1e4], dims)) / 4)
    x[..., 2] = (rng.random(dims) < 0.8).astype(float)
    pred, T = rng.normal(size=dims + (3,)), rng.normal(size=dims + (3,))
    w = (rng.random(dims) < 0.85).astype(float)
    f32 = lambda a: torch.as_tensor(np.asarray(a, np.float32)).cuda().contiguous()
    xd, pd, Td, wd = dev_rows(x), f32(to_rows(pred)), f32(to_rows(T)), f32(to_rows(w[..., None])[:, 0])
    ref, gref = O.edge_loss(x, pred.astype(np.float32), T.astype(np.float32), w, 1e-4, 0.3, 2.0)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    dp = torch.zeros_like(pd)
    _lib.check(_lib.load().feb_net_loss(_lib.FebNetGrid(*dims), _ptr(xd), _ptr(pd), _ptr(Td), _ptr(wd), 1e-4, 0.3, 2.0,
                                        _ptr(loss), _ptr(dp), _stream()))
    assert abs(float(loss.item()) - ref) < 1e-5 * ref
    assert rel(from_rows(host(dp), dims), gref) < 1e-5
    # the head's backward pass for that output gradient
    X = bf16(np.maximum(rng.normal(size=dims + (32,)), 0))
    Wh = rng.normal(0, 0.2, (3, 32))
    Xd = dev_rows(X)
    dX = empty_rows(dims, 32)
    dW = torch.zeros(96, dtype=torch.float32, device="cuda")
    db = torch.zeros(3, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().feb_net_head_grad(_ptr(Xd), 32, Xd.shape[0], _ptr(f32(Wh)), _ptr(dp), _ptr(dX), 32, _ptr(dW),
                                             _ptr(db), _stream()))
    g = from_rows(host(dp), dims)
    assert rel(host(dW).reshape(3, 32), np.einsum("xyzc,xyzk->ck", g, X)) < 1e-5
    assert rel(host(db), g.sum((0, 1, 2))) < 1e-5
    assert rel(from_rows(host(dX), dims), (g @ Wh) * (X > 0)) < 1e-2


def test_energy_loss_matches_oracle():
    """feb_net_energy_loss (the strain energy of the prediction's error with the solve's hex8 element) against the
    oracle, value and gradient, on a box-cell grid with mixed materials, inactive cells and nodes without targets."""
    import torch
    rng = np.random.default_rng(9)
    dims = (5, 4, 6)
    h = np.array([0.8, 0.9, 1.1])
    x = np.zeros(dims + (32,))
    x[..., 0] = bf16(np.log10(rng.choice([1.15, 10.0, 500.0, 1e4], dims)) / 4)
    x[..., 1] = bf16((rng.choice([0.3, 0.4, 0.45], dims) - 0.3) * 4)
    x[..., 2] = (rng.random(dims) < 0.85).astype(float)
    pred = rng.normal(size=dims + (3,)).astype(np.float32)
    T = rng.normal(size=dims + (3,)).astype(np.float32)
    w = (rng.random(dims) < 0.95).astype(float)
    ref, gref = O.energy_loss(x, pred.astype(np.float64), T.astype(np.float64), w, h, 1e-3)
    f32 = lambda a: torch.as_tensor(np.asarray(a, np.float32)).cuda().contiguous()
    xd, pd, Td, wd = dev_rows(x), f32(to_rows(pred)), f32(to_rows(T)), f32(to_rows(w[..., None])[:, 0])
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    dp = torch.zeros_like(pd)
    _lib.check(_lib.load().feb_net_energy_loss(_lib.FebNetGrid(*dims), h.ctypes.data_as(C.c_void_p), _ptr(xd), _ptr(pd),
                                               _ptr(Td), _ptr(wd), 1e-3, _ptr(loss), _ptr(dp), _stream()))
    assert ref > 0
    assert abs(float(loss.item()) - ref) < 1e-4 * ref
    assert rel(from_rows(host(dp), dims), gref) < 1e-4
