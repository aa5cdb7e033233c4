"""The CPU oracle of the warm-start network pinned by finite differences (no GPU): every parameter gradient of
the chain-rule backward pass of oracle/net_oracle.py against central differences of the loss, on a tiny network."""
import numpy as np

from oracle import net_oracle as O


def test_oracle_gradients_match_finite_differences():
    c = (2, 3, 4, 5)
    P = O.init_params(c, cin=3, cin_used=3, seed=1)
    rng = np.random.default_rng(2)
    P["head"] = (rng.normal(0, 0.5, (3, 2)), np.array([0.1, -0.2, 0.3]))
    P = {k: (W, b + rng.normal(0, 0.1, b.shape)) for k, (W, b) in P.items()}
    net = O.Net(P, c)
    x = rng.normal(size=(8, 8, 8, 3))
    T = rng.normal(size=(8, 8, 8, 3))
    w = (rng.random((8, 8, 8)) < 0.7).astype(float)
    loss, g = net.loss_and_grads(x, T, w)
    assert np.isfinite(loss) and loss > 0
    worst = 0.0
    for name in [n for n, _, _, _ in O.layers(c, 3)] + ["head"]:
        for which in (0, 1):
            arr = P[name][which]
            for _ in range(2):
                idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
                num = net.numeric_grad(x, T, w, name, which, idx)
                ana = g[name][which][idx]
                worst = max(worst, abs(num - ana) / max(1e-8, abs(num) + abs(ana)))
    assert worst < 1e-5


def test_layers_are_adjoint():
    """<conv(X), G> = <X, conv_back(G)> for the three layer kinds (the data gradients are the adjoints)."""
    rng = np.random.default_rng(3)
    for fwd, back, xs, taps in ((O.conv3, O.conv3_back, (4, 6, 2, 3), 27), (O.down, O.down_back, (4, 6, 2, 3), 8),
                                (O.up, O.up_back, (2, 3, 1, 3), 8)):
        X = rng.normal(size=xs)
        W = rng.normal(size=(taps, 5, 3))
        Y = fwd(X, W)
        G = rng.normal(size=Y.shape)
        dX, dW, _ = back(X, W, G)
        assert abs((Y * G).sum() - (X * dX).sum()) < 1e-9 * abs((Y * G).sum())
        assert abs((Y * G).sum() - (W * dW).sum()) < 1e-9 * abs((Y * G).sum())


def test_energy_loss_gradient_and_positivity():
    """The oracle's strain-energy loss is non-negative, zero for a rigid-body error, and its gradient matches central
    differences."""
    rng = np.random.default_rng(4)
    dims = (4, 3, 3)
    h = np.array([1.0, 0.8, 1.2])
    x = np.zeros(dims + (32,))
    x[..., 0] = np.log10(rng.choice([1.0, 500.0, 1e4], dims)) / 4
    x[..., 1] = (rng.choice([0.3, 0.45], dims) - 0.3) * 4
    x[..., 2] = 1.0
    w = np.ones(dims)
    T = rng.normal(size=dims + (3,))
    pred = T + rng.normal(size=dims + (3,)) * 0.1
    loss, g = O.energy_loss(x, pred, T, w, h, 1.0)
    assert loss > 0
    # a rigid translation and an infinitesimal rotation carry no strain energy
    X = np.stack(np.meshgrid(*(np.arange(n) * hh for n, hh in zip(dims, h)), indexing="ij"), -1)
    rigid = np.array([0.3, -0.2, 0.5]) + np.cross(np.array([0.01, 0.02, -0.03]), X)
    assert O.energy_loss(x, T + rigid, T, w, h, 1.0)[0] < 1e-12 * loss
    for _ in range(4):
        idx = tuple(int(rng.integers(0, s)) for s in pred.shape)
        eps = 1e-6
        p1 = pred.copy(); p1[idx] += eps
        p2 = pred.copy(); p2[idx] -= eps
        num = (O.energy_loss(x, p1, T, w, h, 1.0)[0] - O.energy_loss(x, p2, T, w, h, 1.0)[0]) / (2 * eps)
        assert abs(num - g[idx]) < 1e-5 * max(1.0, abs(num))


def test_product_and_oracle_describe_the_same_network():
    """The device network (comech_b200.warmnet) and its oracle list the same layers, kinds and widths in the same
    order, and the same parameter count (checked without a GPU)."""
    from comech_b200 import warmnet
    assert warmnet.layer_table() == O.layers(warmnet.WIDTHS, warmnet.CIN)
    n = sum(O.TAPS_OF[k] * ci * co + co for _, k, ci, co in O.layers(warmnet.WIDTHS, warmnet.CIN))
    n += 3 * warmnet.WIDTHS[0] + 3
    import numpy as np
    z = np.load(warmnet.WEIGHTS)
    assert z["theta"].size == n and tuple(z["widths"]) == warmnet.WIDTHS
