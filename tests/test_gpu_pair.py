"""The paired-row level-0 kernel (fine_pair.cu) against the per-cell kernel and the reference assembly, and
the V-cycle with the smoother fused into it against the unfused V-cycle (FEB_KU_PAIR=0 keeps the per-cell
kernels).  Launch shapes are pinned through FEB_PAIR_CONFIG so that tile edges (halo rows and columns, the
z chunks, split-copy tail blocks) fall in different places.

Tolerances: FP64 products 1e-12 relative to the largest entry; FP32 products 2e-6 relative L2 against the FP64
product; solutions at CG tolerance 1e-10 within 1e-8 relative L2 of each other."""
import numpy as np
import pytest

from comech_b200 import engine, _lib, synth
from comech_b200.grid import Grid, lame

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _cases(golden):
    """(name, Problem args, kwargs) of the operator cases: split-node hindfoot with ground springs (SRI,
    cubic cells), block (full integration), a rectilinear grid (SRI, unequal widths), orthotropic
    coefficients on that grid."""
    z = golden("hindfoot_small")
    g = Grid(z["xe"], z["ye"], z["ze"])
    pen_node = z["fixed_nodes"]
    pen_k = np.repeat((z["fixed_area"] * 1e6)[:, None], 3, axis=1)
    yield ("hindfoot", (g, _lib.MAT_ISO_SRI, np.concatenate([z["lam"], z["mu"]]), z["active"]),
           dict(cn=z["cn"], orig=z["orig"], pen_node=pen_node, pen_k=pen_k))
    zb = golden("block_small")
    gb = Grid(zb["xe"], zb["ye"], zb["ze"])
    yield ("block-full", (gb, _lib.MAT_ISO_FULL, np.concatenate([zb["lam"], zb["mu"]]), np.ones(gb.ncell, bool)), {})
    rng = np.random.default_rng(3)
    xe = np.r_[0.0, np.cumsum(rng.uniform(0.5, 1.5, 45))]
    ye = np.r_[0.0, np.cumsum(rng.uniform(0.5, 1.5, 33))]
    ze = np.r_[0.0, np.cumsum(rng.uniform(0.5, 1.5, 20))]
    gr = Grid(xe, ye, ze)
    E = rng.choice([500.0, 1e4, 2e3], gr.ncell)
    lam, mu = lame(E, np.full(gr.ncell, 0.3))
    act = rng.random(gr.ncell) < 0.85
    yield ("rectilinear-sri", (gr, _lib.MAT_ISO_SRI, np.concatenate([lam, mu]), act), {})
    c = np.stack([lam + 2 * mu, lam, lam, lam + 2 * mu, mu, 0.7 * mu], 1)
    yield ("ortho", (gr, _lib.MAT_ORTHO, np.ascontiguousarray(c).ravel(), act), {})


@pytest.mark.parametrize("shape", ["16,5", "8,3", "8,16", "16,40"])
def test_pair_products_match_cell_kernel(golden, monkeypatch, shape):
    import torch
    monkeypatch.setenv("FEB_KU_TC", "0")
    rng = np.random.default_rng(11)
    for name, args, kw in _cases(golden):
        out = {}
        for pair in ("1", "0"):
            monkeypatch.setenv("FEB_KU_PAIR", pair)
            monkeypatch.setenv("FEB_PAIR_CONFIG", shape)
            with engine.Problem(*args, options=dict(max_levels=0), **kw) as P:
                used = P.used_mask()[0].cpu().numpy().astype(bool)
                u = rng.standard_normal((P.ntotal, 3)) * used[:, None] if pair == "1" else out["u"]
                out["u"] = u
                y64 = P.apply(torch.from_numpy(u.ravel()).cuda()).cpu().numpy()
                y32 = P.apply(torch.from_numpy(u.ravel().astype(np.float32)).cuda()).cpu().numpy()
                # a second product: the sparse accumulator must be clear again
                y64b = P.apply(torch.from_numpy(u.ravel()).cuda()).cpu().numpy()
                out[pair] = (y64, y32, y64b)
        y64, y32, y64b = out["1"]
        c64, c32, _ = out["0"]
        tol = 1e-12 * np.abs(c64).max()
        assert np.abs(y64 - c64).max() <= tol, name
        assert np.abs(y64b - c64).max() <= tol, name
        assert rel(y32, c64) < 2e-6, name
        assert rel(c32, c64) < 2e-6, name


def test_pair_operator_matches_reference_assembly(golden, monkeypatch):
    import torch
    monkeypatch.setenv("FEB_KU_TC", "0")
    z = golden("hindfoot_small")
    g = Grid(z["xe"], z["ye"], z["ze"])
    nused = z["nused"]
    with engine.Problem(g, _lib.MAT_ISO_SRI, np.concatenate([z["lam"], z["mu"]]), z["active"], cn=z["cn"],
                        orig=z["orig"], options=dict(max_levels=0)) as P:
        for u, ku in zip(z["u"], z["Ku"]):
            uf = np.zeros((P.ntotal, 3)); uf[nused] = u.reshape(-1, 3)
            y = P.apply(torch.from_numpy(uf.ravel()).cuda()).cpu().numpy().reshape(-1, 3)
            assert np.abs(y[nused].ravel() - ku).max() <= 1e-12 * np.abs(ku).max()
            unused = np.ones(P.ntotal, bool); unused[nused] = False
            assert np.abs(y[unused]).max(initial=0.0) == 0.0


@pytest.mark.parametrize("precision", ["fp64", "mixed", "refine"])
def test_fused_vcycle_matches_unfused(monkeypatch, precision):
    """The same split-node solve with the fused level-0 smoother and with the unfused kernels: iteration counts
    within 2 in FP64 (within 5 % with FP32 V-cycles) and solutions within 1e-8 of each other (each within its own
    1e-10 residual)."""
    monkeypatch.setenv("FEB_KU_TC", "0")
    P = synth.hindfoot_problem(40, 28, 24, h=2.0, seed=5)
    g = P["grid"]
    args = (P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"], P["extra"], P["node_groups"])
    res = {}
    for pair in ("1", "0"):
        monkeypatch.setenv("FEB_KU_PAIR", pair)
        U, info, R = engine.solve_cn(g, *args, tol=1e-10, precision=precision)
        assert info["flag"] == 0 and info["relres"] < 1.5e-10   # CG stops on its recursive residual
        assert info["ku_kind"] == (1 if pair == "1" else 0)
        res[pair] = (U, info)
    ok = ~np.isnan(res["0"][0])
    assert (np.isnan(res["1"][0]) == ~ok).all()
    assert rel(res["1"][0][ok], res["0"][0][ok]) < 1e-8
    # FP32 V-cycles: the count moves by a few with summation order (refinement sums several sweeps)
    bar = 2 if precision == "fp64" else max(3, int(0.05 * res["0"][1]["iters"]))
    assert abs(res["1"][1]["iters"] - res["0"][1]["iters"]) <= bar


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_direct_galerkin_matches_cell_matrices(monkeypatch, precision):
    """The level-1 stencil summed directly from the fine cells (uniform grid, even cell counts) and through the
    coarse-cell matrices (FEB_GALERKIN_DIRECT=0) give the same solve: equal iteration counts within 1 and
    solutions within 1e-9 of each other at CG tolerance 1e-10."""
    P = synth.hindfoot_problem(40, 28, 24, h=2.0, seed=6)
    g = P["grid"]
    args = (P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"], P["extra"], P["node_groups"])
    res = {}
    for direct in ("1", "0"):
        monkeypatch.setenv("FEB_GALERKIN_DIRECT", direct)
        U, info, R = engine.solve_cn(g, *args, tol=1e-10, precision=precision)
        assert info["flag"] == 0 and info["relres"] < 1.5e-10   # CG stops on its recursive residual
        res[direct] = (U, info)
    ok = ~np.isnan(res["0"][0])
    assert rel(res["1"][0][ok], res["0"][0][ok]) < 1e-9
    assert abs(res["1"][1]["iters"] - res["0"][1]["iters"]) <= 1
    assert res["1"][1]["lmax"] == pytest.approx(res["0"][1]["lmax"], rel=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_compressed_level1_stencil_matches_stored(monkeypatch, precision):
    """Level-1 blocks formed on the fly at nodes inside one material (FEB_SYM_COMPRESS=1) and read from the
    stored stencil everywhere (FEB_SYM_COMPRESS=0, the default): the same solve within 1e-9; iterations within 1 in
    FP64, within 3 with the FP32 V-cycle (whose blocks differ from the rounded stored ones in the last bit, and
    whose iteration count moves by a few with such rounding)."""
    P = synth.hindfoot_problem(48, 34, 28, h=80.0 / 48, seed=7)
    g = P["grid"]
    args = (P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"], P["extra"], P["node_groups"])
    res = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("FEB_SYM_COMPRESS", flag)
        U, info, R = engine.solve_cn(g, *args, tol=1e-10, precision=precision)
        assert info["flag"] == 0 and info["relres"] < 1.5e-10   # CG stops on its recursive residual
        res[flag] = (U, info)
    ok = ~np.isnan(res["0"][0])
    assert rel(res["1"][0][ok], res["0"][0][ok]) < 1e-9
    assert abs(res["1"][1]["iters"] - res["0"][1]["iters"]) <= (1 if precision == "fp64" else 3)
