"""Parity of the CUDA path (through the C ABI) with the reference: golden vectors made by running the
reference itself (tests/golden/) and, at larger sizes, the CPU oracle and size-independent properties.

Tolerances: FP64 operator products 1e-12 relative; solutions at CG tolerance 1e-10 within 1e-7 relative
L2 of the reference's; mixed / refined precision at rel-res 1e-8 within 1e-6 (displacement) and 1e-5
(von Mises) against the FP64 reference solution."""
import os

import numpy as np
import pytest

from comech_b200 import engine, _lib
from comech_b200.grid import Grid, face_node_areas, lame
from comech_b200.synth import SpringSet

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _springs(z):
    return SpringSet(pair_a=z["pair_a"], pair_b=z["pair_b"], pair_k=z["pair_k"], line_a=z["line_a"],
                     line_b=z["line_b"], line_d=z["line_d"], line_k=z["line_k"])


def _groups(z):
    return np.split(z["groups"], np.cumsum(z["group_len"])[:-1])


def _hindfoot(golden):
    z = golden("hindfoot_small")
    g = Grid(z["xe"], z["ye"], z["ze"])
    return z, g


def test_fine_operator_matches_reference_assembly(golden):
    import torch
    z, g = _hindfoot(golden)
    mat = np.concatenate([z["lam"], z["mu"]])
    nused = z["nused"]
    with engine.Problem(g, _lib.MAT_ISO_SRI, mat, z["active"], cn=z["cn"], orig=z["orig"],
                        options=dict(max_levels=0)) as P:
        m, n = P.used_mask()
        assert n == len(nused)
        assert (np.flatnonzero(m.cpu().numpy()) == nused).all()
        for u, ku in zip(z["u"], z["Ku"]):
            uf = np.zeros((P.ntotal, 3)); uf[nused] = u.reshape(-1, 3)
            y = P.apply(torch.from_numpy(uf.ravel()).cuda()).cpu().numpy().reshape(-1, 3)
            assert np.abs(y[nused].ravel() - ku).max() <= 1e-12 * np.abs(ku).max()
            unused = np.ones(P.ntotal, bool); unused[nused] = False
            assert np.abs(y[unused]).max(initial=0.0) == 0.0
            y32 = P.apply(torch.from_numpy(uf.ravel().astype(np.float32)).cuda()).cpu().numpy().reshape(-1, 3)
            assert rel(y32[nused].ravel(), ku) < 2e-6


def test_solve_cn_matches_reference(golden):
    z, g = _hindfoot(golden)
    U, info, R = engine.solve_cn(g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                                 (z["fixed_nodes"], z["fixed_area"]),
                                 [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z),
                                 tol=1e-10, maxiter=800)
    ok = ~np.isnan(z["U"])
    assert (np.isnan(U) == ~ok).all()
    assert rel(U[ok], z["U"][ok]) < 1e-7
    assert info["flag"] == 0 and info["relres"] < 1e-10
    assert info["ndof"] == int(z["ndof"]) and info["levels"] == int(z["levels"])
    assert abs(info["iters"] - int(z["iters"])) <= 3
    assert rel(R, z["R"]) < 1e-7
    cells = np.flatnonzero(z["active"])
    sig, vm, eps = engine.cell_stress_cn(g, z["lam"], z["mu"], U, cells, z["cn"])
    assert rel(vm, z["vm"]) < 1e-6


def test_stress_and_element_forces_exact(golden):
    z, g = _hindfoot(golden)
    cells = np.flatnonzero(z["active"])
    sig, vm, eps = engine.cell_stress_cn(g, z["lam"], z["mu"], z["U"], cells, z["cn"])
    np.testing.assert_allclose(sig, z["sig"], rtol=0, atol=1e-10 * np.abs(z["sig"]).max())
    np.testing.assert_allclose(vm, z["vm"], rtol=0, atol=1e-10 * np.abs(z["vm"]).max())
    np.testing.assert_allclose(eps, z["eps"], rtol=0, atol=1e-10 * np.abs(z["eps"]).max())
    F = engine.element_forces_cn(g, z["lam"], z["mu"], z["U"], z["fcells"], z["cn"])
    np.testing.assert_allclose(F, z["F"], rtol=0, atol=1e-10 * np.abs(z["F"]).max())


@pytest.mark.parametrize("tc", ["0", "1"])
@pytest.mark.parametrize("mode", ["sri", "full"])
def test_fp32_operator_on_tensor_cores(golden, monkeypatch, tc, mode):
    """FP32 K.u with the tensor-core kernel forced on (1) or kept off (0): within 2e-6 of the FP64 product
    (the reference assembly's for the SRI split-node model; the integrated model on the block grid)."""
    import torch
    monkeypatch.setenv("FEB_KU_TC", tc)
    if mode == "sri":
        z, g = _hindfoot(golden)
        args = (g, _lib.MAT_ISO_SRI, np.concatenate([z["lam"], z["mu"]]), z["active"])
        kw = dict(cn=z["cn"], orig=z["orig"])
    else:
        z = golden("block_small")
        g = Grid(z["xe"], z["ye"], z["ze"])
        args = (g, _lib.MAT_ISO_FULL, np.concatenate([z["lam"], z["mu"]]), np.ones(g.ncell, bool))
        kw = {}
    rng = np.random.default_rng(7)
    with engine.Problem(*args, options=dict(max_levels=0), **kw) as P:
        m, _ = P.used_mask()
        used = m.cpu().numpy().astype(bool)
        for _ in range(3):
            u = rng.standard_normal((P.ntotal, 3)) * used[:, None]
            y64 = P.apply(torch.from_numpy(u.ravel()).cuda()).cpu().numpy()
            y32 = P.apply(torch.from_numpy(u.ravel().astype(np.float32)).cuda()).cpu().numpy()
            assert rel(y32, y64) < 2e-6
            # a smooth field: the element forces cancel between neighbours
            xyz = np.stack(np.meshgrid(g.xe, g.ye, g.ze, indexing="ij"), -1).transpose(2, 1, 0, 3).reshape(-1, 3)
            us = np.zeros((P.ntotal, 3)); us[: len(xyz)] = np.sin(xyz / 7.0)
            us *= used[:, None]
            y64 = P.apply(torch.from_numpy(us.ravel()).cuda()).cpu().numpy()
            y32 = P.apply(torch.from_numpy(us.ravel().astype(np.float32)).cuda()).cpu().numpy()
            assert rel(y32, y64) < 2e-5


@pytest.mark.parametrize("tc", ["0", "1"])
@pytest.mark.parametrize("precision", ["mixed", "refine"])
def test_reduced_precision_solve_cn(golden, monkeypatch, precision, tc):
    monkeypatch.setenv("FEB_KU_TC", tc)
    z, g = _hindfoot(golden)
    U, info, R = engine.solve_cn(g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                                 (z["fixed_nodes"], z["fixed_area"]),
                                 [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z),
                                 tol=1e-8, maxiter=800, precision=precision)
    assert (info["ku_shape"][0] == 0) == (tc == "1")
    ok = ~np.isnan(z["U"])
    assert info["flag"] == 0 and info["relres"] < 1e-8
    assert rel(U[ok], z["U"][ok]) < 1e-6
    cells = np.flatnonzero(z["active"])
    _, vm, _ = engine.cell_stress_cn(g, z["lam"], z["mu"], U, cells, z["cn"])
    assert rel(vm, z["vm"]) < 1e-5


def _block(golden):
    z = golden("block_small")
    g = Grid(z["xe"], z["ye"], z["ze"])
    springs = [(z["spring_nodes"], z["spring_area"], z["spring_k"])]
    loads = [(z["load_nodes"], z["load_area"], z["load_t"])]
    return z, g, springs, loads


def test_solve_gmg_matches_reference(golden):
    z, g, springs, loads = _block(golden)
    act = np.ones(g.ncell, bool)
    U, info = engine.solve(g, z["lam"], z["mu"], act, springs, loads, method="gmg", tol=1e-10)
    assert rel(U, z["U_gmg"]) < 1e-7
    _, vm, _ = engine.cell_stress(g, z["lam"], z["mu"], U, np.arange(g.ncell))
    assert rel(vm, z["vm_gmg"]) < 1e-6


def test_solve_penalty_ortho_groups_matches_reference(golden):
    z, g, springs, loads = _block(golden)
    act = np.ones(g.ncell, bool)
    pen = [(z["pen_nodes"], z["pen_w"], int(z["pen_comp"]), float(z["pen_k"]))]
    U, info = engine.solve(g, z["lam"], z["mu"], act, springs, loads, method="gmg", tol=1e-10, penalties=pen,
                           coeffs=z["coeffs"], node_groups=[z["group"]])
    assert rel(U, z["U_pen"]) < 1e-7
    _, vm, _ = engine.cell_stress(g, z["lam"], z["mu"], U, np.arange(g.ncell), coeffs=z["coeffs"])
    assert rel(vm, z["vm_pen"]) < 1e-6


def test_solve_cg_method_same_solution(golden):
    z, g, springs, loads = _block(golden)
    act = np.ones(g.ncell, bool)
    U, info = engine.solve(g, z["lam"], z["mu"], act, springs, loads, method="cg", tol=1e-10)
    assert rel(U, z["U_cg"]) < 1e-7


def test_patch_test(golden):
    z = golden("patch")
    g = Grid(z["xe"], z["ye"], z["ze"])
    E, nu = float(z["E"]), float(z["nu"])
    lam, mu = lame(np.full(g.ncell, E), np.full(g.ncell, nu))
    act = np.ones(g.ncell, bool)
    nb, ab = face_node_areas(g, g.cell_nodes, np.flatnonzero(g.cK == 0), "z-")
    nt, at = face_node_areas(g, g.cell_nodes, np.flatnonzero(g.cK == g.nz - 1), "z+")
    U, info = engine.solve(g, lam, mu, act, [(nb, ab, np.array([1e-6, 1e-6, 1e9]))], [(nt, at, np.array([0, 0, -1.0]))],
                           method="direct")
    # uniaxial compression: u_z(top) = -10/E, sigma_zz = -1 everywhere (fe/test_patch.py)
    assert abs(np.nanmin(U[:, 2]) + 10.0 / E) < 1e-9
    sig, vm, _ = engine.cell_stress(g, lam, mu, U, np.arange(g.ncell))
    assert np.abs(sig[:, 2] + 1.0).max() < 1e-8
    assert np.abs(U[:, 2] - z["U"][:, 2]).max() < 1e-10


def test_non_convergence_flag_and_injected_failure(golden, monkeypatch):
    z, g = _hindfoot(golden)
    args = (g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"], (z["fixed_nodes"], z["fixed_area"]),
            [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z))
    U, info, R = engine.solve_cn(*args, tol=1e-12, maxiter=1)
    assert info["flag"] == 1 and info["iters"] == 1 and info["relres"] > 1e-12
    monkeypatch.setenv("FEB_TEST_FAIL", "1")
    with pytest.raises(_lib.FebError) as e:
        engine.solve_cn(*args, tol=1e-8)
    assert e.value.code == -7


def test_block_config1_against_oracle():
    """48x32x24 two-material block (121,275 dofs) at rel-res 1e-8: FP64, mixed and refined precision
    against the CPU oracle (a restatement of fe/solver.py:202 solve(method='gmg'))."""
    from oracle import fe_oracle as O
    from comech_b200 import synth
    P = synth.block_problem(48, 32, 24, h=1.0, seed=0)
    g = P["grid"]
    og = O.OGrid(g.xe, g.ye, g.ze)
    Uo, io = O.solve(og, P["lam"], P["mu"], P["active"], P["springs"], P["loads"], method="gmg", tol=1e-10)
    cells = np.arange(g.ncell)
    _, vmo, _ = O.cell_stress(og, P["lam"], P["mu"], Uo, cells)
    for precision in ("fp64", "mixed", "refine"):
        U, info = engine.solve(g, P["lam"], P["mu"], P["active"], P["springs"], P["loads"], method="gmg", tol=1e-8,
                               precision=precision)
        assert info["flag"] == 0 and info["relres"] < 1e-8, (precision, info)
        assert rel(U, Uo) < 1e-6, precision
        _, vm, _ = engine.cell_stress(g, P["lam"], P["mu"], U, cells)
        assert rel(vm, vmo) < 1e-5, precision


def test_operator_symmetry_and_rigid_nullspace():
    """At a larger size: u^T K v == v^T K u and K annihilates rigid translations / rotations when no
    penalty is present (FP64, size-independent properties)."""
    import torch
    from comech_b200 import synth
    P = synth.hindfoot_problem(64, 48, 40, h=1.25, seed=4)
    g = P["grid"]
    mat = np.concatenate([P["lam"], P["mu"]])
    with engine.Problem(g, _lib.MAT_ISO_SRI, mat, P["active"], cn=P["cn"], orig=P["orig"],
                        options=dict(max_levels=0)) as Pr:
        m, n = Pr.used_mask()
        used = m.cpu().numpy().astype(bool)
        rng = np.random.default_rng(0)
        u = rng.standard_normal((Pr.ntotal, 3)) * used[:, None]
        v = rng.standard_normal((Pr.ntotal, 3)) * used[:, None]
        Ku = Pr.apply(torch.from_numpy(u.ravel()).cuda()).cpu().numpy()
        Kv = Pr.apply(torch.from_numpy(v.ravel()).cuda()).cpu().numpy()
        a, b = v.ravel() @ Ku, u.ravel() @ Kv
        assert abs(a - b) <= 1e-12 * np.sqrt((Ku @ Ku) * (v.ravel() @ v.ravel()))
        xyz = g.node_xyz[P["orig"]]
        for mode in range(6):
            w = np.zeros((Pr.ntotal, 3))
            if mode < 3:
                w[:, mode] = 1.0
            else:
                ax = mode - 3
                w = np.cross(np.eye(3)[ax], xyz - xyz.mean(0))
            w *= used[:, None]
            Kw = Pr.apply(torch.from_numpy(w.ravel()).cuda()).cpu().numpy()
            assert np.linalg.norm(Kw) <= 1e-10 * np.linalg.norm(Ku) * np.linalg.norm(w) / np.linalg.norm(u)


def test_pcg_gmg_on_assembled_matrix(golden):
    """The CSR-accepting plugin point (fe/gmg.py:120 pcg_gmg) on the reference-assembled split-node matrix
    with rigid-body modes, against the reference solution."""
    from oracle import fe_oracle as O
    z, g = _hindfoot(golden)
    og = O.OGrid(z["xe"], z["ye"], z["ze"])
    cells = np.flatnonzero(z["active"])
    K, nmap, nused = O.assemble(og, z["lam"], z["mu"], cells, z["cn"], O.kl_sri(og))
    n = K.shape[0]
    kd = np.zeros(n)
    for c in range(3):
        np.add.at(kd, 3 * nmap[z["fixed_nodes"]] + c, z["fixed_area"] * 1e6)
    K = K + O.sp.diags(kd) + _springs(z)(nmap, n)
    f = np.zeros(n)
    for c in range(3):
        np.add.at(f, 3 * nmap[z["load_nodes"]] + c, z["load_area"] * z["load_t"][c])
    Zm = O.rigid_modes(og.node_xyz[z["orig"]], nmap, n, _groups(z))
    x, info = engine.pcg_gmg(K, f, z["orig"][nused], (g.xe, g.ye, g.ze), tol=1e-10, maxiter=800, Z=Zm)
    assert info["flag"] == 0
    assert rel(x, z["U"][nused].ravel()) < 1e-7
    assert info["gpu_attempt"] == 0 and info["t_hier"] >= 0.0


def _assembled(golden):
    from oracle import fe_oracle as O
    z, g = _hindfoot(golden)
    og = O.OGrid(z["xe"], z["ye"], z["ze"])
    cells = np.flatnonzero(z["active"])
    K, nmap, nused = O.assemble(og, z["lam"], z["mu"], cells, z["cn"], O.kl_sri(og))
    n = K.shape[0]
    kd = np.zeros(n)
    for c in range(3):
        np.add.at(kd, 3 * nmap[z["fixed_nodes"]] + c, z["fixed_area"] * 1e6)
    K = K + O.sp.diags(kd) + _springs(z)(nmap, n)
    f = np.zeros(n)
    for c in range(3):
        np.add.at(f, 3 * nmap[z["load_nodes"]] + c, z["load_area"] * z["load_t"][c])
    Zm = O.rigid_modes(og.node_xyz[z["orig"]], nmap, n, _groups(z))
    return z, g, K, f, Zm, nused


def test_pcg_gmg_with_separate_krylov_operator(golden):
    """pcg_gmg(A_op=...) (fe/gmg.py:127-136): the preconditioner comes from A, the Krylov iteration and the
    rigid-mode coarse matrix from A_op.  With A_op a LinearOperator of the same matrix the solution is the
    reference's; with A_op = 1.01 A it is the reference's divided by 1.01."""
    import scipy.sparse.linalg as spla
    z, g, K, f, Zm, nused = _assembled(golden)
    n = K.shape[0]
    Aop = spla.LinearOperator((n, n), matvec=lambda v: K @ v)
    x, info = engine.pcg_gmg(K, f, z["orig"][nused], (g.xe, g.ye, g.ze), tol=1e-10, maxiter=800, Z=Zm, A_op=Aop)
    assert info["flag"] == 0 and info["relres"] < 1e-9
    assert rel(x, z["U"][nused].ravel()) < 1e-7
    x2, info2 = engine.pcg_gmg(K, f, z["orig"][nused], (g.xe, g.ye, g.ze), tol=1e-10, maxiter=800, A_op=1.01 * K)
    assert info2["flag"] == 0
    assert rel(1.01 * x2, z["U"][nused].ravel()) < 1e-7


def test_pcg_gmg_with_general_coarse_columns(golden):
    """A Z that is not the per-group rigid-mode layout (here: the rigid modes mixed by a random orthogonal
    matrix, same span) runs through the host Krylov loop with the device V-cycle; same solution."""
    z, g, K, f, Zm, nused = _assembled(golden)
    Zd = Zm.toarray() if hasattr(Zm, "toarray") else np.asarray(Zm)
    Q, _ = np.linalg.qr(np.random.default_rng(0).standard_normal((Zd.shape[1], Zd.shape[1])))
    x, info = engine.pcg_gmg(K, f, z["orig"][nused], (g.xe, g.ye, g.ze), tol=1e-10, maxiter=800, Z=Zd @ Q)
    assert info["flag"] == 0
    assert rel(x, z["U"][nused].ravel()) < 1e-7


def test_plugin_swaps_reference_style_modules(golden):
    """plugin.install replaces module attributes the way rb/rbfe.py:21-27 does; the swapped solve_cn is the
    device solver and uninstall restores the originals."""
    import types
    from comech_b200 import plugin
    z, g = _hindfoot(golden)
    mod = types.ModuleType("splitfe_like")
    sentinel = lambda *a, **k: None
    mod.solve_cn = mod.cell_stress_cn = mod.element_forces_cn = sentinel
    plugin.install(splitfe=mod, precision="mixed")
    assert mod._solve_cn_cpu is sentinel and mod.solve_cn is not sentinel
    U, info, R = mod.solve_cn(g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                              (z["fixed_nodes"], z["fixed_area"]), [(z["load_nodes"], z["load_area"], z["load_t"])],
                              _springs(z), _groups(z), tol=1e-8)
    ok = ~np.isnan(z["U"])
    assert info["flag"] == 0 and rel(U[ok], z["U"][ok]) < 1e-6
    plugin.uninstall(splitfe=mod)
    assert mod.solve_cn is sentinel and not hasattr(mod, "_solve_cn_cpu")
    # a module with the split-connectivity entry points gets the device versions (bit-exact)
    zs = golden("split")
    mod.split_connectivity_fast = sentinel
    plugin.install(splitfe=mod)
    gs = Grid(zs["h_edges_x"], zs["h_edges_y"], zs["h_edges_z"])
    cn, orig, ns = mod.split_connectivity_fast(gs, zs["h_active"], zs["h_part"], zs["h_share"])
    assert (cn == zs["h_cn"]).all() and (orig == zs["h_orig"]).all() and ns == int(zs["h_nsplit"])
    plugin.uninstall(splitfe=mod)
    assert mod.split_connectivity_fast is sentinel


@pytest.mark.parametrize("case", ["h", "r"])
def test_split_connectivity_on_device_bit_exact(golden, case):
    from comech_b200.split import split_connectivity_device
    z = golden("split")
    g = Grid(*[z[f"{case}_edges_{a}"] for a in "xyz"])
    cn, orig, ns = split_connectivity_device(g, z[f"{case}_active"], z[f"{case}_part"], z[f"{case}_share"])
    assert cn.dtype == np.int64 and orig.dtype == np.int64
    assert (cn == z[f"{case}_cn"]).all()
    assert (orig == z[f"{case}_orig"]).all()
    assert ns == int(z[f"{case}_nsplit"])


def test_rigid_groups_filtering_on_the_device(golden):
    """feb_set_rigid_groups keeps the used nodes of every group in their given order and drops groups with fewer
    than 4 of them (rb/splitfe.py:105-112): adding a group of unused nodes and a 3-node group, and unused nodes
    inside a real group, leaves the solve unchanged; a node id out of range is an argument error."""
    from comech_b200 import _lib
    z, g = _hindfoot(golden)
    args = (g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"], (z["fixed_nodes"], z["fixed_area"]),
            [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z))
    groups = _groups(z)
    U0, i0, _ = engine.solve_cn(*args, groups, tol=1e-10)
    used = np.zeros(len(z["orig"]), bool)
    used[np.unique(z["cn"][np.flatnonzero(z["active"])])] = True
    unused = np.flatnonzero(~used)
    padded = [np.concatenate([unused[:5], np.asarray(gr), unused[5:9]]) for gr in groups]
    extra = padded + [unused[10:40], np.asarray(groups[0])[:3]]
    U1, i1, _ = engine.solve_cn(*args, extra, tol=1e-10)
    assert i1["flag"] == 0 and abs(i1["iters"] - i0["iters"]) <= 1
    ok = np.isfinite(U0)
    assert rel(U1[ok], U0[ok]) < 1e-10
    with engine.Problem(g, _lib.MAT_ISO_SRI, np.concatenate([z["lam"], z["mu"]]), z["active"], cn=z["cn"],
                        orig=z["orig"], options=dict(max_levels=0)) as P:
        with pytest.raises(_lib.FebError):
            P.set_rigid_groups([np.array([0, 1, 2, len(z["orig"]) + 5])])


def test_deferred_setup_is_joined_before_use(golden):
    """feb_create returns with the dense coarsest inverse and the power iterations still running on side streams.
    A level-0 product taken at once equals the one taken after a solve (it waits for the level-0 power chain,
    which shares its accumulators); handles closed with that work in flight leave the next solve unchanged; rigid
    groups set while it runs give the same solve as rigid groups set after a preconditioner call has joined it."""
    import torch
    z, g = _hindfoot(golden)
    ntotal = len(z["orig"])
    fn = np.asarray(z["fixed_nodes"], np.int64)
    pen_k = np.repeat((np.asarray(z["fixed_area"]) * engine.K_GROUND)[:, None], 3, axis=1)
    coo = engine._extra_entries(_springs(z), None, ntotal)
    mat = np.concatenate([z["lam"], z["mu"]])
    groups = _groups(z)

    def make():
        return engine.Problem(g, _lib.MAT_ISO_SRI, mat, z["active"], cn=z["cn"], orig=z["orig"], pen_node=fn,
                              pen_k=pen_k, extra_coo=coo, precision="mixed", tol=1e-10, maxiter=800)

    for _ in range(3):                      # closed with the deferred work in flight
        make().close()
    u = torch.randn(3 * ntotal, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    with make() as P:
        y0 = P.apply(u)                     # at once
        P.set_rigid_groups(groups)          # beside the deferred work
        f = P.rhs([(z["load_nodes"], z["load_area"], z["load_t"])])
        x1, i1 = P.solve(f)
        y1 = P.apply(u)
        torch.cuda.synchronize()
        assert rel(y0.cpu().numpy(), y1.cpu().numpy()) < 1e-14
        assert i1.flag == 0 and i1.t_setup_ms > 0
        assert i1.t_stage_ms[6] > 0         # the deferred tail was measured when it was joined
    with make() as P:
        f = P.rhs([(z["load_nodes"], z["load_area"], z["load_t"])])
        P.precondition(f)                   # joins the deferred work first
        P.set_rigid_groups(groups)
        x2, i2 = P.solve(f)
    torch.cuda.synchronize()
    assert i2.flag == 0 and abs(i2.iters - i1.iters) <= 2
    ok = x1.abs() > 0
    assert rel(x2[ok].cpu().numpy(), x1[ok].cpu().numpy()) < 1e-7


@pytest.mark.parametrize("kernels", [(9, 10), (8, 12), (8, 0)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_level_kernels_agree(golden, precision, kernels):
    """Forms of the coarse-level products give the same preconditioner (FP32 stencil copies: +8): the slot index
    a run-time value (level_kernel 9) or a compile-time constant (10); the rank-1 term dots accumulated by the
    kernels that write the vectors (8) or formed by a dot pass before each product (12).  z = M r agrees to
    1e-12 (FP64 V-cycle) / 1e-4 (FP32 V-cycle: sums round in other orders) relative, and the solves take the
    same iterations (+-1) to the same solution.  The default FP16 stencil copies (0 against 8; FP32 V-cycle
    only) perturb the coarse operators by the FP16 rounding (2^-12 relative per entry): z agrees to 1e-2, the
    iterations to +-2, the solution to 1e-8."""
    import torch
    z, g = _hindfoot(golden)
    args = (g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"], (z["fixed_nodes"], z["fixed_area"]),
            [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z))
    ntotal = len(z["orig"])
    r = torch.randn(3 * ntotal, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    levels = []
    out = {}
    for lk in kernels:
        # min_dofs 300: levels 1 and 2 of the 24 x 18 x 16 grid are stencil levels carrying the springs' terms
        ctx = engine.prepare_cn(*args, tol=1e-10, precision=precision, options=dict(level_kernel=lk, min_dofs=300))
        try:
            zr = ctx["P"].precondition(r).cpu().numpy()
            x, info = ctx["P"].solve(ctx["f"], ctx["x0"])
            out[lk] = (zr, x.cpu().numpy(), info.iters, info.flag)
            levels.append(int(info.levels))
        finally:
            ctx["P"].close()
    assert min(levels) >= 4              # two stencil levels below the fine level and above the dense one
    (z1, x1, it1, f1), (z2, x2, it2, f2) = out[kernels[0]], out[kernels[1]]
    half = kernels[1] == 0 and precision == "mixed"
    assert f1 == 0 and f2 == 0 and abs(it1 - it2) <= (2 if half else 1)
    assert rel(z2, z1) < (1e-12 if precision == "fp64" else (1e-2 if half else 1e-4))
    assert rel(x2, x1) < 1e-8


def test_pool_reservation_settles(golden):
    """Handles come and go on one device pool: after the first handle of a problem, creating and closing more of
    the same size grows the reservation no further (a reservation that counted itself as a set-up's peak would
    double at every handle)."""
    import ctypes as C
    z, g = _hindfoot(golden)
    args = (g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"], (z["fixed_nodes"], z["fixed_area"]),
            [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z))
    lib = _lib.load()

    def stats():
        res, peak, grows = C.c_int64(), C.c_int64(), C.c_int32()
        _lib.check(lib.feb_pool_stats(C.byref(res), C.byref(peak), C.byref(grows)))
        return res.value, grows.value

    engine.prepare_cn(*args, tol=1e-8, precision="mixed")["P"].close()
    engine.prepare_cn(*args, tol=1e-8, precision="mixed")["P"].close()
    before = stats()
    for _ in range(4):
        ctx = engine.prepare_cn(*args, tol=1e-8, precision="mixed")
        ctx["P"].solve(ctx["f"], ctx["x0"])
        ctx["P"].close()
    assert stats() == before


def test_coarse_failure_is_reported_by_the_solve(golden):
    """The dense coarsest inverse runs after feb_create has returned, so a coarsest matrix that is not positive
    definite (here: zero stiffness, no springs, no penalties: the matrix is exactly zero) is reported by the calls
    that need it, feb_solve and feb_precondition, as FEB_ERR_COARSE, and by every later one."""
    import torch
    z, g = _hindfoot(golden)
    ncell = g.nx * g.ny * g.nz
    ntotal = len(z["orig"])
    f = torch.ones(3 * ntotal, dtype=torch.float64, device="cuda")
    with engine.Problem(g, _lib.MAT_ISO_SRI, np.zeros(2 * ncell), z["active"], cn=z["cn"], orig=z["orig"],
                        precision="mixed") as P:
        for call in (lambda: P.solve(f), lambda: P.precondition(f), lambda: P.solve(f)):
            with pytest.raises(_lib.FebError) as e:
                call()
            assert e.value.code == -5 and "not positive definite" in str(e.value)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_launch_modes_agree(golden, precision):
    """Direct launches (use_graphs 0), one captured graph per CG iteration (1) and the device-side while loop (2)
    run the same iteration, the rigid-mode coefficients on their side stream included (a real fork / join in
    mode 0, captured edges in 1 and 2): iteration counts within 1 (atomic sums round in run-dependent order),
    the same solution."""
    z, g = _hindfoot(golden)
    args = (g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"], (z["fixed_nodes"], z["fixed_area"]),
            [(z["load_nodes"], z["load_area"], z["load_t"])], _springs(z), _groups(z))
    out = [engine.solve_cn(*args, tol=1e-10, precision=precision, options=dict(use_graphs=m)) for m in (0, 1, 2)]
    (U0, i0, _), rest = out[0], out[1:]
    ok = np.isfinite(U0)
    for U, info, _ in rest:
        assert info["flag"] == 0
        assert abs(info["iters"] - i0["iters"]) <= 1
        assert rel(U[ok], U0[ok]) < 1e-8


def test_benchmark_smooth_set(golden):
    """feb_benchmark_smooth_set times the level-0 smoother step (paired K.u with the fused Chebyshev update) over
    rotating buffer sets; a handle without a hierarchy (no Chebyshev coefficients) is an argument error."""
    import ctypes as C
    import torch
    z, g = _hindfoot(golden)
    ntotal = len(z["orig"])
    mat = np.concatenate([z["lam"], z["mu"]])
    sets = [[torch.randn(3 * ntotal, dtype=torch.float32, device="cuda") for _ in range(4)] for _ in range(2)]
    ptr = [(C.c_void_p * 2)(*[st[q].data_ptr() for st in sets]) for q in range(4)]
    lib = _lib.load()
    ms = C.c_float()
    with engine.Problem(g, _lib.MAT_ISO_SRI, mat, z["active"], cn=z["cn"], orig=z["orig"],
                        pen_node=np.asarray(z["fixed_nodes"], np.int64),
                        pen_k=np.repeat((np.asarray(z["fixed_area"]) * engine.K_GROUND)[:, None], 3, axis=1),
                        precision="mixed") as P:
        _lib.check(lib.feb_benchmark_smooth_set(P.h, 2, ptr[0], ptr[1], ptr[2], ptr[3], 4, C.byref(ms)))
        assert ms.value > 0
    with engine.Problem(g, _lib.MAT_ISO_SRI, mat, z["active"], cn=z["cn"], orig=z["orig"],
                        options=dict(max_levels=0)) as P:
        assert lib.feb_benchmark_smooth_set(P.h, 2, ptr[0], ptr[1], ptr[2], ptr[3], 4, C.byref(ms)) == -1
