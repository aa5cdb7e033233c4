"""Pin the CPU oracle (oracle/fe_oracle.py) and the host-side preprocessing of the package against
golden vectors produced by the reference itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import fe_oracle as O
from comech_b200 import grid as G
from comech_b200.split import split_connectivity
from comech_b200.synth import SpringSet


def _springs(z):
    return SpringSet(pair_a=z["pair_a"], pair_b=z["pair_b"], pair_k=z["pair_k"], line_a=z["line_a"],
                     line_b=z["line_b"], line_d=z["line_d"], line_k=z["line_k"])


def _groups(z):
    return np.split(z["groups"], np.cumsum(z["group_len"])[:-1])


def test_element_matrices(golden):
    z = golden("elements")
    for i in range(3):
        d = z[f"dims{i}"]
        for fn in (O.hex8_matrices, G.element_matrices):
            KL, KM, Bc = fn(d)
            np.testing.assert_allclose(KL, z[f"KL{i}"], rtol=0, atol=1e-12 * np.abs(z[f"KL{i}"]).max())
            np.testing.assert_allclose(KM, z[f"KM{i}"], rtol=0, atol=1e-12 * np.abs(z[f"KM{i}"]).max())
            np.testing.assert_allclose(Bc, z[f"Bc{i}"], rtol=0, atol=1e-14 * np.abs(z[f"Bc{i}"]).max())
        for fn in (O.hex8_ortho_basis, G.element_basis):
            np.testing.assert_allclose(fn(d), z[f"KB{i}"], rtol=0, atol=1e-12 * np.abs(z[f"KB{i}"]).max())


def test_grid_indexing_and_sri(golden):
    z = golden("elements")
    edges = (np.r_[0, 1, 3, 4, 7, 10], np.r_[0, 2, 5, 10], np.r_[0, 1, 2, 4, 6, 10])
    og = O.OGrid(*edges)
    pg = G.Grid(*edges)
    for g in (og, pg):
        assert (g.cell_nodes == z["patch_cell_nodes"]).all()
        assert (g.dim_id == z["patch_dim_id"]).all()
        np.testing.assert_array_equal(g.udims, z["patch_udims"])
        np.testing.assert_array_equal(g.node_xyz, z["patch_node_xyz"])
    sri = O.kl_sri(og)
    np.testing.assert_allclose(sri, z["patch_KLsri"], rtol=0, atol=1e-12 * np.abs(sri).max())
    sri2 = np.stack([G.element_lambda_sri(d) for d in pg.udims])
    np.testing.assert_allclose(sri2, z["patch_KLsri"], rtol=0, atol=1e-12 * np.abs(sri).max())


@pytest.mark.parametrize("case", ["h", "r"])
def test_split_connectivity_bit_exact(golden, case):
    z = golden("split")
    edges = [z[f"{case}_edges_{a}"] for a in "xyz"]
    args = (z[f"{case}_active"], z[f"{case}_part"], z[f"{case}_share"])
    for g, fn in ((O.OGrid(*edges), O.split_connectivity), (G.Grid(*edges), split_connectivity)):
        cn, orig, ns = fn(g, *args)
        assert cn.dtype.kind == "i" and orig.dtype.kind == "i"
        assert (cn == z[f"{case}_cn"]).all()
        assert (orig == z[f"{case}_orig"]).all()
        assert ns == int(z[f"{case}_nsplit"])


def test_split_identity_without_bones():
    g = G.Grid(np.arange(5.0), np.arange(4.0), np.arange(3.0))
    cn, orig, ns = split_connectivity(g, np.ones(g.ncell, bool), np.zeros(g.ncell, int), np.zeros((g.ncell, 3)))
    assert ns == 0 and (cn == g.cell_nodes).all() and (orig == np.arange(g.nnode)).all()


def test_oracle_assembly_and_solve_cn(golden):
    z = golden("hindfoot_small")
    g = O.OGrid(z["xe"], z["ye"], z["ze"])
    cells = np.flatnonzero(z["active"])
    K, nmap, nused = O.assemble(g, z["lam"], z["mu"], cells, z["cn"], O.kl_sri(g))
    assert (nused == z["nused"]).all()
    for u, ku in zip(z["u"], z["Ku"]):
        np.testing.assert_allclose(K @ u, ku, rtol=0, atol=1e-12 * np.abs(ku).max())
    U, info, R = O.solve_cn(g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                            (z["fixed_nodes"], z["fixed_area"]), [(z["load_nodes"], z["load_area"], z["load_t"])],
                            _springs(z), _groups(z), tol=1e-10, maxiter=800)
    assert info["ndof"] == int(z["ndof"]) and info["levels"] == int(z["levels"])
    assert abs(info["iters"] - int(z["iters"])) <= 1
    ok = ~np.isnan(z["U"])
    assert (np.isnan(U) == ~ok).all()
    rel = np.linalg.norm(U[ok] - z["U"][ok]) / np.linalg.norm(z["U"][ok])
    assert rel < 1e-8, rel
    np.testing.assert_allclose(R, z["R"], rtol=0, atol=1e-7 * np.abs(z["R"]).max())
    sig, vm, eps = O.cell_stress(g, z["lam"], z["mu"], U, cells, z["cn"], nan_to_zero=True)
    assert np.linalg.norm(vm - z["vm"]) / np.linalg.norm(z["vm"]) < 1e-7
    F = O.element_forces(g, z["lam"], z["mu"], U, z["fcells"], z["cn"])
    assert np.linalg.norm(F - z["F"]) / np.linalg.norm(z["F"]) < 1e-7
    # reaction sum equals the applied load
    assert abs(R[:, 2].sum() + (z["load_area"] * z["load_t"][2]).sum()) < 1e-6 * abs((z["load_area"] * z["load_t"][2]).sum())


def test_oracle_multigrid_internals(golden):
    z = golden("gmg_small")
    h = golden("hindfoot_small")
    g = O.OGrid(h["xe"], h["ye"], h["ze"])
    cells = np.flatnonzero(h["active"])
    K, nmap, nused = O.assemble(g, h["lam"], h["mu"], cells, h["cn"], O.kl_sri(g))
    kd = np.zeros(K.shape[0])
    for c in range(3):
        np.add.at(kd, 3 * nmap[h["fixed_nodes"]] + c, h["fixed_area"] * 1e6)
    K = K + O.sp.diags(kd) + _springs(h)(nmap, K.shape[0])
    mg = O.Multigrid(K, h["orig"][nused], g.xe, g.ye, g.ze, min_dofs=600)
    assert [L.A.shape[0] for L in mg.levels] == list(z["sizes"])
    np.testing.assert_allclose([L.lmax for L in mg.levels], z["lmax"], rtol=1e-10)
    v = mg.vcycle(z["b"])
    assert np.linalg.norm(v - z["vcycle"]) / np.linalg.norm(z["vcycle"]) < 1e-10


def test_oracle_block_solves(golden):
    z = golden("block_small")
    g = O.OGrid(z["xe"], z["ye"], z["ze"])
    springs = [(z["spring_nodes"], z["spring_area"], z["spring_k"])]
    loads = [(z["load_nodes"], z["load_area"], z["load_t"])]
    act = np.ones(g.ncell, bool)
    cells = np.arange(g.ncell)
    U, info = O.solve(g, z["lam"], z["mu"], act, springs, loads, method="gmg", tol=1e-10)
    assert np.linalg.norm(U - z["U_gmg"]) / np.linalg.norm(z["U_gmg"]) < 1e-8
    assert abs(info["iters"] - int(z["iters_gmg"])) <= 1
    pen = [(z["pen_nodes"], z["pen_w"], int(z["pen_comp"]), float(z["pen_k"]))]
    U2, info2 = O.solve(g, z["lam"], z["mu"], act, springs, loads, method="gmg", tol=1e-10, penalties=pen,
                        coeffs=z["coeffs"], node_groups=[z["group"]])
    assert np.linalg.norm(U2 - z["U_pen"]) / np.linalg.norm(z["U_pen"]) < 1e-8
    sig2, vm2, _ = O.cell_stress(g, z["lam"], z["mu"], U2, cells, coeffs=z["coeffs"])
    assert np.linalg.norm(vm2 - z["vm_pen"]) / np.linalg.norm(z["vm_pen"]) < 1e-7
    U3, info3 = O.solve(g, z["lam"], z["mu"], act, springs, loads, method="cg", tol=1e-10)
    assert np.linalg.norm(U3 - z["U_cg"]) / np.linalg.norm(z["U_cg"]) < 1e-8
    assert abs(info3["iters"] - int(z["iters_cg"])) <= 2


def test_oracle_patch(golden):
    z = golden("patch")
    g = O.OGrid(z["xe"], z["ye"], z["ze"])
    lam, mu = O.lame(np.full(g.ncell, float(z["E"])), np.full(g.ncell, float(z["nu"])))
    act = np.ones(g.ncell, bool)
    nb, ab = O.face_node_areas(g, g.cell_nodes, np.flatnonzero(g.cK == 0), "z-")
    nt, at = O.face_node_areas(g, g.cell_nodes, np.flatnonzero(g.cK == g.nz - 1), "z+")
    U, _ = O.solve(g, lam, mu, act, [(nb, ab, np.array([1e-6, 1e-6, 1e9]))], [(nt, at, np.array([0, 0, -1.0]))],
                   method="direct")
    np.testing.assert_allclose(U, z["U"], rtol=0, atol=1e-8)  # lateral springs 1e-6: near-rigid mode
    sig, vm, _ = O.cell_stress(g, lam, mu, U, np.arange(g.ncell))
    np.testing.assert_allclose(sig, z["sig"], rtol=0, atol=1e-9)
    assert abs(np.nanmin(U[:, 2]) + 10.0 / float(z["E"])) < 1e-8


def test_oracle_post_processing(golden):
    """Region forces, rigid fit, relative displacement and both resamplings of the oracle against the
    reference's own outputs (rb/rbfe.py:194-213, rb/rbsim.py:99-161)."""
    z = golden("post")
    g = O.OGrid(z["xe"], z["ye"], z["ze"])
    for t in (1, 2):
        F, p = O.region_forces(g, z["lam"], z["mu"], z["U"], z["cn"], z["active"], z["part"], z["lab"], int(z["nlab"]), t)
        np.testing.assert_allclose(F, z[f"F{t}"], rtol=0, atol=1e-12 * np.abs(z[f"F{t}"]).max())
        assert (p == z[f"present{t}"]).all()
    xyz = g.node_xyz[z["orig"]]
    nodes = z["fit_nodes"]
    t, w, c = O.rigid_fit(xyz[nodes], np.nan_to_num(z["U"][nodes]))
    for a, key in ((t, "fit_t"), (w, "fit_w"), (c, "fit_c")):
        np.testing.assert_allclose(a, z[key], rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal(O.relative_displacement(xyz, z["U"], t, w, c), z["Urel"])
    vm, u, fr, sg = O.sample_fe(g, z["cn"], z["active"], z["VM"], z["SIG"], z["Urel"], (z["ml_xe"], z["ml_ye"], z["ml_ze"]))
    for a, key in ((vm, "vm_c"), (u, "u_c"), (fr, "frac"), (sg, "sig_c")):
        np.testing.assert_array_equal(a, z[key])
    gm = O.OGrid(z["ml_xe"], z["ml_ye"], z["ml_ze"])
    np.testing.assert_array_equal(O.sample_nodes(g, z["cn"], z["active"], z["Urel"], gm.node_xyz), z["u_nodes"])


def _roles(z):
    names = [str(n) for n in z["role_names"]]
    bodies = np.split(z["role_bodies"], np.cumsum(z["role_len"])[:-1])
    return {"bones": {n: tuple(int(b) for b in bb) for n, bb in zip(names, bodies)},
            "bonded_extra": [int(b) for b in z["role_bonded_extra"]]}


def test_oracle_material_mixing(golden):
    """Material mixing of the oracle equals the reference's rb/rbfe.py:75-134, bit for bit."""
    from comech_b200.materials import bone_groups
    z = golden("materials")
    cls = {int(b): int(c) for b, c in zip(z["cls_body"], z["cls_class"])}
    groups, _ = bone_groups(cls, _roles(z))
    shape = (int(z["nx"]), int(z["ny"]), int(z["nz"]))
    for name, kw in (("a", {}), ("b", dict(cart_E=float(z["b_cart_E"]), nu_soft=float(z["b_nu_soft"])))):
        E, nu, active, F, ser = O.mix_materials(cls, z["L"], shape, groups, **kw)
        for a, key in ((E, "E"), (nu, "nu"), (active, "active"), (F, "F"), (ser, "ser")):
            np.testing.assert_array_equal(a, z[f"{name}_{key}"])


# ------------------------------------------------------------------------ spring hook and surgical actions
def spring_hook_inputs(z):
    """Springs and bone-node sets of the spring_hook fixture in the reference's hook form."""
    names = ["talus", "calcaneus", "navicular"]
    bn = np.split(z["bone_nodes"], np.cumsum(z["bone_len"])[:-1])
    bone_nodes = dict(zip(names, bn))
    springs = [dict(a=a, b=b, k=float(k), A=names[e[0]], B=names[e[1]])
               for a, b, k, e in zip(z["spring_a"], z["spring_b"], z["spring_k"], z["spring_ends"])]
    return springs, bone_nodes


def test_oracle_spring_hook_matches_reference(golden):
    z = golden("spring_hook")
    og = O.OGrid(z["xe"], z["ye"], z["ze"])
    springs, bone_nodes = spring_hook_inputs(z)
    hook = O.spring_matrix_cn(og.node_xyz[z["orig"]], springs, bone_nodes)
    cells = np.flatnonzero(z["active"])
    nused = np.unique(z["cn"][cells])
    nmap = -np.ones(len(z["orig"]), np.int64)
    nmap[nused] = np.arange(len(nused))
    M = hook(nmap, 3 * len(nused)).tocoo()
    got = {(3 * nused[r // 3] + r % 3, 3 * nused[c // 3] + c % 3): v for r, c, v in zip(M.row, M.col, M.data)}
    ref = dict(zip(zip(z["hook_rows"], z["hook_cols"]), z["hook_vals"]))
    assert set(got) == set(ref)
    scale = np.abs(z["hook_vals"]).max()
    assert max(abs(got[k] - ref[k]) for k in ref) <= 1e-13 * scale


def test_oracle_solve_with_spring_hook(golden):
    z = golden("spring_hook")
    og = O.OGrid(z["xe"], z["ye"], z["ze"])
    springs, bone_nodes = spring_hook_inputs(z)
    hook = O.spring_matrix_cn(og.node_xyz[z["orig"]], springs, bone_nodes)
    U, info, R = O.solve_cn(og, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                            (z["fixed_nodes"], z["fixed_area"]), [(z["load_nodes"], z["load_area"], z["load_t"])],
                            hook, _groups(z), tol=1e-10)
    ok = ~np.isnan(z["U"])
    assert (np.isnan(U) == ~ok).all()
    assert np.linalg.norm(U[ok] - z["U"][ok]) / np.linalg.norm(z["U"][ok]) < 1e-7
    assert abs(info["iters"] - int(z["iters"])) <= 3


def action_problem(z, action):
    from comech_b200 import synth
    nx, ny, nz, h, seed = z["case"]
    return synth.hindfoot_problem(int(nx), int(ny), int(nz), h=float(h), seed=int(seed), action=action)


def action_digest(P):
    return np.array([P["lam"].sum(), P["mu"].sum(), P["active"].sum(), P["cn"].sum(), len(P["orig"]),
                     P["fixed"][1].sum(), P["loads"][0][1].sum(), P["extra"].node_coo()[4].sum()], float)


@pytest.mark.parametrize("action", ["resection", "osteotomy", "interposition", "fusion", "load"])
def test_action_instances_match_the_fixture(golden, action):
    """The generator still makes the instances the reference solved for the actions fixture."""
    z = golden("actions")
    P = action_problem(z, action)
    np.testing.assert_allclose(action_digest(P), z[f"{action}_digest"], rtol=1e-12, atol=0)
    assert len(P["orig"]) == len(z[f"{action}_U"])
