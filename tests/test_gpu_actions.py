"""Device solve_cn against the reference's own solves (tests/golden/make_golden.py) on the cases that the
batched configuration draws from: the five seeded surgical actions (resection, osteotomy, interposition,
fusion, load scaling) on a mid-size hindfoot, and the reference's multi-node ligament hook
(rb/replica3.py:68-86) passed through the extra argument.

Tolerances: at CG tolerance 1e-10, displacement and reactions within 1e-7 relative L2 of the reference's,
von Mises within 1e-6, iteration counts within 3; in the refined precision at 1e-8, displacement within
1e-6 and von Mises within 1e-5."""
import numpy as np
import pytest

from comech_b200 import engine

from test_oracle_golden import action_problem

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("action", ["resection", "osteotomy", "interposition", "fusion", "load"])
@pytest.mark.parametrize("precision", ["fp64", "refine"])
def test_action_solve_matches_reference(golden, action, precision):
    z = golden("actions")
    P = action_problem(z, action)
    g = P["grid"]
    tol = 1e-10 if precision == "fp64" else 1e-8
    U, info, R = engine.solve_cn(g, P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"],
                                 P["extra"], P["node_groups"], tol=tol, precision=precision)
    Uref = z[f"{action}_U"]
    ok = ~np.isnan(Uref)
    assert (np.isnan(U) == ~ok).all()
    assert info["flag"] == 0 and info["ndof"] == int(z[f"{action}_ndof"])
    cells = np.flatnonzero(P["active"])
    _, vm, _ = engine.cell_stress_cn(g, P["lam"], P["mu"], U, cells, P["cn"])
    if precision == "fp64":
        assert rel(U[ok], Uref[ok]) < 1e-7
        assert rel(R, z[f"{action}_R"]) < 1e-7
        assert rel(vm, z[f"{action}_vm"]) < 1e-6
        assert abs(info["iters"] - int(z[f"{action}_iters"])) <= 3
    else:
        assert rel(U[ok], Uref[ok]) < 1e-6
        assert rel(vm, z[f"{action}_vm"]) < 1e-5


def test_reference_spring_hook_through_extra(golden):
    """The hook's matrix (dense k w w^T blocks of up to ~60 dofs per ligament, coupling two bones) reaches the
    device as non-local entries, is factored into rank-1 terms and projected through the levels."""
    import scipy.sparse as sp
    from comech_b200.grid import Grid
    z = golden("spring_hook")
    g = Grid(z["xe"], z["ye"], z["ze"])
    rows, cols, vals = z["hook_rows"], z["hook_cols"], z["hook_vals"]

    def hook(nmap, n):        # the reference's extra(nmap, n) contract on the fixture's entries
        r = 3 * nmap[rows // 3] + rows % 3
        c = 3 * nmap[cols // 3] + cols % 3
        return sp.csr_matrix((vals, (r, c)), shape=(n, n))

    groups = np.split(z["groups"], np.cumsum(z["group_len"])[:-1])
    U, info, R = engine.solve_cn(g, z["lam"], z["mu"], z["active"], z["cn"], z["orig"],
                                 (z["fixed_nodes"], z["fixed_area"]), [(z["load_nodes"], z["load_area"], z["load_t"])],
                                 hook, groups, tol=1e-10)
    ok = ~np.isnan(z["U"])
    assert (np.isnan(U) == ~ok).all()
    assert info["flag"] == 0 and info["ndof"] == int(z["ndof"])
    assert rel(U[ok], z["U"][ok]) < 1e-7
    assert rel(R, z["R"]) < 1e-7
    assert abs(info["iters"] - int(z["iters"])) <= 3
