"""Batched solves (comech_b200.batch, feb_solve_batch): the five seeded surgical actions of the actions fixture
(resection, osteotomy, interposition, fusion, load scaling on a 32 x 22 x 19 hindfoot; reference solves by
tests/golden/make_golden.py) solved together as one CUDA graph launch, each instance checked against the
reference's own solution; and uneven grids in one batch, whose instances stop at different iteration counts.

Tolerances: CG tolerance 1e-10; displacement and reactions within 1e-7 relative L2 of the reference (FP64), 1e-6
with the FP32 V-cycle at 1e-8; iteration counts within 3 of the reference's (FP64)."""
import numpy as np
import pytest

from comech_b200 import batch, engine, synth

from test_oracle_golden import action_problem

pytestmark = pytest.mark.gpu

ACTIONS = ["resection", "osteotomy", "interposition", "fusion", "load"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_actions_match_reference(golden, precision):
    z = golden("actions")
    items = [action_problem(z, a) for a in ACTIONS]
    tol = 1e-10 if precision == "fp64" else 1e-8
    out = batch.solve_batch(items, precision=precision, tol=tol, concurrency=3)
    for a, (U, info, R) in zip(ACTIONS, out):
        Uref = z[f"{a}_U"]
        ok = ~np.isnan(Uref)
        assert (np.isnan(U) == ~ok).all(), a
        assert info["flag"] == 0 and info["ndof"] == int(z[f"{a}_ndof"]), a
        assert info["relres"] < 1.5 * tol, a
        if precision == "fp64":
            assert rel(U[ok], Uref[ok]) < 1e-7, a
            assert rel(R, z[f"{a}_R"]) < 1e-7, a
            assert abs(info["iters"] - int(z[f"{a}_iters"])) <= 3, a
        else:
            assert rel(U[ok], Uref[ok]) < 1e-6, a
        assert info["batch"]["instances"] == len(ACTIONS)


def test_batch_of_uneven_grids_stops_each_instance_on_its_own():
    """Instances of different sizes need different iteration counts; in the single launch each one stops at
    its own count (the while loop's condition is the instance's flag), equal to its own feb_solve's within 2."""
    items = [synth.hindfoot_problem(nx, ny, nz, h=80.0 / nx, seed=s, action=synth.ACTIONS[1 + s % 5])
             for s, (nx, ny, nz) in enumerate([(24, 16, 14), (40, 28, 24), (20, 14, 12), (32, 22, 18)])]
    out = batch.solve_batch(items, precision="fp64", tol=1e-10, concurrency=2)
    one = [engine.solve_cn(*batch._args(it), tol=1e-10, precision="fp64") for it in items]
    its = [info["iters"] for _, info, _ in out]
    assert len(set(its)) > 1
    for (U, info, R), (U1, info1, R1) in zip(out, one):
        assert info["flag"] == 0
        assert abs(info["iters"] - info1["iters"]) <= 2
        ok = np.isfinite(U1).all(1)
        assert rel(U[ok], U1[ok]) < 1e-8


def test_batch_threads_mode_matches_graph_mode(golden):
    z = golden("actions")
    items = [action_problem(z, a) for a in ACTIONS[:3]]
    g = batch.solve_batch(items, precision="fp64", tol=1e-10, mode="graph")
    t = batch.solve_batch(items, precision="fp64", tol=1e-10, mode="threads", concurrency=2)
    for (U1, i1, _), (U2, i2, _) in zip(g, t):
        ok = np.isfinite(U1).all(1)
        assert rel(U1[ok], U2[ok]) < 1e-8


def test_batch_rejects_refined_precision():
    with pytest.raises(ValueError):
        batch.solve_batch([], precision="refine")
