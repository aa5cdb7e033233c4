"""Batched solves (comech_b200.batch): several instances of uneven size and different surgical actions solved with
three in flight on the GPU give the same displacements as solving them one at a time (each instance has its own
handle, stream and graphs; nothing is shared between solves in flight).  Tolerance: both are FP64 CG to rel-res
1e-10, so they agree to 1e-8 relative L2."""
import numpy as np
import pytest

from comech_b200 import batch, synth

pytestmark = pytest.mark.gpu


def _items():
    out = []
    for seed, (nx, ny, nz) in enumerate([(24, 16, 14), (32, 22, 18), (28, 20, 16), (36, 26, 20), (20, 14, 12)]):
        out.append(synth.hindfoot_problem(nx, ny, nz, h=80.0 / nx, seed=seed, action=synth.ACTIONS[1 + seed % 5]))
    return out


def test_concurrent_batch_equals_sequential():
    items = _items()
    seq = batch.solve_batch(items, precision="fp64", tol=1e-10, concurrency=1)
    par = batch.solve_batch(items, precision="fp64", tol=1e-10, concurrency=3)
    for (U1, i1, R1), (U2, i2, R2) in zip(seq, par):
        assert i1["flag"] == 0 and i2["flag"] == 0
        ok = np.isfinite(U1).all(1)
        np.testing.assert_array_equal(ok, np.isfinite(U2).all(1))
        assert np.linalg.norm(U1[ok] - U2[ok]) <= 1e-8 * np.linalg.norm(U1[ok])
