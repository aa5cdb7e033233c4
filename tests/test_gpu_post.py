"""Post-processing on the device against the reference's own outputs (tests/golden/post.npz, made by
tests/golden/make_golden.py from rb/rbfe.py and rb/rbsim.py): region forces, rigid fit, relative
displacement, resampling on an analysis grid that sticks out of the FE grid.

Tolerances: forces and the fit are FP64 sums in another order (1e-12 relative); the resampled fields are
float32 outputs of FP64/float32 sums in another order (2 ulp of float32 relative to the field's maximum)."""
import numpy as np
import pytest

from comech_b200 import post
from comech_b200.grid import Grid

pytestmark = pytest.mark.gpu


def _case(golden):
    z = golden("post")
    return z, Grid(z["xe"], z["ye"], z["ze"])


def test_region_forces_match_reference(golden):
    z, g = _case(golden)
    for t in (1, 2):
        F, present = post.region_forces_cn(g, z["lam"], z["mu"], z["U"], z["cn"], z["active"], z["part"], z["lab"],
                                           int(z["nlab"]), t)
        np.testing.assert_allclose(F, z[f"F{t}"], rtol=0, atol=1e-12 * np.abs(z[f"F{t}"]).max())
        assert (present == z[f"present{t}"]).all()
    names = [f"r{i}" for i in range(int(z["nlab"]))]
    d = post.forces_on(g, z["lam"], z["mu"], z["U"], z["cn"], z["active"], z["part"], z["lab"], names, 1)
    assert sorted(d) == [names[i] for i in np.flatnonzero(z["present1"])]


def test_rigid_fit_and_relative_displacement_match_reference(golden):
    z, g = _case(golden)
    xyz = g.node_xyz[z["orig"]]
    nodes = z["fit_nodes"]
    t, w, c = post.rigid_fit(xyz[nodes], np.nan_to_num(z["U"][nodes]))
    np.testing.assert_allclose(c, z["fit_c"], rtol=1e-14)
    np.testing.assert_allclose(t, z["fit_t"], rtol=0, atol=1e-10 * np.abs(z["fit_t"]).max())
    np.testing.assert_allclose(w, z["fit_w"], rtol=0, atol=1e-10 * np.abs(z["fit_w"]).max())
    Ur = post.relative_displacement(g, z["orig"], z["U"], z["fit_t"], z["fit_w"], z["fit_c"])
    np.testing.assert_allclose(Ur, z["Urel"], rtol=0, atol=1e-14 * np.abs(z["Urel"]).max())


def test_sample_fe_matches_reference(golden):
    z, g = _case(golden)
    gm = Grid(z["ml_xe"], z["ml_ye"], z["ml_ze"])
    o = dict(g=g, cn=z["cn"], active=z["active"], VM=z["VM"], SIG=z["SIG"])
    vm, u, frac = post.sample_fe(o, gm, z["Urel"], sub=2)
    np.testing.assert_array_equal(frac, z["frac"])
    assert 0 < (frac > 0).mean() < 1                      # the analysis grid sticks out of the FE grid
    ulp = 2 * np.finfo(np.float32).eps
    for a, key in ((vm, "vm_c"), (u, "u_c"), (post.sample_fe.sig, "sig_c")):
        assert a.dtype == np.float32
        np.testing.assert_allclose(a, z[key], rtol=0, atol=ulp * np.abs(z[key]).max())
