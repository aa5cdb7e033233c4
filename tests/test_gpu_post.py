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


def test_nearest_active_matches_scipy_exactly():
    """Integer work: the feature transform equals scipy.ndimage.distance_transform_edt's indices, ties
    included, on random masks of assorted sizes and densities (and a grid without active cells)."""
    from scipy import ndimage
    rng = np.random.default_rng(3)
    for trial in range(25):
        shape = tuple(int(v) for v in rng.integers(2, 23, 3))
        act = rng.random(shape) < rng.uniform(0.01, 0.5)
        if trial == 0:
            act[...] = False
        g = Grid(np.arange(shape[0] + 1.0), np.arange(shape[1] + 1.0), np.arange(shape[2] + 1.0))
        ft = post.nearest_active(g, act.ravel()).cpu().numpy()
        if not act.any():
            assert (ft == -1).all()
            continue
        _, ind = ndimage.distance_transform_edt(~act, return_indices=True)
        ref = ((ind[0] * shape[1] + ind[1]) * shape[2] + ind[2]).ravel()
        np.testing.assert_array_equal(ft, ref)


def test_sample_nodes_matches_reference(golden):
    z, g = _case(golden)
    gm = Grid(z["ml_xe"], z["ml_ye"], z["ml_ze"])
    o = dict(g=g, cn=z["cn"], active=z["active"])
    u = post.sample_nodes(o, gm, z["Urel"])
    assert u.dtype == np.float32 and u.shape == z["u_nodes"].shape
    np.testing.assert_allclose(u, z["u_nodes"], rtol=0, atol=2 * np.finfo(np.float32).eps * np.abs(z["u_nodes"]).max())


def test_material_mixing_on_device_bit_exact(golden):
    """rb/rbfe.py:75-134 on the device: class fractions, joint cells, E, nu and active flags equal the
    reference's bit for bit (two parameter sets)."""
    from comech_b200.materials import materials
    z = golden("materials")
    names = [str(n) for n in z["role_names"]]
    bodies = np.split(z["role_bodies"], np.cumsum(z["role_len"])[:-1])
    roles = {"bones": {n: tuple(int(b) for b in bb) for n, bb in zip(names, bodies)},
             "bonded_extra": [int(b) for b in z["role_bonded_extra"]]}
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    V = dict(cls={str(int(b)): int(c) for b, c in zip(z["cls_body"], z["cls_class"])}, L=z["L"],
             xe=np.arange(nx + 1.0), ye=np.arange(ny + 1.0), ze=np.arange(nz + 1.0))
    for name, kw in (("a", {}), ("b", dict(cart_E=float(z["b_cart_E"]), nu_soft=float(z["b_nu_soft"])))):
        E, nu, active, F, ser = materials(V, roles, **kw)
        for a, key in ((E, "E"), (nu, "nu"), (active, "active"), (F, "F"), (ser, "ser")):
            np.testing.assert_array_equal(a, z[f"{name}_{key}"], err_msg=key)
