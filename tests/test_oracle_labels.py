"""The labelling oracle (oracle/label_oracle.py) against the reference's own label_lattice and label_points
(rb/rbgeom.py:358-524) on seeded synthetic templates (tests/golden/labels.npz, made by tests/golden/make_golden.py):
18 feet and actions that reach every branch of the rule (scale, facet sizes, anterior facet modes, warps, shear,
coalitions I-IV with R1-R4, resection with soft / void / interposition fill, osteotomies, fusion), a whole-foot
lattice and a fine lattice over the joint, and 4000 scattered points.  Integer labels: bit-exact."""
import numpy as np
import pytest

from comech_b200 import labels as LB, synth
from oracle import label_oracle as LO

import sys, os
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from label_cases import LABEL_CASES   # noqa: E402


@pytest.fixture(scope="module")
def templates():
    return {s: synth.synthetic_template(s) for s in (0, 1)}


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_lattices_match_reference(golden, templates, seed):
    z = golden("labels")
    T = templates[seed]
    for name, fk, ak, fill in LABEL_CASES:
        lats = ("foot", "joint") if seed == 0 else ("joint",)
        for ln in lats:
            sx, sy, sz = z[f"s{seed}_{ln}_sx"], z[f"s{seed}_{ln}_sy"], z[f"s{seed}_{ln}_sz"]
            got = LO.label_lattice(sx, sy, sz, LB.Foot(**fk), LB.Action(**ak), T, fill)
            np.testing.assert_array_equal(got, z[f"s{seed}_{name}_{ln}"], err_msg=f"{name} {ln}")


def test_oracle_points_match_reference(golden, templates):
    z = golden("labels")
    for seed in (0, 1):
        P = z[f"s{seed}_points"]
        for name, fk, ak, fill in LABEL_CASES:
            got = LO.label_points(P, LB.Foot(**fk), LB.Action(**ak), templates[seed], fill)
            np.testing.assert_array_equal(got, z[f"s{seed}_{name}_pts"], err_msg=name)


def test_every_case_edits_the_joint(golden):
    """Each case changes labels against the unedited foot on the joint lattice (no case is vacuous)."""
    z = golden("labels")
    base = z["s0_default_joint"]
    for name, fk, ak, fill in LABEL_CASES[1:]:
        assert (z[f"s0_{name}_joint"] != base).sum() > 100, name


def test_synthetic_template_is_deterministic(templates):
    T = synth.synthetic_template(0)
    np.testing.assert_array_equal(T.lab, templates[0].lab)
    np.testing.assert_array_equal(T.dt, templates[0].dt)
    for k in LB.FACETS:
        np.testing.assert_array_equal(T.facets[k]["F0"], templates[0].facets[k]["F0"])
        assert T.facets[k]["gap"] == templates[0].facets[k]["gap"]
