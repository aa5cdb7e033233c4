"""Device labelling (feb_label_lattice, comech_b200.labels) against the reference's own label_lattice on seeded
synthetic templates (tests/golden/labels.npz): every foot and action of tests/golden/label_cases.py on a whole-foot
lattice and a fine joint lattice, both template seeds.  Integer labels: bit-exact."""
import os
import sys

import numpy as np
import pytest

from comech_b200 import labels as LB, synth

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from label_cases import LABEL_CASES   # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1])
def test_device_lattices_match_reference(golden, seed):
    z = golden("labels")
    T = synth.synthetic_template(seed)
    D = LB.DeviceTemplate(T)
    for name, fk, ak, fill in LABEL_CASES:
        for ln in ("foot", "joint"):
            key = f"s{seed}_{name}_{ln}"
            if key not in z:
                continue
            sx, sy, sz = z[f"s{seed}_{ln}_sx"], z[f"s{seed}_{ln}_sy"], z[f"s{seed}_{ln}_sz"]
            got = LB.label_lattice(sx, sy, sz, LB.Foot(**fk), LB.Action(**ak), defect_fill=fill, device_template=D)
            ref = z[key]
            assert got.shape == ref.shape
            bad = np.argwhere(got != ref)
            assert len(bad) == 0, (name, ln, len(bad), bad[:5].tolist())


def test_device_label_rejects_bad_arguments():
    T = synth.synthetic_template(0)
    with pytest.raises(Exception):
        LB.label_lattice(np.zeros(3), np.zeros(3), np.zeros(3), LB.Foot(scale=0.0), LB.Action(), T=T)
