"""Host-side logic around the solve, on the CPU (no GPU): the batch instances' sizes and actions, the warm-start
training schedule and held-out summary, and the generator's box-shaped voxels."""
import numpy as np

import bench
from comech_b200 import synth, warm_train


def test_batch_instances_span_the_stated_sizes_and_actions():
    dims, actions = [], []
    for seed in range(10):
        rng = np.random.default_rng(10_000 + seed)
        f = rng.uniform(0.0, 1.0)
        nx, ny, nz = (int(round(a + f * (b - a))) for a, b in ((64, 128), (48, 96), (40, 80)))
        assert 64 <= nx <= 128 and 48 <= ny <= 96 and 40 <= nz <= 80
        dims.append((nx, ny, nz))
        actions.append(bench.BATCH_ACTIONS[seed % 5])
    assert len(set(dims)) >= 8                               # uneven grids
    assert set(actions) == set(bench.BATCH_ACTIONS)
    P = bench.batch_instance(0)
    assert (P["grid"].nx, P["grid"].ny, P["grid"].nz) == dims[0]
    assert abs(P["grid"].xe[-1] - 80.0) < 1e-9              # an 80-mm-long box whatever the grid


def test_cosine_schedule_and_held_out_summary():
    assert warm_train.cosine(0, 100, 1e-3, 2e-5) == 1e-3
    assert abs(warm_train.cosine(100, 100, 1e-3, 2e-5) - 2e-5) < 1e-15
    assert warm_train.cosine(50, 100, 1e-3, 2e-5) < 1e-3
    rec = lambda a, z, g, s: dict(seed=0, action=a, iters_zero=z, t_zero_s=0.05, solve_zero_ms=30.0,
                                  **{v: dict(iters=g, x0_used=1, x0_scale=s, t_s=0.06, t_predict_s=0.004,
                                             solve_ms=31.0, pred_rel_l2=0.5, relres=9e-9, flag=0)
                                     for v in warm_train.X0_MODES})
    ev = [rec("none", 64, 62, 0.6), rec("osteotomy", 116, 114, 0.7), rec("fusion", 63, 63, 0.5)]
    out = warm_train.summarize(ev)
    assert out["held_iters_zero_median"] == 64
    sm = out["smoothed"]
    assert sm["iters_median"] == 63 and sm["fallback_rate"] == 0.0 and sm["flags"] == [0]
    assert abs(sm["iters_ratio"] - (62 + 114 + 63) / (64 + 116 + 63)) < 1e-12
    assert sm["per_action"]["osteotomy"] == [116.0, 114.0]
    assert warm_train.summarize([]) == {}


def test_box_shaped_voxels_keep_the_box():
    P = synth.hindfoot_problem(24, 16, 12, h=(80 / 24, 56 / 16, 48 / 12), seed=3)
    g = P["grid"]
    assert abs(g.xe[-1] - 80) < 1e-9 and abs(g.ye[-1] - 56) < 1e-9 and abs(g.ze[-1] - 48) < 1e-9
    Q = synth.hindfoot_problem(24, 16, 12, h=2.0, seed=3)
    assert abs(Q["grid"].xe[-1] - 48) < 1e-9 and abs(Q["grid"].ze[-1] - 24) < 1e-9
