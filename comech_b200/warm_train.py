"""Training of the warm-start network on engine-generated FP64 solves, and its evaluation on held-out solves.

    python -m comech_b200.warm_train [--train 2000] [--held 200] [--epochs 12] [--out weights.npz] [--report r.json]

Data: seeded synthetic hindfoot instances on 96 x 64 x 48 voxels over the 80 x 56 x 48 mm box of the full-size
hindfoot (voxels 0.833 x 0.875 x 1.0 mm), one seeded surgical action each (none, resection, osteotomy,
interposition, fusion, load scaling; ``synth.hindfoot_problem``).  The host cores generate the instances (a
process pool started before the first CUDA call); the GPU solves each in FP64 to rel-res 1e-8 (the plain
GMG-PCG) and turns inputs and solution into the network's input and target, kept on the device for training.

Training: Adam on the relative squared error of the displacement (in units of ``u_unit``, scaled by the total
load; weight ``--mse``) plus the relative stiffness-weighted squared error of its differences along the grid edges
(weight ``--h1``; ``feb_net_loss``), the part of the error that the solve's energy norm weighs; gradients
accumulated over ``--batch`` instances, cosine learning-rate decay, all passes in libfeb200.so.  Evaluation on the held-out instances: mixed-precision PCG iterations and time to rel-res 1e-8
from zero and from the network's prediction (as given, and as ``feb_solve`` prepares it by default: one
preconditioner application, then its energy-optimal multiple, or a zero start when that multiple is not positive),
the prediction's relative error, and the fallback rate.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import time

import numpy as np

GRID = (96, 64, 48)
BOX = (80.0, 56.0, 48.0)
H = tuple(b / n for b, n in zip(BOX, GRID))
ACTIONS = ("none", "resection", "osteotomy", "interposition", "fusion", "load")
TOL = 1e-8


def make_instance(seed):
    """One seeded instance (runs in a worker process; no CUDA)."""
    from comech_b200 import synth
    P = synth.hindfoot_problem(*GRID, h=H, seed=int(seed), action=ACTIONS[int(seed) % len(ACTIONS)])
    P["cn"] = P["cn"].astype(np.int32)
    P.pop("bone_share", None)
    P.pop("E", None)
    P.pop("nu", None)
    return int(seed), P


def device_problem(P, precision, options=None):
    """engine.Problem of an instance, with its rigid groups and right-hand side."""
    import torch
    from comech_b200 import engine, _lib
    K_GROUND = engine.K_GROUND
    fn, fa = P["fixed"]
    pen_k = np.repeat((np.asarray(fa) * K_GROUND)[:, None], 3, axis=1)
    nr, cr, nc, cc, v = P["extra"].node_coo()
    mat = torch.from_numpy(np.concatenate([P["lam"], P["mu"]])).cuda()
    pr = engine.Problem(P["grid"], _lib.MAT_ISO_SRI, mat, P["active"], cn=P["cn"].astype(np.int64), orig=P["orig"],
                        pen_node=np.asarray(fn, np.int64), pen_k=pen_k, extra_coo=(3 * nr + cr, 3 * nc + cc, v),
                        precision=precision, tol=TOL, maxiter=800, options=options)
    pr.set_rigid_groups(P["node_groups"])
    f = pr.rhs(P["loads"])
    return pr, f


def load_parts(P):
    (ln, la, lt), = P["loads"]
    return np.asarray(ln, np.int64), np.asarray(la, np.float64) * float(lt[2])


def solve(P, precision, x0=None, options=None):
    pr, f = device_problem(P, precision, options)
    try:
        x, info = pr.solve(f, x0)
        U = pr.export(x)
        return U, info
    finally:
        pr.close()


X0_MODES = {"as_given": 0, "smoothed": 2}


def evaluate(net, items):
    """Held-out instances: the FP64 solution, then mixed-precision PCG iterations / time to rel-res 1e-8 from zero and
    from the network's prediction, used as given (x0_mode 0) and smoothed by one preconditioner application and
    scaled to its energy-optimal multiple (x0_mode 2, the default)."""
    import torch
    ev = []
    for seed, P in items:
        ln, lz = load_parts(P)
        nt = len(P["orig"])
        U64, _ = solve(P, "fp64")
        Ur = U64.view(-1, 3).cpu().numpy()
        used = np.isfinite(Ur).all(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, i0 = solve(P, "mixed")
        torch.cuda.synchronize()
        rec = dict(seed=int(seed), action=ACTIONS[int(seed) % len(ACTIONS)], iters_zero=int(i0.iters),
                   t_zero_s=time.perf_counter() - t0, solve_zero_ms=float(i0.t_solve_ms))
        for variant, mode in X0_MODES.items():
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            x0 = net.predict_x0(P["grid"], P["lam"], P["mu"], P["active"], P["orig"], P["fixed"][0], ln, lz, nt)
            torch.cuda.synchronize()
            tp = time.perf_counter() - t0
            _, i1 = solve(P, "mixed", x0, options=dict(x0_mode=mode))
            torch.cuda.synchronize()
            pr = x0.view(-1, 3).cpu().numpy()
            rec[variant] = dict(iters=int(i1.iters), x0_used=int(i1.x0_used), x0_scale=float(i1.x0_scale),
                                t_s=time.perf_counter() - t0, t_predict_s=tp, solve_ms=float(i1.t_solve_ms),
                                pred_rel_l2=float(np.linalg.norm(pr[used] - Ur[used]) / np.linalg.norm(Ur[used])),
                                relres=float(i1.relres), flag=int(i1.flag))
        ev.append(rec)
    return ev


def summarize(ev):
    if not ev:
        return {}
    med = lambda xs: float(np.median(xs))
    zero = [e["iters_zero"] for e in ev]
    out = dict(held_iters_zero_median=med(zero), held_t_zero_median_s=med([e["t_zero_s"] for e in ev]),
               held_solve_zero_ms_median=med([e["solve_zero_ms"] for e in ev]))
    for v in X0_MODES:
        out[v] = dict(iters_median=med([e[v]["iters"] for e in ev]),
                      iters_ratio=float(np.mean([e[v]["iters"] for e in ev]) / np.mean(zero)),
                      fallback_rate=float(np.mean([1 - e[v]["x0_used"] for e in ev])),
                      pred_rel_l2_median=med([e[v]["pred_rel_l2"] for e in ev]),
                      x0_scale_median=med([e[v]["x0_scale"] for e in ev]),
                      t_median_s=med([e[v]["t_s"] for e in ev]), t_predict_median_s=med([e[v]["t_predict_s"] for e in ev]),
                      solve_ms_median=med([e[v]["solve_ms"] for e in ev]),
                      relres_max=float(max(e[v]["relres"] for e in ev)),
                      flags=sorted({e[v]["flag"] for e in ev}),
                      per_action={a: [round(float(np.mean([e["iters_zero"] for e in ev if e["action"] == a] or [0])), 2),
                                      round(float(np.mean([e[v]["iters"] for e in ev if e["action"] == a] or [0])), 2)]
                                  for a in ACTIONS})
    return out


def cosine(step, total, lr0, lr1):
    return lr1 + 0.5 * (lr0 - lr1) * (1 + math.cos(math.pi * min(step, total) / total))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--held", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--time-budget", type=float, default=0.0, help="stop training after this many seconds (0: none)")
    ap.add_argument("--h1", type=float, default=1.0, help="weight of the stiffness-weighted edge term (0: plain MSE)")
    ap.add_argument("--mse", type=float, default=0.2, help="weight of the squared error when --h1 or --energy > 0")
    ap.add_argument("--energy", type=float, default=0.0, help="weight of the error's strain energy (feb_net_energy_loss)")
    ap.add_argument("--eval-only", default=None, help="evaluate these weights on --held instances (no training)")
    args = ap.parse_args(argv)
    nw = args.workers or max(1, min(32, (os.cpu_count() or 2) - 2))
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(nw)                         # before the first CUDA call
    import torch
    from comech_b200 import warmnet
    if args.eval_only:
        seeds = list(range(args.seed0 + args.train, args.seed0 + args.train + args.held))
        items = pool.map(make_instance, seeds, chunksize=2)
        pool.close()
        ev = evaluate(warmnet.WarmNet.load(args.eval_only), items)
        summary = dict(weights=args.eval_only, held=len(ev), **summarize(ev))
        print(json.dumps(summary), flush=True)
        if args.report:
            with open(args.report, "w") as f:
                json.dump(dict(summary=summary, held=ev), f, indent=1)
        return summary
    t_start = time.perf_counter()
    N, Nh = args.train, args.held
    seeds = list(range(args.seed0, args.seed0 + N + Nh))
    rows = warmnet._rows(GRID)
    X = torch.zeros(N + Nh, rows, warmnet.CIN, dtype=torch.bfloat16, device="cuda")
    T = torch.zeros(N + Nh, rows, 3, dtype=torch.float32, device="cuda")
    Wt = torch.zeros(N + Nh, rows, dtype=torch.float32, device="cuda")
    inv_n = np.zeros(N + Nh)
    inv_h1 = np.zeros(N + Nh)
    inv_en = np.zeros(N + Nh)
    loadf = np.zeros(N + Nh)
    held = {}
    net = warmnet.WarmNet(seed=0, grid=GRID)
    u_unit = None
    t_solve = 0.0
    iters_fp64 = []
    for i, (seed, P) in enumerate(pool.imap(make_instance, seeds, chunksize=2)):
        t0 = time.perf_counter()
        U, info = solve(P, "fp64")
        t_solve += time.perf_counter() - t0
        iters_fp64.append(int(info.iters))
        ln, lz = load_parts(P)
        loadf[i] = float(np.abs(lz).sum()) / warmnet.REF_LOAD
        if u_unit is None:                       # displacement unit: RMS of the first solution at 450 N
            Uh = U.view(-1, 3).cpu().numpy()
            u_unit = float(np.sqrt(np.nanmean(Uh ** 2))) / loadf[i]
            net.u_unit = u_unit
        net.inputs(P["grid"], P["lam"], P["mu"], P["active"], P["orig"], P["fixed"][0], ln, lz, dims=GRID, out=X[i])
        Ti, wi = warmnet.load_targets(GRID, U, u_unit * loadf[i])
        T[i].copy_(Ti)
        Wt[i].copy_(wi)
        inv_n[i] = 1.0 / max(float(wi.sum().item()), 1.0)
        inv_h1[i] = 1.0 / max(warmnet.h1_norm(X[i], GRID, T[i], Wt[i]), 1e-30)
        inv_en[i] = 1.0 / max(warmnet.energy_norm(X[i], GRID, H, T[i], Wt[i]), 1e-30)
        if i >= N:
            held[i] = P
    pool.close()
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t_start

    # ---------------------------------------------------------------------------------------------- training
    def loss_scales(j, nb):
        # relative squared error (weight args.mse) + relative stiffness-weighted edge error (args.h1), averaged over
        # the batch; the relative strain energy of the error (args.energy) is passed separately
        if args.h1 <= 0 and args.energy <= 0:
            return None
        return (args.mse * inv_n[j] / nb, args.h1 * inv_h1[j] / nb)

    def energy_scale(j, nb):
        return None if args.energy <= 0 else (args.energy * inv_en[j] / nb, H)

    rng = np.random.default_rng(0)
    steps_per_epoch = N // args.batch
    total = steps_per_epoch * args.epochs
    B = net.buffers(GRID)
    hist = []
    t1 = time.perf_counter()
    step = 0
    stopped_early = False
    for ep in range(args.epochs):
        perm = rng.permutation(N)
        B["loss"].zero_()
        for s in range(steps_per_epoch):
            for j in perm[s * args.batch:(s + 1) * args.batch]:
                net.forward(X[j], GRID)
                net.backward(X[j], GRID, T[j], Wt[j], inv_n[j] / args.batch, h1=loss_scales(j, args.batch),
                             energy=energy_scale(j, args.batch))
            net.adam(cosine(step, total, args.lr, args.lr * 0.02), clip=10.0)
            step += 1
        train_loss = float(B["loss"].item()) / steps_per_epoch
        # validation loss on the held-out instances
        B["loss"].zero_()
        for j in range(N, N + Nh):
            net.forward(X[j], GRID)
            net.backward(X[j], GRID, T[j], Wt[j], inv_n[j], h1=loss_scales(j, 1), energy=energy_scale(j, 1))
        net.grad.zero_()
        val_loss = float(B["loss"].item()) / max(Nh, 1)
        hist.append(dict(epoch=ep, train_loss=train_loss, val_loss=val_loss, t=round(time.perf_counter() - t1, 1)))
        print(json.dumps(hist[-1]), flush=True)
        if args.time_budget and time.perf_counter() - t1 > args.time_budget:
            stopped_early = True
            break
    net.check_status()
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    t_step = t_train / max(step, 1) / args.batch

    # ---------------------------------------------------------------------------------------------- evaluation
    ev = evaluate(net, [(seeds[j], P) for j, P in held.items()])
    summary = dict(
        grid=GRID, box_mm=BOX, train=N, held=Nh, epochs_run=len(hist), batch=args.batch, params=net.nparam,
        u_unit=u_unit, t_data_s=round(t_data, 1), t_solve_fp64_s=round(t_solve, 1),
        fp64_iters_median=float(np.median(iters_fp64)) if iters_fp64 else None,
        t_train_s=round(t_train, 1), t_per_sample_step_ms=round(1e3 * t_step, 3), stopped_early=stopped_early,
        history=hist, **summarize(ev))
    if args.out:
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        net.save(args.out, train=N, epochs=len(hist), box=np.array(BOX))
    print(json.dumps({k: v for k, v in summary.items() if k != "history"}), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(dict(summary=summary, held=ev), f, indent=1)
    return summary


if __name__ == "__main__":
    main()
