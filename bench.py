#!/usr/bin/env python
"""Seconds per solve to rel-res 1e-8 of the synthetic ~5M-DOF hindfoot (160x112x96 voxels, h = 0.5 mm) on
one B200, mixed precision (FP64 CG around an FP32 multigrid V-cycle; --precision refine: FP64 iterative
refinement around an all-FP32 GMG-PCG) next to the plain FP64 GMG-PCG.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one solve of the same inputs: device set-up of the operator and the multigrid hierarchy
(Galerkin products, power iterations, coarse inverse), CG to rel-res 1e-8, displacement export and
cell stress / von Mises.  ``value`` is timed with CUDA events from device-resident inputs; ``e2e``
times the public API (``engine.solve_cn`` + ``engine.cell_stress_cn``) from pinned host arrays to host
results.  ``--impl reference`` times the CPU oracle (a NumPy/SciPy restatement of the reference's
``rb/splitfe.solve_cn`` + ``cell_stress_cn``) on a bounded sample of the same generator, scaled to the
metric's problem size by the dof ratio.  Under torchrun every rank solves its own seeded instance
(independent units, weak scaling); rank 0 prints one JSON line.

When the packaged warm-start network is present, the same solve started from its prediction (the metric's
learned + mixed configuration) is timed beside the headline in ``learned_warm_start``; it changes the iteration
count by a few percent at most, so the headline ``value`` is the mixed solve from a zero start.  ``--mode batch`` times 64
independent instances of uneven size, one at a time and with 8 / 16 solves in flight.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "s/solve to 1e-8 rel. residual, 5M DOF: learned+mixed vs plain FP64, one B200"
WORKLOAD = dict(nx=160, ny=112, nz=96, h=0.5)
SAMPLE_BIG = dict(nx=64, ny=45, nz=38, h=1.25)     # CPU sample (~25 s of oracle work on 1 core)
SAMPLE_SMALL = dict(nx=40, ny=28, nz=24, h=2.0)    # CPU sample for long reference runs (~5 s)
TOL = 1e-8
SETUP_STAGES = ("cells", "penalties_extra", "diag_blocks", "ku_tuning", "hierarchy", "power_launch",
                "dense_and_power_tail", "host_before_setup")


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler.  It is started before the warm-up steps, so that nvidia-smi's own start-up (NVML
    initialisation over every GPU of the node, which holds the driver's locks for a while) is over before timing
    begins; only the samples inside the timed window (`window`) are summarised."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def window(self, t0, t1):
        self.t0, self.t1 = t0, t1

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        import datetime
        rows = []
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None
            rows.append((ts, f[1:]))
        if self.t0 is not None:   # the timed window, widened by one sampling period so that it holds a sample
            inside = [r for ts, r in rows if ts is not None and self.t0 - 0.2 <= ts <= self.t1 + 0.2]
            self.rows = inside or [r for _, r in rows]
        else:
            self.rows = [r for _, r in rows]

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i, v in enumerate(r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}

def rank_seed(rank):
    """Seed of the instance a rank solves (independent instances, weak scaling)."""
    return int(rank)


def rank_instances(rank, world, n):
    """Round-robin split of n independent instances over the ranks."""
    return list(range(rank, n, world))


def reduce_max(t, dist, device="cuda"):
    """Max over ranks of a per-rank duration (identity without a process group)."""
    if dist is None:
        return float(t)
    import torch
    v = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


def make_problem(seed, dims=WORKLOAD):
    from comech_b200 import synth
    return synth.hindfoot_problem(dims["nx"], dims["ny"], dims["nz"], h=dims["h"], seed=seed)


def cpu_oracle_run(dims, seed=0, P=None):
    """One solve_cn + cell_stress of the CPU oracle on the generator's instance at ``dims``: seconds per phase
    (assembly with penalties and extra entries, multigrid set-up, PCG, stress), dofs, iterations, and the
    solution (U, von Mises) for the parity checks."""
    from oracle import fe_oracle as O
    P = make_problem(seed, dims) if P is None else P
    g = O.OGrid(P["grid"].xe, P["grid"].ye, P["grid"].ze)
    t = time.perf_counter()
    U, info, R = O.solve_cn(g, P["lam"], P["mu"], P["active"], P["cn"], P["orig"], P["fixed"], P["loads"], P["extra"],
                            P["node_groups"], tol=TOL)
    t1 = time.perf_counter()
    _, vm, _ = O.cell_stress(g, P["lam"], P["mu"], U, np.flatnonzero(P["active"]), P["cn"], nan_to_zero=True)
    t2 = time.perf_counter()
    return dict(t=t2 - t, t_assemble=info["t_assemble"], t_setup=info["t_setup"], t_pcg=info["t_pcg"],
                t_stress=t2 - t1, ndof=int(info["ndof"]), iters=int(info["iters"]), U=U, vm=vm)


def cpu_oracle_step(dims, seed=0):
    """One solve_cn + cell_stress of the CPU oracle; returns (seconds, ndof, iterations)."""
    r = cpu_oracle_run(dims, seed)
    return r["t"], r["ndof"], r["iters"]


def extrapolate(sample, ndof, iters):
    """Oracle seconds of a solve of ``ndof`` dofs in ``iters`` iterations from a measured sample: the assembly,
    multigrid set-up and stress phases scale with the dofs, the PCG phase with dofs x iterations."""
    r = ndof / sample["ndof"]
    return ((sample["t_assemble"] + sample["t_setup"] + sample["t_stress"]) * r
            + sample["t_pcg"] * r * iters / sample["iters"])


def parity(U, vm, Uo, vmo):
    """Displacement and von Mises rel-L2 of a device solution against the oracle's (used nodes, active cells)."""
    U = np.asarray(U).reshape(-1, 3)
    Uo = np.asarray(Uo).reshape(-1, 3)
    ok = ~np.isnan(Uo)
    if not (np.isnan(U) == ~ok).all():
        return {"error": "used-node masks differ"}
    return {"disp_rel_l2": float(np.linalg.norm(U[ok] - Uo[ok]) / np.linalg.norm(Uo[ok])),
            "vm_rel_l2": float(np.linalg.norm(np.asarray(vm) - vmo) / np.linalg.norm(vmo))}


def workload_ndof():
    # used nodes of the metric's workload (3 dofs each) -- counted once on the generator output
    P = make_problem(0)
    used = np.unique(P["cn"][np.flatnonzero(P["active"])])
    return 3 * len(used)


def device_inputs(P):
    """Upload the big per-cell / per-node arrays once (value is timed from device-resident inputs)."""
    import torch
    from comech_b200.synth import SpringSet  # noqa: F401
    d = {}
    d["mat"] = torch.from_numpy(np.concatenate([P["lam"], P["mu"]])).cuda()
    d["active"] = torch.from_numpy(P["active"].astype(np.uint8)).cuda()
    d["cn"] = torch.from_numpy(np.ascontiguousarray(P["cn"], dtype=np.int64)).cuda()
    d["orig"] = torch.from_numpy(np.ascontiguousarray(P["orig"], dtype=np.int64)).cuda()
    groups = P["node_groups"]
    d["g_off"] = np.r_[0, np.cumsum([len(x) for x in groups])].astype(np.int64)
    d["g_nodes"] = torch.from_numpy(np.concatenate(groups).astype(np.int64)).cuda()
    (ln, la, lt), = P["loads"]
    d["l_nodes"] = torch.from_numpy(np.asarray(ln, np.int64)).cuda()
    d["l_vals"] = torch.from_numpy(np.asarray(la, np.float64)[:, None] * lt[None, :]).cuda()
    d["load_nodes_h"] = np.asarray(ln, np.int64)
    d["load_z_h"] = np.asarray(la, np.float64) * float(lt[2])
    d["cells"] = torch.from_numpy(np.flatnonzero(P["active"]).astype(np.int64)).cuda()
    fn, fa = P["fixed"]
    d["pen_node"] = np.asarray(fn, np.int64)
    d["pen_k"] = np.repeat((np.asarray(fa) * 1e6)[:, None], 3, axis=1)
    nr, cr, nc, cc, v = P["extra"].node_coo()
    d["extra"] = (3 * nr + cr, 3 * nc + cc, v)
    return d


SOLVER_OPTIONS = {}
# The oracle's FP64 solve of the full 160x112x96 workload (bench.py --cpu-full, one B200 box's host core):
# 72 iterations, 284.3 s (assembly 30.1, multigrid set-up 17.5, PCG 235.4, stress 1.3).  The reference arm
# extrapolates its bounded samples to this iteration count.
ORACLE_FULL_ITERS = 72
ORACLE_FULL_S = 284.3


def device_solve(P, d, precision, x0=None, warm=None):
    """One solve from device-resident inputs (same work as engine.solve_cn + cell_stress_cn); with ``warm`` (a
    trained warmnet.WarmNet) the network's prediction is the initial guess, computed inside the step."""
    from comech_b200 import engine, _lib
    g = P["grid"]
    t = [time.perf_counter()]          # host time stamps of the phases (no synchronisation added)
    pr = engine.Problem(g, _lib.MAT_ISO_SRI, d["mat"], d["active"], cn=d["cn"], orig=d["orig"],
                        pen_node=d["pen_node"], pen_k=d["pen_k"], extra_coo=d["extra"], precision=precision, tol=TOL,
                        maxiter=800, options=SOLVER_OPTIONS)
    t.append(time.perf_counter())
    try:
        pr.set_rigid_groups(d["g_nodes"], offsets=d["g_off"])
        t.append(time.perf_counter())
        f = pr.rhs([(d["l_nodes"], d["l_vals"])])
        if warm is not None and x0 is None:
            nc = g.nx * g.ny * g.nz
            x0 = warm.predict_x0(g, d["mat"][:nc], d["mat"][nc:], d["active"], P["orig"], P["fixed"][0],
                                 d["load_nodes_h"], d["load_z_h"], len(P["orig"]), orig_dev=d["orig"])
        t.append(time.perf_counter())
        x, info = pr.solve(f, x0)
        t.append(time.perf_counter())
        U = pr.export(x)
        sig, vm, eps = engine._stress(g, _lib.MAT_ISO_SRI, d["mat"], U, d["cells"], d["cn"], True, to_host=False)
        t.append(time.perf_counter())
        return U, vm, info
    finally:
        pr.close()
        t.append(time.perf_counter())
        device_solve.host_ms = [round(1e3 * (b - a), 2) for a, b in zip(t, t[1:])]


KU_PROFILE = os.path.join(HERE, "profiles", "k_fine_pair_apply_fp32_hindfoot_160x112x96.md")
SMOOTH_PROFILE = os.path.join(HERE, "profiles", "k_fine_pair_smooth_fp32_hindfoot_160x112x96.md")


def ku_traffic(path=KU_PROFILE):
    """DRAM bytes (read + write) of one launch from a committed ncu summary, or None."""
    import re
    try:
        with open(path) as f:
            m = re.search(r"^traffic_bytes_per_launch:\s*(\d+)", f.read(), re.M)
        return int(m.group(1)) if m else None
    except OSError:
        return None


def flush_l2(buf):
    buf.add_(1.0)


def timed_steps(fn, steps, flush, dist=None, clocks=None, per_step=None):
    """Device time of ``steps`` calls of fn (CUDA events on the current stream, L2 flushed before each); the
    barrier and synchronisation bracket the whole timed region.  Returns (per-step ms, last result);
    ``per_step(result)`` (optional) is appended to the list ``timed_steps.details`` after each step."""
    import gc
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out, ms = None, []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # the interpreter's cyclic collector is run between steps, not inside them: a collection pass over the
    # step's large host arrays stalls the host thread that issues the step's launches
    gc.collect()
    gc.disable()
    try:
        for _ in range(steps):
            flush_l2(flush)
            ev0.record()
            out = fn()
            ev1.record()
            torch.cuda.synchronize()
            ms.append(ev0.elapsed_time(ev1))
            if per_step is not None:
                timed_steps.details.append(per_step(out))
            gc.collect()
    finally:
        gc.enable()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    return ms, out


def special_nodes(P, g):
    """Grid nodes of the level-0 operator that receive a sparse contribution (ground springs, extra entries,
    corners of cells touching split copies) plus the split copies: the nodes that go through the accumulator."""
    cells = np.flatnonzero(P["active"])
    irr = cells[(P["cn"][cells] != g.cell_nodes[cells]).any(1)]
    nr = P["extra"].node_coo()[0]
    nodes = np.unique(np.concatenate([np.asarray(P["fixed"][0]), P["cn"][irr].ravel(), nr]))
    return int(np.count_nonzero(nodes < g.nnode)) + (len(P["orig"]) - g.nnode), len(irr)


def ku_roofline(P, d, lib, engine, _lib, pk, pk_kind):
    """The level-0 operator (sparse pass + paired-row kernel) timed on a rotating set of operand buffers
    larger than L2, with its algorithmic bytes."""
    import ctypes as C
    import torch
    g = P["grid"]
    ntotal = len(P["orig"])
    nact = int(P["active"].sum())
    n_spec, n_irr = special_nodes(P, g)
    n_pen = len(P["fixed"][0])
    n_extra = P["extra"].node_coo()[4].size
    npair = (g.nx + 1) * ((g.ny + 1) // 2 + 1) * (g.nz + 1)
    pr = engine.Problem(g, _lib.MAT_ISO_SRI, d["mat"], d["active"], cn=d["cn"], orig=d["orig"], pen_node=d["pen_node"],
                        pen_k=d["pen_k"], extra_coo=d["extra"], options=dict(max_levels=0))
    roof = {}
    try:
        for name, dt, sv in (("fp32", torch.float32, 4), ("fp64", torch.float64, 8)):
            nbuf = max(2, int(np.ceil(3 * 126e6 / (6 * ntotal * sv))))      # the set exceeds L2 three times over
            us = [torch.randn(3 * ntotal, dtype=dt, device="cuda") for _ in range(nbuf)]
            ys = [torch.empty_like(u) for u in us]
            up = (C.c_void_p * nbuf)(*[u.data_ptr() for u in us])
            yp = (C.c_void_p * nbuf)(*[y.data_ptr() for y in ys])
            ms = C.c_float()
            for nrep in (2 * nbuf, 20 * nbuf):
                _lib.check(lib.feb_benchmark_apply_set(pr.h, 0 if sv == 8 else 1, nbuf, up, yp, nrep, C.byref(ms)))
            # u, y; cell-pair words (2 bytes per pair of node rows); the sparse part: irregular cells (8 node ids +
            # 2 material values), penalties (node + 3 values), extra entries (column + value), and the
            # accumulator of the special nodes (atomic adds, then read and cleared by the owners)
            alg = (6 * ntotal * sv + 2 * npair + n_irr * (32 + 2 * sv) + n_pen * (4 + 3 * sv) + n_extra * (8 + sv)
                   + n_spec * 3 * sv * 3)
            roof[name] = dict(ms=ms.value, bytes=alg, gbs=alg / (ms.value * 1e-3) / 1e9, nbuf=nbuf)
            del us, ys
    finally:
        pr.close()
    # the solve's dominant kernel (its largest share of device time): the level-0 smoother step, the paired K.u
    # with the fused Chebyshev update, as the V-cycle runs it (mixed precision handle with its hierarchy)
    ps = engine.Problem(g, _lib.MAT_ISO_SRI, d["mat"], d["active"], cn=d["cn"], orig=d["orig"], pen_node=d["pen_node"],
                        pen_k=d["pen_k"], extra_coo=d["extra"], precision="mixed", tol=TOL)
    try:
        n3 = 3 * ntotal
        nbuf = max(2, int(np.ceil(3 * 126e6 / (4 * n3 * 4))))            # (d, r, x, d') sets exceed L2 three times over
        sets = [[torch.randn(n3, dtype=torch.float32, device="cuda") for _ in range(2)] +
                [torch.zeros(n3, dtype=torch.float32, device="cuda"), torch.empty(n3, dtype=torch.float32, device="cuda")]
                for _ in range(nbuf)]
        ptr = [(C.c_void_p * nbuf)(*[st[q].data_ptr() for st in sets]) for q in range(4)]
        ms = C.c_float()
        for nrep in (2 * nbuf, 20 * nbuf):
            _lib.check(lib.feb_benchmark_smooth_set(ps.h, nbuf, ptr[0], ptr[1], ptr[2], ptr[3], nrep, C.byref(ms)))
        # d read; r and x read and written; d' written; the 6-value symmetric block-Jacobi inverse; the K.u's
        # cell-pair words and sparse part as above
        sv = 4
        alg_s = (24 * ntotal * sv + 2 * npair + n_irr * (32 + 2 * sv) + n_pen * (4 + 3 * sv) + n_extra * (8 + sv)
                 + n_spec * 3 * sv * 3)
        sm = dict(ms=ms.value, bytes=alg_s, gbs=alg_s / (ms.value * 1e-3) / 1e9, nbuf=nbuf)
        del sets
    finally:
        ps.close()
    r32 = roof["fp32"]
    return {"bound": "hbm", "achieved": round(sm["gbs"], 1), "peak": pk, "unit": "GB/s",
            "frac": round(sm["gbs"] / pk, 4), "traffic": ku_traffic(SMOOTH_PROFILE),
            "kernel": "level-0 smoother step FP32 (k_fine_sparse + k_fine_pair with the fused Chebyshev update), the "
                      "solve's largest share of device time; operands rotated over "
                      f"{sm['nbuf']} buffer sets (> L2)",
            "peak_kind": pk_kind, "ms_per_launch": round(sm["ms"], 4), "algorithmic_bytes": sm["bytes"],
            "active_cells": nact,
            "ku_apply_fp32": {"achieved": round(r32["gbs"], 1), "frac": round(r32["gbs"] / pk, 4),
                              "ms_per_launch": round(r32["ms"], 4), "algorithmic_bytes": r32["bytes"],
                              "traffic": ku_traffic(), "nbuf": r32["nbuf"]},
            "fp64": {"achieved": round(roof["fp64"]["gbs"], 1), "frac": round(roof["fp64"]["gbs"] / pk, 4),
                     "ms_per_launch": round(roof["fp64"]["ms"], 4), "algorithmic_bytes": roof["fp64"]["bytes"]}}


def run_ours(args, rank, world, dist):
    import torch
    from comech_b200 import engine, _lib
    lib = _lib.load()
    dev = torch.cuda.current_device()
    P = make_problem(seed=rank_seed(rank))
    d = device_inputs(P)
    g = P["grid"]
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    prec = args.precision
    warm = None
    if args.warm != "off":
        from comech_b200 import warmnet
        try:
            warm = warmnet.default_net()
        except RuntimeError:
            if args.warm == "on":
                raise
    # the metric's configuration (learned start when the packaged network is present), then the same solve
    # from a zero start and the plain FP64 GMG-PCG; every arm is the mean of the same number of timed steps
    arms = [("headline", prec, warm)]
    if warm is not None:
        arms.append(("zero_start", prec, None))
    arms.append(("plain_fp64", "fp64", None))
    res = {}
    launches = 0
    clk_summary = None
    step_info = {}
    # per step: device set-up and solve ms, iterations, and the host ms of create / rigid groups / rhs (+ the
    # learned start) / solve / export + stress / close
    info_of = lambda out: (round(out[2].t_setup_ms, 2), round(out[2].t_solve_ms, 2), int(out[2].iters),
                           getattr(device_solve, "host_ms", None), round(out[2].t_stage_ms[7], 2))
    for name, pr_, w_ in arms:
        clk = Clocks(dev) if name == "headline" else None
        if clk:
            clk.__enter__()      # before the warm-up: nvidia-smi's start-up is over when timing begins
        # warm-up in the timed loop's form: each step runs while the previous step's results are still held (as
        # timed_steps holds them), so torch's device cache has its two sets of result buffers before timing; a
        # first allocation of the second set inside the timed region waited on cudaMalloc (+45-97 ms in one step)
        prev = None
        for _ in range(args.warmup):
            prev = device_solve(P, d, pr_, warm=w_)
        prev = None
        torch.cuda.synchronize()
        launches0 = lib.feb_launch_count()
        timed_steps.details = []
        if name == "headline":
            try:
                t_a = time.time()
                ms, out = timed_steps(lambda: device_solve(P, d, pr_, warm=w_), args.steps, flush, dist,
                                      per_step=info_of)
                clk.window(t_a, time.time())
            finally:
                clk.__exit__(None, None, None)
            clk_summary = clk.summary()
            launches = (lib.feb_launch_count() - launches0) // max(args.steps, 1)
        else:
            ms, out = timed_steps(lambda: device_solve(P, d, pr_, warm=w_), args.steps, flush, dist, per_step=info_of)
        step_info[name] = timed_steps.details
        U, vm, info = out
        res[name] = dict(ms=ms, U=U.cpu().numpy(), vm=vm, info=info)
    t_total = reduce_max(sum(res["headline"]["ms"]) / 1e3, dist)
    value = t_total / (args.steps * world)
    mean_s = {k: reduce_max(sum(v["ms"]) / 1e3, dist) / (args.steps * world) for k, v in res.items()}
    hinfo = res["headline"]["info"]
    U64h = res["plain_fp64"]["U"]
    vm64 = res["plain_fp64"]["vm"]
    par64 = {}
    for k in res:
        if k != "plain_fp64":
            par64[k] = parity(res[k]["U"], res[k]["vm"].cpu().numpy(), U64h, vm64.cpu().numpy())
    learned = None
    if warm is not None:
        nc = g.nx * g.ny * g.nz
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        x0w = warm.predict_x0(g, d["mat"][:nc], d["mat"][nc:], d["active"], P["orig"], P["fixed"][0],
                              d["load_nodes_h"], d["load_z_h"], len(P["orig"]), orig_dev=d["orig"])
        ev1.record()
        torch.cuda.synchronize()
        xw = x0w.view(-1, 3).cpu().numpy()
        Ur = U64h.reshape(-1, 3)
        okn = ~np.isnan(Ur).any(1)
        zi = res["zero_start"]["info"]
        learned = {"iters": int(hinfo.iters), "zero_start_iters": int(zi.iters),
                   "s_per_solve": round(mean_s["headline"], 5), "zero_start_s_per_solve": round(mean_s["zero_start"], 5),
                   "prediction_ms": round(ev0.elapsed_time(ev1), 3), "x0_used": int(hinfo.x0_used),
                   "x0_scale": float(hinfo.x0_scale),
                   "prediction_rel_l2": float(np.linalg.norm(xw[okn] - Ur[okn]) / np.linalg.norm(Ur[okn])),
                   "network": "3D conv encoder-decoder, 4.26M parameters, trained on 2000 FP64 solves of the "
                              "96x64x48 generator; start = x0 + M(f - K x0), scaled to its energy-optimal multiple"}
    # ---------------------------------------------------------------- e2e through the public API
    pinned = {}
    for k in ("lam", "mu", "cn", "orig"):
        a = np.ascontiguousarray(P[k])
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        pinned[k] = t.numpy()
    act = torch.empty(P["active"].shape, dtype=torch.bool, pin_memory=True)
    act.numpy()[...] = P["active"]
    pinned["active"] = act.numpy()
    cells_h = np.flatnonzero(P["active"])

    def e2e_step():
        t_a = time.perf_counter()
        U, inf, R = engine.solve_cn(g, pinned["lam"], pinned["mu"], pinned["active"], pinned["cn"], pinned["orig"],
                                    P["fixed"], P["loads"], P["extra"], P["node_groups"], tol=TOL, maxiter=800,
                                    precision=prec, keep_device=True, warm_start=warm)
        t_b = time.perf_counter()
        sig, vmh, eps = engine.cell_stress_cn(g, pinned["lam"], pinned["mu"], U, cells_h, pinned["cn"],
                                              device=inf["device"])
        inf["device"]["problem"].close()
        inf["t_host"]["stress"] = round(time.perf_counter() - t_b, 4)
        inf["t_host"]["solve_cn_total"] = round(t_b - t_a, 4)
        return U, vmh, inf

    # warm-up in the timed loop's own form: each step runs while the previous step's results are still held, so
    # torch's page-locked host cache reaches its steady state (two sets of result buffers) before timing starts
    e2e_s = []
    import gc
    gc.collect()
    gc.disable()            # as in timed_steps: the cyclic collector runs between steps
    try:
        n_warm = max(3, args.warmup)
        for i in range(n_warm + max(1, min(args.steps, 5))):
            flush_l2(flush)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Ue, vme, infe = e2e_step()
            torch.cuda.synchronize()
            if i >= n_warm:
                e2e_s.append(time.perf_counter() - t0)
            gc.collect()
    finally:
        gc.enable()
    ncell, ntotal, nact = g.ncell, len(P["orig"]), len(cells_h)
    h2d = (2 * ncell * 8 + ncell + ncell * 64 + ntotal * 8 + 8 * sum(len(x) for x in P["node_groups"])
           + P["loads"][0][0].size * 32 + nact * 8 + P["fixed"][0].size * 32 + P["extra"].node_coo()[4].size * 24)
    d2h = ntotal * 24 + nact * 13 * 8
    e2e_val = reduce_max(sum(e2e_s) / len(e2e_s), dist) / world
    # ---------------------------------------------------------------- roofline of the level-0 operator
    pk, pk_kind = peaks()
    roofline = ku_roofline(P, d, lib, engine, _lib, pk, pk_kind)
    # ---------------------------------------------------------------- CPU baseline and oracle parity (rank 0, N = 1)
    cpu = None
    parity_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        Ps = make_problem(0, SAMPLE_BIG)
        smp = cpu_oracle_run(SAMPLE_BIG, P=Ps)
        ds = device_inputs(Ps)
        parity_oracle = {"workload": (f"hindfoot {SAMPLE_BIG['nx']}x{SAMPLE_BIG['ny']}x{SAMPLE_BIG['nz']} "
                                      f"h={SAMPLE_BIG['h']} ({smp['ndof']} dofs, oracle {smp['iters']} iterations)")}
        for name, pr_, w_ in arms:
            Us, vms, _ = device_solve(Ps, ds, pr_, warm=w_)
            parity_oracle[name] = parity(Us.cpu().numpy(), vms.cpu().numpy(), smp["U"], smp["vm"])
        it_w = int(res["plain_fp64"]["info"].iters)
        est = extrapolate(smp, int(hinfo.ndof), it_w)
        cpu = {"value": round(est, 2), "unit": "s/solve", "cores": 1, "kind": "port",
               "sample": (f"oracle solve_cn + cell_stress (NumPy/SciPy, single-threaded sparse kernels) on hindfoot "
                          f"{SAMPLE_BIG['nx']}x{SAMPLE_BIG['ny']}x{SAMPLE_BIG['nz']} h={SAMPLE_BIG['h']}: {smp['ndof']} "
                          f"dofs, {smp['iters']} iterations, {smp['t']:.1f} s (assembly {smp['t_assemble']:.1f}, "
                          f"multigrid set-up {smp['t_setup']:.1f}, PCG {smp['t_pcg']:.1f}, stress "
                          f"{smp['t_stress']:.1f}); set-up and stress scaled by dofs, PCG by dofs x iterations to "
                          f"{int(hinfo.ndof)} dofs and {it_w} iterations (the FP64 solve's count on the workload)")}
    if args.cpu_full and rank == 0:
        full = cpu_oracle_run(WORKLOAD, P=P)
        cpu_full = {"s_per_solve": round(full["t"], 2), "iters": full["iters"], "ndof": full["ndof"],
                    "phases_s": {k: round(full[k], 2) for k in ("t_assemble", "t_setup", "t_pcg", "t_stress")},
                    "cores": 1}
        parity_full = {k: parity(v["U"], v["vm"].cpu().numpy(), full["U"], full["vm"]) for k, v in res.items()}
    else:
        cpu_full = parity_full = None
    return dict(
        metric=METRIC, value=round(value, 5), unit="s/solve", n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=round(1e3 * t_total / args.steps, 3), higher_is_better=False, scaling="weak", vs_baseline=None,
        dtype=("f32 inner / f64 refinement" if prec == "refine" else
               ("f64" if prec == "fp64" else "f64 CG / f32 V-cycle")),
        data="synthetic (seeded hindfoot generator)",
        config={"workload": (f"hindfoot {WORKLOAD['nx']}x{WORKLOAD['ny']}x{WORKLOAD['nz']} h={WORKLOAD['h']}mm "
                             f"(C2 generator)"), "ndof": int(hinfo.ndof), "precision": prec,
                "warm_start": ("learned (packaged network), prediction inside the step" if warm is not None
                               else "zero (no trained network found)"),
                "tol": TOL, "iters": int(hinfo.iters), "sweeps": int(hinfo.sweeps), "relres": hinfo.relres,
                "levels": int(hinfo.levels), "ku_kernel": ["per-cell", "paired-row", "tensor-core"][int(hinfo.ku_kind)],
                "coarse_stencils": ("f64" if prec == "fp64" else
                                    "f32" if SOLVER_OPTIONS.get("level_kernel", 0) & 8 else "f16 scaled, f32 sums"),
                "l2": "flushed (256 MB write) before every step", "parallelism": f"independent solves x{world}"},
        arms_s_per_solve={k: round(v, 5) for k, v in mean_s.items()},
        arms_step_ms={k: [round(x, 2) for x in v["ms"]] for k, v in res.items()},
        arms_step_setup_solve_iters=step_info,
        arms_iters={k: int(v["info"].iters) for k, v in res.items()},
        plain_fp64={"s_per_solve": round(mean_s["plain_fp64"], 5), "iters": int(res["plain_fp64"]["info"].iters),
                    "relres": res["plain_fp64"]["info"].relres},
        speedup_vs_plain_fp64=round(mean_s["plain_fp64"] / value, 3) if world == 1 else None,
        learned_warm_start=learned, parity_vs_fp64=par64, parity_vs_oracle=parity_oracle,
        cpu_full=cpu_full, parity_vs_oracle_full=parity_full,
        stage_ms={"setup": round(hinfo.t_setup_ms, 3), "solve": round(hinfo.t_solve_ms, 3),
                  "setup_stages": dict(zip(SETUP_STAGES, (round(float(v), 3) for v in hinfo.t_stage_ms)))},
        e2e={"value": round(e2e_val, 5), "unit": "s/solve", "h2d_bytes_per_step": int(h2d),
             "d2h_bytes_per_step": int(d2h), "iters": int(infe["iters"]), "relres": infe["relres"],
             "t_host": infe["t_host"], "steps_s": [round(t, 4) for t in e2e_s]},
        roofline=roofline, cpu_baseline=cpu, gpu_launches=int(launches), clocks=clk_summary,
    )


def run_profile(args):
    """Profiling workloads: one device solve (solve-once) or 3 FP32 + 3 FP64 K.u products (ku)."""
    import ctypes as C
    import torch
    from comech_b200 import engine, _lib
    P = make_problem(seed=0)
    d = device_inputs(P)
    if args.mode == "solve-once":
        warm = None
        if args.warm != "off":
            from comech_b200 import warmnet
            try:
                warm = warmnet.default_net()
            except RuntimeError:
                if args.warm == "on":
                    raise
        for _ in range(args.warmup):
            device_solve(P, d, args.precision, warm=warm)
        U, vm, info = device_solve(P, d, args.precision, warm=warm)
        torch.cuda.synchronize()
        return {"mode": "solve-once", "precision": args.precision, "options": SOLVER_OPTIONS,
                "warm_start": warm is not None, "x0_used": int(info.x0_used), "iters": int(info.iters),
                "sweeps": int(info.sweeps), "relres": info.relres, "t_setup_ms": round(info.t_setup_ms, 2),
                "t_solve_ms": round(info.t_solve_ms, 2), "ndof": int(info.ndof), "ku_shape": list(info.ku_shape),
                "t_stage_ms": [round(float(v), 2) for v in info.t_stage_ms],
                "lmax": [round(float(v), 6) for v in info.lmax[:max(int(info.levels) - 1, 0)]],
                "level_dofs": [int(v) for v in info.level_dofs[:int(info.levels)]]}
    pr = engine.Problem(P["grid"], _lib.MAT_ISO_SRI, d["mat"], d["active"], cn=d["cn"], orig=d["orig"],
                        pen_node=d["pen_node"], pen_k=d["pen_k"], extra_coo=d["extra"], options=dict(max_levels=0))
    if args.mode == "ku-rot":
        pr.close()
        pk, pk_kind = peaks()
        return {"mode": "ku-rot", "pair_config": os.environ.get("FEB_PAIR_CONFIG"),
                "roofline": ku_roofline(P, d, _lib.load(), engine, _lib, pk, pk_kind)}
    out = {"mode": "ku"}
    try:
        ntotal = len(P["orig"])
        for name, dt, prec in (("fp32", torch.float32, 1), ("fp64", torch.float64, 0)):
            u = torch.randn(3 * ntotal, dtype=dt, device="cuda")
            y = torch.empty_like(u)
            ms = C.c_float()
            _lib.check(_lib.load().feb_benchmark_apply(pr.h, prec, C.c_void_p(u.data_ptr()), C.c_void_p(y.data_ptr()),
                                                       3, C.byref(ms)))
            out[name + "_ms"] = ms.value
    finally:
        pr.close()
    return out


BATCH_ACTIONS = ("resection", "osteotomy", "interposition", "fusion", "load")


def batch_instance(seed):
    """One batch instance: a grid drawn from the seed between 64x48x40 and 128x96x80 cells over an 80-mm-long box,
    one surgical action (runs in a worker process; no CUDA)."""
    from comech_b200 import synth
    rng = np.random.default_rng(10_000 + seed)
    f = rng.uniform(0.0, 1.0)
    nx, ny, nz = (int(round(a + f * (b - a))) for a, b in ((64, 128), (48, 96), (40, 80)))
    P = synth.hindfoot_problem(nx, ny, nz, h=80.0 / nx, seed=seed, action=BATCH_ACTIONS[seed % 5])
    for k in ("bone_share", "E", "nu", "part", "bridge", "contact"):
        P.pop(k, None)
    return P


def run_batch(args):
    """64 independent instances of uneven size and seeded action on one GPU: the host thread pool (1, 8 and 16
    whole solve_cn calls in flight) against the batched launch (comech_b200.batch mode "graph": set-up on 16
    threads, one feb_solve_batch graph launch per chunk of 16 instances while the next chunks are being set up,
    then the downloads).  Times are
    wall-clock around the whole batch through the public API (host inputs, uploads, set-up, solves, downloads),
    after one warm-up pass."""
    import multiprocessing as mp
    n = args.batch_n
    with mp.get_context("spawn").Pool(max(1, min(16, (os.cpu_count() or 2) - 1))) as pool:
        items = pool.map(batch_instance, range(n))
    import torch
    from comech_b200 import batch
    batch.solve_batch(items[:4], precision=args.precision, tol=TOL, concurrency=4, mode="threads")   # warm-up
    batch.solve_batch(items[:4], precision=args.precision, tol=TOL, concurrency=4, mode="graph")
    out = {"mode": "batch", "instances": n, "precision": args.precision, "tol": TOL,
           "dims": sorted({(P["grid"].nx, P["grid"].ny, P["grid"].nz) for P in items})[:: max(1, n // 8)],
           "actions": list(BATCH_ACTIONS)}
    runs = {}
    for name, mode, conc in (("threads_1", "threads", 1), ("threads_8", "threads", 8), ("threads_16", "threads", 16),
                             ("graph", "graph", 16)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = batch.solve_batch(items, precision=args.precision, tol=TOL, concurrency=conc, mode=mode)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        runs[name] = dict(seconds=round(dt, 3), solves_per_s=round(n / dt, 2),
                          iters_median=float(np.median([r[1]["iters"] for r in res])),
                          relres_max=float(max(r[1]["relres"] for r in res)),
                          flags=sorted({int(r[1]["flag"]) for r in res}))
        if mode == "graph":
            runs[name]["phases_s"] = res[0][1]["batch"]
    out["ndof_total"] = int(sum(r[1]["ndof"] for r in res))
    out["runs"] = runs
    out["speedup_threads16_vs_1"] = round(runs["threads_1"]["seconds"] / runs["threads_16"]["seconds"], 2)
    out["speedup_graph_vs_threads16"] = round(runs["threads_16"]["seconds"] / runs["graph"]["seconds"], 2)
    return out


LABEL_BENCH_CASES = [
    ("plain foot", {}, {}),
    ("coalition R2, resection", dict(ctype="I", rtype="R2", cov_mid=0.4), dict(resect=1, d_post=0.25)),
    ("warps, valgus, osteotomy", dict(sust_y=14.0, post_dome=3.0, align=6.0), dict(osteo=5.0)),
]


def run_labels(args):
    """Voxel labelling of the FE lattice (rb/rbgeom.py:493-524) on the seeded synthetic template: a 160 x 112 x 96
    lattice at 0.5 mm over the hindfoot, for a plain foot, a coalition with its resection, and warps with a valgus
    shear and an osteotomy.  Device: labels.label_lattice from host lattice axes to host labels (template already
    on the device), median of 5 after a warm-up; CPU: the oracle's label_lattice, one run each; the labels are
    compared."""
    import torch
    from comech_b200 import labels as LB, synth
    from oracle import label_oracle as LO
    T = synth.synthetic_template(0)
    D = LB.DeviceTemplate(T)
    sx = -100.0 + 0.5 * np.arange(160) + 0.13
    sy = -28.0 + 0.5 * np.arange(112) + 0.21
    sz = 20.0 + 0.5 * np.arange(96) + 0.07
    rows, plain = [], None
    for name, fk, ak in LABEL_BENCH_CASES:
        foot, act = LB.Foot(**fk), LB.Action(**ak)
        LB.label_lattice(sx, sy, sz, foot, act, device_template=D)
        ts = []
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Ld = LB.label_lattice(sx, sy, sz, foot, act, device_template=D)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        Lo = LO.label_lattice(sx, sy, sz, foot, act, T)
        tc = time.perf_counter() - t0
        if plain is None:
            plain = Lo
        dev = float(np.median(ts))
        rows.append(dict(case=name, device_ms=round(1e3 * dev, 3), cpu_s=round(tc, 3), speedup=round(tc / dev, 1),
                         mismatches=int((Ld != Lo).sum()), edited_vs_plain=int((Lo != plain).sum())))
    return {"mode": "labels", "lattice": [len(sx), len(sy), len(sz)], "points": int(len(sx) * len(sy) * len(sz)),
            "cases": rows}


def run_post(args):
    """The rows around the solve on the workload: region forces, rigid fit, relative displacement, resampling on a
    2-mm analysis grid, split connectivity and material mixing.  Device: the public calls from host arrays (inputs
    uploaded and results downloaded inside the timed region), median of 5 after one warm-up; CPU: the oracle on
    the same inputs, one run each."""
    import torch
    from comech_b200 import _lib, engine, materials as MX, post
    from comech_b200.grid import Grid
    from comech_b200.split import split_connectivity_device
    from oracle import fe_oracle as O
    P = make_problem(0)
    g = P["grid"]
    d = device_inputs(P)
    U, _, _ = device_solve(P, d, "mixed")
    sig, vm, _ = engine._stress(g, _lib.MAT_ISO_SRI, d["mat"], U, d["cells"], d["cn"], True, to_host=True)
    Uh = U.view(-1, 3).cpu().numpy()
    cells = np.flatnonzero(P["active"])
    VM = np.zeros(g.ncell, np.float32); VM[cells] = vm
    SIG = np.zeros((g.ncell, 6), np.float32); SIG[cells] = sig
    rng = np.random.default_rng(5)
    lab = rng.integers(0, 7, g.ncell).astype(np.int32)
    part = P["part"].astype(np.int32)
    og = O.OGrid(g.xe, g.ye, g.ze)
    xyz = og.node_xyz[P["orig"]]
    nodes = np.unique(P["cn"][cells[part[cells] == 1]].ravel())
    gm = Grid(np.arange(g.xe[0] - 4.0, g.xe[-1] + 4.01, 2.0), np.arange(g.ye[0] - 4.0, g.ye[-1] + 4.01, 2.0),
              np.arange(g.ze[0] - 4.0, g.ze[-1] + 4.01, 2.0))
    ogm = O.OGrid(gm.xe, gm.ye, gm.ze)
    t, w, c = O.rigid_fit(xyz[nodes], np.nan_to_num(Uh[nodes]))
    Urel = O.relative_displacement(xyz, Uh, t, w, c)
    o = dict(g=g, cn=P["cn"], active=P["active"], VM=VM, SIG=SIG)
    # sub-voxel body labels (3^3 per cell): the cell's bone (cortical body of its part), soft tissue in joint
    # cells, void outside; a fifth of the sub-voxels take the label of a neighbouring cell
    body_of_part = np.array([63, 1, 2, 40, 43, 3, 4])
    base = np.where(P["active"], body_of_part[np.clip(part, 0, 6)], 0)
    nbr = np.clip(np.arange(g.ncell)[:, None] + rng.integers(-1, 2, (g.ncell, 27)), 0, g.ncell - 1)
    L = np.where(rng.random((g.ncell, 27)) < 0.2, base[nbr], base[:, None]).astype(np.int32)
    cls = {1: 1, 53: 2, 2: 1, 52: 2, 40: 1, 45: 2, 43: 1, 49: 2, 3: 1, 54: 2, 4: 1, 13: 2, 63: 5}
    roles = {"bones": {"calcaneus": (1, 53), "talus": (2, 52), "fibula": (3, 54), "tibia": (4, 13),
                       "navicular": (40, 45), "cuboid": (43, 49)}, "bonded_extra": [101, 104]}
    V = dict(cls={str(k): v for k, v in cls.items()}, L=L, xe=g.xe, ye=g.ye, ze=g.ze)
    groups, _ = MX.bone_groups(cls, roles)
    steps = {
        "region_forces_2_bones": (lambda: [post.region_forces_cn(g, P["lam"], P["mu"], Uh, P["cn"], P["active"], part,
                                                                 lab, 7, k) for k in (1, 2)],
                                  lambda: [O.region_forces(og, P["lam"], P["mu"], Uh, P["cn"], P["active"], part, lab,
                                                           7, k) for k in (1, 2)]),
        "rigid_fit": (lambda: post.rigid_fit(xyz[nodes], np.nan_to_num(Uh[nodes])),
                      lambda: O.rigid_fit(xyz[nodes], np.nan_to_num(Uh[nodes]))),
        "relative_displacement": (lambda: post.relative_displacement(g, P["orig"], Uh, t, w, c),
                                  lambda: O.relative_displacement(xyz, Uh, t, w, c)),
        "sample_fe": (lambda: post.sample_fe(o, gm, Urel),
                      lambda: O.sample_fe(og, P["cn"], P["active"], VM, SIG, Urel, (gm.xe, gm.ye, gm.ze))),
        "sample_nodes": (lambda: post.sample_nodes(o, gm, Urel),
                         lambda: O.sample_nodes(og, P["cn"], P["active"], Urel, ogm.node_xyz)),
        "split_connectivity": (lambda: split_connectivity_device(g, P["active"], part, P["bone_share"]),
                               lambda: O.split_connectivity(og, P["active"], part, P["bone_share"])),
        "material_mixing": (lambda: MX.materials(V, roles),
                            lambda: O.mix_materials(cls, L, (g.nx, g.ny, g.nz), groups)),
    }
    gpu_ms, cpu_s = {}, {}
    for name, (dev_fn, cpu_fn) in steps.items():
        dev_fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            dev_fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        gpu_ms[name] = round(1e3 * statistics.median(ts), 3)
        t0 = time.perf_counter()
        cpu_fn()
        cpu_s[name] = round(time.perf_counter() - t0, 3)
    return {"mode": "post", "workload": f"hindfoot {g.nx}x{g.ny}x{g.nz}, analysis grid {gm.nx}x{gm.ny}x{gm.nz} (2 mm)",
            "gpu_e2e_ms": gpu_ms, "cpu_oracle_s": cpu_s,
            "speedup": {k: round(cpu_s[k] * 1e3 / max(gpu_ms[k], 1e-6), 1) for k in gpu_ms}}


def run_reference(args, rank, world):
    """The reference's CPU path (the oracle: a NumPy/SciPy restatement of rb/splitfe.solve_cn + cell_stress_cn with
    the reference's GMG-PCG; the reference is pure Python, so this is the implementation being replaced) timed on
    this host.  Its 5M-dof solve takes minutes, so the --steps x --warmup protocol cannot time the full
    configuration: each step is a bounded sample of the same generator, timed by phase and extrapolated to the
    workload (assembly, multigrid set-up and stress by dofs; PCG by dofs x iterations, with the workload's
    iteration count measured once on a mid-size sample and scaled by the measured growth with size)."""
    if rank != 0:
        return None
    dims = SAMPLE_BIG if args.steps <= 4 else SAMPLE_SMALL
    for _ in range(args.warmup):
        cpu_oracle_run(SAMPLE_SMALL)
    runs = [cpu_oracle_run(dims) for _ in range(args.steps)]
    full_ndof = workload_ndof()
    full_iters = ORACLE_FULL_ITERS
    est = [extrapolate(r, full_ndof, full_iters) for r in runs]
    value = float(np.mean(est))
    r0 = runs[0]
    desc = (f"oracle solve_cn + cell_stress (NumPy/SciPy, single-threaded sparse kernels) on hindfoot "
            f"{dims['nx']}x{dims['ny']}x{dims['nz']} h={dims['h']} ({r0['ndof']} dofs, {r0['iters']} iterations, "
            f"{r0['t']:.1f} s: assembly {r0['t_assemble']:.1f}, set-up {r0['t_setup']:.1f}, PCG {r0['t_pcg']:.1f}, "
            f"stress {r0['t_stress']:.1f}), mean of {len(runs)} steps, each extrapolated to {full_ndof} dofs and "
            f"{full_iters} iterations (set-up phases by dofs, PCG by dofs x iterations; the oracle's own count on the "
            f"full workload, measured with --cpu-full, where the whole solve took {ORACLE_FULL_S} s); the full solve "
            f"takes minutes, which the steps x warm-up protocol cannot time")
    return dict(metric=METRIC, value=round(value, 3), unit="s/solve", n_gpus=world, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(1e3 * float(np.mean([r["t"] for r in runs])), 1),
                higher_is_better=False, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic (seeded hindfoot generator)",
                config={"workload": (f"hindfoot {WORKLOAD['nx']}x{WORKLOAD['ny']}x{WORKLOAD['nz']} h={WORKLOAD['h']}mm "
                                     f"(C2 generator)"), "tol": TOL, "parallelism": "CPU, 1 process",
                        "same_config": False, "extrapolated_iters": full_iters},
                impl="reference",
                cpu_baseline={"value": round(value, 3), "unit": "s/solve", "cores": 1, "kind": "port", "sample": desc},
                e2e={"value": round(value, 3), "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed", "refine"], default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-full", action="store_true",
                    help="also run the CPU oracle on the full workload (minutes): true CPU time and parity at full size")
    ap.add_argument("--mode", choices=["full", "solve-once", "ku", "ku-rot", "post", "batch", "labels"], default="full",
                    help="solve-once / ku: one device solve or a few K.u products of the workload (profiling); "
                         "post: the rows around the solve, device against the CPU oracle; batch: 64 uneven "
                         "instances with seeded actions, one at a time and 8 / 16 in flight")
    ap.add_argument("--batch-n", type=int, default=64)
    ap.add_argument("--size", default=None, help="override the workload grid, e.g. 96x64x56x0.833 (profiling)")
    ap.add_argument("--inner-tol", type=float, default=None, help="refinement: FP32 sweep tolerance")
    ap.add_argument("--use-graphs", type=int, default=None, help="0 direct, 1 graph per iteration, 2 device loop")
    ap.add_argument("--level-kernel", type=int, default=None,
                    help="coarse-level stencil slots: 0 auto, 1 run-time slot index, 2 compile-time slot index; "
                         "+4 term-dot passes; +8 FP32 stencil copies instead of FP16")
    ap.add_argument("--warm", choices=["auto", "on", "off"], default="auto",
                    help="learned warm start (auto: when the packaged network is present)")
    args = ap.parse_args()
    if args.inner_tol is not None:
        SOLVER_OPTIONS["inner_tol"] = args.inner_tol
    if args.use_graphs is not None:
        SOLVER_OPTIONS["use_graphs"] = args.use_graphs
    if args.level_kernel is not None:
        SOLVER_OPTIONS["level_kernel"] = args.level_kernel
    if args.size:
        nx, ny, nz, h = args.size.split("x")
        WORKLOAD.update(nx=int(nx), ny=int(ny), nz=int(nz), h=float(h))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.mode == "batch":
        out = run_batch(args)                     # the instance pool starts before the first CUDA call
    else:
        import torch
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        if world > 1:
            import datetime
            import torch.distributed as tdist
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                     device_id=torch.device("cuda", local))
            dist = tdist
        if args.mode == "full":
            out = run_ours(args, rank, world, dist)
        elif args.mode == "post":
            out = run_post(args)
        elif args.mode == "labels":
            out = run_labels(args)
        else:
            out = run_profile(args)
        if dist:
            dist.destroy_process_group()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
