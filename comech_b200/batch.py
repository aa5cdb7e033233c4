"""Batched solves of many independent instances (feet x surgical actions, uneven grids) on one GPU.

The reference solves a bank of (foot, action) instances one per process (exp/rb_run_engine_v4.py:113-147), each
``solve_cn`` alone on its device.  Small instances leave a B200 mostly idle: their coarse multigrid levels are a
few thousand nodes and every CG iteration is a chain of short launches.

``solve_batch(items)`` (mode "graph", the default) runs in three phases:
  1. set-up: ``concurrency`` host threads build the instances' operators and hierarchies (engine.prepare_cn: one
     solver handle each, own non-blocking stream, K.u launch shape from the autotuner, cached per grid shape);
  2. solve: ONE ``feb_solve_batch`` call, i.e. one CUDA graph launch holding every instance's CG as a device-side
     while loop with its own convergence flag, so all instances iterate concurrently with no host round trip;
  3. finish: U and reactions per instance (engine.finish_cn), again on the threads.
Instances are solved ``chunk`` at a time (default: all) to bound device memory.  Mode "threads" keeps the
earlier scheme (each thread runs a whole ``solve_cn``; up to ``concurrency`` in flight).

Returns, in input order, the ``engine.solve_cn`` results (U, info, R) of every item; info["t_item"] is the
item's share of the wall time (phase times of its chunk), info["batch"] the chunk's phase times.
"""
import threading
import time
from concurrent.futures import ThreadPoolExecutor

from . import engine
from .engine import _torch


def _args(item):
    return (item["grid"], item["lam"], item["mu"], item["active"], item["cn"], item["orig"], item["fixed"],
            item["loads"], item.get("extra"), item.get("node_groups"))


def solve_batch(items, precision="mixed", tol=1e-8, maxiter=800, warm_start=None, concurrency=8, mode="graph",
                chunk=None, options=None):
    """Solve every item (a dict of ``solve_cn``'s inputs: grid, lam, mu, active, cn, orig, fixed, loads, extra,
    node_groups).  mode "graph": one batched device launch per chunk (a given ``warm_start`` network predicts
    each start, used as given); "threads": ``concurrency`` concurrent ``solve_cn`` calls."""
    torch = _torch()
    torch.cuda.synchronize()
    if mode == "threads":
        return _solve_threads(items, precision, tol, maxiter, warm_start, concurrency, options)
    if mode != "graph":
        raise ValueError(f"unknown batch mode {mode!r}")
    if precision == "refine":
        raise ValueError("the batched graph solve runs the fp64 and mixed precisions (refine: mode='threads')")
    chunk = len(items) if not chunk else int(chunk)
    out = [None] * len(items)
    for c0 in range(0, len(items), chunk):
        idx = list(range(c0, min(c0 + chunk, len(items))))
        for i, res in zip(idx, _solve_chunk([items[i] for i in idx], precision, tol, maxiter, warm_start,
                                            concurrency, options)):
            out[i] = res
    return out


def _solve_chunk(items, precision, tol, maxiter, warm_start, concurrency, options):
    torch = _torch()
    local = threading.local()

    def on_stream(fn):
        def run(*a):
            if not hasattr(local, "stream"):
                local.stream = torch.cuda.Stream()
            with torch.cuda.stream(local.stream):
                r = fn(*a)
                local.stream.synchronize()
                return r
        return run

    def prep(item):
        return engine.prepare_cn(*_args(item), tol=tol, maxiter=maxiter, precision=precision,
                                 warm_start=warm_start, options=options)

    t0 = time.perf_counter()
    ctxs = []
    try:
        with ThreadPoolExecutor(max_workers=max(1, concurrency)) as ex:
            futs = [ex.submit(on_stream(prep), it) for it in items]
            for fu in futs:          # keep every created context so that a failure closes them all
                ctxs.append(fu.result())
        t1 = time.perf_counter()
        torch.cuda.synchronize()
        res = engine.solve_batch_device([c["P"] for c in ctxs], [c["f"] for c in ctxs],
                                        [c["x0"] for c in ctxs] if any(c["x0"] is not None for c in ctxs) else None)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        for c in ctxs:
            c["stamps"].append(("solve", t2))

        def fin(a):
            c, (x, info) = a
            return engine.finish_cn(c, x, info)

        with ThreadPoolExecutor(max_workers=max(1, concurrency)) as ex:
            outs = list(ex.map(on_stream(fin), zip(ctxs, res)))
        t3 = time.perf_counter()
        phases = dict(setup=round(t1 - t0, 4), solve=round(t2 - t1, 4), finish=round(t3 - t2, 4),
                      instances=len(items))
        for U, info, R in outs:
            info["batch"] = phases
            info["t_item"] = (t3 - t0) / len(items)
        return outs
    finally:
        for c in ctxs:
            c["P"].close()


def _solve_threads(items, precision, tol, maxiter, warm_start, concurrency, options):
    torch = _torch()
    local = threading.local()

    def run(item):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        with torch.cuda.stream(local.stream):
            t0 = time.perf_counter()
            out = engine.solve_cn(*_args(item), tol=tol, maxiter=maxiter, precision=precision,
                                  warm_start=warm_start, options=options)
            local.stream.synchronize()
            out[1]["t_item"] = time.perf_counter() - t0
            return out

    if concurrency <= 1:
        return [run(it) for it in items]
    with ThreadPoolExecutor(max_workers=concurrency) as ex:
        return list(ex.map(run, items))
