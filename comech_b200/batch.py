"""Batched solves of many independent instances (feet x surgical actions, uneven grids) on one GPU.

The reference solves a bank of (foot, action) instances one per process (exp/rb_run_engine_v4.py:113-147), each
``solve_cn`` alone on its device.  Small instances leave a B200 mostly idle: their coarse multigrid levels are a
few thousand nodes and every CG iteration is a chain of short launches.

``solve_batch(items)`` (mode "graph", the default) runs in three phases per chunk of instances:
  1. set-up: ``concurrency`` host threads build the instances' operators and hierarchies (engine.prepare_cn: one
     solver handle each, own non-blocking stream, K.u launch shape from the autotuner, cached per grid shape);
  2. solve: ONE ``feb_solve_batch`` call, i.e. one CUDA graph launch holding every instance's CG as a device-side
     while loop with its own convergence flag, so the chunk's instances iterate concurrently with no host round
     trip;
  3. finish: U and reactions per instance (engine.finish_cn), on a second thread pool.
The chunks are pipelined: every instance's set-up is queued on the pool at the start, so while one chunk's
graph runs the next chunks are being set up (default chunk: a quarter of the items, at least 4; smaller chunks
overlap more of the host-bound set-up, larger ones solve more efficiently: on 64 uneven instances four launches
took 1.81 s where one took 1.32 s, while two chunks left 3.1 s of set-up before the first launch on a box with a
slower host), and each chunk's
handles are closed once it is finished, which also bounds device memory.  Mode "threads" keeps the earlier scheme
(each thread runs a whole ``solve_cn``; up to ``concurrency`` in flight).

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
    n = len(items)
    chunk = max(4, -(-n // 4)) if not chunk else int(chunk)
    return _solve_pipelined(items, precision, tol, maxiter, warm_start, concurrency, options, chunk)


def _solve_pipelined(items, precision, tol, maxiter, warm_start, concurrency, options, chunk):
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

    def fin(a):
        c, (x, info) = a
        try:
            return engine.finish_cn(c, x, info)
        finally:
            c["P"].close()

    n = len(items)
    chunks = [list(range(c0, min(c0 + chunk, n))) for c0 in range(0, n, chunk)]
    out = [None] * n
    t0 = time.perf_counter()
    t_setup = t_solve = 0.0
    futs = []
    handed = set()                 # ids of contexts given to fin (it closes them)
    try:
        with ThreadPoolExecutor(max_workers=max(1, concurrency)) as ex, \
                ThreadPoolExecutor(max_workers=max(1, min(concurrency, 8))) as fx:
            futs = [[ex.submit(on_stream(prep), items[i]) for i in idx] for idx in chunks]   # all set-ups queued
            fins = []
            for ci, idx in enumerate(chunks):
                ta = time.perf_counter()
                ctxs = [fu.result() for fu in futs[ci]]
                tb = time.perf_counter()
                # each set-up synchronised its own stream; the batch launch waits on every handle's stream
                res = engine.solve_batch_device([c["P"] for c in ctxs], [c["f"] for c in ctxs],
                                                [c["x0"] for c in ctxs] if any(c["x0"] is not None for c in ctxs)
                                                else None)
                tc = time.perf_counter()
                t_setup += tb - ta
                t_solve += tc - tb
                for c in ctxs:
                    c["stamps"].append(("solve", tc))
                for i, c, r in zip(idx, ctxs, res):
                    handed.add(id(c))
                    fins.append((i, fx.submit(on_stream(fin), (c, r))))
            for i, fu in fins:
                out[i] = fu.result()
        t3 = time.perf_counter()
    except BaseException:
        # the pools have shut down (every queued set-up ran): close whatever was created and not handed over
        for fl in futs:
            for fu in fl:
                if fu.done() and not fu.cancelled() and fu.exception() is None and id(fu.result()) not in handed:
                    fu.result()["P"].close()
        raise
    phases = dict(setup_wait=round(t_setup, 4), solve=round(t_solve, 4), total=round(t3 - t0, 4), instances=n,
                  chunks=len(chunks))
    for U, info, R in out:
        info["batch"] = phases
        info["t_item"] = (t3 - t0) / n
    return out


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
