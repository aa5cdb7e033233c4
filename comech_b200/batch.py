"""Batched solves of many independent instances (feet x surgical actions, uneven grids) on one GPU.

The reference solves a bank of (foot, action) instances one per process (exp/rb_run_engine_v4.py:123-135), each
``solve_cn`` alone on its device.  Small instances leave a B200 mostly idle: their coarse multigrid levels are a
few thousand nodes and every CG iteration is a chain of short launches.  Here ``concurrency`` host threads each
drive their own solver handle (own non-blocking stream, own CUDA graph per CG iteration, K.u launch shape from the
autotuner, cached per grid shape) and their own torch stream, so the iterations of up to ``concurrency`` instances
run on the GPU at the same time.  ctypes releases the interpreter lock inside every library call, so the host
threads do not serialise.

``solve_batch(items)`` returns, in input order, the ``engine.solve_cn`` results of every item.
"""
import threading
import time
from concurrent.futures import ThreadPoolExecutor

from . import engine
from .engine import _torch


def solve_batch(items, precision="mixed", tol=1e-8, maxiter=800, warm_start=None, concurrency=8):
    """Solve every item (a dict of ``solve_cn``'s inputs: grid, lam, mu, active, cn, orig, fixed, loads, extra,
    node_groups) with up to ``concurrency`` solves in flight on the GPU.  Returns [(U, info, R)] in input order;
    info["t_item"] is the wall time of the item's solve."""
    torch = _torch()
    torch.cuda.synchronize()
    local = threading.local()

    def run(item):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        with torch.cuda.stream(local.stream):
            t0 = time.perf_counter()
            out = engine.solve_cn(item["grid"], item["lam"], item["mu"], item["active"], item["cn"], item["orig"],
                                  item["fixed"], item["loads"], item.get("extra"), item.get("node_groups"), tol=tol,
                                  maxiter=maxiter, precision=precision, warm_start=warm_start)
            local.stream.synchronize()
            out[1]["t_item"] = time.perf_counter() - t0
            return out

    if concurrency <= 1:
        return [run(it) for it in items]
    with ThreadPoolExecutor(max_workers=concurrency) as ex:
        return list(ex.map(run, items))
