"""Build libfeb200.so in-tree with nvcc for sm_100a (no torch extension machinery, no JIT cache).

    python -m comech_b200.build            # incremental
    python -m comech_b200.build --force    # rebuild everything
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfeb200.so")
SOURCES = ["fine.cu", "fine_pair.cu", "fine_tc.cu", "coarse.cu", "vec.cu", "dense.cu", "rigid.cu", "stress.cu", "post.cu", "split.cu", "materials.cu", "net.cu", "labels.cu", "solver.cu"]
# per-file flags: the labelling kernel rounds every product and sum on its own, like NumPy's elementwise operations
FILE_FLAGS = {"labels.cu": ["-fmad=false"]}
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-diag-suppress", "177"]


def _deps(src):
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(os.path.dirname(HERE), "include", "feb200.h"))
    return [os.path.join(CSRC, src)] + hdrs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, force, extra):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    if not force and not _stale(obj, _deps(src)):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(src, []) + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    extra = list(extra)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, extra), SOURCES))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, verbose=True)
    sys.exit(0)
