"""Compile the native library ``_native/libem3d_b200.so`` for sm_100a with nvcc."""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
NATIVE = os.path.join(HERE, "_native")
LIB = os.path.join(NATIVE, "libem3d_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def _run(cmd):
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return proc.stderr


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every ``csrc/*.cu`` (one object each, in parallel; without
    ``force`` only those older than their source or a header) and link them
    into one shared library; returns its path."""
    from concurrent.futures import ThreadPoolExecutor

    if not force and not needs_build():
        return LIB
    os.makedirs(NATIVE, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(NATIVE, "obj")
    os.makedirs(objdir, exist_ok=True)
    jobs = []
    # without force, an object newer than its source and every header is kept
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    newest_header = max((os.path.getmtime(h) for h in headers), default=0.0)
    for src in sources():
        obj = os.path.join(objdir, os.path.splitext(os.path.basename(src))[0] + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        fresh = (not force and os.path.exists(obj)
                 and os.path.getmtime(obj) > max(os.path.getmtime(src), newest_header))
        jobs.append((cmd, obj, fresh))
    todo = [j for j in jobs if not j[2]]
    workers = max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as pool:
        logs = list(pool.map(lambda j: _run(j[0]), todo))
    if verbose:
        for (cmd, _, _), log in zip(todo, logs):
            print(" ".join(cmd))
            if log:
                print(log)
    tmp = LIB + ".tmp"
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *[o for _, o, _ in jobs]])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force=True))
