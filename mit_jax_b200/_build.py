"""Build libcg2d.so in-tree for sm_100a with nvcc (python -m mit_jax_b200._build)."""

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = [HERE / "csrc" / "cg2d_solver.cu", HERE / "csrc" / "cg2d_capi.cu", HERE / "csrc" / "cg2d_adjoint.cu",
           HERE / "csrc" / "cg2d_pressure.cu"]
OUT = HERE / "libcg2d.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC"]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def build(force=False, verbose=False):
    """Compile the translation units side by side into objects next to the library, then link libcg2d.so."""
    deps = SOURCES + [HERE / "csrc" / "cg2d_internal.cuh", HERE.parent / "include" / "cg2d.h"]
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    objs = [HERE / "csrc" / (src.stem + ".o") for src in SOURCES]
    procs = []
    for src, obj in zip(SOURCES, objs):
        cmd = [nvcc(), *NVCC_FLAGS, "-c", "-o", str(obj), str(src)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, pr in procs if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    subprocess.run([nvcc(), *NVCC_FLAGS, "-shared", "-o", str(OUT) + ".tmp", *map(str, objs)], check=True)
    os.replace(str(OUT) + ".tmp", OUT)
    for obj in objs:
        obj.unlink()
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
