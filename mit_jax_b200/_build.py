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


FFI_SRC = HERE / "csrc" / "cg2d_ffi.cc"
FFI_OUT = HERE / "libcg2d_ffi.so"


def jax_ffi_include():
    """jaxlib's XLA FFI header directory, or None where jax is not installed (then the FFI handlers are not built)."""
    try:
        import jax.ffi
        d = Path(jax.ffi.include_dir())
    except Exception:
        return None
    return d if (d / "xla" / "ffi" / "api" / "ffi.h").exists() else None


def build_ffi(force=False):
    """libcg2d_ffi.so: the XLA FFI handlers of csrc/cg2d_ffi.cc over libcg2d.so (host code only). Skipped, returning
    None, where jax.ffi's headers are absent."""
    inc = jax_ffi_include()
    if inc is None:
        return None
    deps = [FFI_SRC, OUT, HERE.parent / "include" / "cg2d.h"]
    if not force and FFI_OUT.exists() and all(FFI_OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return FFI_OUT
    cuda_inc = Path(nvcc()).resolve().parent.parent / "include"
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-shared", "-fPIC", f"-I{inc}", f"-I{cuda_inc}",
           f"-I{HERE.parent / 'include'}", str(FFI_SRC), f"-L{HERE}", "-lcg2d", "-Wl,-rpath,$ORIGIN",
           "-o", str(FFI_OUT) + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(str(FFI_OUT) + ".tmp", FFI_OUT)
    return FFI_OUT


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
    print(build_ffi(force="--force" in sys.argv) or "libcg2d_ffi.so not built: jax.ffi headers absent")
