"""In-tree build of libstt.so (CUDA, sm_100a) and the C++ drop-in layer.

``python spacetimetomography_b200/build.py [--force]`` compiles

* ``spacetimetomography_b200/libstt.so``  -- kernels + the C ABI of include/stt.h
* ``spacetimetomography_b200/libstt_facade.so`` and ``bin/st_tomography`` -- the
  C++ classes and command line that keep the reference's names (built only when
  their sources exist)

with nvcc for ``arch=compute_100a,code=sm_100a``.  Outputs stay inside the
package directory so they travel with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libstt.so"

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]

KERNEL_SOURCES = ["stt_capi.cu", "stt_solver.cu", "stt_batch.cu", "stt_noalloc.cu", "stt_flow.cu", "stt_tune.cu",
                  "k_project.cu",
                  "k_fp_slab.cu", "k_bp_slab.cu", "k_voxel.cu", "k_persist.cu", "k_warp.cu", "k_flow.cu"]
# Per-file flags.  The optical-flow kernels keep the reference's float
# rounding operation by operation, so no multiply-add contraction there.
FILE_FLAGS = {"k_flow.cu": ["-fmad=false"]}
OBJ_DIR = PKG / "_build"


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: libstt.so cannot be built")
    return found


def _host_compiler() -> list[str]:
    # The image exports CXX=/opt/gcc/bin/g++; nvcc is pinned to the system g++.
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if Path(gxx).exists() else []


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str], verbose: bool) -> None:
    cmd = [_nvcc(), *GENCODE, *NVCC_FLAGS, *_host_compiler(), *FILE_FLAGS.get(src.name, []), "-c",
           f"-I{INCLUDE}", f"-I{CSRC}", "-o", str(obj), str(src), *extra]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build_libstt(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles every kernel source to an object (in parallel) and links libstt.so."""
    from concurrent.futures import ThreadPoolExecutor

    extra = list(extra or [])
    srcs = [CSRC / s for s in KERNEL_SOURCES]
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "stt.h"]
    if not force and not _stale(LIB, srcs + headers):
        return LIB
    OBJ_DIR.mkdir(exist_ok=True)
    objs = [OBJ_DIR / (s.stem + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or extra or _stale(o, [s] + headers)]
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        for fut in [pool.submit(_compile, s, o, extra, verbose) for s, o in todo]:
            fut.result()
    cmd = [_nvcc(), *GENCODE, *_host_compiler(), "-shared", "-o", str(LIB), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_libstt(force=force, verbose=verbose)
    facade = CSRC / "facade"
    if facade.exists():
        import importlib.util

        spec = importlib.util.spec_from_file_location("stt_build_facade", PKG / "build_facade.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build(force=force, verbose=verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
