"""Second build stage: the C++ layer that keeps the reference's names.

Compiles, with the host C++ compiler against libstt.so and the CUDA runtime,

* ``spacetimetomography_b200/libstt_facade.so`` -- csrc/facade/*.cpp except the
  command line: the host-pointer C entry points of include/stt_host.h, the
  TIFF / Analyze codec and the classes of include/reference/ (VolumeData,
  TypicalRayProducer, ST_Tomography, ...);
* ``spacetimetomography_b200/bin/st_tomography`` -- the ST-Tomography command
  line (csrc/facade/st_tomography_main.cpp).

Called by build.py when csrc/facade exists; outputs stay inside the package.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
FACADE = PKG / "csrc" / "facade"
INCLUDE = ROOT / "include"
LIB = PKG / "libstt.so"
FACADE_LIB = PKG / "libstt_facade.so"
CLI = PKG / "bin" / "st_tomography"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
LIB_SOURCES = ["host_api.cpp", "host_solver.cpp", "tiff_io.cpp", "reference_api.cpp"]
CLI_SOURCES = ["st_tomography_main.cpp"]


def _cxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def _flags() -> list[str]:
    return ["-std=c++17", "-O2", "-fPIC", "-Wall", f"-I{INCLUDE}", f"-I{INCLUDE / 'reference'}",
            f"-I{CUDA / 'include'}"]


def _links(rpath_pkg: str) -> list[str]:
    return [f"-L{PKG}", f"-L{CUDA / 'lib64'}", "-lstt", "-lcudart", f"-Wl,-rpath,{rpath_pkg}",
            f"-Wl,-rpath,{CUDA / 'lib64'}"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> None:
    headers = list(INCLUDE.glob("*.h")) + list((INCLUDE / "reference").glob("*.h"))
    lib_srcs = [FACADE / s for s in LIB_SOURCES]
    if force or _stale(FACADE_LIB, lib_srcs + headers + [LIB]):
        cmd = [_cxx(), *_flags(), "-shared", "-o", str(FACADE_LIB), *map(str, lib_srcs), *_links("$ORIGIN")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    cli_srcs = [FACADE / s for s in CLI_SOURCES]
    if force or _stale(CLI, cli_srcs + headers + [FACADE_LIB]):
        CLI.parent.mkdir(exist_ok=True)
        cmd = [_cxx(), *_flags(), "-o", str(CLI), *map(str, cli_srcs), "-lstt_facade",
               *_links("$ORIGIN/..")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
