"""Build recipe for the native library: every CUDA source under csrc/ compiled
for sm_100a with nvcc into one shared object, in-tree
(reformulation_b200/_lib/libreform_b200.so), with the C ABI of include/*.h.

Run as ``python -m reformulation_b200.build`` (or through
``__graft_entry__.build()``).  Incremental: a source newer than the library
triggers a rebuild of the whole library (the sources are few and nvcc runs per
file in parallel).

The file CLIs of cli/ (praq_solve_file, pria_solve_file: host C++ over the C
ABI) are linked against the library into the same folder, with an rpath to it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
LIB = OUT / "libreform_b200.so"
OBJ = OUT / "obj"
CLI_SRC = PKG / "cli"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-Xcompiler", "-Wall", f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the native library cannot be built")
    return exe


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + headers())


def _compile(src: Path, verbose: bool, objdir: Path = OBJ, extra: tuple = ()) -> Path:
    obj = objdir / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def cli_targets() -> list[tuple[Path, Path]]:
    return [(src, OUT / src.stem) for src in sorted(CLI_SRC.glob("*.cpp"))]


def build_cli(force: bool = False) -> list[Path]:
    """Link each cli/*.cpp against the library (host code only: g++)."""
    out = []
    cxx = shutil.which("g++") or "g++"
    for src, exe in cli_targets():
        deps = [src, LIB] + sorted((ROOT / "include").glob("*.h")) + sorted(CLI_SRC.glob("*.hpp"))
        if not force and exe.exists() and all(d.stat().st_mtime <= exe.stat().st_mtime for d in deps):
            out.append(exe)
            continue
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-Wextra", f"-I{ROOT / 'include'}", f"-I{CLI_SRC}",
               f"-I{CUDA_HOME / 'include'}",
               str(src), "-o", str(exe), f"-L{OUT}", "-lreform_b200", f"-L{CUDA_HOME / 'lib64'}", "-lcudart",
               "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{CUDA_HOME / 'lib64'}"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"building {src.name} failed:\n{res.stderr}")
        out.append(exe)
    return out


def _link(objdir: Path, lib: Path, verbose: bool, extra: tuple = ()) -> Path:
    objdir.mkdir(parents=True, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as pool:
        objs = list(pool.map(lambda s: _compile(s, verbose, objdir, extra), srcs))
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    tmp.replace(lib)
    return lib


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        build_cli()
        return LIB
    _link(OBJ, LIB, verbose)
    build_cli(force=True)
    return LIB


# The checked build (RB200_DEBUG_BOUNDS, csrc/common.cuh): every gather and
# scatter index that comes from data is range-checked on the device; a bad one
# is skipped and reported through the run's status.  A library of its own, for
# tests and debugging; nothing loads it unless asked (REFORM_B200_LIB).
DEBUG_LIB = OUT / "libreform_b200_debug_bounds.so"
DEBUG_OBJ = OUT / "obj_debug_bounds"


def build_debug_bounds(force: bool = False, verbose: bool = False) -> Path:
    if not force and DEBUG_LIB.exists():
        t = DEBUG_LIB.stat().st_mtime
        if not any(p.stat().st_mtime > t for p in sources() + headers()):
            return DEBUG_LIB
    return _link(DEBUG_OBJ, DEBUG_LIB, verbose, ("-DRB200_DEBUG_BOUNDS",))


if __name__ == "__main__":
    if "--debug-bounds" in sys.argv:
        print(build_debug_bounds(force="--force" in sys.argv, verbose="-v" in sys.argv))
    else:
        print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
