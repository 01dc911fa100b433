"""In-tree build of the egg_b200 native libraries.

* ``egg_b200/libegg_b200.so``  CUDA kernels + C-ABI, nvcc for sm_100a only;
* ``egg_b200/cpp_core<EXT>``   pybind11 surface over the C-ABI (g++, rpath $ORIGIN).

Run ``python -m egg_b200.build`` (or ``__graft_entry__.build()``).
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = PKG / "libegg_b200.so"
EXT = sysconfig.get_config_var("EXT_SUFFIX")
CORE = PKG / f"cpp_core{EXT}"

OBJ_DIR = ROOT / "_build"
# Translation units of libegg_b200.so: the sweep core (session.cu with every
# kernel header) and the device-side wire builder (wire.cu, standalone).  Each
# compiles to its own object, in parallel, and only when its inputs changed.
CU_UNITS = {
    "session": (CSRC / "session.cu",
                sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inc")) + [INCLUDE / "egg_b200.h"]),
    "wire": (CSRC / "wire.cu", [INCLUDE / "egg_b200.h"]),
}
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
              f"-I{INCLUDE}", f"-I{CSRC}"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, **kw):
    print("+", " ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True, **kw)


def _compile(name: str, force: bool) -> Path:
    src, deps = CU_UNITS[name]
    obj = OBJ_DIR / f"{name}.o"
    if force or _stale(obj, [src, *deps, Path(__file__)]):
        OBJ_DIR.mkdir(exist_ok=True)
        tmp = obj.with_suffix(".o.tmp")
        _run([NVCC, *NVCC_FLAGS, "-c", src, "-o", tmp])
        os.replace(tmp, obj)
    return obj


def build_lib(force: bool = False) -> Path:
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(len(CU_UNITS)) as ex:
        objs = list(ex.map(lambda n: _compile(n, force), CU_UNITS))
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", *objs, "-o", tmp, "-lcudart"])
        os.replace(tmp, LIB)
    return LIB


def build_core(force: bool = False) -> Path:
    src = CSRC / "cpp_core.cpp"
    if force or _stale(CORE, [src, INCLUDE / "egg_b200.h", LIB, Path(__file__)]):
        import pybind11

        tmp = CORE.with_suffix(".tmp")
        _run(
            ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
             f"-I{INCLUDE}", f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}",
             src, "-o", tmp, f"-L{PKG}", "-legg_b200", "-Wl,-rpath,$ORIGIN"]
        )
        os.replace(tmp, CORE)
    return CORE


def build(force: bool = False) -> None:
    build_lib(force)
    build_core(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
