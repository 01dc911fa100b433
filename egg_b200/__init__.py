"""egg_b200: B200-native (sm_100a) structured TMOP smoother/untangler core.

The compute path is ``libegg_b200.so`` (hand-written CUDA kernels behind a
C-ABI, ``include/egg_b200.h``); ``cpp_core`` is the pybind11 surface that
mirrors the reference module ``egg._cpp.cpp_core``.  There is no CPU
implementation: importing ``cpp_core`` fails loudly when the native build is
missing, and sessions raise when no CUDA device is present.
"""

from __future__ import annotations

import importlib
from pathlib import Path

__all__ = ["load_core", "lib_path", "PACKAGE_DIR"]

PACKAGE_DIR = Path(__file__).resolve().parent


def lib_path() -> Path:
    return PACKAGE_DIR / "libegg_b200.so"


def load_core():
    """Import the native ``cpp_core`` module (raises ImportError if unbuilt)."""
    try:
        return importlib.import_module("egg_b200.cpp_core")
    except ImportError as exc:  # pragma: no cover - depends on the build
        raise ImportError(
            "egg_b200.cpp_core is not built: run `python -m egg_b200.build` "
            f"(or __graft_entry__.build()); original error: {exc}"
        ) from exc


def __getattr__(name):
    if name == "cpp_core":
        return load_core()
    raise AttributeError(name)
