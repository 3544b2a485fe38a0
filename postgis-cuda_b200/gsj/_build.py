"""Locate (and, when missing, build) the in-tree shared libraries of the package."""
from __future__ import annotations

import os
import subprocess
import threading

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD_DIR = os.path.join(PKG_DIR, "_build")
_lock = threading.Lock()


def build(targets=("all",)) -> None:
    """Run the package Makefile (nvcc for sm_100a, g++ for the host code)."""
    subprocess.run(["make", "-C", PKG_DIR, "-j8", *targets], check=True)


def lib_path(name: str) -> str:
    p = os.path.join(BUILD_DIR, name)
    if not os.path.exists(p):
        with _lock:
            if not os.path.exists(p):
                build()
    if not os.path.exists(p):
        raise RuntimeError(f"{name} was not built (make -C {PKG_DIR})")
    return p
