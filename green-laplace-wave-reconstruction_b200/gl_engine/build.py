"""Build the engine's shared library for sm_100a with nvcc.

The library is a plain C-ABI ``.so`` (no torch types in its signatures),
compiled in-tree so it travels with the source tree: ``gl_engine/_native/
libgl_b200.so``.  Its translation units compile in parallel into
``_build/`` at the repository root (a changed unit, or any changed header,
recompiles what depends on it) and are then linked.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG.parent / "csrc"
NATIVE = PKG / "_native"
LIB = NATIVE / "libgl_b200.so"
OBJ = PKG.parent.parent / "_build"
SOURCES = ["gl_engine.cu", "gl_launch_cols.cu", "gl_rows_pair.cu", "gl_rows_wide.cu", "gl_rows_adj.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the GL engine needs the CUDA toolkit to build")


def _headers() -> list:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [PKG.parent.parent / "include" / "gl_engine.h"]


def _obj(src: str) -> Path:
    return OBJ / (Path(src).stem + ".o")


def _obj_stale(src: str) -> bool:
    o = _obj(src)
    if not o.exists():
        return True
    t = o.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in [CSRC / src] + _headers())


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + _headers()
    return any(d.exists() and d.stat().st_mtime > built for d in deps)


def _compile(src: str, verbose: bool) -> None:
    o = _obj(src)
    tmp = o.with_suffix(".o.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, "-c", "-o", str(tmp), str(CSRC / src)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src} ({proc.returncode}):\n{proc.stderr[-4000:]}")
    tmp.replace(o)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile ``libgl_b200.so`` if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    NATIVE.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    todo = [s for s in SOURCES if force or _obj_stale(s)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, s, verbose) for s in todo]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp)]
    cmd += [str(_obj(s)) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({proc.returncode}):\n{proc.stderr[-4000:]}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
