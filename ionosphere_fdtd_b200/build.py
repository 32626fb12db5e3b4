"""Build the in-tree CUDA library ``libifdtd.so`` for sm_100a with nvcc.

``python -m ionosphere_fdtd_b200.build`` compiles every CUDA source of the
package into one shared library next to this file.  The library exports the
C ABI declared in ``include/ifdtd.h``; the Python host binds it with ctypes.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
SOURCES = [PACKAGE / "csrc" / "ifdtd.cu", PACKAGE / "csrc" / "surrogate.cu", PACKAGE / "csrc" / "gemm_tcgen05.cu"]
HEADERS = [
    PACKAGE / "csrc" / "step_kernels.cuh",
    PACKAGE / "csrc" / "pipe_kernels.cuh",
    PACKAGE / "csrc" / "fused_kernels.cuh",
    PACKAGE / "csrc" / "errors.cuh",
    ROOT / "include" / "ifdtd.h",
    ROOT / "include" / "ifdtd_surrogate.h",
]
LIBRARY = PACKAGE / "libifdtd.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libifdtd.so")


def command(output: Path = LIBRARY, extra: list[str] | None = None) -> list[str]:
    return [
        nvcc(),
        *ARCH,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-shared",
        "-I",
        str(ROOT / "include"),
        *(extra or []),
        "-o",
        str(output),
        *map(str, SOURCES),
    ]


def stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(p.stat().st_mtime > built for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if force or stale():
        cmd = command(extra=["-Xptxas", "-v"] if verbose else None)
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + result.stdout + result.stderr)
        if verbose:
            sys.stderr.write(result.stderr)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIBRARY)
