"""Build recipe of libb200fe.so (nvcc, sm_100a only), in-tree."""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
SOURCES = ["b200fe.cu", "slopes.cu", "noalloc.cu", "kss.cu", "learned.cu"]
HEADERS = ["limits.cuh", "context.cuh", "common_kernels.cuh", "kernels.cuh", "setup_kernels.cuh",
           "ols_kernels.cuh", "prep_kernels.cuh", "slope_kernels.cuh", "sparse_kernels.cuh",
           "pcg_kernels.cuh", "mlp_kernels.cuh", "ws_kernels.cuh", "stream_kernels.cuh"]
OUT = HERE / "libb200fe.so"
OBJ_DIR = HERE / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "b200fe.h", Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every translation unit for sm_100a (in parallel), then link."""
    if not force and not _stale():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    OBJ_DIR.mkdir(exist_ok=True)
    inc = [f"-I{ROOT / 'include'}", f"-I{CSRC}"]
    cmds = [[nvcc(), *NVCC_FLAGS, *inc, "-c", "-o", str(OBJ_DIR / (Path(src).stem + ".o")),
             str(CSRC / src)] for src in SOURCES]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(OUT),
            *[str(OBJ_DIR / (Path(src).stem + ".o")) for src in SOURCES]]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
