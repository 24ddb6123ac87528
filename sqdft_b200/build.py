"""Build the sqdft_b200 shared library for sm_100a with nvcc.

    python -m sqdft_b200.build [--verbose-ptxas] [--bounds-check]

Produces ``sqdft_b200/_build/libsqdft_b200.so`` in the source tree (it travels
with the tree to the GPU host; it is not installed anywhere), and with
--bounds-check the index-checking variant ``libsqdft_b200_bc.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = BUILD / "libsqdft_b200.so"
INCLUDE = HERE.parent / "include"

SOURCES = ["sqb_api.cu", "sqb_node.cu", "sqb_node_forces.cu", "sqb_node_vjp.cu", "sqb_node_mixed.cu", "sqb_node_lq.cu",
           "sqb_fermi.cu", "sqb_sweep.cu", "sqb_sweep_forces.cu", "sqb_fermi_dev.cu", "sqb_local.cu"]
# Sources that need flags of their own: the device-side Fermi solver rounds
# every operation as the host solver does, and the pseudocharge kernels as
# the reference's x86 build does (no multiply-add contraction).
EXTRA = {"sqb_fermi_dev.cu": ["-fmad=false"], "sqb_local.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


LIB_BC = BUILD / "libsqdft_b200_bc.so"


def build(verbose_ptxas: bool = False, force: bool = False, bounds_check: bool = False) -> Path:
    """The library; with bounds_check the index-checking variant
    (-DSQB_BOUNDS_CHECK, libsqdft_b200_bc.so: a failed device index check
    returns SQB_ERR_BOUNDS; load it with SQDFT_B200_LIB)."""
    out_dir = BUILD / "bc" if bounds_check else BUILD
    lib = LIB_BC if bounds_check else LIB
    out_dir.mkdir(parents=True, exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "sqdft_b200.h"]
    if lib.exists() and not force and all(lib.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return lib
    cmds, objs = [], []
    for src in SOURCES:
        obj = out_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
               *EXTRA.get(src, []), *(["-DSQB_BOUNDS_CHECK"] if bounds_check else []), f"-I{INCLUDE}", "-c",
               str(CSRC / src), "-o", str(obj)]
        if verbose_ptxas:
            cmd.insert(-4, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, check=False), cmds):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = lib.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    tmp.replace(lib)
    return lib


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv,
                bounds_check="--bounds-check" in sys.argv))
