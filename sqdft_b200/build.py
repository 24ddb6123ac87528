"""Build the sqdft_b200 shared library for sm_100a with nvcc.

    python -m sqdft_b200.build [--verbose-ptxas]

Produces ``sqdft_b200/_build/libsqdft_b200.so`` in the source tree (it travels
with the tree to the GPU host; it is not installed anywhere).
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
           "sqb_fermi.cu", "sqb_sweep.cu", "sqb_sweep_forces.cu", "sqb_fermi_dev.cu"]
# Sources that need flags of their own: the device-side Fermi solver rounds
# every operation as the host solver does (no multiply-add contraction).
EXTRA = {"sqb_fermi_dev.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "sqdft_b200.h"]
    if LIB.exists() and not force and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    cmds, objs = [], []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
               *EXTRA.get(src, []), f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)]
        if verbose_ptxas:
            cmd.insert(-4, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, check=False), cmds):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
