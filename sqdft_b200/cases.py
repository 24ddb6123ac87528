"""Benchmark and test cases exported by the drop-in program.

``make_case(name)`` writes the system's ``.input``/``.atoms``
(configs/gen_configs.py), runs ``sqdft_gpu`` (the SQDFT program with this
package's SQ step, sqdft_b200/dropin) in export mode -- the reference's own
set-up (ChargeDensity, Replica_atoms_Rcut, Poisson, XC) up to the first SQ
call, which writes its inputs and exits without touching a GPU -- and keeps
the case container under ``sqdft_b200/_data/cases``.  The Veff in a case is
the reference's first-SCF-iteration Veff; projector tables are not stored
(the GPU computes them from the radial tables).

    python -m sqdft_b200.cases c1 c2 ...
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

from .case import load_case
from .configs.gen_configs import write_system

HERE = Path(__file__).resolve().parent
DATA = HERE / "_data"
CASES = DATA / "cases"
POT = DATA / "pot"
DROPIN = HERE / "_build" / "dropin" / "sqdft_gpu"


def case_path(name: str) -> Path:
    return CASES / f"{name}.sqc"


def make_case(name: str, force: bool = False) -> Path:
    out = case_path(name)
    if out.exists() and not force:
        return out
    if not DROPIN.exists():
        raise RuntimeError(f"drop-in program not built: {DROPIN} (make -C sqdft_b200/dropin)")
    if not any(POT.glob("*.pot")):
        raise RuntimeError(f"pseudopotential tables missing in {POT}")
    CASES.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        run = write_system(name, Path(td))
        for pot in POT.glob("*.pot"):
            (run / pot.name).symlink_to(pot)
        env = dict(os.environ, SQDFT_B200_EXPORT=str(out))
        subprocess.run([str(DROPIN), "-name", name], cwd=run, env=env, check=True, stdout=subprocess.DEVNULL)
    return out


def load(name: str):
    """The case of a named system (exported first if needed)."""
    return load_case(make_case(name))


if __name__ == "__main__":
    import time

    for nm in sys.argv[1:]:
        t = time.time()
        p = make_case(nm, force=True)
        print(f"{p}: {p.stat().st_size / 2**20:.1f} MiB in {time.time() - t:.1f} s")
