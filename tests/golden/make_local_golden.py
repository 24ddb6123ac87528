"""Regenerate the pseudocharge fixtures tests/golden/<system>_local.npz from
the reference itself.

Runs the reference SQDFT, compiled from its own sources by ``make -C oracle``
(oracle/_ref/sqref_driver ``--local``), on the small systems of
``sqdft_b200/configs/gen_configs.py`` and stores, per system:

* the grid parameters (``params_i``, ``params_d``, ``coeff_lap``,
  ``coeff_grad`` of the SQ-step container);
* the pseudocharge inputs: the replicas of Replica_atoms (initialize.cpp:21-160)
  in the loop order of ChargeDensity and ForcesLocal, with their
  intersection boxes; per type the radial grid, rVloc, uu and the reference's
  spline derivatives of both (getYD_gen); the valence charges; rc_tilda;
* ChargeDensity's outputs as the call leaves them (initialize.cpp:470-784):
  b, b_tilda, Vc, rho_at, Eself, Ncharge, Ecorr (``cd_*``);
* the fields ForcesLocal reads (phi with its FDn halo, Vc, b, b_tilda;
  ``loc_*``) and its outputs, the local and correction forces
  (forces.cpp:20-315; ``fl_floc``, ``fl_fcorr``).

    python tests/golden/make_local_golden.py [system ...]
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from sqdft_b200.case import read_container  # noqa: E402
from sqdft_b200.configs.gen_configs import write_system  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "sqref_driver"
POT = ROOT / "oracle" / "_ref" / "pot"
SYSTEMS = ["tiny", "lihs", "mid"]
GRID_KEYS = ("params_i", "params_d", "coeff_lap", "coeff_grad")


def main(names: list[str]) -> None:
    for name in names or SYSTEMS:
        with tempfile.TemporaryDirectory() as td:
            run = write_system(name, Path(td))
            for pot in POT.glob("*.pot"):
                (run / pot.name).symlink_to(pot)
            out = Path(td) / f"{name}_ref"
            subprocess.run([str(DRIVER), str(run), name, str(out), "--no-forces", "--local"], check=True,
                           stdout=subprocess.DEVNULL)
            inp = read_container(f"{out}_in.sqc")
            loc = read_container(f"{out}_local.sqc")
        arrays = {k: inp[k] for k in GRID_KEYS}
        arrays.update({k: v for k, v in loc.items() if not k.startswith("t_")})
        dest = Path(__file__).parent / f"{name}_local.npz"
        np.savez_compressed(dest, **arrays)
        print(f"{dest}: {dest.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main(sys.argv[1:])
