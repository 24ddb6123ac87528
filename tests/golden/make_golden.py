"""Regenerate the golden fixtures of tests/golden from the reference itself.

Runs the reference SQDFT, compiled from its own sources by ``make -C oracle``
(oracle/_ref/sqref_driver), on the small systems of
``sqdft_b200/configs/gen_configs.py`` and stores, per system, the SQ-step
inputs the reference used (Veff with its halo, replica atoms, projector
tables UdVtm, grid parameters) and its outputs (rho, rho_pj, Ci, chi, zee,
lambda_f, Ebs, Eent, nonlocal forces, and HsubTimesVec on seeded vectors).
The radial pseudopotential tables are not stored.

    SQDFT_REFERENCE=/path/to/SQDFT python tests/golden/make_golden.py [system ...]

SQDFT_REFERENCE (a checkout of the reference) is needed for the system ``al``,
which reads the reference's own regression input.
"""
from __future__ import annotations

import os
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
SYSTEMS = {"tiny": ["--hv", "3"], "lihs": ["--hv", "2"], "mid": ["--hv", "1"], "al": ["--no-forces"]}
# The reference's own regression input tests/Al (4-atom Al, 10^3 grid, npl 28);
# its published log (tests/Al/results_Al:82) gives the first-SCF Fermi level.


def ref_tests() -> Path:
    """tests/ of the reference checkout named by SQDFT_REFERENCE."""
    ref = os.environ.get("SQDFT_REFERENCE")
    if not ref or not (Path(ref) / "tests").is_dir():
        raise SystemExit("set SQDFT_REFERENCE=/path/to/SQDFT (a checkout of the reference sources)")
    return Path(ref) / "tests"


def run_reference(name: str, extra: list[str], workdir: Path) -> tuple[dict, dict]:
    if name == "al":
        run = workdir / "al"
        run.mkdir()
        (run / "al.input").write_text((ref_tests() / "Al" / "test_Al.input").read_text())
        atoms = (ref_tests() / "Al" / "Al_eq.atoms").read_text().replace("../../pseudopotentials/", "")
        (run / "Al_eq.atoms").write_text(atoms)
    else:
        run = write_system(name, workdir)
    for pot in POT.glob("*.pot"):
        (run / pot.name).symlink_to(pot)
    out = workdir / f"{name}_ref"
    subprocess.run([str(DRIVER), str(run), name, str(out), *extra], check=True, stdout=subprocess.DEVNULL)
    return read_container(f"{out}_in.sqc"), read_container(f"{out}_out.sqc")


def main(names: list[str]) -> None:
    for name in names or list(SYSTEMS):
        with tempfile.TemporaryDirectory() as td:
            inp, out = run_reference(name, SYSTEMS[name], Path(td))
        arrays = {f"in_{k}": v for k, v in inp.items() if not k.startswith("psd")}
        keep = (lambda k: k in ("lambda_f", "Ebs", "Eent", "chi", "zee", "rho")) if name == "al" else (lambda k: True)
        arrays.update({f"out_{k}": v for k, v in out.items() if not k.startswith("t_") and keep(k)})
        dest = Path(__file__).parent / f"{name}.npz"
        np.savez_compressed(dest, **arrays)
        print(f"{dest}: {dest.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main(sys.argv[1:])
