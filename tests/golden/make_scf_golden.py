"""Regenerate tests/golden/al_ref_scf.json: a whole SQDFT run of the
reference's regression system tests/Al, by the reference itself.

Runs the unmodified reference program, compiled from its own sources by
``make -C oracle ref`` (oracle/_ref/sqdft_ref, one rank), on the system
``al_ref`` of ``sqdft_b200/configs/gen_configs.py`` (the geometry and
parameters of tests/Al/test_Al.input and Al_eq.atoms) and stores what its log
reports: every SCF iteration (error, Fermi level, total energy), the free
energy, the atomic forces and the Lanczos / Brent iteration counts.  The
reference's own published log of that system (tests/Al/results_Al) is parsed
the same way and stored beside it as ``published``.

    SQDFT_REFERENCE=/path/to/SQDFT python tests/golden/make_scf_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from sqdft_b200.configs.gen_configs import write_system  # noqa: E402
from sqdft_b200.runlog import parse  # noqa: E402

PROGRAM = ROOT / "oracle" / "_ref" / "sqdft_ref"
POT = ROOT / "oracle" / "_ref" / "pot"


def main() -> None:
    with tempfile.TemporaryDirectory() as td:
        run = write_system("al_ref", Path(td))
        for pot in POT.glob("*.pot"):
            (run / pot.name).symlink_to(pot)
        out = subprocess.run([str(PROGRAM), "-name", "al_ref"], cwd=run, check=True, capture_output=True, text=True)
    golden = {"system": "al_ref", "program": "reference SQDFT built from source, 1 rank", **parse(out.stdout)}
    ref = os.environ.get("SQDFT_REFERENCE")
    if not ref:
        raise SystemExit("set SQDFT_REFERENCE=/path/to/SQDFT (a checkout of the reference sources)")
    golden["published"] = parse((Path(ref) / "tests" / "Al" / "results_Al").read_text())
    dest = Path(__file__).parent / "al_ref_scf.json"
    dest.write_text(json.dumps(golden, indent=1) + "\n")
    print(f"{dest}: {len(golden['scf'])} SCF iterations, free energy {golden['free_energy']}")


if __name__ == "__main__":
    main()
