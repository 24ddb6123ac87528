"""Regenerate tests/golden/io/: the restart and output files the reference
program writes (readfiles.cpp:1230-1651), from a 2-step MD run of the tiny
system with prnt_atoms, prnt_scf and prnt_md on.

Runs the reference program compiled from its own sources by
``make -C oracle`` (oracle/_ref/sqdft_ref) and keeps tiny.aout,
tiny.restart and tiny.restartMD.

    python tests/golden/make_io_golden.py
"""
from __future__ import annotations

import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from sqdft_b200.configs.gen_configs import write_system  # noqa: E402

PROGRAM = ROOT / "oracle" / "_ref" / "sqdft_ref"
POT = ROOT / "oracle" / "_ref" / "pot"
FLAGS = {"prnt_atoms": "1", "prnt_scf": "1", "prnt_md": "1", "MaxMDsteps": "2"}


def main() -> None:
    dest = Path(__file__).parent / "io"
    dest.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        run = write_system("tiny", Path(td))
        inp = run / "tiny.input"
        lines = []
        for line in inp.read_text().splitlines():
            key = line.split()[0] if line.split() else ""
            lines.append(f"{key} {FLAGS[key]}" if key in FLAGS else line)
        inp.write_text("\n".join(lines) + "\n")
        for pot in POT.glob("*.pot"):
            (run / pot.name).symlink_to(pot)
        subprocess.run([str(PROGRAM), "-name", "tiny"], cwd=run, check=True, stdout=subprocess.DEVNULL)
        for ext in ("aout", "restart", "restartMD"):
            shutil.copyfile(run / f"tiny.{ext}", dest / f"tiny.{ext}")
            print(dest / f"tiny.{ext}")


if __name__ == "__main__":
    main()
