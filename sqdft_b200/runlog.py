"""Read the numbers an SQDFT run prints to standard output.

The SCF loop prints one line per iteration (scf.cpp:202, e.g.
``Iter:9,SCF_err = 1.56619e-05, Fermi energy (Ha) : 0.277377479887  and Total
energy (Ha/atom) : -2.453313155422``), the free energy once the SCF has
converged (scf.cpp:314), and the atomic forces after ``Atomic forces:`` (forces.cpp:635-640,
three columns per atom, at most 8 atoms).  ``parse`` returns them as plain
Python values; it reads the drop-in program's log and the reference's alike.
"""
from __future__ import annotations

import re

_ITER = re.compile(
    r"Iter:(\d+),SCF_err = ([-+0-9.eE]+), Fermi energy \(Ha\) : ([-+0-9.eE]+)\s+and Total energy \(Ha/atom\) : ([-+0-9.eE]+)")
_FREE = re.compile(r"Free energy \(Ha/atom\)\s*:\s*([-+0-9.eE]+)")
_LANCZOS = re.compile(r"Lanczos took (\d+) iterations")
_FERMI_ITERS = re.compile(r"(?:Brent's algorithm|Newton-Raphson) took (\d+) iterations")


def parse(text: str) -> dict:
    """SCF iterations, free energy, forces and iteration counts of one run's log.

    Only the first MD step is read (the log of a single-point run has one).
    """
    scf = [{"iter": int(m[1]), "scf_err": float(m[2]), "fermi": float(m[3]), "etot": float(m[4])}
           for m in _ITER.finditer(text)]
    free = _FREE.search(text)
    forces = []
    lines = text.splitlines()
    for i, line in enumerate(lines):
        if line.strip().startswith("Atomic forces:"):
            for row in lines[i + 1:]:
                parts = row.split()
                if len(parts) != 3:
                    break
                try:
                    forces.append([float(p) for p in parts])
                except ValueError:
                    break
            break
    return {
        "scf": scf,
        "free_energy": float(free[1]) if free else None,
        "forces": forces,
        "lanczos_iters": [int(m[1]) for m in _LANCZOS.finditer(text)],
        "fermi_iters": [int(m[1]) for m in _FERMI_ITERS.finditer(text)],
    }
