"""The reference's restart and output files, read and written byte for byte.

SQDFT writes, at the end of an SCF or an MD step (readfiles.cpp:1230-1651):

* ``<stem>.restart`` (PrintSCF / RestartSCF): the number of ranks, then the
  electron density of every rank's block, rank by rank, each block z-major
  with x fastest, one ``%.14f`` value per line;
* ``<stem>.aout`` (PrintAtoms): atom count, types, per type its symbol,
  valence charge, mass, count, local component, rb and pseudopotential file,
  the positions (``%.16f``, fractional when the input's are) and the atomic
  forces (``%.14f``);
* ``<stem>.restartMD`` (PrintMD / RestartMD): the MD step count, velocities,
  forces and positions (``%.15f``) and the running energy and temperature
  statistics.

The writers produce the same bytes as the reference's fprintf calls (Python's
``%``-formatting of a double is correctly rounded, like glibc's), so a run
of this package can hand its density, forces and MD state to the reference
program and back.  Arrays of per-atom triples are [n_atm, 3] in the
reference's type-major atom order.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


# -- .restart ---------------------------------------------------------------------

def write_restart(path, rho: np.ndarray, nproc: int = 1) -> None:
    """PrintSCF (readfiles.cpp:1328-1383): ``rho`` is the whole density in the
    file's order (rank blocks one after another, each z-major), e.g. from
    :func:`rank_order`."""
    rho = np.asarray(rho, np.float64).reshape(-1)
    with open(path, "w") as f:
        f.write("%d\n" % nproc)
        f.write("".join("%.14f\n" % v for v in rho))


def read_restart(path) -> tuple[int, np.ndarray]:
    """RestartSCF (readfiles.cpp:1386-1441): (rank count, density in file order)."""
    with open(path) as f:
        nproc = int(f.readline())
        rho = np.array([float(x) for x in f.read().split()], np.float64)
    return nproc, rho


def rank_order(blocks: list[np.ndarray]) -> np.ndarray:
    """The .restart order of per-rank density blocks ([np_z, np_y, np_x] each,
    rank order): each block flattened z-major, blocks concatenated."""
    return np.concatenate([np.ascontiguousarray(b, np.float64).reshape(-1) for b in blocks])


# -- .aout ------------------------------------------------------------------------

@dataclass
class AtomType:
    symb: str
    Z: int
    mass: float
    lloc: int
    rb: float
    pseudo_path: str
    positions: np.ndarray  # [natm, 3], as printed (divided by the lattice constant when fractional)


@dataclass
class AtomsOut:
    types: list
    forces: np.ndarray      # [n_atm, 3] Ha/bohr
    frac_coord: int = 0

    @property
    def n_atm(self) -> int:
        return sum(len(t.positions) for t in self.types)


def write_aout(path, out: AtomsOut) -> None:
    """PrintAtoms (readfiles.cpp:1230-1288)."""
    lines = ["%u\n" % out.n_atm, "n_typ %u\n" % len(out.types), "frac_coord %u\n" % out.frac_coord]
    if out.frac_coord == 1:
        lines.append("Note: Atom positions below are in fractional coordinates. \n")
    lines.append("\n%s\n" % "Atoms")
    for t in out.types:
        lines.append("%s %u %f %u %u %f\n" % (t.symb, t.Z, t.mass, len(t.positions), t.lloc, t.rb))
        lines.append("%s\n" % t.pseudo_path)
        lines.extend("%.16f %.16f %.16f\n" % tuple(p) for p in np.asarray(t.positions, np.float64))
    lines.extend([" \n", "Atomic Forces (Ha/Bohr): \n", " \n"])
    k = 0
    for t in out.types:
        lines.append("%s\n" % t.symb)
        for _ in range(len(t.positions)):
            lines.append("%.14f %.14f %.14f\n" % tuple(out.forces[k]))
            k += 1
    Path(path).write_text("".join(lines))


def read_aout(path) -> AtomsOut:
    lines = Path(path).read_text().split("\n")
    n_atm = int(lines[0])
    n_typ = int(lines[1].split()[1])
    frac = int(lines[2].split()[1])
    i = lines.index("Atoms") + 1
    types = []
    for _ in range(n_typ):
        symb, Z, mass, natm, lloc, rb = lines[i].split()
        path_line = lines[i + 1]
        pos = np.array([[float(x) for x in lines[i + 2 + a].split()] for a in range(int(natm))])
        types.append(AtomType(symb, int(Z), float(mass), int(lloc), float(rb), path_line, pos))
        i += 2 + int(natm)
    i = next(j for j in range(i, len(lines)) if lines[j].startswith("Atomic Forces")) + 2
    forces = []
    for t in types:
        i += 1  # the type's symbol
        for _ in range(len(t.positions)):
            forces.append([float(x) for x in lines[i].split()])
            i += 1
    out = AtomsOut(types=types, forces=np.array(forces), frac_coord=frac)
    assert out.n_atm == n_atm
    return out


# -- .restartMD -------------------------------------------------------------------

@dataclass
class MDState:
    step: int                  # MDstepCount + MDrestartCount
    velocities: np.ndarray     # [n_atm, 3]
    forces: np.ndarray         # [n_atm, 3]
    positions: np.ndarray      # [n_atm, 3] (main-domain atoms)
    stats: np.ndarray = field(default_factory=lambda: np.zeros((4, 2)))  # mean/std of TE, PE, KE, T


def write_restart_md(path, md: MDState) -> None:
    """PrintMD (readfiles.cpp:1444-1503)."""
    lines = ["MDstepCount\n", "%d\n" % md.step, "MD velocities\n"]
    lines.extend("%.15f %.15f %.15f\n" % tuple(v) for v in md.velocities)
    lines.append("MD forces\n")
    lines.extend("%.15f %.15f %.15f\n" % tuple(v) for v in md.forces)
    lines.append("Atom positions\n")
    lines.extend("%.15f %.15f %.15f\n" % tuple(v) for v in md.positions)
    lines.append("MD stats\n")
    lines.extend("%.15f %.15f\n" % tuple(v) for v in md.stats)
    Path(path).write_text("".join(lines))


def read_restart_md(path) -> MDState:
    """RestartMD (readfiles.cpp:1506-1600): the sections by their headers."""
    lines = Path(path).read_text().split("\n")

    def section(name, count, width):
        i = lines.index(name) + 1
        return np.array([[float(x) for x in lines[i + r].split()[:width]] for r in range(count)])

    step = int(lines[lines.index("MDstepCount") + 1])
    i = lines.index("MD velocities") + 1
    n_atm = lines.index("MD forces") - i
    return MDState(step=step, velocities=section("MD velocities", n_atm, 3), forces=section("MD forces", n_atm, 3),
                   positions=section("Atom positions", n_atm, 3), stats=section("MD stats", 4, 2))
