"""Write SQDFT ``.input`` / ``.atoms`` files for the benchmark and test systems.

Every system is a periodic supercell written with explicit, seeded-Gaussian
displaced coordinates (``perturb 0``, ``ncell 1``), so that the reference
program and this package read identical geometry.  Keywords and file layout
follow the reference's own parser (readfiles.cpp:86-391 for ``.input``,
readfiles.cpp:409-602 for ``.atoms``); the pseudopotential path in ``.atoms``
is the bare file name, resolved in the run directory.

    python -m sqdft_b200.configs.gen_configs [out_dir]
"""
from __future__ import annotations

import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

KB_EV = 8.617343e-5  # Boltzmann constant in eV/K, readfiles.cpp:309

FCC = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])
# Species: symbol, valence Z, mass (amu), lloc, rb, pseudopotential file.
SPECIES = {
    "Al": ("Al", 3, 26.9815385, 1, 6.0, "psd_Al.pot"),
    "Li": ("Li", 1, 6.941, 0, 8.0, "psd_Li.pot"),
    "H": ("H", 1, 1.00794, 0, 8.0, "psd_H.pot"),
}


@dataclass
class System:
    name: str
    lattice: float  # conventional cubic cell edge (bohr)
    cells: int  # supercell repeats per direction
    n_int_cell: int  # grid intervals per cell edge
    kt_ev: float
    npl: int
    rcut: float
    sigma: float  # Gaussian displacement (bohr)
    seed: int
    basis: list[tuple[str, tuple[float, float, float]]]
    max_md: int = 1
    note: str = ""
    xyz: tuple | None = None  # explicit Cartesian positions (bohr), in basis order

    @property
    def domain(self) -> float:
        return self.lattice * self.cells

    @property
    def n_int(self) -> int:
        return self.n_int_cell * self.cells


def _al_basis():
    return [("Al", tuple(p)) for p in FCC]


def _lih_basis():
    return [("Li", tuple(p)) for p in FCC] + [("H", tuple((p + [0.5, 0.0, 0.0]) % 1.0)) for p in FCC]


SYSTEMS = {
    # Small systems whose reference SQ step runs in well under a minute on one
    # core: golden fixtures and CPU-suite parity cases.
    "tiny": System("tiny", 7.78, 1, 8, 5.0, 16, 3.0, 0.05, 11, _al_basis(), note="Al 4 atoms, 9^3 window"),
    "lihs": System("lihs", 7.72, 1, 10, 3.0, 16, 3.0, 0.1, 12, _lih_basis(), note="LiH 8 atoms, 9^3 window"),
    "mid": System("mid", 7.78, 1, 12, 5.0, 24, 4.5, 0.05, 13, _al_basis(), note="Al 4 atoms, 15^3 window"),
    # The five benchmark configurations.
    "c1": System("c1", 7.78, 1, 16, 5.0, 64, 6.0, 0.05, 1, _al_basis(), note="FCC Al 4 atoms, 16^3"),
    "c2": System("c2", 7.78, 3, 16, 5.0, 96, 7.0, 0.15, 2, _al_basis(), note="FCC Al 108 atoms, 48^3"),
    "c3": System("c3", 7.72, 2, 20, 3.0, 128, 6.0, 0.1, 3, _lih_basis(), note="rocksalt LiH 64 atoms, 40^3"),
    "c4": System("c4", 7.78, 2, 16, 5.0, 64, 6.0, 0.05, 4, _al_basis(), note="FCC Al 32 atoms, 32^3"),
    "c5": System("c5", 7.78, 5, 16, 10.0, 128, 7.0, 0.05, 5, _al_basis(), max_md=10,
                 note="FCC Al 500 atoms, 80^3, NVE"),
    # The reference's regression system tests/Al (test_Al.input, Al_eq.atoms):
    # 4 Al atoms, one displaced, 10^3 grid, T = 46418.02 K, npl 28, Rcut 6.
    "al_ref": System("al_ref", 7.78, 1, 10, 46418.02 * KB_EV, 28, 6.0, 0.0, 0, _al_basis(),
                     note="reference regression Al, 4 atoms, 17^3 window",
                     xyz=((0.0, 0.0, 0.0), (0.0, 3.89, 3.89), (3.89, 0.0, 3.89), (3.74, 3.49, 0.37))),
    # The same geometry on finer grids at npl 64: the adjoint's atom gradient
    # against the reference's nonlocal forces as the grid is refined.
    "al_ref14": System("al_ref14", 7.78, 1, 14, 46418.02 * KB_EV, 64, 6.0, 0.0, 0, _al_basis(),
                       note="reference regression Al geometry, 14^3 grid, 23^3 window",
                       xyz=((0.0, 0.0, 0.0), (0.0, 3.89, 3.89), (3.89, 0.0, 3.89), (3.74, 3.49, 0.37))),
    "al_ref20": System("al_ref20", 7.78, 1, 20, 46418.02 * KB_EV, 64, 6.0, 0.0, 0, _al_basis(),
                       note="reference regression Al geometry, 20^3 grid, 33^3 window",
                       xyz=((0.0, 0.0, 0.0), (0.0, 3.89, 3.89), (3.89, 0.0, 3.89), (3.74, 3.49, 0.37))),
}


def positions(s: System) -> dict[str, np.ndarray]:
    """Cartesian positions per species: lattice sites plus seeded Gaussian noise, wrapped."""
    if s.xyz is not None:
        per: dict[str, list] = {}
        for (sym, _), xyz in zip(s.basis, s.xyz):
            per.setdefault(sym, []).append(xyz)
        return {sym: np.array(v, dtype=float) for sym, v in per.items()}
    rng = np.random.default_rng(s.seed)
    per: dict[str, list] = {}
    for cz in range(s.cells):
        for cy in range(s.cells):
            for cx in range(s.cells):
                for sym, frac in s.basis:
                    per.setdefault(sym, []).append((np.array(frac) + [cx, cy, cz]) * s.lattice)
    out = {}
    for sym in per:  # species in first-appearance order of the basis
        xyz = np.array(per[sym])
        xyz = xyz + rng.normal(0.0, s.sigma, size=xyz.shape)
        out[sym] = np.mod(xyz, s.domain)
    return out


def input_text(s: System) -> str:
    t_kelvin = s.kt_ev / KB_EV
    lines = [
        f"atoms_file {s.name}",
        f"domain {s.domain:.10f} {s.domain:.10f} {s.domain:.10f}",
        f"n_int {s.n_int} {s.n_int} {s.n_int}",
        "ncell 1",
        "perturb 0.0",
        "rand_seed 2",
        f"T {t_kelvin:.6f}",
        f"npl {s.npl}",
        f"Rcut {s.rcut}",
        "FD_order 12",
        "poisson_tol 1e-6",
        "poisson_maxiter 1000",
        "lanczos_tol 1e-6",
        "fermi_tol 1e-6",
        "scf_tol 1e-4",
        "scf_miniter 3",
        "scf_maxiter 40",
        "beta_aaj 0.6",
        "m_aaj 7",
        "p_aaj 6",
        "beta_scf 0.1",
        "m_scf 7",
        "p_scf 2",
        "non_blocking 0",
        "prnt_atoms 0",
        "restart_scf 0",
        "prnt_scf 0",
        "fermi_alg 1",
        "Correction 1",
        "qmass 1",
        "vel_dstr 1",
        "ensemble 2",
        "time_step 1",
        f"MaxMDsteps {s.max_md}",
        "ChgExtrap 1",
        "restart_md 0",
        "name Position2.txt",
        "prnt_md 0",
        "RelaxAtoms 0",
    ]
    return "\n".join(lines) + "\n"


def atoms_text(s: System) -> str:
    pos = positions(s)
    n = sum(len(v) for v in pos.values())
    out = [f"{n}", f"n_typ {len(pos)}", "", "Atoms"]
    for sym, xyz in pos.items():
        symb, z, mass, lloc, rb, pot = SPECIES[sym]
        out.append(f"{symb} {z} {mass} {len(xyz)} {lloc} {rb}")
        out.append(pot)
        out += [f"{x:.12f} {y:.12f} {zz:.12f}" for x, y, zz in xyz]
    return "\n".join(out) + "\n"


def write_system(name: str, out_dir: Path) -> Path:
    s = SYSTEMS[name]
    d = out_dir / name
    d.mkdir(parents=True, exist_ok=True)
    (d / f"{name}.input").write_text(input_text(s))
    (d / f"{name}.atoms").write_text(atoms_text(s))
    return d


def main(argv: list[str]) -> None:
    out = Path(argv[1]) if len(argv) > 1 else Path(__file__).parent
    for name in SYSTEMS:
        write_system(name, out)


if __name__ == "__main__":
    main(sys.argv)
