"""Pseudocharge replicas and fields of ChargeDensity and ForcesLocal.

The reference forms the nuclear pseudocharge density b = -(1/4 pi) Lap V_J
of every atom J whose rb-box meets the processor block (ChargeDensity,
initialize.cpp:470-784), the smooth reference density b_tilda of radius
rc_tilda with its correction potential Vc, and the superposed atomic
densities rho_at; ForcesLocal (forces.cpp:20-315) differentiates the same
per-atom fields for the local and correction forces.  :class:`LocalAtoms`
holds what both need: the replicas of Replica_atoms (initialize.cpp:21-160)
in the functions' loop order (type, main atom, replica) with their
intersection boxes, and per type the radial tables with the reference's
spline derivatives.  Case containers written by the drop-in program's export
mode and the fixtures of tests/golden carry them as ``loc_*`` arrays.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class LocalAtoms:
    tables: list          # per type [5, size]: radial grid, rVloc, DVloc, uu, Duu
    Z: np.ndarray         # valence charge per type
    rep_type: np.ndarray  # [n_rep] int32
    rep_atom: np.ndarray  # [n_rep] int32, global (type-major) atom index
    rep_xyz: np.ndarray   # [n_rep, 3]
    rep_box: np.ndarray   # [n_rep, 6] int32: xstart, xend, ystart, yend, zstart, zend (global nodes)
    rc_tilda: float

    @property
    def n_rep(self) -> int:
        return len(self.rep_type)


@dataclass
class LocalGrid:
    np_: tuple
    pnode_s: tuple
    fdn: int
    delta: float
    coeff_lap: np.ndarray
    coeff_grad: np.ndarray
    n_atm: int


def local_from_arrays(a: dict) -> LocalAtoms:
    """LocalAtoms from container arrays (``loc_tab<t>``, ``loc_rep_*``,
    ``loc_Z``, ``loc_rc_tilda``)."""
    Z = np.asarray(a["loc_Z"], np.float64).reshape(-1)
    return LocalAtoms(tables=[np.asarray(a[f"loc_tab{t}"], np.float64) for t in range(len(Z))], Z=Z,
                      rep_type=np.asarray(a["loc_rep_type"], np.int32).reshape(-1),
                      rep_atom=np.asarray(a["loc_rep_atom"], np.int32).reshape(-1),
                      rep_xyz=np.asarray(a["loc_rep_xyz"], np.float64).reshape(-1, 3),
                      rep_box=np.asarray(a["loc_rep_box"], np.int32).reshape(-1, 6),
                      rc_tilda=float(np.asarray(a["loc_rc_tilda"]).reshape(-1)[0]))


def grid_from_arrays(a: dict) -> LocalGrid:
    """The block grid of a container (``params_i``, ``params_d``,
    ``coeff_lap``, ``coeff_grad``; the layout of sqdft_b200.case)."""
    pi, pd = np.asarray(a["params_i"]), np.asarray(a["params_d"])
    return LocalGrid(np_=tuple(int(x) for x in pi[3:6]), pnode_s=tuple(int(x) for x in pi[6:9]), fdn=int(pi[10]),
                     delta=float(pd[0]), coeff_lap=np.asarray(a["coeff_lap"], np.float64),
                     coeff_grad=np.asarray(a["coeff_grad"], np.float64), n_atm=int(pi[14]))


def fields_from_arrays(a: dict) -> dict:
    """The block fields a container holds for ForcesLocal: phi (with its FDn
    halo), Vc, b, b_tilda."""
    return {k: np.asarray(a[f"loc_{k}"], np.float64) for k in ("phi", "vc", "b", "b_tilda")}
