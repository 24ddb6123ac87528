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

import math
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


_TEMP_TOL = 1e-12  # TEMP_TOL of the reference


def _c_round(x: float) -> int:
    """C's round(): to nearest, halves away from zero (exact for |x| < 2^52)."""
    a = abs(x)
    f = math.floor(a)
    r = f + (1 if a - f >= 0.5 else 0)
    return int(r) if x >= 0 else -int(r)


def pseudocharge_replicas(atoms_xyz, atom_type, rb, domain, n_int, pnode_s, np_):
    """Replica_atoms (initialize.cpp:21-160): every periodic image of every
    atom whose rb-box, centred on the image's nearest grid node, meets the
    block [pnode_s, pnode_s + np_), with the intersection box.

    ``atoms_xyz`` [n_atm, 3] are the main-domain positions (DS_coord::main_atm)
    in type-major order with types ``atom_type``; ``rb`` the per-type cutoffs
    as the .atoms file gives them (rounded up to a multiple of the mesh size
    here, readfiles.cpp:513); ``domain`` the three domain lengths of the
    .input file.  Returns (rep_type, rep_atom, rep_xyz, rep_box) in the
    reference's loop order (type, main atom, image z-y-x), as
    :class:`LocalAtoms` holds them."""
    domain = [float(d) for d in domain]
    delta = domain[0] / int(n_int[0])  # readfiles.cpp:294-303
    rb_eff = [math.ceil(r / delta) * delta for r in rb]
    ps = [int(p) for p in pnode_s]
    pe = [int(pnode_s[d]) + int(np_[d]) - 1 for d in range(3)]
    xyz = np.asarray(atoms_xyz, np.float64).reshape(-1, 3)
    types = np.asarray(atom_type, np.int64).reshape(-1)
    rt, ra, rx, rbox = [], [], [], []

    def nearest(c):
        n = _c_round(c / delta)
        if abs(abs(n * delta - c) - delta * 0.5) < _TEMP_TOL:
            n = math.floor((c / delta) - 10 * _TEMP_TOL)
        return n

    def overlap(lo, hi, s, e):
        start = lo if s <= lo <= e else (s if lo <= s <= hi else -1)
        end = hi if s <= hi <= e else (e if lo <= e <= hi else -1)
        return start, end

    atom = 0
    for t in range(len(rb)):
        r_b = rb_eff[t]
        half = _c_round(r_b / delta)
        for a in np.nonzero(types == t)[0]:
            c = xyz[a]
            hi = [math.floor(((domain[d] + r_b - c[d]) / domain[d]) + _TEMP_TOL) for d in range(3)]
            lo = [math.ceil(((-r_b - c[d]) / domain[d]) - _TEMP_TOL) for d in range(3)]
            for rr in range(lo[2], hi[2] + 1):
                for qq in range(lo[1], hi[1] + 1):
                    for pp in range(lo[0], hi[0] + 1):
                        img = (c[0] + pp * domain[0], c[1] + qq * domain[1], c[2] + rr * domain[2])
                        box = []
                        for d in range(3):
                            n = nearest(img[d])
                            box.extend(overlap(n - half, n + half, ps[d], pe[d]))
                        if -1 not in box:
                            rt.append(t)
                            ra.append(atom)
                            rx.append(img)
                            rbox.append(box)
            atom += 1
    return (np.array(rt, np.int32), np.array(ra, np.int32), np.array(rx, np.float64).reshape(-1, 3),
            np.array(rbox, np.int32).reshape(-1, 6))


def projector_replicas(atoms_xyz, atom_type, rc, domain, n_int, pnode_s, np_, nloc):
    """Replica_atoms_Rcut (initialize.cpp:1003-1196): every periodic image of
    every atom whose rc-box, centred on the image's nearest grid node, meets
    the block widened by the truncation half-width nloc on every side -- the
    replicas whose projectors the SQ windows of the block can see
    (sqb_set_atoms).  ``rc`` are the per-type projector radii as DS_Psd holds
    them (the case container's ``typ_d[:, 0]``), Rcut = nloc * delta
    (readfiles.cpp:306-307).  Returns (rep_type, rep_atom, rep_xyz) in the
    reference's loop order."""
    domain = [float(d) for d in domain]
    delta = domain[0] / int(n_int[0])
    rcut = nloc * delta
    ps = [int(pnode_s[d]) - nloc for d in range(3)]
    pe = [int(pnode_s[d]) + int(np_[d]) - 1 + nloc for d in range(3)]
    xyz = np.asarray(atoms_xyz, np.float64).reshape(-1, 3)
    types = np.asarray(atom_type, np.int64).reshape(-1)
    rt, ra, rx = [], [], []

    def nearest(c):
        n = _c_round(c / delta)
        if abs(abs(n * delta - c) - delta * 0.5) < _TEMP_TOL:
            n = math.floor((c / delta) - 10 * _TEMP_TOL)
        return n

    def meets(lo, hi, s, e):
        start = s <= lo <= e or lo <= s <= hi
        end = s <= hi <= e or lo <= e <= hi
        return start and end

    atom = 0
    for t in range(len(rc)):
        half = math.ceil(rc[t] / delta)
        for a in np.nonzero(types == t)[0]:
            c = xyz[a]
            hi = [math.floor(((domain[d] + rcut + rc[t] - c[d]) / domain[d]) + _TEMP_TOL) for d in range(3)]
            lo = [math.ceil(((-(rcut + rc[t]) - c[d]) / domain[d]) - _TEMP_TOL) for d in range(3)]
            for rr in range(lo[2], hi[2] + 1):
                for qq in range(lo[1], hi[1] + 1):
                    for pp in range(lo[0], hi[0] + 1):
                        img = (c[0] + pp * domain[0], c[1] + qq * domain[1], c[2] + rr * domain[2])
                        if all(meets(nearest(img[d]) - half, nearest(img[d]) + half, ps[d], pe[d]) for d in range(3)):
                            rt.append(t)
                            ra.append(atom)
                            rx.append(img)
            atom += 1
    return np.array(rt, np.int32), np.array(ra, np.int32), np.array(rx, np.float64).reshape(-1, 3)
