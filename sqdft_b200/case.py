"""SQ-step case files: the inputs (and reference outputs) of one SQ call.

A case holds what ``ClenshawCurtisSpectralQuadrature`` (sq.cpp:377),
``NonlocalProjectors`` (nonlocal.cpp:317) and ``ForcesNonLocal``
(forces.cpp:318) read from ``DS_SQ`` (ds_sq.h:128-238).  The binary layout is
the named-array container of ``sqdft_b200/csrc/sq_case.h``; this module reads
and writes it with numpy and gives the arrays their reference meaning.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_MAGIC = b"SQBCASE1"
_DT = {1: np.float64, 2: np.int32, 3: np.float32}
_DT_CODE = {np.dtype(np.float64): 1, np.dtype(np.int32): 2, np.dtype(np.float32): 3}


def read_container(path) -> dict[str, np.ndarray]:
    """Read every record of a case container into a dict of numpy arrays."""
    out: dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        if f.read(8) != _MAGIC:
            raise ValueError(f"{path}: not a case container")
        while True:
            raw = f.read(48)
            if len(raw) < 48:
                raise ValueError(f"{path}: truncated")
            name = raw.split(b"\0", 1)[0].decode()
            dtype, ndim = struct.unpack("<ii", f.read(8))
            dims = struct.unpack(f"<{ndim}q", f.read(8 * ndim)) if ndim else ()
            if name == "__end__":
                return out
            dt = np.dtype(_DT[dtype])
            n = int(np.prod(dims)) if dims else 1
            out[name] = np.frombuffer(f.read(n * dt.itemsize), dtype=dt).reshape(dims).copy()


def write_container(path, arrays: dict[str, np.ndarray]) -> None:
    """Write a dict of numpy arrays as a case container."""
    with open(path, "wb") as f:
        f.write(_MAGIC)
        for name, a in arrays.items():
            a = np.ascontiguousarray(a)
            if a.dtype not in _DT_CODE:
                a = a.astype(np.float64)
            nm = name.encode()[:47].ljust(48, b"\0")
            f.write(nm + struct.pack("<ii", _DT_CODE[a.dtype], a.ndim))
            f.write(struct.pack(f"<{a.ndim}q", *a.shape))
            f.write(a.tobytes())
        f.write(b"__end__".ljust(48, b"\0") + struct.pack("<ii", 2, 1) + struct.pack("<q", 0))


@dataclass
class AtomType:
    """One pseudopotential / atom type (DS_Psd + DS_Atm, ds_sq.h:54-102)."""

    natm: int
    lmax: int
    lloc: int
    nlocc: int  # ceil(rc / delta), nonlocal.cpp:43
    nproj: int  # sum over l != lloc, l <= lmax of (2l + 1)
    rc: float
    denom: np.ndarray  # Denom_s, Denom_p, Denom_d, Denom_f
    z: float
    tables: np.ndarray  # [19, size]: grid, rVloc, rV_spdf, rU_spdf, DVloc, DV_spdf, DU_spdf

    @property
    def ball(self) -> int:
        return 2 * self.nlocc + 1

    @property
    def lm_list(self) -> list[tuple[int, int]]:
        """(l, m) of each projector in the reference's order (nonlocal.cpp:365-374)."""
        return [(l, m) for l in range(self.lmax + 1) if l != self.lloc for m in range(-l, l + 1)]


@dataclass
class Case:
    """Inputs of one SQ step on one processor block (the whole grid on 1 GPU)."""

    n_int: tuple[int, int, int]
    np_: tuple[int, int, int]  # np_x, np_y, np_z
    pnode_s: tuple[int, int, int]
    nloc: int
    fdn: int
    npl: int
    fermi_alg: int
    n_atm: int
    scf_iter: int
    delta: float
    bet: float
    lanczos_tol: float
    fermi_tol: float
    ncharge: float
    lambda_f: float
    temperature: float
    rcut: float
    coeff_lap: np.ndarray
    coeff_grad: np.ndarray
    veff: np.ndarray  # [np_z + 2nloc, np_y + 2nloc, np_x + 2nloc], halo filled
    types: list[AtomType]
    rep_type: np.ndarray  # [n_rep]
    rep_atom: np.ndarray  # [n_rep] global (type-major) atom index
    rep_xyz: np.ndarray  # [n_rep, 3]
    atoms_xyz: np.ndarray  # [n_atm, 3]
    atom_type: np.ndarray  # [n_atm]
    udvtm: np.ndarray | None = None  # reference projector tables, replica order
    extra: dict = field(default_factory=dict)

    @property
    def nw(self) -> int:
        return 2 * self.nloc + 1

    @property
    def n_nodes(self) -> int:
        return self.np_[0] * self.np_[1] * self.np_[2]

    @property
    def veff_block(self) -> np.ndarray:
        """Veff on the processor block only (no halo), [np_z, np_y, np_x]."""
        nl = self.nloc
        nx, ny, nz = self.np_
        return self.veff[nl:nl + nz, nl:nl + ny, nl:nl + nx]

    def with_veff_block(self, block: np.ndarray) -> "Case":
        """Copy of the case with a new Veff interior and its periodic halo.

        Valid when the block is the whole periodic domain (one processor),
        where the reference's halo exchange (sq.cpp:400-492) is a wrap-around.
        """
        if tuple(self.np_) != tuple(self.n_int):
            raise ValueError("periodic halo fill needs the whole domain in one block")
        nl = self.nloc
        nx, ny, nz = self.np_
        kz = (np.arange(nz + 2 * nl) - nl) % nz
        ky = (np.arange(ny + 2 * nl) - nl) % ny
        kx = (np.arange(nx + 2 * nl) - nl) % nx
        ext = np.ascontiguousarray(block[np.ix_(kz, ky, kx)], dtype=np.float64)
        import dataclasses

        return dataclasses.replace(self, veff=ext)

    def replica_offsets(self) -> np.ndarray:
        """Start of each replica's table in the concatenated UdVtm array."""
        sizes = np.array([self.types[t].nproj * self.types[t].ball ** 3 for t in self.rep_type], dtype=np.int64)
        return np.concatenate([[0], np.cumsum(sizes)])[:-1] if len(sizes) else np.zeros(0, np.int64)


def load_case(path) -> Case:
    """Read a case container written by the reference driver or the exporter."""
    return case_from_arrays(read_container(path))


def case_from_arrays(a: dict) -> Case:
    """Build a Case from container arrays; the radial tables ``psd<t>`` may be
    absent (then only supplied projector tables can be used)."""
    pi = a["params_i"]
    pd = a["params_d"]
    n_typ = int(pi[13])
    types = []
    for t in range(n_typ):
        ti = a["typ_i"][t]
        td = a["typ_d"][t]
        types.append(AtomType(natm=int(ti[0]), lmax=int(ti[1]), lloc=int(ti[2]), nlocc=int(ti[3]),
                              nproj=int(ti[5]), rc=float(td[0]), denom=td[1:5].copy(), z=float(td[5]),
                              tables=a.get(f"psd{t}", np.zeros((19, 0)))))
    return Case(
        n_int=tuple(int(x) for x in pi[0:3]), np_=tuple(int(x) for x in pi[3:6]),
        pnode_s=tuple(int(x) for x in pi[6:9]), nloc=int(pi[9]), fdn=int(pi[10]), npl=int(pi[11]),
        fermi_alg=int(pi[12]), n_atm=int(pi[14]), scf_iter=int(pi[15]),
        delta=float(pd[0]), bet=float(pd[1]), lanczos_tol=float(pd[2]), fermi_tol=float(pd[3]),
        ncharge=float(pd[4]), lambda_f=float(pd[5]), temperature=float(pd[6]), rcut=float(pd[7]),
        coeff_lap=a["coeff_lap"], coeff_grad=a["coeff_grad"], veff=a["veff"], types=types,
        rep_type=a["rep_i"][:, 0].copy(), rep_atom=a["rep_i"][:, 2].copy(), rep_xyz=a["rep_xyz"],
        atoms_xyz=a["atoms_xyz"], atom_type=a["atom_type"], udvtm=a.get("udvtm"),
    )


def save_case(path, c: Case) -> None:
    """Write a Case back into the container layout that ``load_case`` reads."""
    pi = np.array([*c.n_int, *c.np_, *c.pnode_s, c.nloc, c.fdn, c.npl, c.fermi_alg, len(c.types), c.n_atm,
                   c.scf_iter, 1], dtype=np.int32)
    pd = np.array([c.delta, c.bet, c.lanczos_tol, c.fermi_tol, c.ncharge, c.lambda_f, c.temperature, c.rcut])
    arrays = {"params_i": pi, "params_d": pd, "coeff_lap": c.coeff_lap, "coeff_grad": c.coeff_grad,
              "veff": c.veff}
    for t, ty in enumerate(c.types):
        arrays[f"psd{t}"] = ty.tables
    arrays["typ_i"] = np.array([[ty.natm, ty.lmax, ty.lloc, ty.nlocc, ty.tables.shape[1], ty.nproj]
                                for ty in c.types], dtype=np.int32)
    arrays["typ_d"] = np.array([[ty.rc, *ty.denom, ty.z] for ty in c.types])
    rep_local = np.zeros(len(c.rep_type), np.int32)
    arrays["rep_i"] = np.stack([c.rep_type.astype(np.int32), rep_local, c.rep_atom.astype(np.int32)], axis=1)
    arrays["rep_xyz"] = c.rep_xyz
    arrays["atoms_xyz"] = c.atoms_xyz
    arrays["atom_type"] = c.atom_type.astype(np.int32)
    if c.udvtm is not None:
        arrays["udvtm"] = c.udvtm
    write_container(path, arrays)


def nearest_node(coord: float, delta: float) -> int:
    """Nearest grid index of an atom coordinate with the reference's tie rule.

    nonlocal.cpp:54-64: round(), but an atom within 1e-12 of the midpoint
    between two nodes is assigned to the left node.
    """
    x = coord / delta
    ax = abs(x)
    r = math.floor(ax)
    n = int(r + 1 if ax - r >= 0.5 else r)  # C round(): half away from zero
    n = -n if x < 0 else n
    if abs(abs(n * delta - coord) - delta * 0.5) < 1e-12:
        n = int(math.floor(coord / delta - 1e-11))
    return n
