"""ctypes front-end of the C restatement (oracle/sq_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg, never by the library.  It builds the
``sqo_problem`` struct from a :class:`sqdft_b200.case.Case` and exposes the
restated reference functions with numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libsqoracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Problem(C.Structure):
    _fields_ = [
        ("np", C.c_int * 3), ("pnode_s", C.c_int * 3), ("nloc", C.c_int), ("fdn", C.c_int), ("npl", C.c_int),
        ("fermi_alg", C.c_int), ("delta", C.c_double), ("bet", C.c_double), ("lanczos_tol", C.c_double),
        ("fermi_tol", C.c_double), ("ncharge", C.c_double), ("coeff_lap", _dp), ("coeff_grad", _dp),
        ("veff", _dp), ("n_typ", C.c_int), ("typ_nlocc", _ip), ("typ_nproj", _ip), ("typ_lmax", _ip),
        ("typ_lloc", _ip), ("typ_denom", _dp), ("n_rep", C.c_int), ("rep_type", _ip), ("rep_atom", _ip),
        ("rep_xyz", _dp), ("udvtm", _dp), ("rep_off", C.POINTER(C.c_longlong)), ("n_atm", C.c_int),
    ]


class _Local(C.Structure):
    _fields_ = [("n_typ", C.c_int), ("typ_size", _ip), ("typ_tab", C.POINTER(_dp)), ("Z", _dp), ("n_rep", C.c_int),
                ("rep_type", _ip), ("rep_atom", _ip), ("rep_xyz", _dp), ("rep_box", _ip), ("rc_tilda", C.c_double)]


class _Psd(C.Structure):
    _fields_ = [("size", C.c_int), ("lmax", C.c_int), ("lloc", C.c_int), ("nlocc", C.c_int), ("tables", _dp)]


def _lib():
    if not LIB_PATH.exists():
        raise RuntimeError(f"oracle library missing: build it with `make -C oracle oracle` ({LIB_PATH})")
    lib = C.CDLL(str(LIB_PATH))
    P = C.POINTER(_Problem)
    lib.sqo_set_threads.argtypes = [C.c_int]
    lib.sqo_projectors.argtypes = [P, C.POINTER(_Psd), _dp]
    lib.sqo_hsub_times_vec.argtypes = [P, C.c_int, _dp, _dp]
    lib.sqo_lanczos.argtypes = [P, C.c_int, _dp, _dp]
    lib.sqo_tridiag_eigen.argtypes = [_dp, _dp, C.c_int, _dp, _dp]
    lib.sqo_moments.argtypes = [P, C.c_int, C.c_double, C.c_double, _dp]
    lib.sqo_lanczos_moments.argtypes = [P, _ip, C.c_int, _dp, _dp, _dp, _ip, _dp, _dp]
    lib.sqo_chebyshev_coeff.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int]
    lib.sqo_ne_constraint.argtypes = [P, _dp, _dp, _dp, C.c_double]
    lib.sqo_ne_constraint.restype = C.c_double
    lib.sqo_fermi_level.argtypes = [P, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _ip]
    lib.sqo_density_energy.argtypes = [P, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp]
    lib.sqo_forces_nonlocal.argtypes = [P, _ip, C.c_int, _dp, _dp, _dp, _dp]
    LP = C.POINTER(_Local)
    lib.sqo_charge_density.argtypes = [P, LP, _dp, _dp, _dp, _dp, _dp]
    lib.sqo_forces_local.argtypes = [P, LP, _dp, _dp, _dp, _dp, _dp, _dp]
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Oracle:
    """The C restatement bound to one case's inputs."""

    def __init__(self, case, udvtm: np.ndarray | None = None, threads: int | None = None):
        self.lib = _lib()
        self.case = case
        c = case
        self._keep = []
        self.coeff_lap = np.ascontiguousarray(c.coeff_lap, np.float64)
        self.coeff_grad = np.ascontiguousarray(c.coeff_grad, np.float64)
        self.veff = np.ascontiguousarray(c.veff, np.float64)
        self.typ_nlocc = np.array([t.nlocc for t in c.types], np.int32)
        self.typ_nproj = np.array([t.nproj for t in c.types], np.int32)
        self.typ_lmax = np.array([t.lmax for t in c.types], np.int32)
        self.typ_lloc = np.array([t.lloc for t in c.types], np.int32)
        self.typ_denom = np.ascontiguousarray(np.array([t.denom for t in c.types]).reshape(-1), np.float64)
        self.rep_type = np.ascontiguousarray(c.rep_type, np.int32)
        self.rep_atom = np.ascontiguousarray(c.rep_atom, np.int32)
        self.rep_xyz = np.ascontiguousarray(c.rep_xyz, np.float64)
        self.rep_off = np.ascontiguousarray(c.replica_offsets(), np.int64)
        total = int(sum(c.types[t].nproj * c.types[t].ball ** 3 for t in c.rep_type))
        if udvtm is None:
            udvtm = c.udvtm if c.udvtm is not None else np.zeros(total)
        self.udvtm = np.ascontiguousarray(udvtm, np.float64)
        if self.udvtm.size < total:
            raise ValueError("projector table size mismatch")
        p = _Problem()
        p.np[:] = list(c.np_)
        p.pnode_s[:] = list(c.pnode_s)
        p.nloc, p.fdn, p.npl, p.fermi_alg = c.nloc, c.fdn, c.npl, c.fermi_alg
        p.delta, p.bet, p.lanczos_tol, p.fermi_tol, p.ncharge = c.delta, c.bet, c.lanczos_tol, c.fermi_tol, c.ncharge
        p.coeff_lap, p.coeff_grad, p.veff = _d(self.coeff_lap), _d(self.coeff_grad), _d(self.veff)
        p.n_typ = len(c.types)
        p.typ_nlocc, p.typ_nproj, p.typ_lmax, p.typ_lloc = (_i(self.typ_nlocc), _i(self.typ_nproj),
                                                             _i(self.typ_lmax), _i(self.typ_lloc))
        p.typ_denom = _d(self.typ_denom)
        p.n_rep = len(self.rep_type)
        p.rep_type, p.rep_atom, p.rep_xyz = _i(self.rep_type), _i(self.rep_atom), _d(self.rep_xyz)
        p.udvtm = _d(self.udvtm)
        p.rep_off = self.rep_off.ctypes.data_as(C.POINTER(C.c_longlong))
        p.n_atm = c.n_atm
        self.p = p
        self.lib.sqo_set_threads(threads if threads else max(1, os.cpu_count() or 1))

    # -- projectors ---------------------------------------------------------
    def projectors(self) -> np.ndarray:
        c = self.case
        tabs = [np.ascontiguousarray(t.tables, np.float64) for t in c.types]
        psd = (_Psd * len(c.types))()
        for k, t in enumerate(c.types):
            psd[k].size, psd[k].lmax, psd[k].lloc, psd[k].nlocc = t.tables.shape[1], t.lmax, t.lloc, t.nlocc
            psd[k].tables = _d(tabs[k])
        out = np.zeros_like(self.udvtm)
        rc = self.lib.sqo_projectors(C.byref(self.p), psd, _d(out))
        if rc != 0:
            raise RuntimeError("spline out of range in projector evaluation")
        return out

    # -- kernels ------------------------------------------------------------
    def hsub_times_vec(self, node: int, v: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64).reshape(-1)
        out = np.zeros_like(v)
        self.lib.sqo_hsub_times_vec(C.byref(self.p), int(node), _d(v), _d(out))
        return out

    def lanczos(self, node: int):
        lo, hi = C.c_double(), C.c_double()
        it = self.lib.sqo_lanczos(C.byref(self.p), int(node), C.byref(lo), C.byref(hi))
        return lo.value, hi.value, it

    def lanczos_moments(self, nodes=None):
        c = self.case
        n = c.n_nodes
        nodes = np.arange(n, dtype=np.int32) if nodes is None else np.ascontiguousarray(nodes, np.int32)
        chi, zee = np.zeros(n), np.zeros(n)
        lmin, lmax = np.zeros(n), np.zeros(n)
        rpj = np.zeros((n, c.npl + 1))
        its = np.zeros(n, np.int32)
        self.lib.sqo_lanczos_moments(C.byref(self.p), _i(nodes), len(nodes), _d(chi), _d(zee), _d(rpj), _i(its),
                                     _d(lmin), _d(lmax))
        return dict(chi=chi, zee=zee, rho_pj=rpj, lanczos_iters=its, lmin=lmin, lmax=lmax)

    def chebyshev_coeff(self, lambda_fp: float, bet: float, kind: int = 0) -> np.ndarray:
        out = np.zeros(self.case.npl + 1)
        self.lib.sqo_chebyshev_coeff(self.case.npl, lambda_fp, bet, _d(out), kind)
        return out

    def ne_constraint(self, m, lam: float) -> float:
        return self.lib.sqo_ne_constraint(C.byref(self.p), _d(m["chi"]), _d(m["zee"]), _d(m["rho_pj"]), lam)

    def fermi_level(self, m, scf_iter: int = 1, lambda_warm: float = 0.0):
        lam, it = C.c_double(), C.c_int()
        rc = self.lib.sqo_fermi_level(C.byref(self.p), _d(m["chi"]), _d(m["zee"]), _d(m["rho_pj"]), scf_iter,
                                      lambda_warm, float(m["lmin"].min()), float(m["lmax"].max()),
                                      C.byref(lam), C.byref(it))
        if rc != 0:
            raise RuntimeError(f"Fermi level solve failed ({rc})")
        return lam.value, it.value

    def density_energy(self, m, lam: float):
        c = self.case
        rho = np.zeros(c.n_nodes)
        ci = np.zeros((c.n_nodes, c.npl + 1))
        ebs, eent = C.c_double(), C.c_double()
        rc = self.lib.sqo_density_energy(C.byref(self.p), _d(m["chi"]), _d(m["zee"]), _d(m["rho_pj"]), lam,
                                         _d(rho), _d(ci), C.byref(ebs), C.byref(eent))
        return dict(rho=rho.reshape(c.np_[2], c.np_[1], c.np_[0]), Ci=ci, Ebs=ebs.value, Eent=eent.value,
                    status=rc)

    def forces_nonlocal(self, chi, zee, ci, nodes=None) -> np.ndarray:
        c = self.case
        nodes = np.arange(c.n_nodes, dtype=np.int32) if nodes is None else np.ascontiguousarray(nodes, np.int32)
        f = np.zeros((c.n_atm, 3))
        self.lib.sqo_forces_nonlocal(C.byref(self.p), _i(nodes), len(nodes), _d(chi), _d(zee),
                                     _d(np.ascontiguousarray(ci)), _d(f))
        return f

    def spectral_quadrature(self, scf_iter: int | None = None, lambda_warm: float | None = None):
        """ClenshawCurtisSpectralQuadrature (sq.cpp:377-834) end to end."""
        c = self.case
        m = self.lanczos_moments()
        lam, it = self.fermi_level(m, c.scf_iter if scf_iter is None else scf_iter,
                                   c.lambda_f if lambda_warm is None else lambda_warm)
        out = self.density_energy(m, lam)
        out.update(m)
        out["lambda_f"] = lam
        out["fermi_iters"] = it
        return out


class LocalOracle:
    """ChargeDensity (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315)
    of the C restatement on one block.  ``loc`` is a
    :class:`sqdft_b200.pseudocharge.LocalAtoms`; the grid comes from ``grid``,
    an object with ``np_``, ``pnode_s``, ``fdn``, ``delta``, ``coeff_lap``,
    ``coeff_grad`` and ``n_atm``."""

    def __init__(self, grid, loc):
        self.lib = _lib()
        self.grid, self.loc = grid, loc
        self.coeff_lap = np.ascontiguousarray(grid.coeff_lap, np.float64)
        self.coeff_grad = np.ascontiguousarray(grid.coeff_grad, np.float64)
        p = _Problem()
        p.np[:] = list(grid.np_)
        p.pnode_s[:] = list(grid.pnode_s)
        p.fdn, p.delta, p.n_atm = grid.fdn, grid.delta, grid.n_atm
        p.coeff_lap, p.coeff_grad = _d(self.coeff_lap), _d(self.coeff_grad)
        self.p = p
        self.tabs = [np.ascontiguousarray(t, np.float64) for t in loc.tables]
        self.sizes = np.array([t.shape[1] for t in self.tabs], np.int32)
        self.tab_ptrs = (_dp * len(self.tabs))(*[_d(t) for t in self.tabs])
        self.Z = np.ascontiguousarray(loc.Z, np.float64)
        self.rep_type = np.ascontiguousarray(loc.rep_type, np.int32)
        self.rep_atom = np.ascontiguousarray(loc.rep_atom, np.int32)
        self.rep_xyz = np.ascontiguousarray(loc.rep_xyz, np.float64)
        self.rep_box = np.ascontiguousarray(loc.rep_box, np.int32)
        L = _Local()
        L.n_typ, L.typ_size, L.typ_tab, L.Z = len(self.tabs), _i(self.sizes), self.tab_ptrs, _d(self.Z)
        L.n_rep = len(self.rep_type)
        L.rep_type, L.rep_atom, L.rep_xyz, L.rep_box = (_i(self.rep_type), _i(self.rep_atom), _d(self.rep_xyz),
                                                        _i(self.rep_box))
        L.rc_tilda = loc.rc_tilda
        self.L = L

    def _shape(self):
        return tuple(self.grid.np_[::-1])

    def charge_density(self) -> dict:
        sh = self._shape()
        b, bt, vc, ra = (np.zeros(sh) for _ in range(4))
        scal = np.zeros(7)
        rc = self.lib.sqo_charge_density(C.byref(self.p), C.byref(self.L), _d(b), _d(bt), _d(vc), _d(ra), _d(scal))
        if rc != 0:
            raise RuntimeError("spline out of range in ChargeDensity")
        return dict(b=b, b_tilda=bt, vc=vc, rho_at=ra, Eself=scal[0], Ncharge=scal[1], Nelectron_at=scal[2],
                    Ncharge_tilda=scal[3], Eself_tilda=scal[4], Vcon=scal[5], Ecorr=scal[6])

    def forces_local(self, phi, vc, b, b_tilda):
        n = self.grid.n_atm
        floc, fcorr = np.zeros((n, 3)), np.zeros((n, 3))
        arrs = [np.ascontiguousarray(a, np.float64) for a in (phi, vc, b, b_tilda)]
        rc = self.lib.sqo_forces_local(C.byref(self.p), C.byref(self.L), *[_d(a) for a in arrs], _d(floc), _d(fcorr))
        if rc != 0:
            raise RuntimeError("spline out of range in ForcesLocal")
        return floc, fcorr
