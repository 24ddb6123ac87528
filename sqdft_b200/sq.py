"""Python host mirror of SQDFT's SQ entry points over the sqdft_b200 C ABI.

``SQState`` carries the DS_SQ fields the SQ step reads and writes
(ds_sq.h:128-238) as numpy arrays; the functions ``NonlocalProjectors``,
``ClenshawCurtisSpectralQuadrature`` and ``ForcesNonLocal`` fill the same
fields as their reference namesakes (nonlocal.cpp:317, sq.cpp:377,
forces.cpp:318).  All computation runs in the CUDA library
(``sqdft_b200/_build/libsqdft_b200.so``); there is no CPU path, and a missing
library is an error.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .case import Case

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("SQDFT_B200_LIB", HERE / "_build" / "libsqdft_b200.so"))

SQB_FP64 = 0
SQB_FP32_MIXED = 1
SQB_FP64_LANCZOS_QUAD = 2
SQB_SUM, SQB_MIN, SQB_MAX = 0, 1, 2
SQB_KERNEL_AUTO, SQB_KERNEL_PLANE, SQB_KERNEL_SWEEP = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# Names of the functions include/sqdft_b200.h declares (checked by the tests).
EXPORTS = [
    "sqb_create", "sqb_destroy", "sqb_set_precision", "sqb_set_allreduce", "sqb_set_launch", "sqb_set_veff",
    "sqb_set_atoms", "sqb_nonlocal_projectors", "sqb_set_projectors", "sqb_hsub_times_vec",
    "sqb_lanczos_moments", "sqb_ne_constraint", "sqb_fermi_level", "sqb_density_energy",
    "sqb_spectral_quadrature", "sqb_forces_nonlocal", "sqb_get_stats", "sqb_status_string", "sqb_version",
    "sqb_lanczos_moments_noalloc", "sqb_moments_at", "sqb_moments_vjp", "sqb_autotune",
    "sqb_set_graph", "sqb_set_mixed_lanczos", "sqb_set_defect_check", "sqb_lanczos_moments_nodes",
    "sqb_set_node_kernel", "sqb_set_veff_device", "sqb_test_stage_wait", "sqb_density_loss",
    "sqb_density_loss_vjp", "sqb_set_sweep_rows", "sqb_autotune_sweep", "sqb_set_local_atoms",
    "sqb_charge_density", "sqb_forces_local",
]


class SqbLocalSpecies(C.Structure):
    _fields_ = [("size", C.c_int), ("Z", C.c_double), ("tables", _dp)]


class SqbGrid(C.Structure):
    _fields_ = [("np", C.c_int * 3), ("pnode_s", C.c_int * 3), ("n_int", C.c_int * 3), ("nloc", C.c_int),
                ("fdn", C.c_int), ("npl", C.c_int), ("fermi_alg", C.c_int), ("delta", C.c_double),
                ("bet", C.c_double), ("lanczos_tol", C.c_double), ("fermi_tol", C.c_double),
                ("ncharge", C.c_double), ("coeff_lap", C.c_double * 8), ("coeff_grad", C.c_double * 8)]


class SqbSpecies(C.Structure):
    _fields_ = [("natm", C.c_int), ("lmax", C.c_int), ("lloc", C.c_int), ("nlocc", C.c_int), ("size", C.c_int),
                ("rc", C.c_double), ("denom", C.c_double * 4), ("tables", _dp)]


class SqbStats(C.Structure):
    _fields_ = [("ms_lanczos_moments", C.c_double), ("ms_fermi", C.c_double), ("ms_density", C.c_double),
                ("ms_forces", C.c_double), ("ms_projectors", C.c_double), ("matvecs", C.c_longlong),
                ("lanczos_iters", C.c_longlong), ("window_points", C.c_longlong), ("proj_points", C.c_longlong),
                ("proj_points_cheb", C.c_longlong),
                ("fermi_iters", C.c_int), ("max_lanczos_iters", C.c_int), ("kernel_launches", C.c_int),
                ("ms_vjp", C.c_double), ("ms_defect", C.c_double), ("defect_nodes", C.c_longlong),
                ("lanczos_maxiter_nodes", C.c_longlong), ("proj_points_window", C.c_longlong),
                ("node_kernel", C.c_int), ("ms_charge_density", C.c_double), ("ms_forces_local", C.c_double)]


ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, _dp, C.c_int, C.c_int, C.c_void_p)


class SQBError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {status_string(code)} (status {code})")
        self.code = code


_LIB = None


def library() -> C.CDLL:
    """Load the CUDA library; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"sqdft_b200 CUDA library not built: {LIB_PATH} (run python -m sqdft_b200.build)")
        lib = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        lib.sqb_create.argtypes = [C.POINTER(SqbGrid), C.c_int, C.POINTER(P)]
        lib.sqb_destroy.argtypes = [P]
        lib.sqb_set_precision.argtypes = [P, C.c_int]
        lib.sqb_set_mixed_lanczos.argtypes = [P, C.c_double, C.c_double]
        lib.sqb_set_defect_check.argtypes = [P, C.c_double]
        lib.sqb_set_allreduce.argtypes = [P, ALLREDUCE_FN, C.c_void_p]
        lib.sqb_set_launch.argtypes = [P, C.c_int, C.c_int]
        lib.sqb_set_veff.argtypes = [P, _dp]
        lib.sqb_set_atoms.argtypes = [P, C.c_int, C.POINTER(SqbSpecies), C.c_int, _ip, _ip, _dp, C.c_int]
        lib.sqb_nonlocal_projectors.argtypes = [P, _dp]
        lib.sqb_set_projectors.argtypes = [P, _dp]
        lib.sqb_hsub_times_vec.argtypes = [P, C.c_int, _ip, _dp, _dp]
        lib.sqb_lanczos_moments.argtypes = [P, _dp, _dp, _dp, _ip, _dp, _dp]
        lib.sqb_lanczos_moments_nodes.argtypes = [P, C.c_int, _ip, _dp, _dp, _dp, _ip]
        lib.sqb_ne_constraint.argtypes = [P, C.c_double, _dp]
        lib.sqb_fermi_level.argtypes = [P, C.c_int, C.c_double, _dp, _ip]
        lib.sqb_density_energy.argtypes = [P, C.c_double, _dp, _dp, _dp, _dp]
        lib.sqb_spectral_quadrature.argtypes = [P, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.sqb_forces_nonlocal.argtypes = [P, _dp, _dp, _dp, _dp]
        lib.sqb_get_stats.argtypes = [P, C.POINTER(SqbStats), C.c_size_t]
        lib.sqb_lanczos_moments_noalloc.argtypes = [P, C.c_int, _ip, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.sqb_moments_at.argtypes = [P, _dp, _dp, _dp]
        lib.sqb_autotune.argtypes = [P, C.c_int, _ip, _dp]
        lib.sqb_set_graph.argtypes = [P, C.c_int]
        lib.sqb_set_node_kernel.argtypes = [P, C.c_int]
        lib.sqb_set_veff_device.argtypes = [P, C.c_void_p]
        lib.sqb_test_stage_wait.argtypes = [P, C.c_uint, C.c_double]
        lib.sqb_density_loss.argtypes = [P, _dp, _dp]
        lib.sqb_set_sweep_rows.argtypes = [P, C.c_int]
        lib.sqb_autotune_sweep.argtypes = [P, C.c_int, _ip, _dp]
        lib.sqb_density_loss_vjp.argtypes = [P, _dp, C.c_int, C.c_double, _dp, _dp]
        lib.sqb_moments_vjp.argtypes = [P, _dp, _dp, _dp]
        lib.sqb_set_local_atoms.argtypes = [P, C.c_int, C.POINTER(SqbLocalSpecies), C.c_int, _ip, _ip, _dp, _ip,
                                            C.c_double, C.c_int]
        lib.sqb_charge_density.argtypes = [P, _dp, _dp, _dp, _dp, _dp]
        lib.sqb_forces_local.argtypes = [P, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.sqb_status_string.argtypes = [C.c_int]
        lib.sqb_status_string.restype = C.c_char_p
        lib.sqb_version.restype = C.c_char_p
        _LIB = lib
    return _LIB


def status_string(code: int) -> str:
    return library().sqb_status_string(code).decode()


def _check(code: int, where: str) -> None:
    if code != 0:
        raise SQBError(code, where)


def _d(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_ip)


class Context:
    """One sqb_ctx: a processor block of the grid resident on one GPU."""

    def __init__(self, case: Case, device: int = 0, precision: int = SQB_FP64, allreduce=None):
        self.lib = library()
        self.case = case
        g = SqbGrid()
        g.np[:] = list(case.np_)
        g.pnode_s[:] = list(case.pnode_s)
        g.n_int[:] = list(case.n_int)
        g.nloc, g.fdn, g.npl, g.fermi_alg = case.nloc, case.fdn, case.npl, case.fermi_alg
        g.delta, g.bet, g.lanczos_tol, g.fermi_tol, g.ncharge = (case.delta, case.bet, case.lanczos_tol,
                                                                case.fermi_tol, case.ncharge)
        for k in range(case.fdn + 1):
            g.coeff_lap[k] = float(case.coeff_lap[k])
            g.coeff_grad[k] = float(case.coeff_grad[k])
        self.ptr = C.c_void_p()
        _check(self.lib.sqb_create(C.byref(g), device, C.byref(self.ptr)), "sqb_create")
        self._cb = None
        if allreduce is not None:
            self.set_allreduce(allreduce)
        self.set_precision(precision)
        self._keep = []
        self.local_shape = tuple(case.np_[::-1])
        self.set_veff(case.veff)
        self.set_atoms(case)

    def close(self):
        if self.ptr:
            self.lib.sqb_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- set-up --------------------------------------------------------------
    def set_precision(self, precision: int):
        _check(self.lib.sqb_set_precision(self.ptr, precision), "sqb_set_precision")

    def set_mixed_lanczos(self, tol: float = 0.0, checkerboard: float = 0.5):
        """Lanczos of the FP32-mixed path: stop and margin in Ha (0: the grid's
        lanczos_tol) and the checkerboard weight of the start vector."""
        _check(self.lib.sqb_set_mixed_lanczos(self.ptr, float(tol), float(checkerboard)), "sqb_set_mixed_lanczos")

    def set_defect_check(self, budget: float = 1e-6):
        """Turn on the fast forms' defect check with this density budget (0: off, the default)."""
        _check(self.lib.sqb_set_defect_check(self.ptr, float(budget)), "sqb_set_defect_check")

    def set_launch(self, ctas_per_sm: int = 0, cols_per_thread: int = 0):
        _check(self.lib.sqb_set_launch(self.ptr, ctas_per_sm, cols_per_thread), "sqb_set_launch")

    def set_node_kernel(self, kernel: int = SQB_KERNEL_AUTO):
        """Kernel of the Lanczos bounds and moments: auto, plane-streaming or sweep."""
        _check(self.lib.sqb_set_node_kernel(self.ptr, int(kernel)), "sqb_set_node_kernel")

    def set_graph(self, on=True):
        """sqb_set_graph: False/0 plain launches, True/1 the node-kernel sequence from a graph,
        2 the whole SQ step (Fermi solve included) as one graph."""
        _check(self.lib.sqb_set_graph(self.ptr, int(on)), "sqb_set_graph")

    def autotune(self, sample: int = 0):
        """Pick the node kernel's layout by timing a node sample; returns the
        chosen layout and {layout: ms} for the layouts that apply."""
        chosen = C.c_int()
        ms = np.zeros(3)
        _check(self.lib.sqb_autotune(self.ptr, sample, C.byref(chosen), _d(ms)), "sqb_autotune")
        return chosen.value, {k: v for k, v in zip((1, 2, -2), ms) if v >= 0}

    def set_allreduce(self, fn):
        """fn(values: np.ndarray, op: int) -> None, reducing in place across ranks."""

        def cb(ptr, count, op, user):
            try:
                arr = np.ctypeslib.as_array(ptr, shape=(count,))
                fn(arr, op)
                return 0
            except Exception:  # reported to the library as a failed reduction
                return 1

        self._cb = ALLREDUCE_FN(cb)
        _check(self.lib.sqb_set_allreduce(self.ptr, self._cb, None), "sqb_set_allreduce")

    def _veff_ext_shape(self) -> tuple[int, int, int]:
        """Veff block with its halo: [np_z + 2nloc][np_y + 2nloc][np_x + 2nloc]."""
        c, nl = self.case, self.case.nloc
        return (c.np_[2] + 2 * nl, c.np_[1] + 2 * nl, c.np_[0] + 2 * nl)

    def set_veff(self, veff_ext: np.ndarray):
        v = np.ascontiguousarray(veff_ext, np.float64)
        if v.size != int(np.prod(self._veff_ext_shape())):
            raise ValueError(f"Veff with halo must have shape {self._veff_ext_shape()}, got {v.shape}")
        _check(self.lib.sqb_set_veff(self.ptr, _d(v)), "sqb_set_veff")

    def set_sweep_rows(self, rows: int = 0):
        """sqb_set_sweep_rows: window rows per sweep-kernel thread (0 automatic, 2, 3)."""
        _check(self.lib.sqb_set_sweep_rows(self.ptr, int(rows)), "sqb_set_sweep_rows")

    def autotune_sweep(self, sample: int = 0):
        """sqb_autotune_sweep: (rows chosen, [ms with 2 rows, ms with 3 rows])."""
        rows = C.c_int()
        ms = np.zeros(2)
        _check(self.lib.sqb_autotune_sweep(self.ptr, int(sample), C.byref(rows), _d(ms)), "sqb_autotune_sweep")
        return rows.value, ms

    def density_loss(self, w: np.ndarray) -> float:
        """sqb_density_loss: sum_p w_p rho_p of the last density."""
        w = np.ascontiguousarray(w, np.float64).reshape(-1)
        out = C.c_double()
        _check(self.lib.sqb_density_loss(self.ptr, _d(w), C.byref(out)), "sqb_density_loss")
        return out.value

    def density_loss_vjp(self, w: np.ndarray, fixed_electrons: bool = True, grad_l: float = 1.0,
                         atoms: bool = False):
        """sqb_density_loss_vjp: grad_l dL/dVeff (Veff block with halo), and dL/dR with atoms=True."""
        w = np.ascontiguousarray(w, np.float64).reshape(-1)
        g = np.zeros(self._veff_ext_shape())
        ga = np.zeros((self.case.n_atm, 3)) if atoms else None
        _check(self.lib.sqb_density_loss_vjp(self.ptr, _d(w), int(bool(fixed_electrons)), float(grad_l), _d(g),
                                             _d(ga)), "sqb_density_loss_vjp")
        return (g, ga) if atoms else g

    def test_stage_wait(self, extra_bytes: int = 0, wait_ms: float = 0.0):
        """sqb_test_stage_wait (test hook of the plane-streaming kernel's bounded waits)."""
        _check(self.lib.sqb_test_stage_wait(self.ptr, int(extra_bytes), float(wait_ms)), "sqb_test_stage_wait")

    def set_veff_device(self, ptr: int):
        """sqb_set_veff_device: Veff with halo from a device pointer (e.g. a torch tensor's data_ptr())."""
        _check(self.lib.sqb_set_veff_device(self.ptr, C.c_void_p(ptr)), "sqb_set_veff_device")

    def set_atoms(self, case: Case):
        types = (SqbSpecies * max(1, len(case.types)))()
        tabs = []
        for k, t in enumerate(case.types):
            tab = np.ascontiguousarray(t.tables, np.float64)
            tabs.append(tab)
            types[k].natm, types[k].lmax, types[k].lloc, types[k].nlocc = t.natm, t.lmax, t.lloc, t.nlocc
            types[k].size = tab.shape[1]
            types[k].rc = t.rc
            types[k].denom[:] = [float(x) for x in t.denom]
            types[k].tables = _d(tab)
        rt = np.ascontiguousarray(case.rep_type, np.int32)
        ra = np.ascontiguousarray(case.rep_atom, np.int32)
        rx = np.ascontiguousarray(case.rep_xyz, np.float64)
        _check(self.lib.sqb_set_atoms(self.ptr, len(case.types), types, len(rt), _i(rt), _i(ra), _d(rx), case.n_atm),
               "sqb_set_atoms")
        self._keep = tabs

    def nonlocal_projectors(self, copy_out: bool = False) -> np.ndarray | None:
        out = np.zeros(self.table_size()) if copy_out else None
        _check(self.lib.sqb_nonlocal_projectors(self.ptr, _d(out)), "sqb_nonlocal_projectors")
        return out

    def set_projectors(self, udvtm: np.ndarray):
        u = np.ascontiguousarray(udvtm, np.float64)
        _check(self.lib.sqb_set_projectors(self.ptr, _d(u)), "sqb_set_projectors")

    def table_size(self) -> int:
        c = self.case
        return int(sum(c.types[t].nproj * c.types[t].ball ** 3 for t in c.rep_type))

    # -- kernels ---------------------------------------------------------------
    def hsub_times_vec(self, nodes, vin: np.ndarray) -> np.ndarray:
        nodes = np.ascontiguousarray(nodes, np.int32)
        vin = np.ascontiguousarray(vin, np.float64).reshape(len(nodes), -1)
        out = np.zeros_like(vin)
        _check(self.lib.sqb_hsub_times_vec(self.ptr, len(nodes), _i(nodes), _d(vin), _d(out)), "sqb_hsub_times_vec")
        return out

    def lanczos_moments(self):
        c = self.case
        n = c.n_nodes
        r = dict(chi=np.zeros(n), zee=np.zeros(n), rho_pj=np.zeros((n, c.npl + 1)),
                 lanczos_iters=np.zeros(n, np.int32), lmin=np.zeros(n), lmax=np.zeros(n))
        _check(self.lib.sqb_lanczos_moments(self.ptr, _d(r["chi"]), _d(r["zee"]), _d(r["rho_pj"]),
                                            _i(r["lanczos_iters"]), _d(r["lmin"]), _d(r["lmax"])),
               "sqb_lanczos_moments")
        return r

    def lanczos_moments_nodes(self, nodes):
        """Bounds and moments of the listed nodes only (arrays per listed node)."""
        nodes = np.ascontiguousarray(nodes, np.int32)
        k = len(nodes)
        r = dict(chi=np.zeros(k), zee=np.zeros(k), rho_pj=np.zeros((k, self.case.npl + 1)),
                 lanczos_iters=np.zeros(k, np.int32))
        _check(self.lib.sqb_lanczos_moments_nodes(self.ptr, k, _i(nodes), _d(r["chi"]), _d(r["zee"]),
                                                  _d(r["rho_pj"]), _i(r["lanczos_iters"])),
               "sqb_lanczos_moments_nodes")
        return r

    def moments_at(self, chi: np.ndarray, zee: np.ndarray) -> np.ndarray:
        """Chebyshev moments rho_pj [nnode][npl+1] with the given spectral bounds."""
        c = self.case
        chi = np.ascontiguousarray(chi, np.float64)
        zee = np.ascontiguousarray(zee, np.float64)
        rho_pj = np.zeros((c.n_nodes, c.npl + 1))
        _check(self.lib.sqb_moments_at(self.ptr, _d(chi), _d(zee), _d(rho_pj)), "sqb_moments_at")
        return rho_pj

    def moments_vjp(self, g_mu: np.ndarray, atoms: bool = False):
        """dL/dVeff on the Veff block with halo for dL/drho_pj = g_mu (bounds of the
        last moments held fixed); with atoms=True also dL/dR [n_atm][3]."""
        c = self.case
        g = np.ascontiguousarray(g_mu, np.float64).reshape(c.n_nodes, c.npl + 1)
        out = np.zeros(self._veff_ext_shape())
        gat = np.zeros((c.n_atm, 3)) if atoms else None
        _check(self.lib.sqb_moments_vjp(self.ptr, _d(g), _d(out), _d(gat)), "sqb_moments_vjp")
        return (out, gat) if atoms else out

    def ne_constraint(self, lam: float) -> float:
        v = C.c_double()
        _check(self.lib.sqb_ne_constraint(self.ptr, lam, C.byref(v)), "sqb_ne_constraint")
        return v.value

    def fermi_level(self, scf_iter: int = 1, lambda_warm: float = 0.0):
        lam, it = C.c_double(), C.c_int()
        _check(self.lib.sqb_fermi_level(self.ptr, scf_iter, lambda_warm, C.byref(lam), C.byref(it)),
               "sqb_fermi_level")
        return lam.value, it.value

    def density_energy(self, lam: float):
        c = self.case
        rho = np.zeros(c.n_nodes)
        ci = np.zeros((c.n_nodes, c.npl + 1))
        ebs, eent = C.c_double(), C.c_double()
        _check(self.lib.sqb_density_energy(self.ptr, lam, _d(rho), _d(ci), C.byref(ebs), C.byref(eent)),
               "sqb_density_energy")
        return dict(rho=rho.reshape(c.np_[2], c.np_[1], c.np_[0]), Ci=ci, Ebs=ebs.value, Eent=eent.value)

    def spectral_quadrature(self, scf_iter: int, lambda_f: float, outputs: bool = True):
        """sqb_spectral_quadrature; with outputs=False only the scalars come back."""
        c = self.case
        n = c.n_nodes
        lam = C.c_double(lambda_f)
        ebs, eent = C.c_double(), C.c_double()
        arr = {}
        if outputs:
            arr = dict(rho=np.zeros(n), rho_pj=np.zeros((n, c.npl + 1)), Ci=np.zeros((n, c.npl + 1)),
                       chi=np.zeros(n), zee=np.zeros(n))
        _check(self.lib.sqb_spectral_quadrature(self.ptr, scf_iter, C.byref(lam), _d(arr.get("rho")),
                                                _d(arr.get("rho_pj")), _d(arr.get("Ci")), _d(arr.get("chi")),
                                                _d(arr.get("zee")), C.byref(ebs), C.byref(eent)),
               "sqb_spectral_quadrature")
        if outputs:
            arr["rho"] = arr["rho"].reshape(c.np_[2], c.np_[1], c.np_[0])
        arr.update(lambda_f=lam.value, Ebs=ebs.value, Eent=eent.value)
        return arr

    def forces_nonlocal(self, chi=None, zee=None, ci=None) -> np.ndarray:
        f = np.zeros((self.case.n_atm, 3))
        args = [None, None, None]
        if chi is not None:
            args = [np.ascontiguousarray(chi, np.float64), np.ascontiguousarray(zee, np.float64),
                    np.ascontiguousarray(ci, np.float64)]
        _check(self.lib.sqb_forces_nonlocal(self.ptr, _d(args[0]), _d(args[1]), _d(args[2]), _d(f)),
               "sqb_forces_nonlocal")
        return f

    def stats(self) -> dict:
        s = SqbStats()
        _check(self.lib.sqb_get_stats(self.ptr, C.byref(s), C.sizeof(s)), "sqb_get_stats")
        return {k: getattr(s, k) for k, _ in SqbStats._fields_}

    # -- pseudocharge density and local forces ---------------------------------
    def set_local_atoms(self, loc, n_atm: int | None = None):
        """sqb_set_local_atoms with a :class:`sqdft_b200.pseudocharge.LocalAtoms`."""
        _set_local_atoms(self, loc, self.case.n_atm if n_atm is None else n_atm)

    def charge_density(self) -> dict:
        """sqb_charge_density: ChargeDensity's pseudocharge part (initialize.cpp:470-784)."""
        return _charge_density(self)

    def forces_local(self, phi, vc, b, b_tilda):
        """sqb_forces_local (forces.cpp:20-315): (floc, fcorr), [n_atm, 3] each."""
        return _forces_local(self, phi, vc, b, b_tilda)


def _set_local_atoms(ctx, loc, n_atm: int) -> None:
    tabs = [np.ascontiguousarray(t, np.float64) for t in loc.tables]
    sp = (SqbLocalSpecies * len(tabs))()
    for t, tab in enumerate(tabs):
        sp[t].size, sp[t].Z, sp[t].tables = tab.shape[1], float(loc.Z[t]), _d(tab)
    arrs = (np.ascontiguousarray(loc.rep_type, np.int32), np.ascontiguousarray(loc.rep_atom, np.int32),
            np.ascontiguousarray(loc.rep_xyz, np.float64), np.ascontiguousarray(loc.rep_box, np.int32))
    _check(ctx.lib.sqb_set_local_atoms(ctx.ptr, len(tabs), sp, len(arrs[0]), _i(arrs[0]), _i(arrs[1]), _d(arrs[2]),
                                       _i(arrs[3]), float(loc.rc_tilda), int(n_atm)), "sqb_set_local_atoms")
    ctx._local_natm = int(n_atm)


def _charge_density(ctx) -> dict:
    sh = tuple(ctx.local_shape)
    b, bt, vc, ra = (np.zeros(sh) for _ in range(4))
    scal = np.zeros(7)
    _check(ctx.lib.sqb_charge_density(ctx.ptr, _d(b), _d(bt), _d(vc), _d(ra), _d(scal)), "sqb_charge_density")
    return dict(b=b, b_tilda=bt, vc=vc, rho_at=ra, Eself=scal[0], Ncharge=scal[1], Nelectron_at=scal[2],
                Ncharge_tilda=scal[3], Eself_tilda=scal[4], Vcon=scal[5], Ecorr=scal[6])


def _forces_local(ctx, phi, vc, b, b_tilda):
    arrs = [np.ascontiguousarray(a, np.float64) for a in (phi, vc, b, b_tilda)]
    n = ctx._local_natm
    floc, fcorr = np.zeros((n, 3)), np.zeros((n, 3))
    _check(ctx.lib.sqb_forces_local(ctx.ptr, *[_d(a) for a in arrs], _d(floc), _d(fcorr)), "sqb_forces_local")
    return floc, fcorr


class LocalContext:
    """An sqb_ctx used for the pseudocharge calls only: the block grid of a
    :class:`sqdft_b200.pseudocharge.LocalGrid` and the replicas of a
    :class:`~sqdft_b200.pseudocharge.LocalAtoms` (no Veff or projectors)."""

    def __init__(self, grid, loc, device: int = 0, allreduce=None):
        self.lib = library()
        g = SqbGrid()
        g.np[:] = list(grid.np_)
        g.pnode_s[:] = list(grid.pnode_s)
        g.n_int[:] = list(grid.np_)
        g.nloc, g.fdn, g.npl, g.fermi_alg = 1, grid.fdn, 4, 1
        g.delta, g.bet, g.lanczos_tol, g.fermi_tol, g.ncharge = grid.delta, 1.0, 1e-6, 1e-6, 0.0
        for k in range(grid.fdn + 1):
            g.coeff_lap[k] = float(grid.coeff_lap[k])
            g.coeff_grad[k] = float(grid.coeff_grad[k])
        self.ptr = C.c_void_p()
        _check(self.lib.sqb_create(C.byref(g), device, C.byref(self.ptr)), "sqb_create")
        self.local_shape = tuple(grid.np_[::-1])
        self._cb = None
        if allreduce is not None:
            Context.set_allreduce(self, allreduce)
        _set_local_atoms(self, loc, grid.n_atm)

    def close(self):
        if self.ptr:
            self.lib.sqb_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def charge_density(self) -> dict:
        return _charge_density(self)

    def forces_local(self, phi, vc, b, b_tilda):
        return _forces_local(self, phi, vc, b, b_tilda)

    def stats(self) -> dict:
        s = SqbStats()
        _check(self.lib.sqb_get_stats(self.ptr, C.byref(s), C.sizeof(s)), "sqb_get_stats")
        return {k: getattr(s, k) for k, _ in SqbStats._fields_}


@dataclass
class SQState:
    """The DS_SQ fields of the SQ step (ds_sq.h:128-238) for one block."""

    case: Case
    lambda_f: float = 0.0
    rho: np.ndarray | None = None
    rho_pj: np.ndarray | None = None
    Ci: np.ndarray | None = None
    chi: np.ndarray | None = None
    zee: np.ndarray | None = None
    Ebs: float = 0.0
    Eent: float = 0.0
    fnloc: np.ndarray | None = None
    UdVtm: np.ndarray | None = None
    precision: int = SQB_FP64
    device: int = 0
    ctx: Context | None = field(default=None, repr=False)

    def context(self) -> Context:
        if self.ctx is None:
            self.ctx = Context(self.case, self.device, self.precision)
        return self.ctx


def NonlocalProjectors(s: SQState) -> None:
    """nonlocal.cpp:317-518: projector tables of every replica atom (on the GPU)."""
    s.UdVtm = s.context().nonlocal_projectors(copy_out=True)


def ClenshawCurtisSpectralQuadrature(s: SQState, scf_iter: int) -> None:
    """sq.cpp:377-834: rho, rho_pj, Ci, chi, zee, lambda_f, Ebs, Eent."""
    ctx = s.context()
    if s.UdVtm is None:
        NonlocalProjectors(s)
    out = ctx.spectral_quadrature(scf_iter, s.lambda_f)
    s.rho, s.rho_pj, s.Ci, s.chi, s.zee = out["rho"], out["rho_pj"], out["Ci"], out["chi"], out["zee"]
    s.lambda_f, s.Ebs, s.Eent = out["lambda_f"], out["Ebs"], out["Eent"]


def ForcesNonLocal(s: SQState) -> None:
    """forces.cpp:318-578: fnloc[n_atm][3] from the state's chi, zee, Ci."""
    s.fnloc = s.context().forces_nonlocal(s.chi, s.zee, s.Ci)
