"""The C restatement (oracle/) against the reference's own outputs.

The golden fixtures were produced by the reference SQDFT compiled from its
sources (tests/golden/make_golden.py).  The restatement keeps the reference's
arithmetic order, so on these inputs it must agree to rounding level; the
shipped regression log pins the Al case's Fermi level.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.pyoracle import Oracle

# tests/Al/results_Al:82 -- "Iter:1 ... Fermi energy (Ha) : 0.236781162275"
RESULTS_AL_ITER1_FERMI = 0.236781162275


@pytest.mark.parametrize("name", ["tiny", "lihs", "mid"])
def test_oracle_matches_reference(golden, name):
    case, ref = golden(name)
    orc = Oracle(case)
    out = orc.spectral_quadrature()
    assert np.abs(out["chi"] - ref["chi"]).max() <= 1e-12
    assert np.abs(out["zee"] - ref["zee"]).max() <= 1e-12
    assert np.abs(out["rho_pj"] - ref["rho_pj"]).max() <= 1e-12 * np.abs(ref["rho_pj"]).max()
    assert np.abs(out["Ci"] - ref["Ci"]).max() <= 1e-12
    assert np.abs(out["rho"] - ref["rho"]).max() <= 1e-13
    assert abs(out["lambda_f"] - ref["lambda_f"][0]) <= 1e-13
    assert abs(out["Ebs"] - ref["Ebs"][0]) <= 1e-11
    assert abs(out["Eent"] - ref["Eent"][0]) <= 1e-11
    f = orc.forces_nonlocal(out["chi"], out["zee"], out["Ci"])
    assert np.abs(f - ref["fnloc"]).max() <= 1e-12


@pytest.mark.parametrize("name", ["tiny", "lihs"])
def test_oracle_hsub_matches_reference(golden, name):
    case, ref = golden(name)
    orc = Oracle(case, threads=1)
    for node, vin, vout in zip(ref["hv_nodes"], ref["hv_in"], ref["hv_out"]):
        hv = orc.hsub_times_vec(int(node), vin)
        assert np.abs(hv - vout).max() <= 1e-13 * np.abs(vout).max()


def test_oracle_pinned_to_results_al(golden):
    """First SQ call of the shipped Al regression (tests/Al) reproduces its log."""
    case, ref = golden("al")
    orc = Oracle(case)
    m = orc.lanczos_moments()
    assert np.abs(m["chi"] - ref["chi"]).max() <= 1e-12
    lam, _ = orc.fermi_level(m, scf_iter=1)
    assert abs(lam - ref["lambda_f"][0]) <= 1e-13
    assert round(lam, 12) == RESULTS_AL_ITER1_FERMI
    out = orc.density_energy(m, lam)
    assert np.abs(out["rho"] - ref["rho"]).max() <= 1e-13


def test_tridiagonal_eigensolver_against_numpy():
    from oracle.pyoracle import _lib
    import ctypes as C

    lib = _lib()
    rng = np.random.default_rng(7)
    for n in (2, 5, 17, 60):
        d = rng.normal(size=n) * 5
        e = np.abs(rng.normal(size=n))
        lo, hi = C.c_double(), C.c_double()
        rc = lib.sqo_tridiag_eigen(d.ctypes.data_as(C.POINTER(C.c_double)), e.ctypes.data_as(C.POINTER(C.c_double)),
                                   n, C.byref(lo), C.byref(hi))
        assert rc == 0
        T = np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1)
        w = np.linalg.eigvalsh(T)
        assert abs(lo.value - w[0]) <= 1e-12 * max(1, abs(w[0]))
        assert abs(hi.value - w[-1]) <= 1e-12 * max(1, abs(w[-1]))


def test_chebyshev_coefficients_interpolate_fermi_dirac():
    """ChebyshevCoeff reproduces f at the Chebyshev-Gauss nodes (discrete orthogonality)."""
    from sqdft_b200.case import case_from_arrays  # noqa: F401  (import check)

    npl = 32
    bet, lf = 20.0, 0.1
    import ctypes as C
    from oracle.pyoracle import _lib

    lib = _lib()
    ci = np.zeros(npl + 1)
    lib.sqo_chebyshev_coeff(npl, lf, bet, ci.ctypes.data_as(C.POINTER(C.c_double)), 0)
    k = np.arange(npl + 1)
    x = np.cos(np.pi * (k + 0.5) / (npl + 1))
    T = np.cos(np.outer(np.arange(npl + 1), np.arccos(x)))
    f = 1 / (1 + np.exp(bet * (x - lf)))
    assert np.abs(ci @ T - f).max() < 1e-12
