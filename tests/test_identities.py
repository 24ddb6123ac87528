"""The two identities the fast SQ forms rest on, checked on the CPU with the
same recurrences the kernels use (no GPU needed).

* Gauss-quadrature moments (the Lanczos-quadrature form, `lanczos_quadrature`
  in sqdft_b200/csrc/sqb_node.cuh): a Lanczos run of m steps from e_c gives a
  tridiagonal T_m with e_c^T T_j(Ht) e_c = e_1^T T_j(That_m) e_1 for j <= 2m - 1.
* Re-expansion (the defect check, `rho_at_bounds` in sqb_fermi.cu): the
  Chebyshev moments at bounds (chi', zee') follow exactly from those at
  (chi, zee) through P_j+1 = 2 (al X + be) P_j - P_j-1.
"""
from __future__ import annotations

import numpy as np


def _hamiltonian(n=80, seed=3):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n))
    h = 0.5 * (a + a.T) + np.diag(rng.uniform(-2.0, 4.0, n))
    return h


def _moments(h, e, chi, zee, npl):
    """mu_j = e^T T_j((H - chi)/zee) e by the three-term recurrence (sq.cpp:564-655)."""
    ht = (h - chi * np.eye(len(h))) / zee
    t0, t1 = e.copy(), ht @ e
    mu = [e @ t0, e @ t1]
    for _ in range(2, npl + 1):
        t0, t1 = t1, 2 * ht @ t1 - t0
        mu.append(e @ t1)
    return np.array(mu)


def _bounds(h, margin=1e-3):
    w = np.linalg.eigvalsh(h)
    lo, hi = w[0] - margin, w[-1] + margin
    return 0.5 * (hi + lo), 0.5 * (hi - lo)


def test_gauss_quadrature_moments():
    """The kernel's recurrence on the m x m tridiagonal gives the moments of H
    itself for every j <= 2m - 1 (full reorthogonalisation here, so the
    identity is tested without rounding drift)."""
    h = _hamiltonian()
    n, npl = len(h), 24
    e = np.zeros(n)
    e[n // 2] = 1.0
    chi, zee = _bounds(h)
    m = npl // 2 + 1
    q = np.zeros((n, m))
    q[:, 0] = e
    al, be = np.zeros(m), np.zeros(m)
    for k in range(m):
        w = h @ q[:, k]
        al[k] = q[:, k] @ w
        w -= q[:, : k + 1] @ (q[:, : k + 1].T @ w)
        w -= q[:, : k + 1] @ (q[:, : k + 1].T @ w)
        if k + 1 < m:
            be[k] = np.linalg.norm(w)
            q[:, k + 1] = w / be[k]
    # the kernel's recurrence: v_j+1 = 2 That v_j - v_j-1 on k-vectors, mu_j = v_j[0]
    d, off = (al - chi) / zee, be[: m - 1] / zee

    def that(v):
        r = d * v
        r[1:] += off * v[:-1]
        r[:-1] += off * v[1:]
        return r

    v0 = np.zeros(m)
    v0[0] = 1.0
    v1 = that(v0)
    mu_q = [v0[0], v1[0]]
    for _ in range(1, npl):
        v0, v1 = v1, 2 * that(v1) - v0
        mu_q.append(v1[0])
    mu = _moments(h, e, chi, zee, npl)
    assert np.abs(np.array(mu_q) - mu).max() <= 1e-11
    # and one order past 2m - 1 the identity no longer holds
    far = _moments(h, e, chi, zee, 2 * m + 2)
    v0[:] = 0.0
    v0[0] = 1.0
    v1 = that(v0)
    for _ in range(1, 2 * m + 2):
        v0, v1 = v1, 2 * that(v1) - v0
    assert abs(v1[0] - far[-1]) > 1e-8


def test_reexpansion_to_other_bounds():
    """The defect check's re-expansion reproduces the moments at moved bounds."""
    h = _hamiltonian(seed=5)
    n, npl = len(h), 48
    e = np.zeros(n)
    e[7] = 1.0
    chi, zee = _bounds(h)
    mu = _moments(h, e, chi, zee, npl)
    for dchi, dzee in ((-0.002, 0.002), (0.002, 0.002), (0.01, -0.003)):
        chi2, zee2 = chi + dchi, zee + dzee
        alpha, beta = zee / zee2, (chi - chi2) / zee2
        k = npl + 1
        pm = np.zeros(k)
        pm[0] = 1.0
        pc = np.zeros(k)
        pc[0], pc[1] = beta, alpha
        mu2 = [mu[0], alpha * mu[1] + beta * mu[0]]
        for _ in range(1, npl):
            up = np.append(pc[1:], 0.0)
            down = np.insert(pc[:-1], 0, 0.0)
            xp = 0.5 * (down + up)
            xp[0] = 0.5 * pc[1]
            xp[1] = pc[0] + 0.5 * pc[2]
            pn = 2 * (alpha * xp + beta * pc) - pm
            mu2.append(pn @ mu)
            pm, pc = pc, pn
        direct = _moments(h, e, chi2, zee2, npl)
        assert np.abs(np.array(mu2) - direct).max() <= 1e-10
