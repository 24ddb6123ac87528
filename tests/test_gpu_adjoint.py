"""Adjoint of the SQ moments (sqb_moments_vjp) on the B200.

The gradient of a scalar L of the Chebyshev moments with respect to the grid
Veff comes from the reverse Chebyshev (Clenshaw) recursion with checkpoints;
the spectral bounds chi, zee are held fixed.  Checked against:
  * central finite differences (step 1e-4) of L through sqb_moments_at, on
    points of the periodic grid (the gradient on the Veff block with its halo
    is summed over each point's periodic images);
  * the Hellmann-Feynman identity: for the band grand potential
    Omega = sum_nodes h^3 2 sum_j d_j mu_j (d_j the Chebyshev coefficients of
    -(1/beta) log(1 + exp(-beta (e - lambda))) on the node's interval),
    dOmega/dVeff(x) = rho(x) h^3, exact for the untruncated Hamiltonian and
    approximate for the SQ windows.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(case):
    from sqdft_b200 import sq

    ctx = sq.Context(case, device=0)
    if case.udvtm is not None:
        ctx.set_projectors(case.udvtm)
    else:
        ctx.nonlocal_projectors()
    return ctx


def _images(case):
    """Extended-block index -> periodic grid index (single block, whole grid)."""
    nl = case.nloc
    nz, ny, nx = case.n_int[2], case.n_int[1], case.n_int[0]
    ez, ey, ex = case.veff.shape
    kz = (np.arange(ez) - nl) % nz
    ky = (np.arange(ey) - nl) % ny
    kx = (np.arange(ex) - nl) % nx
    return (kz[:, None, None] * ny + ky[None, :, None]) * nx + kx[None, None, :]


def _fold(case, g_ext):
    """Gradient with respect to the periodic grid Veff: sum over images."""
    n = int(np.prod(case.n_int))
    return np.bincount(_images(case).ravel(), weights=g_ext.ravel(), minlength=n)


def _perturbed(case, idx, eps):
    ext = case.veff.copy()
    ext[_images(case) == idx] += eps
    return ext


def _fd(ctx, case, chi, zee, g, idx, eps=1e-4):
    vals = []
    for s in (+1, -1):
        ctx.set_veff(_perturbed(case, idx, s * eps))
        vals.append(float(np.sum(g * ctx.moments_at(chi, zee))))
    ctx.set_veff(case.veff)
    return (vals[0] - vals[1]) / (2 * eps)


@pytest.mark.parametrize("name", ["tiny", "lihs"])
def test_vjp_matches_central_differences(golden, name):
    case, _ = golden(name)
    rng = np.random.default_rng(7)
    with _ctx(case) as ctx:
        m = ctx.lanczos_moments()
        chi, zee = m["chi"], m["zee"]
        g = rng.uniform(-1.0, 1.0, size=m["rho_pj"].shape)
        ctx.moments_at(chi, zee)
        grad = _fold(case, ctx.moments_vjp(g))
        scale = np.abs(grad).max()
        pts = rng.choice(grad.size, 4, replace=False)
        for idx in pts:
            fd = _fd(ctx, case, chi, zee, g, idx)
            assert abs(fd - grad[idx]) <= 1e-6 * scale, (idx, fd, grad[idx], scale)


def test_density_loss_gradient(golden):
    """L = sum_x w(x) rho(x) at fixed Fermi level and bounds (the loss of the
    adjoint configuration), g_mu = 2 w c_j from the density coefficients."""
    case, _ = golden("tiny")
    rng = np.random.default_rng(11)
    with _ctx(case) as ctx:
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        st = ctx.lanczos_moments()
        chi, zee = st["chi"], st["zee"]
        dens = ctx.density_energy(out["lambda_f"])
        w = rng.uniform(0.0, 1.0, size=case.n_nodes)
        sign = np.sign(2.0 * np.sum(dens["Ci"] * st["rho_pj"], axis=1))
        g = 2.0 * (w * sign)[:, None] * dens["Ci"]
        ctx.moments_at(chi, zee)
        grad = _fold(case, ctx.moments_vjp(g))
        scale = np.abs(grad).max()
        for idx in rng.choice(grad.size, 3, replace=False):
            fd = _fd(ctx, case, chi, zee, g, idx)
            assert abs(fd - grad[idx]) <= 1e-6 * scale, (idx, fd, grad[idx], scale)


def _grand_potential_coeffs(chi, zee, lam, beta, npl):
    """Chebyshev coefficients of -(1/beta) log(1 + exp(-beta (e - lam))) on
    [chi - zee, chi + zee], by the Clenshaw-Curtis sums of ChebyshevCoeff
    (sq.cpp:1230-1259)."""
    k = np.arange(npl + 1)
    xk = np.cos(np.pi * (k + 0.5) / (npl + 1))
    e = chi[:, None] + zee[:, None] * xk[None, :]
    t = -beta * (e - lam)
    gv = -(1.0 / beta) * (np.maximum(t, 0) + np.log1p(np.exp(-np.abs(t))))
    cosm = np.cos(np.pi * np.outer(np.arange(npl + 1), k + 0.5) / (npl + 1))
    d = 2.0 / (npl + 1) * gv @ cosm.T
    d[:, 0] /= 2.0
    return d


def _derivative_coeffs(d):
    """T-coefficients e_k of P'(x) for P = sum_j d_j T_j (T_j' = j U_j-1 and
    U_m = sum over k = m, m-2, ... >= 0 of (2 - [k = 0]) T_k)."""
    npl = d.shape[1] - 1
    j = np.arange(npl + 1)
    e = np.zeros_like(d)
    for k in range(npl):
        js = j[(j > k) & ((j - 1 - k) % 2 == 0)]
        e[:, k] = (2.0 - (k == 0)) * (d[:, js] * js).sum(axis=1)
    return e


def _omega_gradient(case):
    """dOmega_band/dVeff on the periodic grid, rho h^3, and the derivative
    polynomial's density (P'(Ht)/zee at the node's own moments) times h^3."""
    h3 = case.delta ** 3
    with _ctx(case) as ctx:
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        st = ctx.lanczos_moments()
        d = _grand_potential_coeffs(st["chi"], st["zee"], out["lambda_f"], case.bet, case.npl)
        ctx.moments_at(st["chi"], st["zee"])
        grad = _fold(case, ctx.moments_vjp(2.0 * h3 * d))
    rho_h3 = out["rho"].reshape(-1) * h3
    poly_h3 = (2.0 / st["zee"]) * np.sum(_derivative_coeffs(d) * st["rho_pj"], axis=1) * h3
    return grad, rho_h3, poly_h3


def test_hellmann_feynman_order64():
    """The 4,096-node Al cell (27^3 windows, npl 64): dOmega/dVeff = rho h^3 to
    2.3e-4 of max(rho h^3) (measured on B200)."""
    from sqdft_b200.cases import load

    case = load("c1")  # projector tables computed on the GPU (the case stores none)
    grad, rho_h3, _ = _omega_gradient(case)
    rel = np.abs(grad - rho_h3).max() / np.abs(rho_h3).max()
    print(f"Hellmann-Feynman (c1): {rel:.3e}")
    assert rel <= 5e-4


def test_hellmann_feynman_window_locality(golden):
    """At low order the gap to rho h^3 is the Chebyshev truncation (2.9e-2 at
    npl 24); against the derivative of the same polynomial only the window
    truncation remains (1.9e-3 on 15^3 windows, measured on B200)."""
    case, _ = golden("mid")
    grad, rho_h3, poly_h3 = _omega_gradient(case)
    rel = np.abs(grad - poly_h3).max() / np.abs(poly_h3).max()
    print(f"Hellmann-Feynman vs derivative polynomial (mid): {rel:.3e}")
    assert rel <= 5e-3


def _directional(case, runner, w, d_periodic, eps=1e-4):
    """Central difference of runner.forward along a periodic Veff direction."""
    ext = d_periodic.reshape(-1)[_images(case)]
    lp = runner.forward(case.veff + eps * ext, w)
    lm = runner.forward(case.veff - eps * ext, w)
    return (lp - lm) / (2 * eps)


@pytest.mark.parametrize("fixed_electrons", [True, False])
def test_density_loss_with_fermi_level(golden, fixed_electrons):
    """L = sum w rho with the electron count fixed (the Fermi level follows
    Veff, as in the SCF) or the Fermi level fixed; directional central
    differences of the whole forward (moments, Fermi solve, density)."""
    import dataclasses

    from sqdft_b200.adjoint import DensityLoss, density_coeffs

    case, _ = golden("tiny")
    case = dataclasses.replace(case, fermi_tol=1e-14)
    rng = np.random.default_rng(5)
    with _ctx(case) as ctx:
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        st = ctx.lanczos_moments()
        h3 = case.delta ** 3
        runner = DensityLoss(ctx, st["chi"], st["zee"], case.bet, h3, fixed_electrons=fixed_electrons,
                             scf_iter=2, lambda_warm=out["lambda_f"])
        w = rng.uniform(0.0, 1.0, size=case.n_nodes)
        runner.forward(case.veff, w)
        ci_host = density_coeffs(st["chi"], st["zee"], runner.lam, case.bet, case.npl)
        assert np.abs(ci_host - runner.saved[1]).max() <= 1e-12
        grad = _fold(case, runner.backward(1.0))
        for trial in range(2):
            d = rng.uniform(-1.0, 1.0, size=int(np.prod(case.n_int)))
            fd = _directional(case, runner, w, d)
            an = float(np.dot(grad, d))
            assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9, (trial, fd, an)


def test_torch_autograd_contract(golden):
    """The forward/backward pair bound to torch.autograd.Function (the
    gradient test harness is the only place torch is bound)."""
    torch = pytest.importorskip("torch")
    from sqdft_b200.adjoint import DensityLoss

    class SQDensityLoss(torch.autograd.Function):
        @staticmethod
        def forward(fctx, veff, w, runner):
            fctx.runner = runner
            return torch.tensor(runner.forward(veff.detach().numpy(), w.numpy()), dtype=torch.float64)

        @staticmethod
        def backward(fctx, grad_out):
            g = fctx.runner.backward(float(grad_out))
            return torch.from_numpy(g), None, None

    case, _ = golden("tiny")
    rng = np.random.default_rng(3)
    with _ctx(case) as ctx:
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        st = ctx.lanczos_moments()
        runner = DensityLoss(ctx, st["chi"], st["zee"], case.bet, case.delta ** 3, scf_iter=2,
                             lambda_warm=out["lambda_f"])
        veff = torch.tensor(case.veff, dtype=torch.float64, requires_grad=True)
        w = torch.from_numpy(rng.uniform(0.0, 1.0, size=case.n_nodes))
        loss = SQDensityLoss.apply(veff, w, runner)
        (3.0 * loss).backward()
        direct = runner.backward(3.0)
    assert veff.grad is not None and veff.grad.shape == case.veff.shape
    assert np.abs(veff.grad.numpy() - direct).max() <= 1e-12 * np.abs(direct).max()


@pytest.mark.parametrize("name", ["tiny", "lihs"])
def test_atom_gradient_matches_central_differences(name):
    """dL/dR through the projectors: moving atom J (all its periodic replicas)
    by +-1e-4 bohr, recomputing the projector tables on the GPU and the
    moments at the fixed bounds; LiH exercises l = 1 projectors.  The cases
    come from the drop-in's export (they carry the radial tables the
    projector kernel needs)."""
    import dataclasses

    from sqdft_b200 import sq
    from sqdft_b200.cases import load

    case = load(name)
    rng = np.random.default_rng(9)
    with sq.Context(case, device=0) as ctx:
        ctx.nonlocal_projectors()
        m = ctx.lanczos_moments()
        chi, zee = m["chi"], m["zee"]
        g = rng.uniform(-1.0, 1.0, size=m["rho_pj"].shape)
        ctx.moments_at(chi, zee)
        gv_only = ctx.moments_vjp(g)
        gv, gat = ctx.moments_vjp(g, atoms=True)
        assert np.abs(gv - gv_only).max() <= 1e-12 * np.abs(gv).max()
        scale = np.abs(gat).max()
        assert scale > 0
        eps = 1e-4
        for atom, al in ((0, 0), (1, 2), (case.n_atm - 1, 1)):
            vals = []
            for s in (+1, -1):
                xyz = case.rep_xyz.copy()
                xyz[case.rep_atom == atom, al] += s * eps
                ctx.set_atoms(dataclasses.replace(case, rep_xyz=xyz))
                ctx.nonlocal_projectors()
                vals.append(float(np.sum(g * ctx.moments_at(chi, zee))))
            fd = (vals[0] - vals[1]) / (2 * eps)
            assert abs(fd - gat[atom, al]) <= 1e-5 * scale, (atom, al, fd, gat[atom, al], scale)


def _nonlocal_force_gap(name):
    """max|(-dOmega_band/dR) - F_nonlocal| and max|F_nonlocal| on one system:
    the adjoint's atom gradient of the band grand potential (Veff, bounds and
    Fermi level fixed) against the force of ForcesNonLocal (forces.cpp:318)."""
    from sqdft_b200 import sq
    from sqdft_b200.cases import load

    case = load(name)
    h3 = case.delta ** 3
    with sq.Context(case, device=0) as ctx:
        ctx.nonlocal_projectors()
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        f = ctx.forces_nonlocal()
        m = ctx.lanczos_moments()
        d = _grand_potential_coeffs(m["chi"], m["zee"], out["lambda_f"], case.bet, case.npl)
        ctx.moments_at(m["chi"], m["zee"])
        _, gat = ctx.moments_vjp(2.0 * h3 * d, atoms=True)
    return float(np.abs(gat + f).max()), float(np.abs(f).max())


def test_atom_gradient_converges_to_reference_nonlocal_forces():
    """-dOmega_band/dR is the nonlocal Hellmann-Feynman force.  ForcesNonLocal
    moves the position derivative onto the density-matrix column as its
    12th-order grid gradient (summation by parts), the adjoint differentiates
    the grid-sampled projector itself; the two differ by the grid's
    translation error, which vanishes with the spacing.  On the regression Al
    geometry (npl 64, Rcut 6; measured on B200) the gap is 0.164 of max|F| at
    h = 0.556 and 0.052 at h = 0.389, while a 4 -> 8 bohr window or npl
    32 -> 128 moves it by under 0.07."""
    gap14, f14 = _nonlocal_force_gap("al_ref14")
    gap20, f20 = _nonlocal_force_gap("al_ref20")
    print(f"nonlocal force gap: h=0.556 {gap14 / f14:.3e}, h=0.389 {gap20 / f20:.3e}")
    assert abs(f20 - f14) <= 0.05 * f20  # the same physical force on both grids
    assert gap20 <= 0.08 * f20
    assert gap20 <= 0.45 * gap14


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64_bounds", "fp32_mixed_bounds"])
def test_density_loss_adjoint_configuration(precision):
    """The adjoint configuration c4 (32 Al atoms, 32^3 grid, 27^3 windows,
    npl 64, kT 5 eV): L = sum_x w(x) rho(x) with seeded uniform w in [0, 1] at
    a fixed electron count, the bounds of the FP64 or the FP32-mixed Lanczos
    held fixed (the FP32-mixed form's moments and adjoint recursion are FP64,
    so its adjoint is this one at its own bounds).  The C++ pair
    (sqb_density_loss, sqb_density_loss_vjp: Fermi-level response and moment
    weights on the device, checkpoints every 8 recursion steps) gives the
    gradient the host-formed weights give to 1e-12; it matches central
    differences (step 1e-4) of the whole forward along random Veff directions
    to 1e-6 relative, and the atom gradient matches central differences of
    moved atoms (tables recomputed on the GPU) to 1e-6 of max |dL/dR|."""
    import dataclasses

    from sqdft_b200 import sq
    from sqdft_b200.adjoint import DensityLoss
    from sqdft_b200.cases import load

    case = dataclasses.replace(load("c4"), fermi_tol=1e-14)
    rng = np.random.default_rng(44)
    h3 = case.delta ** 3
    with sq.Context(case, device=0, precision=precision) as ctx:
        ctx.set_mixed_lanczos(0.0)
        ctx.nonlocal_projectors()
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        m = ctx.lanczos_moments()
        runner = DensityLoss(ctx, m["chi"], m["zee"], case.bet, h3, fixed_electrons=True, scf_iter=2,
                             lambda_warm=out["lambda_f"])
        w = rng.uniform(0.0, 1.0, size=case.n_nodes)
        runner.forward(case.veff, w)
        g_ext = runner.backward(1.0)
        g_host = runner.backward_host(1.0)
        assert np.abs(g_ext - g_host).max() <= 1e-12 * np.abs(g_ext).max()
        g_v, g_at = ctx.density_loss_vjp(w, fixed_electrons=True, grad_l=1.0, atoms=True)
        assert np.abs(g_v - g_ext).max() <= 1e-12 * np.abs(g_ext).max()
        grad = _fold(case, g_ext)
        for trial in range(2):
            d = rng.uniform(-1.0, 1.0, size=int(np.prod(case.n_int)))
            fd = _directional(case, runner, w, d)
            an = float(np.dot(grad, d))
            assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
        scale = np.abs(g_at).max()
        assert scale > 0
        eps = 1e-4
        for atom, al in ((0, 0), (case.n_atm // 2, 2)):
            vals = []
            for s in (+1, -1):
                xyz = case.rep_xyz.copy()
                xyz[case.rep_atom == atom, al] += s * eps
                ctx.set_atoms(dataclasses.replace(case, rep_xyz=xyz))
                ctx.nonlocal_projectors()
                vals.append(runner.forward(case.veff, w))
            ctx.set_atoms(case)
            ctx.nonlocal_projectors()
            fd = (vals[0] - vals[1]) / (2 * eps)
            assert abs(fd - g_at[atom, al]) <= 1e-6 * scale, (atom, al, fd, g_at[atom, al], scale)
