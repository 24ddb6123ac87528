"""Gradients of scalars of the SQ density with respect to Veff.

The GPU computes the moment adjoint (``Context.moments_vjp``, the reverse
Chebyshev / Clenshaw recursion of sqb_moments_vjp); this module turns a loss
of the density into the moment weights that adjoint takes, including the
response of the Fermi level when the electron count is held fixed (as the SCF
does), and gives the forward/backward pair of a ``torch.autograd.Function``
without importing torch.

For a node p with bounds chi, zee (held fixed) the density is
``rho_p = 2 sum_j c_j(lambda) mu_j`` (sq.cpp:743-797) with ``c_j`` the
Chebyshev coefficients of the Fermi-Dirac function on the node's interval
(ChebyshevCoeff, sq.cpp:1230-1259: beta_p = beta zee, lambda' = (lambda -
chi)/zee).  For ``L = sum_p w_p rho_p``:

* at fixed lambda, dL/dmu_j(p) = 2 w_p c_j(p);
* at fixed electron count N = h^3 sum_p rho_p, lambda moves with Veff:
  dL/dVeff = dL/dVeff|_lambda - kappa dN/dVeff|_lambda with
  kappa = (dL/dlambda)/(dN/dlambda), and dc_j/dlambda are the Chebyshev
  coefficients of beta f (1 - f).  Both terms are moment adjoints, so the
  gradient is one call with weights 2 (w_p - kappa h^3) c_j(p).
"""
from __future__ import annotations

import numpy as np


def chebyshev_coeffs(values: np.ndarray) -> np.ndarray:
    """c_j = 2/(npl+1) sum_k v_k cos(pi j (k + 1/2)/(npl+1)), c_0 halved, per row of
    ``values`` [nodes][npl+1] sampled at x_k = cos(pi (k + 1/2)/(npl+1))
    (ChebyshevCoeff, sq.cpp:1230-1259)."""
    npl = values.shape[1] - 1
    k = np.arange(npl + 1)
    cosm = np.cos(np.pi * np.outer(np.arange(npl + 1), k + 0.5) / (npl + 1))
    c = (2.0 / (npl + 1)) * values @ cosm.T
    c[:, 0] /= 2.0
    return c


def fermi_values(chi, zee, lam, beta, npl):
    """Fermi-Dirac occupations f(x_k) on each node's interval, [nodes][npl+1]."""
    k = np.arange(npl + 1)
    xk = np.cos(np.pi * (k + 0.5) / (npl + 1))
    e = np.asarray(chi)[:, None] + np.asarray(zee)[:, None] * xk[None, :]
    t = np.clip(beta * (e - lam), -700.0, 700.0)
    return 1.0 / (1.0 + np.exp(t))


def density_coeffs(chi, zee, lam, beta, npl):
    """c_j(lambda) of every node (the library's Ci)."""
    return chebyshev_coeffs(fermi_values(chi, zee, lam, beta, npl))


def density_coeffs_dlambda(chi, zee, lam, beta, npl):
    """dc_j/dlambda of every node: coefficients of beta f (1 - f)."""
    f = fermi_values(chi, zee, lam, beta, npl)
    return chebyshev_coeffs(beta * f * (1.0 - f))


class DensityLoss:
    """L(Veff) = sum_p w_p rho_p(Veff) with the spectral bounds held fixed and
    either the Fermi level fixed or the electron count fixed.

    ``forward`` runs the SQ step on the GPU (moments at the bounds, Fermi level,
    density) and returns L; ``backward(grad_L)`` returns grad_L * dL/dVeff on
    the Veff block with its halo (the layout of ``Context.set_veff``).  This is
    the forward/backward pair a ``torch.autograd.Function`` wraps.
    """

    def __init__(self, ctx, chi, zee, beta, h3, fixed_electrons: bool = True, scf_iter: int = 1,
                 lambda_warm: float = 0.0):
        self.ctx, self.chi, self.zee = ctx, np.asarray(chi), np.asarray(zee)
        self.beta, self.h3, self.fixed_electrons = beta, h3, fixed_electrons
        self.scf_iter, self.lam = scf_iter, lambda_warm
        self.saved = None

    def forward(self, veff_ext: np.ndarray, w: np.ndarray) -> float:
        ctx = self.ctx
        ctx.set_veff(veff_ext)
        mu = ctx.moments_at(self.chi, self.zee)
        if self.fixed_electrons:
            self.lam, _ = ctx.fermi_level(self.scf_iter, self.lam)
        dens = ctx.density_energy(self.lam)
        w = np.ascontiguousarray(w, np.float64).reshape(-1)
        self.saved = (mu, dens["Ci"], dens["rho"].reshape(-1), w)
        return ctx.density_loss(w)  # sqb_density_loss

    def backward(self, grad_l: float = 1.0) -> np.ndarray:
        """grad_l dL/dVeff by sqb_density_loss_vjp (the lambda response and the
        moment weights on the device, then the moment adjoint)."""
        w = self.saved[3]
        return self.ctx.density_loss_vjp(w, fixed_electrons=self.fixed_electrons, grad_l=grad_l)

    def backward_host(self, grad_l: float = 1.0) -> np.ndarray:
        """The same gradient with the moment weights formed on the host (the
        check of sqb_density_loss_vjp's weights)."""
        mu, ci, rho, w = self.saved
        sign = np.sign(rho)
        weight = w * sign
        if self.fixed_electrons:
            npl = ci.shape[1] - 1
            dc = density_coeffs_dlambda(self.chi, self.zee, self.lam, self.beta, npl)
            drho_dlam = 2.0 * np.sum(dc * mu, axis=1) * sign
            dl_dlam = float(np.dot(w, drho_dlam))
            dn_dlam = self.h3 * float(np.sum(drho_dlam))
            kappa = dl_dlam / dn_dlam
            weight = (w - kappa * self.h3) * sign
        g_mu = 2.0 * grad_l * weight[:, None] * ci
        return self.ctx.moments_vjp(g_mu)
