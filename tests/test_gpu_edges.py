"""Edge cases of the CUDA path (needs a B200): node lists, low quadrature
orders, and the reference's outputs (the C oracle restates sq.cpp's
arithmetic) away from the orders of the fixtures.

Tolerances as in test_gpu_parity.py: chi, zee 1e-10; rho_pj 1e-10 of max;
rho 1e-10; the Fermi level 1e-10.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(case, precision=0):
    from sqdft_b200 import sq

    ctx = sq.Context(case, device=0, precision=precision)
    ctx.set_projectors(case.udvtm)
    return ctx


def test_node_lists_empty_duplicate_and_out_of_range(golden):
    """sqb_lanczos_moments_nodes: an empty list does nothing and succeeds; a
    node listed twice gets the same bounds and moments both times, equal to
    the whole step's; an id outside the block is rejected on the host
    (SQB_ERR_ARG) before anything runs."""
    from sqdft_b200 import sq

    case, _ = golden("lihs")
    with _ctx(case) as ctx:
        full = ctx.lanczos_moments()
        empty = ctx.lanczos_moments_nodes(np.zeros(0, np.int32))
        assert empty["chi"].shape == (0,)
        nodes = np.array([5, 17, 5, case.n_nodes - 1, 17], np.int32)
        part = ctx.lanczos_moments_nodes(nodes)
        with pytest.raises(sq.SQBError) as err:
            ctx.lanczos_moments_nodes(np.array([0, case.n_nodes], np.int32))
        assert err.value.code == 1
    for key in ("chi", "zee", "rho_pj", "lanczos_iters"):
        assert np.array_equal(part[key][0], part[key][2]), key
        assert np.array_equal(part[key][1], part[key][4]), key
        assert np.array_equal(part[key], full[key][nodes]), key


@pytest.mark.parametrize("npl", [4, 8, 12])
def test_low_quadrature_orders_match_the_oracle(golden, npl):
    """The smallest quadrature orders (npl a multiple of 4 down to 4: a
    single doubling step, round(npl/4) = 1) on the Al cell: the sweep kernel's
    bounds, moments, Fermi level and density equal the oracle's.  At npl 4
    the expansion is too coarse for this cell and some node's density comes
    out below -1e-6: the reference exits there ("Element of rho is negative",
    sq.cpp:763-764), the oracle reports it, and the step returns
    SQB_ERR_NEGATIVE_RHO after bounds, moments and Fermi level that still
    equal the oracle's."""
    from oracle.pyoracle import Oracle
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    case = dataclasses.replace(case, npl=npl)
    ref = Oracle(case).spectral_quadrature()
    with _ctx(case) as ctx:
        if ref["status"] != 0:
            with pytest.raises(sq.SQBError) as err:
                ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
            assert err.value.code == 6  # SQB_ERR_NEGATIVE_RHO
            out = ctx.lanczos_moments()
            out["lambda_f"], _ = ctx.fermi_level(case.scf_iter, case.lambda_f)
        else:
            out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
    assert np.abs(out["chi"] - ref["chi"]).max() <= 1e-10
    assert np.abs(out["zee"] - ref["zee"]).max() <= 1e-10
    assert np.abs(out["rho_pj"] - ref["rho_pj"]).max() <= 1e-10 * np.abs(ref["rho_pj"]).max()
    assert abs(out["lambda_f"] - ref["lambda_f"]) <= 1e-10
    if ref["status"] == 0:
        assert np.abs(out["rho"].ravel() - np.asarray(ref["rho"]).ravel()).max() <= 1e-10
