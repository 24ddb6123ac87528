"""FP64 CUDA path against the reference on the benchmark configurations.

Fixtures (tests/golden/make_config_golden.py, from the reference compiled
from its own sources):
  c1  4-atom Al cell, 16^3 grid, 27^3 windows, npl 64: the whole SQ step
      (sq.cpp:377-834) and the nonlocal forces (forces.cpp:318-578);
  c2  108-atom Al cell, 48^3 grid, 31^3 windows, npl 96: the reference's
      Lanczos bounds and Chebyshev moments (sq.cpp:530-661) of 512 nodes;
  c3  64-atom LiH cell (Li with three l=1 projectors beside projector-less
      H), 40^3 grid, 33^3 windows, npl 128: the same on 512 nodes.
The GPU runs on the cases the drop-in program exports from the same input
files; the fixtures' Veff checksums pin that the inputs are the reference's
bit for bit.  The projector tables are computed on the GPU from the radial
tables (sqb_nonlocal_projectors).  Tolerances as in test_gpu_parity.py:
chi, zee 1e-10; rho_pj 1e-10 of max |rho_pj|; rho 1e-10; Ebs, Eent 1e-8
Ha/atom; forces 1e-7 Ha/bohr.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _fixture(name):
    return dict(np.load(GOLDEN / f"{name}_ref.npz"))


def _context(name):
    import sys

    sys.path.insert(0, str(GOLDEN))
    from make_config_golden import veff_checksums

    from sqdft_b200 import sq
    from sqdft_b200.cases import load

    case = load(name)
    ref = _fixture(name)
    assert np.array_equal(veff_checksums(case.veff_block), ref["veff_checksums"]), "case Veff differs from the reference's"
    ctx = sq.Context(case, device=0)
    ctx.nonlocal_projectors()
    return case, ctx, ref


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_sampled_nodes_match_reference(name):
    case, ctx, ref = _context(name)
    with ctx:
        m = ctx.lanczos_moments_nodes(ref["sample_nodes"])
        st = ctx.stats()
    assert np.abs(m["chi"] - ref["sample_chi"]).max() <= 1e-10
    assert np.abs(m["zee"] - ref["sample_zee"]).max() <= 1e-10
    scale = np.abs(ref["sample_rho_pj"]).max()
    assert np.abs(m["rho_pj"] - ref["sample_rho_pj"]).max() <= 1e-10 * scale
    assert st["lanczos_maxiter_nodes"] == 0


def test_c1_whole_step_and_forces_match_reference():
    case, ctx, ref = _context("c1")
    n_atm = case.n_atm
    with ctx:
        out = ctx.spectral_quadrature(1, 0.0)
        f = ctx.forces_nonlocal()
    assert np.abs(out["chi"] - ref["chi"]).max() <= 1e-10
    assert np.abs(out["zee"] - ref["zee"]).max() <= 1e-10
    nodes = ref["sample_nodes"]
    scale = np.abs(ref["sample_rho_pj"]).max()
    assert np.abs(out["rho_pj"][nodes] - ref["sample_rho_pj"]).max() <= 1e-10 * scale
    assert np.abs(out["rho"].ravel() - ref["rho"].ravel()).max() <= 1e-10
    assert abs(out["lambda_f"] - float(ref["lambda_f"])) <= 1e-10
    assert abs(out["Ebs"] - float(ref["Ebs"])) / n_atm <= 1e-8
    assert abs(out["Eent"] - float(ref["Eent"])) / n_atm <= 1e-8
    assert np.abs(f - ref["fnloc"]).max() <= 1e-7


@pytest.mark.parametrize("name", ["tiny", "lihs"])
def test_projector_tables_match_reference_udvtm(golden, name):
    """NonlocalProjectors (nonlocal.cpp:317-518) on the GPU from the radial
    tables against the reference's own UdVtm of the same replicas (Al: one l=0
    projector; LiH: three l=1 projectors per Li, none for H)."""
    from sqdft_b200 import sq
    from sqdft_b200.cases import load

    case = load(name)  # radial tables as the reference parsed them
    gcase, _ = golden(name)
    assert np.array_equal(case.rep_xyz, gcase.rep_xyz)
    with sq.Context(case, device=0) as ctx:
        u = ctx.nonlocal_projectors(copy_out=True)
    want = gcase.udvtm
    assert u.shape == want.shape
    assert np.abs(u - want).max() <= 1e-14 * np.abs(want).max()
