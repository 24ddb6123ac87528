"""Error reporting of the CUDA path: every failure the reference exits on is a
status code here, produced from the host side (no GPU fault is provoked)."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _err(fn):
    from sqdft_b200 import sq

    with pytest.raises(sq.SQBError) as ei:
        fn()
    return ei.value.code


def test_nan_veff_rejected(golden):
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    veff = case.veff.copy()
    veff[3, 4, 5] = np.nan
    with sq.Context(case) as ctx:
        assert _err(lambda: ctx.set_veff(veff)) == 11


def test_zero_denominator_rejected(golden):
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    t0 = dataclasses.replace(case.types[0], denom=np.zeros(4))
    bad = dataclasses.replace(case, types=[t0])
    assert _err(lambda: sq.Context(bad)) == 8  # nonlocal.cpp:163


def test_unbracketed_fermi_level(golden):
    """An electron count no Fermi level can reach: Brent's bracket check (sq.cpp:1307)."""
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    bad = dataclasses.replace(case, ncharge=-1e6)
    with sq.Context(bad) as ctx:
        ctx.set_projectors(case.udvtm)
        assert _err(lambda: ctx.spectral_quadrature(1, 0.0)) == 4


def test_calls_out_of_order(golden):
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    with sq.Context(case) as ctx:
        assert _err(lambda: ctx.lanczos_moments()) == 12  # projectors not set
        ctx.set_projectors(case.udvtm)
        assert _err(lambda: ctx.ne_constraint(0.1)) == 12  # no moments yet


def test_lanczos_cap_is_a_counted_warning(golden):
    """A Lanczos that cannot meet its tolerance (-1: |dl| > -1 always holds)
    stops at the 500-iteration cap and carries on with its last Ritz values,
    as the reference prints and carries on (sq.cpp:1073-1074): no error
    status, the nodes are counted in the stats, and the bounds are the
    oracle's after the same 500 iterations."""
    from oracle.pyoracle import Oracle
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    capped = dataclasses.replace(case, lanczos_tol=-1.0)
    nodes = np.array([0, 100, 511], np.int32)
    with sq.Context(capped) as ctx:
        ctx.set_projectors(case.udvtm)
        m = ctx.lanczos_moments_nodes(nodes)
        st = ctx.stats()
    assert st["lanczos_maxiter_nodes"] == len(nodes)
    assert np.all(m["lanczos_iters"] == 500)
    ref = Oracle(capped, case.udvtm).lanczos_moments(nodes)
    assert np.all(ref["lanczos_iters"][nodes] == 500)
    assert np.abs(m["chi"] - ref["chi"][nodes]).max() <= 1e-9
    assert np.abs(m["zee"] - ref["zee"][nodes]).max() <= 1e-9
