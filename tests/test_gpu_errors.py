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
