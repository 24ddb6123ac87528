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


def test_metrics_record_per_call(golden, tmp_path, monkeypatch):
    """SQDFT_B200_METRICS names a file that receives one JSON line per SQ step
    and per force pass: phase times, iteration counts, status."""
    import json

    from sqdft_b200 import sq

    case, _ = golden("tiny")
    path = tmp_path / "metrics.jsonl"
    monkeypatch.setenv("SQDFT_B200_METRICS", str(path))
    with sq.Context(case, device=0) as ctx:
        ctx.set_projectors(case.udvtm)
        out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        ctx.forces_nonlocal()
        st = ctx.stats()
    lines = [json.loads(s) for s in path.read_text().splitlines()]
    assert [r["call"] for r in lines] == ["spectral_quadrature", "forces_nonlocal"]
    sq_rec = lines[0]
    assert sq_rec["status"] == 0 and sq_rec["nodes"] == case.n_nodes and sq_rec["npl"] == case.npl
    assert sq_rec["lambda_f"] == out["lambda_f"]
    assert sq_rec["lanczos_iters"] > 0 and sq_rec["ms_lanczos_moments"] > 0.0
    assert abs(lines[1]["ms_forces"] - st["ms_forces"]) <= 1e-5


def test_bounded_stage_wait_runs_out_cleanly(golden):
    """The plane-streaming kernel's waits for its bulk-copied table planes are
    bounded: with the test hook every stage expects 16 bytes more than its
    copies bring, each wait gives up after 1 ms (plus the 1 ms grace for the
    copies already issued), the call returns SQB_ERR_CUDA, and the context
    runs the next step normally with the hook off."""
    from sqdft_b200 import sq

    case, ref = golden("tiny")
    with sq.Context(case, device=0) as ctx:
        ctx.set_projectors(case.udvtm)
        ctx.set_node_kernel(sq.SQB_KERNEL_PLANE)
        ctx.test_stage_wait(16, 1.0)
        with pytest.raises(sq.SQBError) as err:
            ctx.lanczos_moments()
        assert err.value.code == 2  # SQB_ERR_CUDA
        ctx.test_stage_wait(0, 0.0)
        m = ctx.lanczos_moments()
    assert np.abs(m["chi"] - ref["chi"]).max() <= 1e-10
    assert np.abs(m["zee"] - ref["zee"]).max() <= 1e-10
