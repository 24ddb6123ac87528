"""The bounds-check build (libsqdft_b200_bc.so, -DSQB_BOUNDS_CHECK) on the B200.

Every global index of the sweep kernel (window vectors, extended-grid fields,
projector coefficients, flush-buffer slots, the force pass's gradient and
projector reads) is checked against its buffer; a failed check sets a status
bit and the call returns SQB_ERR_BOUNDS.  The test runs the SQ step in all
three forms and the nonlocal forces on the golden systems and the c1
configuration through that library, in a subprocess (the library is chosen at
load time through SQDFT_B200_LIB), and requires a clean status and the normal
library's results.  The checks stand in for a memory checker, which is not
available on this hardware.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
BC_LIB = ROOT / "sqdft_b200" / "_build" / "libsqdft_b200_bc.so"

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import load_golden
from sqdft_b200 import sq
from sqdft_b200.cases import load

out = {}
for name in ("tiny", "lihs", "mid", "c1"):
    if name == "c1":
        case, udvtm = load("c1"), None
    else:
        case, _ = load_golden(name)
        udvtm = case.udvtm
    for prec in (0, 1, 2):
        with sq.Context(case, device=0, precision=prec) as ctx:
            if udvtm is not None:
                ctx.set_projectors(udvtm)
            else:
                ctx.nonlocal_projectors()
            r = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
            f = ctx.forces_nonlocal()
        out[f"{name}-{prec}"] = dict(rho=float(np.abs(r["rho"]).sum()), lam=r["lambda_f"], ebs=r["Ebs"],
                                     chi=float(np.abs(r["chi"]).sum()), f=float(np.abs(f).sum()))
print("RESULT " + json.dumps(out))
"""


def _run(env_lib):
    env = dict(os.environ)
    if env_lib:
        env["SQDFT_B200_LIB"] = str(env_lib)
    else:
        env.pop("SQDFT_B200_LIB", None)
    p = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    line = [s for s in p.stdout.splitlines() if s.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):])


def test_bounds_check_build_runs_clean_and_agrees():
    assert BC_LIB.exists(), f"bounds-check library not built: {BC_LIB}"
    checked = _run(BC_LIB)
    normal = _run(None)
    assert checked.keys() == normal.keys()
    for key in normal:
        for q in ("rho", "lam", "ebs", "chi", "f"):
            a, b = checked[key][q], normal[key][q]
            assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (key, q, a, b)
