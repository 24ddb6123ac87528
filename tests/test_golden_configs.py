"""The benchmark-configuration fixtures pin the inputs the GPU tests run on.

tests/golden/{c1,c2,c3}_ref.npz hold the reference's outputs together with
checksums of the Veff block it ran on; the GPU tests run on the cases the
drop-in program exports from the same input files.  Where those cases exist
(built by __graft_entry__.build), their Veff must equal the reference's bit
for bit.  The fixtures' own consistency is checked without them.
"""
from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, str(GOLDEN))


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_fixture_shapes(name):
    z = np.load(GOLDEN / f"{name}_ref.npz")
    nodes = z["sample_nodes"]
    assert len(nodes) == 512 and len(np.unique(nodes)) == 512
    assert z["sample_rho_pj"].shape[0] == 512
    if name == "c1":
        assert z["chi"].shape == (4096,) and z["fnloc"].shape == (4, 3)
        # mu_0 = 1/h^3 for every node (sq.cpp:588)
        assert np.allclose(z["sample_rho_pj"][:, 0], z["sample_rho_pj"][0, 0], rtol=1e-15)
    else:
        assert z["sample_chi"].shape == (512,) and np.all(z["sample_zee"] > 0)


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_exported_case_veff_matches_reference(name):
    from make_config_golden import veff_checksums

    from sqdft_b200.case import load_case
    from sqdft_b200.cases import case_path

    path = case_path(name)
    if not path.exists():
        pytest.skip(f"{path} not built")
    z = np.load(GOLDEN / f"{name}_ref.npz")
    assert np.array_equal(veff_checksums(load_case(path).veff_block), z["veff_checksums"])
