"""The C restatement of ChargeDensity and ForcesLocal against the reference.

The fixtures tests/golden/<system>_local.npz hold the reference's own
outputs (tests/golden/make_local_golden.py runs the reference build).  The
restatement follows the reference's arithmetic order, so the per-point
fields agree to the last bits; the sums (energies, charges, forces) run in
the reference's order too.  Tolerances: fields 1e-14 of their largest
magnitude, Eself/Ncharge/Ecorr 1e-12 relative, forces 1e-12 Ha/bohr.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
SYSTEMS = ["tiny", "lihs", "mid"]


def _load(name):
    from sqdft_b200.pseudocharge import fields_from_arrays, grid_from_arrays, local_from_arrays

    a = dict(np.load(GOLDEN / f"{name}_local.npz"))
    return grid_from_arrays(a), local_from_arrays(a), fields_from_arrays(a), a


def _close(x, y, rel):
    x, y = np.asarray(x), np.asarray(y)
    return np.abs(x - y).max() <= rel * max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("name", SYSTEMS)
def test_charge_density_matches_reference(name):
    from oracle.pyoracle import LocalOracle

    grid, loc, _, a = _load(name)
    out = LocalOracle(grid, loc).charge_density()
    for key in ("b", "b_tilda", "vc", "rho_at"):
        assert _close(out[key], a[f"cd_{key}"], 1e-14), key
    for key in ("Eself", "Ncharge", "Ecorr"):
        ref = float(a[f"cd_{key}"].reshape(-1)[0])
        assert abs(out[key] - ref) <= 1e-12 * max(1.0, abs(ref)), (key, out[key], ref)
    # the reference sets Nelectron = -Ncharge after scaling rho to integral(b)
    assert out["Ncharge"] < 0 and out["Nelectron_at"] > 0


@pytest.mark.parametrize("name", SYSTEMS)
def test_forces_local_matches_reference(name):
    from oracle.pyoracle import LocalOracle

    grid, loc, f, a = _load(name)
    floc, fcorr = LocalOracle(grid, loc).forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
    assert np.abs(floc - a["fl_floc"]).max() <= 1e-12
    assert np.abs(fcorr - a["fl_fcorr"]).max() <= 1e-12
    assert np.abs(a["fl_floc"]).max() > 1e-6  # the fixture holds real forces


@pytest.mark.parametrize("config", ["c1", "c2"])
def test_charge_density_matches_reference_on_configurations(config):
    """The benchmark configurations' case files hold the reference's own
    ChargeDensity output (the drop-in program's export runs the reference
    function): the restatement reproduces b, b_tilda, Vc and rho_at of c1
    (4 atoms, 16^3 grid) and c2 (108 atoms, 48^3 grid, 364 replicas)."""
    from oracle.pyoracle import LocalOracle
    from sqdft_b200.case import read_container
    from sqdft_b200.cases import case_path
    from sqdft_b200.pseudocharge import grid_from_arrays, local_from_arrays

    path = case_path(config)
    if not path.exists():
        pytest.skip(f"case file not built: {path}")
    a = read_container(path)
    if "loc_b" not in a:
        pytest.skip("case file exported without the pseudocharge data")
    out = LocalOracle(grid_from_arrays(a), local_from_arrays(a)).charge_density()
    for key in ("b", "b_tilda", "vc", "rho_at"):
        assert _close(out[key], a[f"loc_{key}"], 1e-14), key


@pytest.mark.parametrize("name", ["tiny", "lihs", "c1", "c2", "c5"])
def test_pseudocharge_replicas_match_reference(name):
    """sqdft_b200.pseudocharge.pseudocharge_replicas restates Replica_atoms
    (initialize.cpp:21-160): from the main-domain positions, the .atoms
    cutoffs rb and the .input domain it gives the reference's own replica
    list (exported by the drop-in program from DS_coord::ProcAtm) exactly:
    types, atoms, image coordinates and intersection boxes."""
    from sqdft_b200.case import read_container
    from sqdft_b200.cases import case_path
    from sqdft_b200.configs.gen_configs import SPECIES, SYSTEMS, positions
    from sqdft_b200.pseudocharge import grid_from_arrays, local_from_arrays, pseudocharge_replicas

    path = case_path(name)
    if not path.exists():
        pytest.skip(f"case file not built: {path}")
    a = read_container(path)
    if "loc_rep_box" not in a:
        pytest.skip("case file exported without the pseudocharge data")
    s = SYSTEMS[name]
    rb = [SPECIES[sym][4] for sym in positions(s)]
    domain = [float(f"{s.domain:.10f}")] * 3  # as the .input file writes it
    grid, loc = grid_from_arrays(a), local_from_arrays(a)
    n_int = a["params_i"][0:3]
    rt, ra, rx, box = pseudocharge_replicas(a["atoms_xyz"], a["atom_type"], rb, domain, n_int, grid.pnode_s,
                                            grid.np_)
    assert np.array_equal(rt, loc.rep_type)
    assert np.array_equal(ra, loc.rep_atom)
    assert np.array_equal(rx, loc.rep_xyz)
    assert np.array_equal(box, loc.rep_box)


@pytest.mark.parametrize("name", ["tiny", "lihs", "c1", "c2", "c3", "c5"])
def test_projector_replicas_match_reference(name):
    """sqdft_b200.pseudocharge.projector_replicas restates Replica_atoms_Rcut
    (initialize.cpp:1003-1196) and gives the replica list of the SQ step
    (sqb_set_atoms) that the reference built, exactly."""
    from sqdft_b200.case import read_container
    from sqdft_b200.cases import case_path
    from sqdft_b200.configs.gen_configs import SYSTEMS
    from sqdft_b200.pseudocharge import projector_replicas

    path = case_path(name)
    if not path.exists():
        pytest.skip(f"case file not built: {path}")
    a = read_container(path)
    s = SYSTEMS[name]
    pi = a["params_i"]
    rt, ra, rx = projector_replicas(a["atoms_xyz"], a["atom_type"], a["typ_d"][:, 0], [float(f"{s.domain:.10f}")] * 3,
                                    pi[0:3], pi[6:9], pi[3:6], int(pi[9]))
    assert np.array_equal(rt, a["rep_i"][:, 0])
    assert np.array_equal(ra, a["rep_i"][:, 2])
    assert np.array_equal(rx, a["rep_xyz"])
