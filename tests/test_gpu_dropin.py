"""The whole SQDFT program with this package's SQ step, against the reference.

``sqdft_gpu`` (sqdft_b200/dropin) is the reference program -- SCF loop,
Poisson, mixing, exchange-correlation, local forces -- linked with the GPU
ClenshawCurtisSpectralQuadrature, NonlocalProjectors and ForcesNonLocal.  It
runs the reference's regression system tests/Al (4 Al atoms, 10^3 grid,
npl 28, Rcut 6; system ``al_ref``) and its log must reproduce, SCF iteration
by SCF iteration, the log of the unmodified reference program on the same
input (tests/golden/al_ref_scf.json, made by make_scf_golden.py): the same
number of SCF iterations and Brent iterations, Fermi levels and total
energies within 1e-9 Ha, the free energy within 1e-8 Ha/atom and the forces
within 1e-7 Ha/bohr.  The golden run itself is pinned to the reference's
published log (tests/Al/results_Al) by the CPU test below.
"""
from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).parent / "golden" / "al_ref_scf.json"
PROGRAM = ROOT / "sqdft_b200" / "_build" / "dropin" / "sqdft_gpu"
POT = ROOT / "sqdft_b200" / "_data" / "pot"


def test_golden_run_matches_published_log():
    """The reference built here reproduces its own published log of tests/Al."""
    g = json.loads(GOLDEN.read_text())
    pub = g["published"]
    assert len(g["scf"]) == len(pub["scf"]) == 9
    for a, b in zip(g["scf"], pub["scf"]):
        assert a["iter"] == b["iter"]
        assert abs(a["fermi"] - b["fermi"]) <= 2e-12
        assert abs(a["etot"] - b["etot"]) <= 2e-12
    assert abs(g["free_energy"] - pub["free_energy"]) <= 2e-12
    assert np.abs(np.array(g["forces"]) - np.array(pub["forces"])).max() <= 2e-12
    assert g["fermi_iters"] == pub["fermi_iters"]


def run_program(tmp_path: Path, precision: str | None = None, graph: int = 0, local: bool = False) -> dict:
    from sqdft_b200.configs.gen_configs import write_system
    from sqdft_b200.runlog import parse

    assert PROGRAM.exists(), f"drop-in program not built: {PROGRAM}"
    run = write_system("al_ref", tmp_path)
    for pot in POT.glob("*.pot"):
        (run / pot.name).symlink_to(pot)
    env = dict(os.environ)
    env.pop("SQDFT_B200_EXPORT", None)
    if precision:
        env["SQDFT_B200_PRECISION"] = precision
    if graph:
        env["SQDFT_B200_GRAPH"] = str(graph)
    if local:
        env["SQDFT_B200_LOCAL"] = "1"
    out = subprocess.run([str(PROGRAM), "-name", "al_ref"], cwd=run, env=env, capture_output=True, text=True,
                         timeout=900)
    (tmp_path / "sqdft_gpu.log").write_text(out.stdout + out.stderr)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return parse(out.stdout)


@pytest.mark.gpu
def test_dropin_program_reproduces_reference_run(tmp_path):
    g = json.loads(GOLDEN.read_text())
    got = run_program(tmp_path)
    assert len(got["scf"]) == len(g["scf"])
    for a, b in zip(got["scf"], g["scf"]):
        assert a["iter"] == b["iter"]
        assert abs(a["fermi"] - b["fermi"]) <= 1e-9, (a, b)
        assert abs(a["etot"] - b["etot"]) <= 1e-9, (a, b)
    assert got["fermi_iters"] == g["fermi_iters"]
    assert abs(got["free_energy"] - g["free_energy"]) <= 1e-8
    assert np.abs(np.array(got["forces"]) - np.array(g["forces"])).max() <= 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "lq"])
def test_dropin_program_fast_forms(tmp_path, precision):
    """The whole program with the FP32-mixed or the Lanczos-quadrature SQ step
    (at the input's Lanczos tolerance) converges like the reference run: the
    same number of SCF iterations, the free energy within 1e-6 Ha/atom and the
    forces within 1e-5 Ha/bohr."""
    g = json.loads(GOLDEN.read_text())
    got = run_program(tmp_path, precision)
    de = abs(got["free_energy"] - g["free_energy"])
    df = np.abs(np.array(got["forces"]) - np.array(g["forces"])).max()
    print(f"drop-in {precision}: {len(got['scf'])} SCF iterations, free energy {de:.1e} Ha/atom, forces {df:.1e}")
    assert len(got["scf"]) == len(g["scf"])
    assert de <= 1e-6
    assert df <= 1e-5


@pytest.mark.gpu
def test_dropin_program_scf_loop_on_step_graphs(tmp_path):
    """The reference's SCF loop (Poisson, XC, Anderson mixing on the host) with
    every SQ step replayed from one CUDA graph (SQDFT_B200_GRAPH=2: node kernel,
    Fermi solve on the device, density): the same SCF history as the reference
    run, to the tolerances of the plain drop-in run."""
    g = json.loads(GOLDEN.read_text())
    got = run_program(tmp_path, graph=2)
    assert len(got["scf"]) == len(g["scf"])
    for a, b in zip(got["scf"], g["scf"]):
        assert abs(a["fermi"] - b["fermi"]) <= 1e-9, (a, b)
        assert abs(a["etot"] - b["etot"]) <= 1e-9, (a, b)
    assert got["fermi_iters"] == g["fermi_iters"]
    assert abs(got["free_energy"] - g["free_energy"]) <= 1e-8
    assert np.abs(np.array(got["forces"]) - np.array(g["forces"])).max() <= 1e-7


@pytest.mark.gpu
def test_dropin_program_with_local_path_on_device(tmp_path):
    """SQDFT_B200_LOCAL=1: ChargeDensity's per-atom loop and ForcesLocal run on
    the GPU too (sqb_charge_density, sqb_forces_local), the rest of
    ChargeDensity on the host.  The SCF history, free energy and forces match
    the reference run to the tolerances of the plain drop-in run."""
    g = json.loads(GOLDEN.read_text())
    got = run_program(tmp_path, local=True)
    assert len(got["scf"]) == len(g["scf"])
    for a, b in zip(got["scf"], g["scf"]):
        assert abs(a["fermi"] - b["fermi"]) <= 1e-9, (a, b)
        assert abs(a["etot"] - b["etot"]) <= 1e-9, (a, b)
    assert got["fermi_iters"] == g["fermi_iters"]
    assert abs(got["free_energy"] - g["free_energy"]) <= 1e-8
    assert np.abs(np.array(got["forces"]) - np.array(g["forces"])).max() <= 1e-7
