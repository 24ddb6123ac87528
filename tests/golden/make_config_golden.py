"""Regenerate the reference fixtures of the benchmark configurations.

Runs the reference SQDFT compiled from its own sources (``make -C oracle``,
oracle/_ref/sqref_driver) on the systems c1, c2 and c3 of
``sqdft_b200/configs/gen_configs.py`` and keeps, per system:

* c2, c3 (110,592 and 64,000 nodes; hours of CPU for a whole step): the
  reference's per-node work -- LanczosAlgorithm (sq.cpp:965) and the moment
  loop of sq.cpp:564-655 -- on a seeded, evenly spread sample of 512 nodes:
  their chi, zee and rho_pj (``sample.sqc`` of the driver's ``--sample``);
* c1 (4,096 nodes): the whole ClenshawCurtisSpectralQuadrature (sq.cpp:377)
  and ForcesNonLocal (forces.cpp:318): rho, chi, zee, lambda_f, Ebs, Eent,
  the nonlocal forces, and rho_pj of 512 of its nodes.

Each fixture also stores checksums of the Veff block the reference ran on,
so the GPU tests can confirm they run on identical inputs (the cases the GPU
tests load are exported by the drop-in program from the same input files).

    python tests/golden/make_config_golden.py [c1 c2 c3]
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from sqdft_b200.case import load_case, read_container  # noqa: E402
from sqdft_b200.configs.gen_configs import write_system  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "sqref_driver"
POT = ROOT / "oracle" / "_ref" / "pot"
SAMPLE = 512


def veff_checksums(block: np.ndarray) -> np.ndarray:
    """Plain and index-weighted sums of a Veff block interior (z-major)."""
    v = np.asarray(block, np.float64).ravel()
    w = np.arange(1, v.size + 1, dtype=np.float64) / v.size
    return np.array([v.sum(), (w * v).sum(), np.abs(v).max()])


def run(name: str, extra: list[str], workdir: Path) -> Path:
    run_dir = write_system(name, workdir)
    for pot in POT.glob("*.pot"):
        (run_dir / pot.name).symlink_to(pot)
    out = workdir / f"{name}_ref"
    subprocess.run([str(DRIVER), str(run_dir), name, str(out), *extra], check=True, stdout=subprocess.DEVNULL)
    return out


def make(name: str) -> None:
    threads = str(os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        if name == "c1":
            out = run(name, [], td)
            block = load_case(f"{out}_in.sqc").veff_block
            res = read_container(f"{out}_out.sqc")
            n = res["chi"].size
            nodes = (np.arange(SAMPLE) * n // SAMPLE + (n // SAMPLE) // 2) % n
            arrays = dict(rho=res["rho"], chi=res["chi"], zee=res["zee"], lambda_f=res["lambda_f"],
                          Ebs=res["Ebs"], Eent=res["Eent"], fnloc=res["fnloc"], sample_nodes=nodes.astype(np.int32),
                          sample_rho_pj=res["rho_pj"][nodes])
        else:
            out = run(name, ["--sample", str(SAMPLE), "--threads", threads], td)
            smp = read_container(f"{out}_sample.sqc")
            block = smp["veff_block"]
            arrays = dict(sample_nodes=smp["sample_nodes"], sample_chi=smp["sample_chi"],
                          sample_zee=smp["sample_zee"], sample_rho_pj=smp["sample_rho_pj"])
    arrays["veff_checksums"] = veff_checksums(block)
    dest = Path(__file__).parent / f"{name}_ref.npz"
    np.savez_compressed(dest, **{k: np.asarray(v) for k, v in arrays.items()})
    print(f"{dest}: {dest.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    for nm in sys.argv[1:] or ["c2", "c3", "c1"]:
        make(nm)
