"""The multi-rank path on CPU: two gloo ranks, z-slab decomposition.

Each rank builds its slab of the grid exactly as bench.py does for N GPUs
(sqdft_b200.dist.slab) and runs the oracle on it in place of the CUDA kernel;
the gathered per-node results must equal the single-rank reference outputs
bit for bit (nodes are independent given Veff and the projectors), and the
electron-count constraint summed over ranks through the library's reduction
hook (sqdft_b200.dist.allreduce_fn) must equal the single-rank one.
"""
from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank: int, world: int, init_file: str, out_dir: str) -> None:
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch.distributed as dist

    from conftest import load_golden
    from oracle.pyoracle import Oracle
    from sqdft_b200.dist import MAX, MIN, SUM, allreduce_fn, global_nodes, slab

    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world)
    try:
        case, ref = load_golden("lihs")
        block = slab(case, rank, world)
        orc = Oracle(block, threads=1)
        m = orc.lanczos_moments()
        gids = global_nodes(case, block)
        reduce = allreduce_fn(dist)
        lam = float(ref["lambda_f"][0])
        # NeConstraint returns g + Ncharge (sq.cpp:1226); the reference's
        # MPI_Allreduce (sq.cpp:1219) sums the per-rank g
        part = np.array([orc.ne_constraint(m, lam) - case.ncharge])
        reduce(part, SUM)
        bounds = np.array([m["lmin"].min(), m["lmax"].max()])
        lo, hi = bounds[:1].copy(), bounds[1:].copy()
        reduce(lo, MIN)
        reduce(hi, MAX)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), gids=gids, chi=m["chi"], zee=m["zee"],
                 rho_pj=m["rho_pj"], ne=part + case.ncharge, lo=lo, hi=hi)
    finally:
        dist.destroy_process_group()


def test_two_rank_slabs_match_single_rank(golden):
    import torch.multiprocessing as mp

    case, ref = golden("lihs")
    with tempfile.TemporaryDirectory() as td:
        init = os.path.join(td, "init")
        mp.start_processes(_worker, args=(2, init, td), nprocs=2, start_method="spawn", join=True)
        parts = [np.load(os.path.join(td, f"rank{r}.npz")) for r in range(2)]
    gids = np.concatenate([p["gids"] for p in parts])
    assert np.array_equal(np.sort(gids), np.arange(case.n_nodes))  # every node once
    for key in ("chi", "zee", "rho_pj"):
        got = np.concatenate([p[key] for p in parts])
        assert np.array_equal(got, ref[key][gids]), key
    from oracle.pyoracle import Oracle

    orc = Oracle(case)
    full = orc.lanczos_moments()
    ne1 = orc.ne_constraint(full, float(ref["lambda_f"][0]))
    for p in parts:
        assert abs(float(p["ne"][0]) - ne1) <= 1e-12 * max(1.0, abs(case.ncharge))
        assert float(p["lo"][0]) == full["lmin"].min() and float(p["hi"][0]) == full["lmax"].max()


def test_slab_rejects_uneven_split(golden):
    from sqdft_b200.dist import slab

    case, _ = golden("lihs")
    with pytest.raises(ValueError):
        slab(case, 0, 3)  # 10 planes over 3 ranks
