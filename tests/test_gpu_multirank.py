"""The multi-rank path through the library: two gloo ranks, one GPU.

Each rank builds its z-slab of the grid (sqdft_b200.dist.slab, as bench.py
does for N GPUs), creates its own context on cuda:0 with the library's
reduction hook wired to torch.distributed (sqb_set_allreduce through
sqdft_b200.dist.allreduce_fn), and runs sqb_spectral_quadrature and
sqb_forces_nonlocal.  The reductions are the reference's MPI_Allreduce calls
(NeConstraint sq.cpp:1219, the Lanczos bracket, the energies sq.cpp:792,
the forces forces.cpp:623).  Nodes are independent given Veff and the
projectors, so the gathered per-node bounds and moments must equal the
single-rank run bit for bit; the Fermi level, energies, density and forces,
summed over ranks in another order, to 1e-12.  The two ranks' kernels never
wait on each other: every exchange goes through the host.
"""
from __future__ import annotations

import datetime
import os
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CASE = "lihs"


def _worker(rank: int, world: int, init_file: str, out_dir: str, precision: int) -> None:
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch.distributed as dist

    from conftest import load_golden
    from sqdft_b200 import sq
    from sqdft_b200.dist import allreduce_fn, global_nodes, slab

    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        case, _ = load_golden(CASE)
        block = slab(case, rank, world)
        with sq.Context(block, device=0, precision=precision, allreduce=allreduce_fn(dist)) as ctx:
            ctx.set_projectors(case.udvtm)
            out = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
            f = ctx.forces_nonlocal()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), gids=global_nodes(case, block), chi=out["chi"],
                 zee=out["zee"], rho_pj=out["rho_pj"], rho=out["rho"].ravel(), lam=out["lambda_f"],
                 ebs=out["Ebs"], eent=out["Eent"], f=f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", [0, 1])
def test_two_rank_library_matches_single_rank(golden, precision):
    import torch.multiprocessing as mp

    from sqdft_b200 import sq

    case, _ = golden(CASE)
    with sq.Context(case, device=0, precision=precision) as ctx:
        ctx.set_projectors(case.udvtm)
        one = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        f1 = ctx.forces_nonlocal()
    with tempfile.TemporaryDirectory() as td:
        init = os.path.join(td, "init")
        mp.start_processes(_worker, args=(2, init, td, precision), nprocs=2, start_method="spawn", join=True)
        parts = [np.load(os.path.join(td, f"rank{r}.npz")) for r in range(2)]
    gids = np.concatenate([p["gids"] for p in parts])
    assert np.array_equal(np.sort(gids), np.arange(case.n_nodes))
    for key in ("chi", "zee", "rho_pj"):
        got = np.concatenate([p[key] for p in parts])
        assert np.array_equal(got, one[key][gids]), key
    rho = np.concatenate([p["rho"] for p in parts])
    assert np.abs(rho - one["rho"].ravel()[gids]).max() <= 1e-12 * np.abs(one["rho"]).max()
    for p in parts:
        assert abs(float(p["lam"]) - one["lambda_f"]) <= 1e-12
        assert abs(float(p["ebs"]) - one["Ebs"]) <= 1e-12 * max(1.0, abs(one["Ebs"]))
        assert abs(float(p["eent"]) - one["Eent"]) <= 1e-12 * max(1.0, abs(one["Eent"]))
        assert np.abs(p["f"] - f1).max() <= 1e-12


def test_veff_from_device_memory(golden):
    """sqb_set_veff_device with a slab gathered on the GPU from the whole-grid
    Veff (what each rank does after the broadcast) gives the same step as the
    host slab through sqb_set_veff, bit for bit."""
    import torch

    from sqdft_b200 import sq
    from sqdft_b200.dist import slab, slab_indices

    case, _ = golden(CASE)
    block = slab(case, 1, 2)
    _, _, kz, ky, kx = slab_indices(case, 1, 2)
    grid = torch.from_numpy(np.ascontiguousarray(case.veff_block)).cuda()
    dev = grid.index_select(0, torch.from_numpy(kz).cuda()).index_select(1, torch.from_numpy(ky).cuda())
    dev = dev.index_select(2, torch.from_numpy(kx).cuda()).contiguous()
    assert np.array_equal(dev.cpu().numpy(), block.veff)
    with sq.Context(block, device=0) as ctx:
        ctx.set_projectors(case.udvtm)
        host = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
        ctx.set_veff(np.zeros_like(block.veff) + 0.25)  # something else in between
        ctx.set_veff_device(dev.data_ptr())
        devd = ctx.spectral_quadrature(case.scf_iter, case.lambda_f)
    for key in ("chi", "zee", "rho_pj", "rho"):
        assert np.array_equal(host[key], devd[key]), key
    assert host["lambda_f"] == devd["lambda_f"]
