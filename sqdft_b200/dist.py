"""Multi-rank decomposition of the SQ step (one process per GPU).

The grid is split into z-slabs, one per rank, the way the reference splits it
into processor blocks (initialize.cpp:219-282): each rank's case carries its
block (``np``, ``pnode_s``) and the Veff block with its Rcut halo, which for a
periodic grid is the wrap-around the reference's halo exchange produces
(sq.cpp:400-492).  The only exchange of the SQ step is the scalar reductions
the reference does with MPI (Fermi-level sums, energies, Lanczos bracket);
``allreduce_fn`` gives the library's hook over ``torch.distributed``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .case import Case

SUM, MIN, MAX = 0, 1, 2


def slab_indices(case: Case, rank: int, world: int):
    """(z0, planes, kz, ky, kx): the first plane and plane count of `rank`'s
    z-slab and, per axis, the whole-grid indices of its Veff block with the
    Rcut halo (periodic wrap), so that veff_slab = veff_grid[kz][:, ky][:, :, kx]."""
    if tuple(case.np_) != tuple(case.n_int):
        raise ValueError("slab decomposition starts from the whole grid")
    nz = case.n_int[2]
    if nz % world:
        raise ValueError(f"grid of {nz} planes does not split over {world} ranks")
    sz, z0 = nz // world, rank * (nz // world)
    nl = case.nloc
    kz = np.arange(z0 - nl, z0 + sz + nl) % nz
    ky = (np.arange(case.n_int[1] + 2 * nl) - nl) % case.n_int[1]
    kx = (np.arange(case.n_int[0] + 2 * nl) - nl) % case.n_int[0]
    return z0, sz, kz, ky, kx


def slab(case: Case, rank: int, world: int) -> Case:
    """The z-slab of the (whole, periodic) grid that `rank` of `world` owns."""
    if world == 1:
        return case
    z0, sz, kz, ky, kx = slab_indices(case, rank, world)
    veff = np.ascontiguousarray(case.veff_block[np.ix_(kz, ky, kx)])
    return dataclasses.replace(case, np_=(case.n_int[0], case.n_int[1], sz), pnode_s=(0, 0, z0), veff=veff)


def global_nodes(case: Case, block: Case) -> np.ndarray:
    """Global node ids (x fastest) of the nodes of `block`, in block order."""
    nx, ny, nz = block.np_
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    gi, gj, gk = i + block.pnode_s[0], j + block.pnode_s[1], k + block.pnode_s[2]
    return ((gk * case.n_int[1] + gj) * case.n_int[0] + gi).reshape(-1)


def allreduce_fn(dist, device: str = "cpu"):
    """The library's reduction hook over a torch.distributed process group."""
    import torch

    ops = {SUM: dist.ReduceOp.SUM, MIN: dist.ReduceOp.MIN, MAX: dist.ReduceOp.MAX}

    def reduce(values: np.ndarray, op: int) -> None:
        t = torch.from_numpy(np.array(values, dtype=np.float64)).to(device)
        dist.all_reduce(t, op=ops[op])
        values[:] = t.cpu().numpy()

    return reduce
