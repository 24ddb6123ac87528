"""Pseudocharge density and local forces on the B200 (sqb_charge_density,
sqb_forces_local) against the reference.

The fixtures tests/golden/<system>_local.npz hold the reference's own
ChargeDensity (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315)
outputs.  Each node sums its replicas in the reference's order with the
reference's expressions and no multiply-add contraction, so b and rho_at
must equal the reference bit for bit.  b_tilda and Vc go through pow(),
whose last bit may differ from the host libm: 1e-14 of their largest
magnitude.  The sums over the block (Eself, Ncharge) and the forces reduce
in another order: 1e-12 relative, 1e-12 Ha/bohr.  Ecorr is the small
difference of the correction sum, Eself and Eself_tilda (O(100) Ha each,
Ecorr O(1e-5) Ha): it is checked to 1e-13 of |Eself| + |Eself_tilda|, a few
1e-12 Ha, far inside the 1e-8 Ha/atom energy tolerance.  The c1
configuration is checked against the C restatement the same way, and a
block split in two against the whole.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
SYSTEMS = ["tiny", "lihs", "mid"]


def _fixture(name):
    from sqdft_b200.pseudocharge import fields_from_arrays, grid_from_arrays, local_from_arrays

    a = dict(np.load(GOLDEN / f"{name}_local.npz"))
    return grid_from_arrays(a), local_from_arrays(a), fields_from_arrays(a), a


def _ecorr_tol(cd):
    return 1e-13 * (abs(cd["Eself"]) + abs(cd["Eself_tilda"]))


def _rel(x, y):
    return float(np.abs(np.asarray(x) - np.asarray(y)).max() / max(np.abs(np.asarray(y)).max(), 1e-300))


@pytest.mark.parametrize("name", SYSTEMS)
def test_charge_density_matches_reference(name):
    from sqdft_b200 import sq

    grid, loc, _, a = _fixture(name)
    with sq.LocalContext(grid, loc) as ctx:
        out = ctx.charge_density()
        st = ctx.stats()
    assert np.array_equal(out["b"], a["cd_b"])
    assert np.array_equal(out["rho_at"], a["cd_rho_at"])
    assert _rel(out["b_tilda"], a["cd_b_tilda"]) <= 1e-14
    assert _rel(out["vc"], a["cd_vc"]) <= 1e-14
    for key in ("Eself", "Ncharge"):
        ref = float(a[f"cd_{key}"].reshape(-1)[0])
        assert abs(out[key] - ref) <= 1e-12 * max(1.0, abs(ref)), (key, out[key], ref)
    ref = float(a["cd_Ecorr"].reshape(-1)[0])
    assert abs(out["Ecorr"] - ref) <= _ecorr_tol(out), (out["Ecorr"], ref)
    assert st["ms_charge_density"] > 0


@pytest.mark.parametrize("name", SYSTEMS)
def test_forces_local_matches_reference(name):
    from sqdft_b200 import sq

    grid, loc, f, a = _fixture(name)
    with sq.LocalContext(grid, loc) as ctx:
        floc, fcorr = ctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
    assert np.abs(floc - a["fl_floc"]).max() <= 1e-12
    assert np.abs(fcorr - a["fl_fcorr"]).max() <= 1e-12


def test_c1_matches_the_oracle():
    """The c1 configuration (its pseudocharge replicas and fields as the
    drop-in program's export writes them) against the C restatement."""
    from oracle.pyoracle import LocalOracle
    from sqdft_b200 import sq
    from sqdft_b200.case import read_container
    from sqdft_b200.cases import make_case
    from sqdft_b200.pseudocharge import fields_from_arrays, grid_from_arrays, local_from_arrays

    a = read_container(make_case("c1"))
    grid, loc, f = grid_from_arrays(a), local_from_arrays(a), fields_from_arrays(a)
    ref = LocalOracle(grid, loc)
    cd_ref = ref.charge_density()
    fl_ref = ref.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
    with sq.LocalContext(grid, loc) as ctx:
        cd = ctx.charge_density()
        fl = ctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
    assert np.array_equal(cd["b"], cd_ref["b"])
    assert np.array_equal(cd["rho_at"], cd_ref["rho_at"])
    assert _rel(cd["b_tilda"], cd_ref["b_tilda"]) <= 1e-14 and _rel(cd["vc"], cd_ref["vc"]) <= 1e-14
    # the exported fields are the reference's own ChargeDensity output
    assert np.array_equal(cd["b"], f["b"])
    assert abs(cd["Ecorr"] - cd_ref["Ecorr"]) <= _ecorr_tol(cd_ref)
    for got, want in zip(fl, fl_ref):
        assert np.abs(got - want).max() <= 1e-12


def test_block_split_in_two_matches_the_whole():
    """Two z-slabs of the LiH block, each with its replicas' boxes clipped to
    the slab (what Replica_atoms gives each rank), run as separate blocks
    without a reduction: b, Vc and rho_at are the whole block's slices bit
    for bit, the partial Eself and Ncharge add up to the whole's, and the
    two blocks' local and correction forces add up to the whole's."""
    import dataclasses

    from sqdft_b200 import sq

    grid, loc, f, _ = _fixture("lihs")
    with sq.LocalContext(grid, loc) as ctx:
        whole = ctx.charge_density()
        fw = ctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
    nz = grid.np_[2]
    cut = nz // 2
    parts, forces = [], []
    for z0, z1 in ((0, cut), (cut, nz)):
        g = dataclasses.replace(grid, np_=(grid.np_[0], grid.np_[1], z1 - z0),
                                pnode_s=(grid.pnode_s[0], grid.pnode_s[1], grid.pnode_s[2] + z0))
        box = loc.rep_box.copy()
        lo, hi = g.pnode_s[2], g.pnode_s[2] + g.np_[2] - 1
        keep = (box[:, 5] >= lo) & (box[:, 4] <= hi)
        box[:, 4] = np.maximum(box[:, 4], lo)
        box[:, 5] = np.minimum(box[:, 5], hi)
        sub = dataclasses.replace(loc, rep_type=loc.rep_type[keep], rep_atom=loc.rep_atom[keep],
                                  rep_xyz=loc.rep_xyz[keep], rep_box=np.ascontiguousarray(box[keep]))
        fd = grid.fdn
        phi = f["phi"][z0:z1 + 2 * fd]
        with sq.LocalContext(g, sub) as ctx:
            parts.append(ctx.charge_density())
            forces.append(ctx.forces_local(phi, f["vc"][z0:z1], f["b"][z0:z1], f["b_tilda"][z0:z1]))
    for key in ("b", "rho_at"):
        assert np.array_equal(np.concatenate([p[key] for p in parts]), whole[key]), key
    for key in ("Eself", "Ncharge", "Nelectron_at"):
        assert abs(sum(p[key] for p in parts) - whole[key]) <= 1e-12 * abs(whole[key]), key
    for q in range(2):
        assert np.abs(forces[0][q] + forces[1][q] - fw[q]).max() <= 1e-12


def _slab(grid, loc, z0, z1):
    """The block's z-slab [z0, z1) with its replicas' boxes clipped to it
    (what Replica_atoms gives the rank that holds the slab)."""
    import dataclasses

    g = dataclasses.replace(grid, np_=(grid.np_[0], grid.np_[1], z1 - z0),
                            pnode_s=(grid.pnode_s[0], grid.pnode_s[1], grid.pnode_s[2] + z0))
    box = loc.rep_box.copy()
    lo, hi = g.pnode_s[2], g.pnode_s[2] + g.np_[2] - 1
    keep = (box[:, 5] >= lo) & (box[:, 4] <= hi)
    box[:, 4] = np.maximum(box[:, 4], lo)
    box[:, 5] = np.minimum(box[:, 5], hi)
    sub = dataclasses.replace(loc, rep_type=loc.rep_type[keep], rep_atom=loc.rep_atom[keep],
                              rep_xyz=loc.rep_xyz[keep], rep_box=np.ascontiguousarray(box[keep]))
    return g, sub


def _rank_worker(rank: int, world: int, init_file: str, out_dir: str) -> None:
    import datetime
    import os
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import torch.distributed as dist

    from sqdft_b200 import sq
    from sqdft_b200.dist import allreduce_fn
    from test_gpu_local import _fixture, _slab

    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        grid, loc, _, _ = _fixture("lihs")
        cut = grid.np_[2] // 2
        z0, z1 = (0, cut) if rank == 0 else (cut, grid.np_[2])
        g, sub = _slab(grid, loc, z0, z1)
        with sq.LocalContext(g, sub, allreduce=allreduce_fn(dist)) as ctx:
            out = ctx.charge_density()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **{k: np.asarray(v) for k, v in out.items()})
    finally:
        dist.destroy_process_group()


def test_two_ranks_through_the_allreduce_hook():
    """Two gloo ranks on one GPU, each with its z-slab of the LiH block: the
    sums go through sqb_set_allreduce (the reference's MPI_Allreduce of
    initialize.cpp:717-723 and 770), V000 and Vcon come from the rank whose
    block starts the main domain.  b and rho_at are the single-rank slices
    bit for bit; the scaled b_tilda, the shifted Vc, Eself, Ncharge and Ecorr
    agree with the single-rank call to rounding.  The ranks' kernels never
    wait on each other: every exchange goes through the host."""
    import os
    import tempfile

    import torch.multiprocessing as mp

    from sqdft_b200 import sq

    grid, loc, _, _ = _fixture("lihs")
    with sq.LocalContext(grid, loc) as ctx:
        whole = ctx.charge_density()
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank_worker, args=(2, os.path.join(td, "init"), td), nprocs=2, start_method="spawn",
                           join=True)
        parts = [dict(np.load(os.path.join(td, f"rank{r}.npz"))) for r in range(2)]
    for key in ("b", "rho_at"):
        assert np.array_equal(np.concatenate([p[key] for p in parts]), whole[key]), key
    for key in ("b_tilda", "vc"):
        assert _rel(np.concatenate([p[key] for p in parts]), whole[key]) <= 1e-13, key
    for p in parts:
        for key in ("Eself", "Ncharge", "Ncharge_tilda", "Eself_tilda"):
            assert abs(float(p[key]) - whole[key]) <= 1e-12 * abs(whole[key]), key
        assert abs(float(p["Ecorr"]) - whole["Ecorr"]) <= _ecorr_tol(whole)
        assert float(p["Vcon"]) == whole["Vcon"]


def test_argument_and_state_errors():
    """A replica box outside the block is rejected on the host (SQB_ERR_ARG)
    before anything runs, and the pseudocharge calls before
    sqb_set_local_atoms return SQB_ERR_STATE."""
    import ctypes
    import dataclasses

    from sqdft_b200 import sq

    grid, loc, f, _ = _fixture("tiny")
    bad = loc.rep_box.copy()
    bad[0, 1] = grid.pnode_s[0] + grid.np_[0]  # one node past the block
    with pytest.raises(sq.SQBError) as err:
        sq.LocalContext(grid, dataclasses.replace(loc, rep_box=bad))
    assert err.value.code == 1
    with sq.LocalContext(grid, loc) as ctx:
        # a second context of the same grid, without replicas
        g = sq.SqbGrid()
        g.np[:] = list(grid.np_)
        g.pnode_s[:] = list(grid.pnode_s)
        g.n_int[:] = list(grid.np_)
        g.nloc, g.fdn, g.npl, g.fermi_alg = 1, grid.fdn, 4, 1
        g.delta, g.bet = grid.delta, 1.0
        ptr = ctypes.c_void_p()
        assert ctx.lib.sqb_create(ctypes.byref(g), 0, ctypes.byref(ptr)) == 0
        try:
            scal = np.zeros(7)
            assert ctx.lib.sqb_charge_density(ptr, None, None, None, None, sq._d(scal)) == 12  # SQB_ERR_STATE
            out = np.zeros((grid.n_atm, 3))
            args = [np.ascontiguousarray(f[k]) for k in ("phi", "vc", "b", "b_tilda")]
            assert ctx.lib.sqb_forces_local(ptr, *[sq._d(x) for x in args], sq._d(out), sq._d(out)) == 12
        finally:
            ctx.lib.sqb_destroy(ptr)
