"""sqb_lanczos_moments_noalloc: the node kernel run with the library's fixed
device scratch array instead of GPU memory allocated during the call.

It is meant for callers that must not allocate device memory while they run
(a framework whose allocator owns the GPU memory, a loop that keeps its
footprint fixed).  The test gives it caller-owned device outputs, calls it
twice in a row through the C ABI in each precision form, and checks both
results against sqb_lanczos_moments run in the same form on the same
context, with the parity tolerances of test_gpu_parity.py; it also checks
that the second call leaves the device's free memory unchanged.  The file
sorts last so that a run stopping at the first failure has run every other
test first; it also passes alone.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1, 2], ids=["fp64", "fp32_mixed", "lanczos_quad"])
def test_noalloc_matches_lanczos_moments_twice(golden, precision):
    import torch

    from sqdft_b200 import sq

    case, _ = golden("lihs")  # two species, 1000 nodes
    n, K = case.n_nodes, case.npl + 1
    with sq.Context(case) as ctx:
        ctx.set_projectors(case.udvtm)
        ctx.set_precision(precision)
        ref = ctx.lanczos_moments()
        nodes = np.ascontiguousarray(np.arange(n)[::-1], np.int32)  # any order, each node once
        chi = torch.empty((n,), dtype=torch.float64, device="cuda")
        zee = torch.empty((n,), dtype=torch.float64, device="cuda")
        rpj = torch.empty((n, K), dtype=torch.float64, device="cuda")
        its = torch.empty((n,), dtype=torch.int32, device="cuda")
        for call in range(2):
            # poison the outputs on torch's stream; the call orders itself after it
            chi.fill_(float("nan"))
            zee.fill_(float("nan"))
            rpj.fill_(float("nan"))
            its.fill_(-1)
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = ctx.lib.sqb_lanczos_moments_noalloc(ctx.ptr, n, nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                     chi.data_ptr(), zee.data_ptr(), rpj.data_ptr(), its.data_ptr())
            assert rc == 0, sq.status_string(rc)
            free1 = torch.cuda.mem_get_info()[0]
            if call == 1:  # the first call may set up the array's address; the second allocates nothing
                assert free1 == free0, (free0, free1)
            torch.cuda.synchronize()
            assert np.abs(chi.cpu().numpy() - ref["chi"]).max() <= 1e-10, call
            assert np.abs(zee.cpu().numpy() - ref["zee"]).max() <= 1e-10, call
            assert np.abs(rpj.cpu().numpy() - ref["rho_pj"]).max() <= 1e-10 * np.abs(ref["rho_pj"]).max(), call
            assert np.array_equal(its.cpu().numpy(), ref["lanczos_iters"]), call


def test_noalloc_orders_after_queued_writes(golden):
    """Outputs poisoned on torch's stream and the call made without a
    synchronize in between: the kernel's results must still win."""
    import torch

    from sqdft_b200 import sq

    case, _ = golden("tiny")
    n, K = case.n_nodes, case.npl + 1
    with sq.Context(case) as ctx:
        ctx.set_projectors(case.udvtm)
        ref = ctx.lanczos_moments()
        nodes = np.ascontiguousarray(np.arange(n), np.int32)
        rpj = torch.empty((n, K), dtype=torch.float64, device="cuda")
        chi = torch.empty((n,), dtype=torch.float64, device="cuda")
        zee = torch.empty((n,), dtype=torch.float64, device="cuda")
        big = torch.empty((64 << 20,), dtype=torch.float64, device="cuda")
        for _ in range(3):
            big.fill_(1.0)  # keep torch's stream busy ahead of the poison
            rpj.fill_(float("nan"))
            chi.fill_(float("nan"))
            zee.fill_(float("nan"))
            rc = ctx.lib.sqb_lanczos_moments_noalloc(ctx.ptr, n, nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                     chi.data_ptr(), zee.data_ptr(), rpj.data_ptr(), None)
            assert rc == 0, sq.status_string(rc)
            torch.cuda.synchronize()
            assert np.abs(rpj.cpu().numpy() - ref["rho_pj"]).max() <= 1e-10 * np.abs(ref["rho_pj"]).max()
            assert np.abs(chi.cpu().numpy() - ref["chi"]).max() <= 1e-10


def test_noalloc_rejects_bad_node_ids(golden):
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    with sq.Context(case) as ctx:
        ctx.set_projectors(case.udvtm)
        bad = np.array([0, case.n_nodes], np.int32)
        null = ctypes.c_void_p(0)
        rc = ctx.lib.sqb_lanczos_moments_noalloc(ctx.ptr, 2, bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 null, null, null, null)
        assert rc == 1  # SQB_ERR_ARG: checked on the host before anything runs
