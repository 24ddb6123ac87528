"""SQ-step throughput of sqdft_b200 on B200 (grid nodes per second).

One step is ClenshawCurtisSpectralQuadrature on the whole grid of a
benchmark system: Lanczos bounds and Chebyshev moments of every node,
Fermi-level solve, density and energies.  The default workload is the
108-atom FCC Al cell (48^3 = 110,592 nodes, 31^3 truncation windows,
Chebyshev order 96) with the reference's own first-SCF-iteration Veff.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2]
                    [--precision all|fp64|mixed|lq] [--mixed-lanczos-tol T]
                    [--impl ours|reference]

The default (--precision all) times three forms of the step (W untimed and K
timed steps for the first, 1 and 1 for the two it is compared with) and
prints one line:
  value       the FP64 Lanczos-quadrature step (SQB_FP64_LANCZOS_QUAD: bounds
              and all Chebyshev moments of a node from one Lanczos run started
              at the node, Lanczos stop at T Ha)
  fp32_mixed  the FP32-mixed step (FP32 Lanczos vectors from a checkerboard-
              weighted start, stop at T Ha; FP64 Chebyshev moments)
  fp64        the FP64 parity step
`accuracy` holds each fast form's density, Fermi-level and band-energy
differences from the FP64 arm's last step.  --precision lq|mixed alone states
them against one untimed FP64 step.

value  nodes / (device time of the step), inputs resident in HBM
e2e    nodes / (wall time of the C-ABI call with host buffers: Veff copied
       in from pinned memory, rho, rho_pj, Ci, chi, zee copied out)
With N > 1 (torchrun, NCCL), rank r owns a z-slab of the grid; the
Fermi-level sums and energies are all-reduced through the library's hook.
--impl reference times the reference SQDFT compiled from its sources
(oracle/_ref/sqref_driver: its LanczosAlgorithm and HsubTimesVec per node)
on a node sample across all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def algorithmic_bytes(stats, case, precision, lq=False, n_nodes=None, window=False):
    """Bytes per node-kernel launch by the roofline's accounting: per matvec
    step n_w (3 s_v + s_V) plus the projector tables of every atom whose ball
    meets the window, steps = Lanczos iterations + 1 + npl/2 per node.  Veff
    and the tables are FP64 in both paths; the Lanczos vectors (s_v) are FP32
    in the mixed path, the Chebyshev vectors FP64 in both."""
    nw = stats["window_points"]
    n = case.n_nodes if n_nodes is None else n_nodes
    lz_steps = stats["lanczos_iters"] + n
    ch_steps = 0 if lq else n * (case.npl // 2)
    sv_lz = 8 if precision == 0 else 4
    vectors = lz_steps * nw * (3 * sv_lz + 8) + ch_steps * nw * 32
    if window:  # projector values of each ball clipped to the window (what a matvec reads)
        return vectors + stats["proj_points_window"] * 8
    return vectors + stats["proj_points"] * 8


def run_sample(args):
    """Node kernel alone on K evenly spaced nodes of a configuration (the
    Lanczos bounds and Chebyshev moments of sq.cpp:530-661 for those nodes),
    W untimed and S timed runs; prints one JSON line with the kernel time and
    its algorithmic bytes.  For profiling a full-size configuration on a
    subset of its nodes."""
    import torch

    from sqdft_b200 import sq
    from sqdft_b200.cases import load as load_named

    torch.cuda.set_device(0)
    case = load_named(args.config)
    prec = {"fp64": sq.SQB_FP64, "mixed": sq.SQB_FP32_MIXED, "lq": sq.SQB_FP64_LANCZOS_QUAD}[args.precision]
    k = min(args.sample_nodes, case.n_nodes)
    nodes = (np.arange(k, dtype=np.int64) * case.n_nodes // k).astype(np.int32)
    with sq.Context(case, device=0, precision=prec) as ctx:
        ctx.set_mixed_lanczos(args.mixed_lanczos_tol)
        ctx.set_sweep_rows(args.sweep_rows)
        ctx.nonlocal_projectors()
        for _ in range(args.warmup):
            ctx.lanczos_moments_nodes(nodes)
        ms = []
        for _ in range(args.steps):
            ctx.lanczos_moments_nodes(nodes)
            st = ctx.stats()
            ms.append(st["ms_lanczos_moments"])
    kern = float(np.mean(ms)) * 1e-3
    abytes = algorithmic_bytes(st, case, prec, lq=(args.precision == "lq"), n_nodes=k)
    peak, peak_kind = hbm_peak()
    print(json.dumps({"mode": "sample", "config": args.config, "precision": args.precision, "nodes": k,
                      "kernel_ms": kern * 1e3, "nodes_per_s": k / kern,
                      "lanczos_iters_per_node": st["lanczos_iters"] / k, "algorithmic_bytes": abytes,
                      "achieved_gbs": abytes / kern / 1e9, "peak": peak, "peak_kind": peak_kind,
                      "frac": abytes / kern / 1e9 / peak}), flush=True)


def run_scf(args):
    """The reference program's SCF loop on a configuration -- the drop-in
    program (Poisson, exchange-correlation and Anderson mixing on the host,
    the SQ step and forces through this library) -- for exactly
    --scf-steps SCF iterations, each SQ step replayed from one CUDA graph
    (--graph 2, the default here) or launched plainly (--graph 0).  One JSON
    line: the device time of every SQ step from the library's metrics record,
    the Brent iterations, the force pass and the program's wall time."""
    import subprocess
    import tempfile

    from sqdft_b200.configs.gen_configs import write_system

    prog = ROOT / "sqdft_b200" / "_build" / "dropin" / "sqdft_gpu"
    pot = ROOT / "sqdft_b200" / "_data" / "pot"
    n = args.scf_steps
    with tempfile.TemporaryDirectory() as td:
        run = write_system(args.config, Path(td))
        inp = run / f"{args.config}.input"
        text = inp.read_text().replace("scf_miniter 3", f"scf_miniter {n}").replace("scf_maxiter 40",
                                                                                   f"scf_maxiter {n}")
        inp.write_text(text)
        for p in pot.glob("*.pot"):
            (run / p.name).symlink_to(p)
        metrics = Path(td) / "metrics.jsonl"
        env = dict(os.environ, SQDFT_B200_GRAPH=str(args.graph), SQDFT_B200_METRICS=str(metrics))
        env.pop("SQDFT_B200_EXPORT", None)
        if args.precision in ("mixed", "lq"):
            env["SQDFT_B200_PRECISION"] = "fp32" if args.precision == "mixed" else "lq"
            env["SQDFT_B200_LANCZOS_TOL"] = str(args.mixed_lanczos_tol)
        t0 = time.perf_counter()
        out = subprocess.run([str(prog), "-name", args.config], cwd=run, env=env, capture_output=True, text=True,
                             timeout=3600)
        wall = time.perf_counter() - t0
        recs = [json.loads(x) for x in metrics.read_text().splitlines()] if metrics.exists() else []
    steps = [r for r in recs if r["call"] == "spectral_quadrature"]
    forces = [r for r in recs if r["call"] == "forces_nonlocal"]
    print(json.dumps({"mode": "scf", "config": args.config, "precision": args.precision, "graph": args.graph,
                      "program_rc": out.returncode, "scf_iterations": len(steps),
                      "sq_step_ms": [r["ms_lanczos_moments"] + r["ms_fermi"] + r["ms_density"] + r["ms_defect"]
                                     for r in steps],
                      "kernel_launches_per_step": [r["kernel_launches"] for r in steps],
                      "fermi_iters": [r["fermi_iters"] for r in steps], "lambda_f": [r["lambda_f"] for r in steps],
                      "forces_ms": [r["ms_forces"] for r in forces], "wall_s": wall,
                      "nodes": steps[0]["nodes"] if steps else 0}), flush=True)
    if out.returncode:
        print(out.stdout[-2000:] + out.stderr[-2000:], file=sys.stderr)


def run_forces(args):
    """ForcesNonLocal (forces.cpp:318-578) alone on a configuration after one
    SQ step of the given precision: W untimed and S timed force passes; one
    JSON line with the kernel time.  For profiling the force kernel."""
    import torch

    from sqdft_b200 import sq
    from sqdft_b200.cases import load as load_named

    torch.cuda.set_device(0)
    case = load_named(args.config)
    prec = {"fp64": sq.SQB_FP64, "mixed": sq.SQB_FP32_MIXED, "all": sq.SQB_FP64}[args.precision]
    with sq.Context(case, device=0, precision=prec) as ctx:
        ctx.set_sweep_rows(args.sweep_rows)
        ctx.nonlocal_projectors()
        ctx.spectral_quadrature(case.scf_iter, case.lambda_f, outputs=False)
        for _ in range(args.warmup):
            ctx.forces_nonlocal()
        ms = []
        for _ in range(args.steps):
            f = ctx.forces_nonlocal()
            st = ctx.stats()
            ms.append(st["ms_forces"])
    kern = float(np.mean(ms)) * 1e-3
    print(json.dumps({"mode": "forces", "config": args.config, "precision": args.precision, "nodes": case.n_nodes,
                      "kernel_ms": kern * 1e3, "nodes_per_s": case.n_nodes / kern,
                      "kernel": "sweep_force_kernel" if st["node_kernel"] == sq.SQB_KERNEL_SWEEP else "node_kernel",
                      "max_abs_force": float(np.abs(f).max())}), flush=True)


def run_local(args):
    """Pseudocharge density and local forces of a configuration: the per-atom
    loops of ChargeDensity (initialize.cpp:470-784) and ForcesLocal
    (forces.cpp:20-315) through sqb_charge_density and sqb_forces_local.  W
    untimed and S timed calls of each; device time from the library's CUDA
    events, e2e with host buffers in and out (phi, Vc, b, b_tilda up; fields
    and forces down).  CPU baseline: the C restatement (single thread, the
    reference's own loops) on a sample of replicas spread over the list,
    scaled to all of them.  Prints one JSON line."""
    import time

    from oracle.pyoracle import LocalOracle
    from sqdft_b200 import sq
    from sqdft_b200.case import read_container
    from sqdft_b200.cases import make_case
    from sqdft_b200.pseudocharge import fields_from_arrays, grid_from_arrays, local_from_arrays

    a = read_container(make_case(args.config))
    grid, loc, f = grid_from_arrays(a), local_from_arrays(a), fields_from_arrays(a)
    cd_ms, fl_ms, wall = [], [], []
    with sq.LocalContext(grid, loc) as ctx:
        for _ in range(args.warmup):
            ctx.charge_density()
            ctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
        for _ in range(args.steps):
            t0 = time.perf_counter()
            cd = ctx.charge_density()
            fl = ctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
            wall.append((time.perf_counter() - t0) * 1e3)
            st = ctx.stats()
            cd_ms.append(st["ms_charge_density"])
            fl_ms.append(st["ms_forces_local"])
    dev_ms = float(np.mean(cd_ms) + np.mean(fl_ms))
    n = loc.n_rep
    line = {"mode": "local", "config": args.config, "replicas": n, "atoms": grid.n_atm,
            "nodes": int(np.prod(grid.np_)), "charge_density_ms": float(np.mean(cd_ms)),
            "forces_local_ms": float(np.mean(fl_ms)), "replicas_per_s": n / (dev_ms * 1e-3),
            "e2e": {"ms": float(np.mean(wall)), "replicas_per_s": n / (float(np.mean(wall)) * 1e-3)},
            "b_matches_export": bool(np.array_equal(cd["b"], f["b"])),
            "max_abs_floc": float(np.abs(fl[0]).max())}
    if not args.no_cpu:
        # the restatement on k replicas spread over the list, per replica
        k = min(n, args.cpu_sample or 16)
        pick = np.unique((np.arange(k) * n) // k)
        import dataclasses

        sub = dataclasses.replace(loc, rep_type=loc.rep_type[pick], rep_atom=loc.rep_atom[pick],
                                  rep_xyz=loc.rep_xyz[pick], rep_box=np.ascontiguousarray(loc.rep_box[pick]))
        o = LocalOracle(grid, sub)
        t0 = time.perf_counter()
        o.charge_density()
        o.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
        secs = time.perf_counter() - t0
        per = secs / len(pick)
        line["cpu_baseline"] = {"value": 1.0 / per, "unit": "replicas/s", "cores": 1, "kind": "port",
                                "sample": f"{len(pick)} of {n} replicas, {secs:.1f} s"}
        line["vs_cpu"] = line["replicas_per_s"] / line["cpu_baseline"]["value"]
    print(json.dumps(line), flush=True)


def run_ours(args):
    if args.precision != "all" and args.sample_nodes > 0:
        return run_sample(args)
    import torch
    import torch.distributed as dist

    from sqdft_b200 import sq
    from sqdft_b200.cases import load as load_named
    from sqdft_b200.dist import allreduce_fn, slab, slab_indices

    rank, ws, local = dist_env()
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    case = load_named(args.config)
    my = slab(case, rank, ws)
    arms = {"all": ["mixed", "lq", "fp64"], "fp64": ["fp64"], "mixed": ["mixed"], "lq": ["lq"]}[args.precision]
    prec_of = {"fp64": sq.SQB_FP64, "mixed": sq.SQB_FP32_MIXED, "lq": sq.SQB_FP64_LANCZOS_QUAD}
    first = prec_of[arms[0]]

    ctx = sq.Context(my, device=local, precision=first, allreduce=allreduce_fn(dist, "cuda") if ws > 1 else None)
    ctx.set_mixed_lanczos(args.mixed_lanczos_tol)
    ctx.set_sweep_rows(args.sweep_rows)
    ctx.nonlocal_projectors()
    n = my.n_nodes
    K1 = my.npl + 1
    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    veff_host = pin(my.veff.shape)
    veff_host[...] = my.veff
    outs = dict(rho=pin((n,)), rho_pj=pin((n, K1)), Ci=pin((n, K1)), chi=pin((n,)), zee=pin((n,)))
    flush = torch.empty(256 * 2**20, dtype=torch.uint8, device="cuda")
    if ws > 1:
        # every step: rank 0 uploads the whole-grid Veff, NCCL broadcasts it,
        # each rank gathers its slab with the Rcut halo on its GPU and hands it
        # to the library (sqb_set_veff_device); after the step the ranks'
        # densities are all-gathered and rank 0 reads the whole grid back
        grid_host = pin(case.veff_block.shape)
        grid_host[...] = case.veff_block
        grid_dev = torch.empty(case.veff_block.shape, dtype=torch.float64, device="cuda")
        _, _, kz, ky, kx = slab_indices(case, rank, ws)
        kz_d, ky_d, kx_d = (torch.from_numpy(k).cuda() for k in (kz, ky, kx))
        rho_dev = torch.empty(n, dtype=torch.float64, device="cuda")
        rho_all = torch.empty(n * ws, dtype=torch.float64, device="cuda")
        rho_all_host = torch.empty(n * ws, dtype=torch.float64).pin_memory()

    import ctypes as C

    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))

    def step():
        flush.fill_(1)  # evict L2 (126 MB) between steps
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        t0 = time.perf_counter()
        if ws > 1:
            if rank == 0:
                grid_dev.copy_(torch.from_numpy(grid_host), non_blocking=True)
            dist.broadcast(grid_dev, src=0)
            vslab = grid_dev.index_select(0, kz_d).index_select(1, ky_d).index_select(2, kx_d).contiguous()
            ctx.set_veff_device(vslab.data_ptr())
        else:
            ctx.set_veff(veff_host)
        lamv = C.c_double(case.lambda_f)
        ebs, eent = C.c_double(), C.c_double()
        rc = ctx.lib.sqb_spectral_quadrature(ctx.ptr, 1, C.byref(lamv), dp(outs["rho"]), dp(outs["rho_pj"]),
                                             dp(outs["Ci"]), dp(outs["chi"]), dp(outs["zee"]), C.byref(ebs),
                                             C.byref(eent))
        if rc:
            raise sq.SQBError(rc, "sqb_spectral_quadrature")
        if ws > 1:
            rho_dev.copy_(torch.from_numpy(outs["rho"]))
            dist.all_gather_into_tensor(rho_all, rho_dev)
            if rank == 0:
                rho_all_host.copy_(rho_all)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        st = ctx.stats()
        dev_ms = st["ms_lanczos_moments"] + st["ms_fermi"] + st["ms_density"] + st["ms_defect"]
        return wall, dev_ms, st, lamv.value, ebs.value

    peak, peak_kind = hbm_peak()
    # DRAM bytes per node matvec step of the node kernel, measured with ncu on
    # a node sample of the configuration (profiles/sweep_kernel_c2_traffic.md)
    traffic = {}
    tr = ROOT / "profiles" / "sweep_kernel_traffic.json"
    if tr.exists():
        traffic = json.loads(tr.read_text()).get(args.config, {})

    def measure(arm, warmup, steps):
        """warmup untimed and steps timed SQ steps of one precision; max over ranks."""
        prec = prec_of[arm]
        ctx.set_precision(prec)
        for _ in range(warmup):
            step()
        walls, devs, node_ms = [], [], []
        with ClockSampler(local) as clocks:
            for _ in range(steps):
                wall, dev_ms, st, lam, ebs = step()
                walls.append(wall)
                devs.append(dev_ms)
                node_ms.append(st["ms_lanczos_moments"])
        t = torch.tensor([np.mean(walls), np.mean(devs) * 1e-3, np.mean(node_ms) * 1e-3], dtype=torch.float64,
                         device="cuda")
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall, dev, kern = t.tolist()
        abytes = algorithmic_bytes(st, my, prec, lq=(arm == "lq"))
        wbytes = algorithmic_bytes(st, my, prec, lq=(arm == "lq"), window=True)
        achieved = abytes / kern / 1e9
        steps_local = st["lanczos_iters"] + n + (0 if arm == "lq" else n * (my.npl // 2))
        per_step = traffic.get(arm)
        return dict(prec=prec, wall=wall, dev=dev, kern=kern, st=st, lam=lam, ebs=ebs, rho=outs["rho"].copy(),
                    clocks=clocks.summary(),
                    roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                              "frac": achieved / peak, "peak_kind": peak_kind,
                              "traffic": (per_step * steps_local) if per_step else None, "algorithmic_bytes": abytes,
                              "frac_window": wbytes / kern / 1e9 / peak, "algorithmic_bytes_window": wbytes,
                              "kernel": "sweep_kernel" if st["node_kernel"] == sq.SQB_KERNEL_SWEEP else "node_kernel",
                              "kernel_ms": kern * 1e3})

    # the line's value: W untimed + K timed steps; the comparison arms: 1 + 1
    # (their kernels are already loaded), which keeps the timed work near a
    # minute on one GPU
    res_arms = {}
    for i, arm in enumerate(arms):
        res_arms[arm] = measure(arm, args.warmup if i == 0 else 1, args.steps if i == 0 else 1)
    head = res_arms[arms[0]]

    def accuracy_of(arm):
        """Differences of an arm's last step from the FP64 arm's (or from one
        untimed FP64 step when the FP64 arm is not run)."""
        r = res_arms[arm]
        if "fp64" in res_arms:
            ref = res_arms["fp64"]
            ref_rho, ref_lam, ref_ebs = ref["rho"], ref["lam"], ref["ebs"]
        else:
            ctx.set_precision(sq.SQB_FP64)
            out = ctx.spectral_quadrature(1, case.lambda_f)
            ref_rho, ref_lam, ref_ebs = out["rho"].reshape(-1), out["lambda_f"], out["Ebs"]
        t = torch.tensor([np.abs(r["rho"] - ref_rho).max(), np.abs(ref_rho).max()], dtype=torch.float64,
                         device="cuda")
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return {"rho_rel_err_vs_fp64": float(t[0] / t[1]), "lambda_f_diff": abs(r["lam"] - ref_lam),
                "ebs_diff_per_atom": abs(r["ebs"] - ref_ebs) / case.n_atm, "lanczos_tol": args.mixed_lanczos_tol}

    acc = {arm: accuracy_of(arm) for arm in arms if arm != "fp64"}

    # nonlocal forces (ForcesNonLocal, forces.cpp:318-578) after the FP64 step,
    # timed; with a fast form run too, its force error against FP64
    forces = None
    if "fp64" in res_arms and not args.no_forces:
        def force_bytes(st, sv):
            # per node and recursion step: t_k, t_k-1 read, t_k+1 written (sv
            # bytes each), Veff, D read and written (FP64); plus the projector
            # balls meeting the window
            return n * my.npl * st["window_points"] * (3 * sv + 24) + st["proj_points"] * 8

        # the context still holds the FP64 arm's last step (the last arm run)
        f64 = ctx.forces_nonlocal()
        st64 = ctx.stats()
        t = torch.tensor([st64["ms_forces"]], dtype=torch.float64, device="cuda")
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fms = float(t[0])
        fb = force_bytes(st64, 8)
        forces = {"step": "ForcesNonLocal after the FP64 SQ step (npl-step Chebyshev recursion of the density-matrix "
                          "column per node, FD gradient, projector contraction)", "nodes_per_s": n * ws / (fms * 1e-3),
                  "kernel_ms": fms, "max_abs_force": float(np.abs(f64).max()), "unit": "nodes/s",
                  "kernel": "sweep_force_kernel" if st64["node_kernel"] == sq.SQB_KERNEL_SWEEP else "node_kernel",
                  "roofline": {"bound": "hbm", "achieved": fb / (fms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                               "frac": fb / (fms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                               "algorithmic_bytes": fb}}
        fast = arms[0] if arms[0] != "fp64" else None
        if fast:
            ctx.set_precision(prec_of[fast])
            ctx.spectral_quadrature(1, case.lambda_f, outputs=False)
            ff = ctx.forces_nonlocal()
            stf = ctx.stats()
            t = torch.tensor([float(np.abs(ff - f64).max()), stf["ms_forces"]], dtype=torch.float64, device="cuda")
            if ws > 1:
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
            forces[f"force_err_{fast}_vs_fp64"] = float(t[0])
            forces[f"{fast}"] = {"nodes_per_s": n * ws / (float(t[1]) * 1e-3), "kernel_ms": float(t[1]),
                                 "recursion_vectors": "fp32" if fast == "mixed" else "fp64"}

    # FP64 arm against the reference's own per-node outputs on a seeded node
    # sample of this configuration (tests/golden/<config>_ref.npz, made by the
    # reference compiled from its sources): bounds and moments
    parity = None
    gold = ROOT / "tests" / "golden" / f"{args.config}_ref.npz"
    if "fp64" in res_arms and ws == 1 and gold.exists():
        z = np.load(gold)
        if "sample_nodes" in z.files and "sample_rho_pj" in z.files:
            ctx.set_precision(sq.SQB_FP64)
            m = ctx.lanczos_moments_nodes(z["sample_nodes"])
            rchi = z["sample_chi"] if "sample_chi" in z.files else z["chi"][z["sample_nodes"]]
            rzee = z["sample_zee"] if "sample_zee" in z.files else z["zee"][z["sample_nodes"]]
            parity = {"nodes": int(len(z["sample_nodes"])), "chi_max_abs": float(np.abs(m["chi"] - rchi).max()),
                      "zee_max_abs": float(np.abs(m["zee"] - rzee).max()),
                      "rho_pj_max_rel": float(np.abs(m["rho_pj"] - z["sample_rho_pj"]).max()
                                              / np.abs(z["sample_rho_pj"]).max()),
                      "reference": f"tests/golden/{args.config}_ref.npz"}

    steps_desc = {
        "fp64": "FP64 SQ step (Lanczos bounds + Chebyshev moments + Fermi level + density), the parity path",
        "mixed": "FP32-mixed SQ step (FP32 Lanczos vectors from a checkerboard-weighted start, looser Lanczos stop; "
                 "FP64 Chebyshev moments, Fermi level, density)",
        "lq": "FP64 Lanczos-quadrature SQ step (bounds and all Chebyshev moments from one Lanczos run per node "
              "through the Gauss-quadrature identity, looser Lanczos stop; Fermi level, density)",
    }
    res = None
    if rank == 0:
        nodes = case.n_nodes
        if ws > 1:  # the whole-grid Veff to rank 0's GPU, each rank's rho up for the gather; outputs down
            h2d = case.veff_block.nbytes + outs["rho"].nbytes * ws
            d2h = sum(a.nbytes for a in outs.values()) * ws + outs["rho"].nbytes * ws
        else:
            h2d = my.veff.nbytes
            d2h = sum(a.nbytes for a in outs.values())
        cpu = cpu_baseline(args) if (ws == 1 and not args.no_cpu) else None
        st = head["st"]
        res = {
            "metric": "SQ grid nodes/s",
            "step": steps_desc[arms[0]] + (" at <= 1e-6 relative rho error vs FP64" if arms[0] != "fp64" else ""),
            "value": nodes / head["dev"], "unit": "nodes/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["dev"] * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64 (mixed)" if arms[0] == "mixed" else "f64",
            "data": "synthetic (seeded-Gaussian-displaced FCC Al; reference first-SCF Veff)",
            "config": {"workload": f"{args.config}: {case.n_int[0]}^3 grid, {nodes} nodes, {case.nw}^3 windows, "
                       f"npl {case.npl}, {case.n_atm} atoms", "nodes": nodes, "window": case.nw, "npl": case.npl,
                       "precision": arms[0], "parallelism": f"z-slabs x{ws}", "l2": "flushed (256 MB write) "
                       "before every step"},
            "e2e": {"value": nodes / head["wall"], "unit": "nodes/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": head["roofline"],
            "gpu_launches": int(st["kernel_launches"]),
            "clocks": head["clocks"],
            "lanczos_iters_per_node": st["lanczos_iters"] / n, "fermi_iters": st["fermi_iters"],
            "lambda_f": head["lam"], "defect_check": {"nodes_redone_fp64": int(st["defect_nodes"]),
                                                      "ms": st["ms_defect"]},
        }
        if arms[0] in acc:
            res["accuracy"] = acc[arms[0]]
        for arm in arms[1:]:
            f = res_arms[arm]
            sub = {"step": steps_desc[arm], "warmup": 1, "steps": 1, "value": nodes / f["dev"], "e2e": nodes / f["wall"],
                   "ms_per_step": f["dev"] * 1e3, "roofline": f["roofline"], "clocks": f["clocks"],
                   "lanczos_iters_per_node": f["st"]["lanczos_iters"] / n,
                   "gpu_launches": int(f["st"]["kernel_launches"]),
                   "defect_check": {"nodes_redone_fp64": int(f["st"]["defect_nodes"]), "ms": f["st"]["ms_defect"]}}
            if arm in acc:
                sub["accuracy"] = acc[arm]
            res[{"fp64": "fp64", "mixed": "fp32_mixed", "lq": "lanczos_quadrature"}[arm]] = sub
        if "fp64" in res_arms and arms[0] != "fp64":
            res["speedup_vs_fp64"] = res_arms["fp64"]["dev"] / head["dev"]
        if parity:
            res["fp64_parity_vs_reference"] = parity
        if forces:
            res["forces"] = forces
        if cpu:
            res["cpu_baseline"] = cpu
    ctx.close()
    if res and ws == 1:
        res["pseudocharge"] = pseudocharge_timing(args.config)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if res:
        print(json.dumps(res), flush=True)


def pseudocharge_timing(config: str, steps: int = 2) -> dict:
    """Device time of one sqb_charge_density and one sqb_forces_local (the
    per-atom loops of ChargeDensity and ForcesLocal) on the configuration,
    after one untimed call; reported beside the SQ step, outside its timed
    region."""
    try:
        from sqdft_b200 import sq
        from sqdft_b200.case import read_container
        from sqdft_b200.cases import make_case
        from sqdft_b200.pseudocharge import fields_from_arrays, grid_from_arrays, local_from_arrays

        a = read_container(make_case(config))
        grid, loc, f = grid_from_arrays(a), local_from_arrays(a), fields_from_arrays(a)
        cd, fl = [], []
        with sq.LocalContext(grid, loc) as lctx:
            for it in range(steps + 1):
                out = lctx.charge_density()
                lctx.forces_local(f["phi"], f["vc"], f["b"], f["b_tilda"])
                if it:
                    st = lctx.stats()
                    cd.append(st["ms_charge_density"])
                    fl.append(st["ms_forces_local"])
        ms = float(np.mean(cd) + np.mean(fl))
        return {"replicas": loc.n_rep, "charge_density_ms": float(np.mean(cd)), "forces_local_ms": float(np.mean(fl)),
                "replicas_per_s": loc.n_rep / (ms * 1e-3), "b_matches_reference_export": bool(np.array_equal(out["b"], f["b"]))}
    except Exception as e:  # reported, never fatal for the SQ line
        return {"unavailable": f"{type(e).__name__}: {e}"[:200]}


def reference_rate(config: str, sample: int, threads: int):
    """Nodes/s of the reference's per-node SQ work on a node sample."""
    from sqdft_b200.case import read_container
    from sqdft_b200.configs.gen_configs import write_system

    drv = ROOT / "oracle" / "_ref" / "sqref_driver"
    pot = ROOT / "oracle" / "_ref" / "pot"
    if not drv.exists():
        return None, "reference build missing (make -C oracle ref)"
    with tempfile.TemporaryDirectory() as td:
        run = write_system(config, Path(td))
        for p in pot.glob("*.pot"):
            (run / p.name).symlink_to(p)
        out = Path(td) / "ref"
        subprocess.run([str(drv), str(run), config, str(out), "--sample", str(sample), "--threads", str(threads)],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        r = read_container(f"{out}_sample.sqc")
    return sample / float(r["t_sample"][0]), None


def cpu_baseline(args):
    threads = os.cpu_count() or 1
    sample = max(2 * threads, 16) if args.cpu_sample <= 0 else args.cpu_sample
    rate, err = reference_rate(args.config, sample, threads)
    if rate is None:
        return {"value": None, "unit": "nodes/s", "cores": threads, "kind": "reference", "sample": err}
    return {"value": rate, "unit": "nodes/s", "cores": threads, "kind": "reference",
            "sample": f"{sample} nodes of {args.config} (reference LanczosAlgorithm + Chebyshev moment loop over "
                      f"HsubTimesVec, g++ -O2), {threads} threads; Fermi solve and density excluded (<1% of the step)"}


def run_reference(args):
    rank, ws, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample = max(2 * threads, 16) if args.cpu_sample <= 0 else args.cpu_sample
    rates = []
    for _ in range(args.warmup):
        reference_rate(args.config, sample, threads)
    for _ in range(args.steps):
        rate, err = reference_rate(args.config, sample, threads)
        if rate is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        rates.append(rate)
    v = float(np.mean(rates))
    desc = (f"{sample} nodes of {args.config} per step (reference LanczosAlgorithm + Chebyshev moment loop over "
            f"HsubTimesVec, g++ -O2), {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": "SQ grid nodes/s",
        "step": "reference FP64 per-node SQ work (LanczosAlgorithm + Chebyshev moment loop)", "value": v, "unit": "nodes/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sample / v * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded-Gaussian-displaced FCC Al; reference first-SCF Veff)",
        "config": {"workload": args.config, "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c2")
    ap.add_argument("--precision", default="all", choices=["all", "fp64", "mixed", "lq"])
    ap.add_argument("--mixed-lanczos-tol", type=float, default=1e-3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forces", action="store_true", help="skip the nonlocal-force timing")
    ap.add_argument("--sample-nodes", type=int, default=0,
                    help="time the node kernel alone on this many nodes (needs --precision fp64|mixed|lq)")
    ap.add_argument("--sweep-rows", type=int, default=0, choices=[0, 2, 3],
                    help="window rows per sweep-kernel thread (0: the library's choice)")
    ap.add_argument("--forces-only", action="store_true",
                    help="one SQ step, then time ForcesNonLocal alone (needs --precision fp64|mixed)")
    ap.add_argument("--scf-steps", type=int, default=0,
                    help="run the drop-in program's SCF loop for this many iterations on --config")
    ap.add_argument("--graph", type=int, default=2, choices=[0, 1, 2],
                    help="with --scf-steps: graph mode of the SQ step (sqb_set_graph)")
    ap.add_argument("--local", action="store_true",
                    help="time the pseudocharge density and local forces (sqb_charge_density, sqb_forces_local)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.scf_steps > 0:
        run_scf(args)
    elif args.forces_only:
        run_forces(args)
    elif args.local:
        run_local(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
