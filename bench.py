"""Throughput of the implicit finite-volume iteration on B200.

Workload (default): the laminar flat plate, 256 x 96 x 2 hexahedra (49,152
cells), Re_L = 1e5, Mach 0.3, Roe flux, Sutherland viscosity, Pr 0.72,
second-order LSQ reconstruction with the Barth-Jespersen limiter, backward
Euler with 5x5 block Jacobians and 10 block point-relaxation sweeps per step,
FP64.  A "step" is one backward-Euler iteration (CFL ramp, local time step,
gradients, face loop + Jacobian assembly, 10 sweeps, update, state + BCs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed]

Multi-GPU: one process per GPU, each advancing its own replica of the case
(the cases are independent; no collective on the data path), value = all
cells x steps / max-over-ranks device time.  The 49k-cell working set fits
the 126 MB L2, so L2 is flushed (a 256 MB write) between timed steps, outside
the timed events.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SWEEPS = 10
WORKLOAD = "laminar flat plate 256x96x2 hex (49,152 cells), Roe + Sutherland, 5x5 blocks, 10 relaxation sweeps/step"


def plate_case():
    from myjoe_b200 import case
    raw, g, prm = case.plate_case(256, 96, 2)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="JACOBI", LS_MAX_ITER=SWEEPS, CFL=1.0,
                              CFL_RAMP=(10, 5, 1.2, 100.0))
    return raw, g, prm


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(g, precision):
    """Compulsory bytes per cell (each array counted once per pass): the face
    loop (residual + Jacobian assembly) and one relaxation sweep, with this
    mesh's internal faces per cell f, blocks per row m = 1 + f_cell, B = 5."""
    d, i = 8, 4
    s = 4 if precision == "mixed" else 8
    B = 5
    f = (g.nfa - g.nfa_b) / g.ncv            # internal faces per cell
    m = 1.0 + 2.0 * f                        # blocks per row (diagonal + one per internal face of the cell)
    face = d * (5 + 15 + 3 + 5) + f * (d * 6 + 4 * i) + s * (B * B + 2 * f * B * B)
    sweep = s * m * B * B + d * 3 * B + i * (m - 1)
    return face, sweep, f, m


class ClockSampler:
    """Read-only NVML samples of the SM clock and the clock-event reasons of the
    GPU this process runs on, every `period` seconds in a thread, until stop().
    The GPU is found by its UUID (from the CUDA device this process uses), so a
    remapping by CUDA_VISIBLE_DEVICES cannot point the query at another GPU."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index, period=0.02):
        import threading
        self.samples, self.uuid, self.error = [], None, None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            u = str(torch.cuda.get_device_properties(device_index).uuid)
            self.uuid = u if u.startswith("GPU-") else "GPU-" + u
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByUUID(self.uuid)
            self._max = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: the line says why
            self.error = "%s: %s" % (type(e).__name__, e)
            return
        self._thread = threading.Thread(target=self._run, args=(period,), daemon=True)
        self._thread.start()

    def _run(self, period):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self._h))
                self.samples.append((sm, rs))
            except Exception as e:
                self.error = "%s: %s" % (type(e).__name__, e)
                return
            self._stop.wait(period)

    def stop(self):
        if self._thread is None:
            return {"error": self.error} if self.error else None
        self._stop.set()
        self._thread.join(timeout=5)
        if not self.samples:
            return {"gpu_uuid": self.uuid, "samples": 0, "error": self.error}
        sm = sorted(x for x, _ in self.samples)
        reasons = sorted({nm for _, rs in self.samples for nm, bit in self.REASONS if rs & bit})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self._max, "reasons": reasons,
                "samples": len(sm), "gpu_uuid": self.uuid}


def reference_run(raw, prm, nsteps, nproc):
    """The reference's own runBackwardEuler (oracle/_ref/ref_harness, built
    from its sources) on the same mesh, BCGSTAB with MAX_ITER = 10; nproc
    independent processes, one per host core.  Returns (cells*steps/s, secs)."""
    from myjoe_b200 import meshgen
    from oracle import refrun
    if not refrun.available():
        return None
    rp = dataclasses.replace(prm, LINEAR_SOLVER_NS="BCGSTAB", LS_MAX_ITER=SWEEPS, NSTEPS=nsteps)
    with tempfile.TemporaryDirectory(prefix="joe_ref_bench_") as d:
        meshgen.write_msh(os.path.join(d, "mesh.msh"), raw)
        with open(os.path.join(d, "Joe.in"), "w") as f:
            f.write(rp.joe_in("mesh.msh"))
        procs = []
        for k in range(nproc):
            wd = os.path.join(d, "r%d" % k)
            os.mkdir(wd)
            os.symlink(os.path.join(d, "mesh.msh"), os.path.join(wd, "mesh.msh"))
            os.symlink(os.path.join(d, "Joe.in"), os.path.join(wd, "Joe.in"))
            os.mkdir(os.path.join(wd, "out"))
            procs.append(subprocess.Popen([refrun.HARNESS, "Joe.in", "0", "run", "out"], cwd=wd,
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        secs = []
        for p in procs:
            out, _ = p.communicate(timeout=1800)
            for line in out.splitlines():
                if line.startswith("HARNESS_SECONDS"):
                    secs.append(float(line.split()[1]))
        if len(secs) != nproc:
            return None
    ncv = raw.ncv
    return nproc * ncv * nsteps / max(secs), max(secs)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    raw, g, prm = plate_case()
    nproc = os.cpu_count() or 1
    # bounded sample: the reference takes ~0.3-0.5 s per iteration of this case on one core
    nsteps = max(1, min(args.steps, 20))
    r = reference_run(raw, prm, nsteps, nproc)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref/ref_harness not built"}))
        return
    value, secs = r
    line = {"metric": "cell-iters/s", "value": value, "unit": "cell-iters/s", "n_gpus": args.gpus,
            "steps": nsteps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / nsteps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seed-generated mesh)", "impl": "reference",
            "config": {"workload": WORKLOAD + " (reference: BCGSTAB MAX_ITER=10)", "cells": raw.ncv},
            "cpu_baseline": {"value": value, "unit": "cell-iters/s", "cores": nproc, "kind": "reference",
                             "sample": "%d backward-Euler iterations per process, %d independent processes "
                                       "(one per host core)" % (nsteps, nproc)},
            "e2e": {"value": value, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


CONVERGE_WORKLOAD = ("burst of seeded channel-bump cases (hex, 2 cell layers; cells log-uniform, Mach U(0.3,0.8), "
                     "AoA U(+-4 deg), bump U(0.05,0.12)), inviscid HLLC, second order, far field, SGS x10, "
                     "CFL 1 -> 20, each retired at a 1e-8 drop of its L1 energy residual")


HBM_WORKLOAD = ("channel bump 1400x700x2 hex (1,960,000 cells), HLLC, second order, far field, JACOBI x10, "
                "cells grouped by Gauss-Seidel colour in RCM order; the working set (~4 GB FP64) is far above L2")


def build_hbm_case():
    from myjoe_b200 import case
    _, g, prm = case.bump_case(1400, 700, 2, inlet="FARFIELD")
    return g, prm, case.perturbed_state(g.x_cv, prm, 0.0)


def hbm_leg(hcase, nsteps=20):
    """The 5x5 path at HBM scale, FP64 and mixed: ms per step and the face-loop and sweep roofline
    from the in-graph events (the matrix and the state do not fit L2, so no flush is needed)."""
    import torch
    from myjoe_b200 import solver
    g, prm, st0 = hcase
    peak, _ = measured_peaks()
    out = {"workload": HBM_WORKLOAD, "cells": g.ncv, "l2": "working set above L2 (no flush)"}
    p = dataclasses.replace(prm, LINEAR_SOLVER_NS="JACOBI", LS_MAX_ITER=SWEEPS, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 20.0))
    for prec, name in ((0, "fp64"), (1, "mixed")):
        j = solver.JoeGpu(g, p, precision=prec, renumber=2)
        j.set_state(*st0)
        cl, rv, _ = j.autotune(3)
        j.set_state(*st0)
        j.set_profiling(True)
        j.runBackwardEuler(3)
        stream = torch.cuda.ExternalStream(j.stream)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        fm, sm = [], []
        for e0, e1 in ev:
            e0.record(stream)
            j.step_async(1)
            e1.record(stream)
            pr = j.profile()
            fm.append(pr["face_loop_ms"])
            sm.append(pr["linear_solve_ms"])
        torch.cuda.synchronize()
        step_ms = sum(a.elapsed_time(b) for a, b in ev) / nsteps
        face_b, sweep_b, f_int, _ = algorithmic_bytes(g, name)
        face_ms, sweep_ms = sum(fm) / nsteps, sum(sm) / nsteps / SWEEPS
        out[name] = {"ms_per_step": step_ms, "cell_iters_per_s": g.ncv / (step_ms * 1e-3),
                     "launch_shape": {"face_loop": cl, "sweep_kernel": rv},
                     "face_loop": {"ms": face_ms, "bytes_per_cell": face_b,
                                   "achieved_gbs": face_b * g.ncv / (face_ms * 1e-3) / 1e9,
                                   "frac": face_b * g.ncv / (face_ms * 1e-3) / 1e9 / peak},
                     "sweep": {"ms": sweep_ms, "bytes_per_cell": sweep_b,
                               "achieved_gbs": sweep_b * g.ncv / (sweep_ms * 1e-3) / 1e9,
                               "frac": sweep_b * g.ncv / (sweep_ms * 1e-3) / 1e9 / peak}}
        j.close()
    out["peak_gbs"] = peak
    return out


CONFIG3_WORKLOAD = ("precision form: SA-RANS channel bump M 0.7, Re 3e6, shuffled mixed prism/hex mesh 512x400x8 "
                    "(88 prism rows, stretch 1.02; 1,998,848 cells) renumbered by the handle (RCM, each LINE line's cells "
                    "consecutive), HLLC + viscous, "
                    "6x6 coupled blocks, LINE x10, FP64 and mixed")


def run_config3(args):
    """--workload config3: the precision form's 2M-cell workload, FP64 and mixed, one JSON line."""
    import numpy as np
    import torch
    from myjoe_b200 import build, case, solver
    if build.needs_build():
        build.build()
    _, g, prm = case.sa_bump_case(512, 400, 8, mach=0.7, re=3.0e6, bump_h=0.05, stretch=1.02, n_prism=88,
                                  shuffle=True, seed=0)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="LINE", LS_MAX_ITER=SWEEPS, CFL=1.0,
                              CFL_RAMP=(10, 5, 1.2, 1000.0), SECOND_ORDER=False)
    st0 = case.perturbed_state(g.x_cv, prm, 0.0)
    out = {"metric": "cell-iters/s", "unit": "cell-iters/s", "workload": CONFIG3_WORKLOAD, "cells": g.ncv,
           "steps": args.steps, "l2": "working set above L2 (no flush)"}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        j = solver.JoeGpu(g, prm, precision=prec, renumber=args.config3_renumber)
        j.set_state(*st0)
        j.set_scalars(np.full(g.ncv, prm.NUSA_INITIAL))
        j.runBackwardEuler(max(args.warmup, 3))
        j.set_profiling(True)
        stream = torch.cuda.ExternalStream(j.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fm, sm = [], []
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            j.step_async(1)
            pr = j.profile()
            fm.append(pr["face_loop_ms"])
            sm.append(pr["linear_solve_ms"])
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out[name] = {"ms_per_step": ms, "cell_iters_per_s": g.ncv / (ms * 1e-3), "face_loop_ms": sum(fm) / len(fm),
                     "relaxation_ms": sum(sm) / len(sm), "device_bytes": j.device_bytes()}
        j.close()
    out["value"] = out["mixed"]["cell_iters_per_s"]
    print(json.dumps(out))


def build_converge_cases(args, rank, world):
    """This rank's share of one seeded case list of converge_cases cases per GPU (weak scaling in
    cases): each case runs whole on one GPU, balanced by cells (serve.partition_cases)."""
    import multiprocessing as mp
    from myjoe_b200 import serve
    lo, hi = (int(x) for x in args.converge_cells.split(","))
    specs = serve.partition_cases(serve.case_specs(args.converge_cases * world, lo, hi, seed=1000), world, rank)
    with mp.get_context("spawn").Pool(min(len(specs), os.cpu_count() or 1)) as pool:
        return pool.map(serve.build_request, specs)


def converge_leg(cases, args):
    """Converged solves per hour on one GPU: the same case list through the plain FP64 drop-in
    (one case at a time, Jacobian every step) and through the serving form (mixed precision,
    lagged Jacobian, many cases resident)."""
    from myjoe_b200 import serve
    cfg = serve.BurstConfig(jac_lag=args.jac_lag)
    plain = serve.run_burst("plain", cases, cfg)
    served = serve.run_burst("serve", cases, cfg)
    return {"workload": CONVERGE_WORKLOAD, "cases": len(cases), "cells": args.converge_cells,
            "cells_total": int(sum(c[0].ncv for c in cases)),
            "solves_per_hour": served["solves_per_hour"], "p50_s": served["p50_s"], "p99_s": served["p99_s"],
            "plain_fp64": plain, "serving": served,
            "ratio_vs_plain_fp64": served["solves_per_hour"] / plain["solves_per_hour"]
            if plain["solves_per_hour"] > 0 else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--face-loop", default="auto", choices=["auto", "1", "2", "4", "17", "33", "34", "36", "40"],
                    help="face loop shape: autotuned; fused 1/2/4 lanes per cell or 17 (one lane, 3 blocks per SM); "
                         "split 32 + lanes per cell of the residual kernel")
    ap.add_argument("--converge-cases", type=int, default=24,
                    help="cases of the time-to-converge leg (0: skip it)")
    ap.add_argument("--converge-cells", default="5000,500000", help="cells log-uniform on lo,hi")
    ap.add_argument("--jac-lag", type=int, default=4, help="serving arm: flux Jacobian every k-th step")
    ap.add_argument("--no-hbm-leg", dest="hbm_leg", action="store_false",
                    help="skip the 2M-cell HBM-scale leg")
    ap.add_argument("--config3-renumber", type=int, default=3, choices=[1, 3],
                    help="config3's cell order: 1 RCM, 3 RCM with each LINE line consecutive (default)")
    ap.add_argument("--workload", default="plate", choices=["plate", "config3"],
                    help="plate: the headline line; config3: the 2M-cell precision-form workload (own line)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.workload == "config3":
        run_config3(args)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the HBM-scale case is meshed in a spawn process while the time-to-converge cases are meshed by a
    # spawn pool on the host cores, all outside every timed region
    import multiprocessing as mp
    hpool = mp.get_context("spawn").Pool(1) if args.hbm_leg else None
    hjob = hpool.apply_async(build_hbm_case) if hpool else None
    conv_cases = build_converge_cases(args, rank, world) if args.converge_cases > 0 else None
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from myjoe_b200 import build, case, solver
    if build.needs_build():
        build.build()
    raw, g, prm = plate_case()
    precision = 1 if args.precision == "mixed" else 0
    j = solver.JoeGpu(g, prm, precision=precision)
    st0 = case.perturbed_state(g.x_cv, prm, 0.0)
    j.set_state(*st0)
    # launch shapes picked on this mesh before any timing (jg_autotune; a set-up step of the API)
    tuned_cl, tuned_sweep, _ = j.autotune(5)
    if args.face_loop != "auto":
        tuned_cl = int(args.face_loop)
        j.set_launch_config(tuned_cl, tuned_sweep)
    j.set_state(*st0)
    kernels_per_step = j.step_kernel_count()
    stream = torch.cuda.ExternalStream(j.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(max(args.warmup, 3)):
        j.step_async(1)
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            starts[k].record(stream)
            j.step_async(1)
            ends[k].record(stream)
            flush.add_(1.0)   # > L2: evict the case before the next timed step
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    # the face loop and the relaxation, from CUDA events inside the step graph, over a second pass
    # of the same K steps under the same L2 flush: event nodes between the kernels lengthen a step
    # (they split the graph's launch stream), so the timed steps above run without them
    face_ms, solve_ms = [], []
    j.set_profiling(True)
    j.step_async(2)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            j.step_async(1)
        prof = j.profile()
        face_ms.append(prof["face_loop_ms"])
        solve_ms.append(prof["linear_solve_ms"])
        with torch.cuda.stream(stream):
            flush.add_(1.0)
    torch.cuda.synchronize()
    j.set_profiling(False)
    total_s = sum(step_ms) / 1000.0
    if world > 1:
        t = torch.tensor([total_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_s = float(t.item())
    value = world * g.ncv * args.steps / total_s
    res = j.runBackwardEuler(1)
    finite = bool(np.all(np.isfinite(res)))

    # end to end through the C ABI from pinned host buffers: upload, step, download
    n = g.ncv
    h_rho = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    h_rhou = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    h_rhoE = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    h_res = torch.empty((1, 5), dtype=torch.float64, pin_memory=True).numpy()
    rho, rhou, rhoE = j.get_state()
    h_rho[:], h_rhou[:], h_rhoE[:] = rho, rhou, rhoE
    import ctypes as C
    from myjoe_b200.abi import dptr
    L = solver.lib()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        # jg_step_host: the state up from the pinned arrays, the preamble and one step, the new state
        # and the step's residual back into pinned memory, one synchronisation
        solver._ck(L.jg_step_host(j.h, dptr(h_rho), dptr(h_rhou), dptr(h_rhoE), 1, dptr(h_res)))
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * n * args.steps / e2e_s

    # like for like with the reference arm: the same case with the GPU's BiCGSTAB x10 (the
    # reference's LINEAR_SOLVER_NS_TRESHOLDS MAX_ITER=10), FP64, host-driven iterations
    jb = solver.JoeGpu(g, dataclasses.replace(prm, LINEAR_SOLVER_NS="BCGSTAB", LS_MAX_ITER=SWEEPS), precision=0)
    jb.set_state(*st0)
    jb.runBackwardEuler(max(args.warmup, 3))
    nb = max(5, min(args.steps, 50))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    jb.runBackwardEuler(nb)
    torch.cuda.synchronize()
    bcg_s = time.perf_counter() - t0
    jb.close()
    bicgstab = {"value": g.ncv * nb / bcg_s, "unit": "cell-iters/s", "steps": nb,
                "linear_solver": "BCGSTAB MAX_ITER=%d (the reference arm's solver), FP64" % SWEEPS,
                "timing": "wall clock around synchronised host-driven steps"}

    conv = converge_leg(conv_cases, args) if conv_cases else None
    hbm = None
    if hjob is not None:
        hcase = hjob.get()
        hpool.close()
        hbm = hbm_leg(hcase)
        del hcase
    if world > 1 and conv is not None:
        from myjoe_b200 import serve
        allc = [None] * world
        dist.all_gather_object(allc, conv)
        conv = serve.merge_rank_results(allc)
    clk = clocks.stop()
    if clk is not None:
        clk["window"] = "the timed steps, the e2e, BiCGSTAB, time-to-converge and HBM-scale legs"

    # roofline of the dominant kernel, from the live in-graph events
    face_b, sweep_b, f_int, m_blk = algorithmic_bytes(g, args.precision)
    peak, peak_kind = measured_peaks()
    face_avg = sum(face_ms) / len(face_ms)
    solve_avg = sum(solve_ms) / len(solve_ms)
    sweep_avg = solve_avg / SWEEPS
    sweep_gbs = sweep_b * n / (sweep_avg * 1e-3) / 1e9
    face_gbs = face_b * n / (face_avg * 1e-3) / 1e9
    split = tuned_cl >= 32
    face_name = ("face loop: k_res (residual, %d lanes per cell) beside k_jac (Jacobian blocks) on a second stream"
                 % (tuned_cl - 32) if split else "k_flux (fused face loop + Jacobian assembly)")
    if solve_avg >= face_avg:
        dom = {"kernel": "k_jacobi (block point-relaxation sweep)", "bound": "hbm", "achieved": sweep_gbs,
               "peak": peak, "unit": "GB/s", "frac": sweep_gbs / peak, "traffic": None,
               "bytes_per_cell": sweep_b, "launch_ms": sweep_avg}
        other = {"kernel": face_name, "achieved": face_gbs, "frac": face_gbs / peak,
                 "bytes_per_cell": face_b, "launch_ms": face_avg}
    else:
        dom = {"kernel": face_name, "bound": "hbm", "achieved": face_gbs,
               "peak": peak, "unit": "GB/s", "frac": face_gbs / peak, "traffic": None,
               "bytes_per_cell": face_b, "launch_ms": face_avg}
        other = {"kernel": "k_jacobi (block point-relaxation sweep)", "achieved": sweep_gbs, "frac": sweep_gbs / peak,
                 "bytes_per_cell": sweep_b, "launch_ms": sweep_avg}
    dom["launch_ms_source"] = ("CUDA events inside the step graph, averaged over a second pass of the same "
                               "steps (the timed steps run without the event nodes)")
    dom["peak_source"] = peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind
    prof_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_path):
        with open(prof_path) as f:
            tr = json.load(f)
        key = "k_jacobi" if dom["kernel"].startswith("k_jacobi") else "face_loop"
        if key in tr and args.precision in tr[key]:
            entry = tr[key][args.precision]
            if key == "face_loop":  # per launch shape
                entry = entry.get(str(tuned_cl))
            if entry:
                dom["traffic"] = entry["bytes_per_cell"] * n
                dom["traffic_source"] = entry["source"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = reference_run(raw, prm, 6, 1)
        if r is not None:
            cpu = {"value": r[0], "unit": "cell-iters/s", "cores": 1, "kind": "reference",
                   "sample": "6 backward-Euler iterations of the same 49,152-cell case by the reference "
                             "(BCGSTAB MAX_ITER=10), one process"}

    if rank == 0:
        line = {"metric": "cell-iters/s", "value": value, "unit": "cell-iters/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": 1000.0 * total_s / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64 residual / f32 Jacobian+relaxation",
                "data": "synthetic (seed-generated mesh, uniform free-stream start)",
                "config": {"workload": WORKLOAD, "cells": n, "internal_faces_per_cell": round(f_int, 4),
                           "precision": args.precision, "l2": "flushed between timed steps (256 MB write)",
                           "parallelism": "replicas" if world > 1 else "single case",
                           "launch_shape": {"face_loop": (("split: residual %d lanes per cell + Jacobian kernel"
                                                           % (tuned_cl - 32)) if split else
                                                          "fused, 1 lane per cell, 3 blocks per SM" if tuned_cl == 17
                                                          else "fused, %d lanes per cell" % tuned_cl),
                                            "code": tuned_cl, "sweep_kernel": tuned_sweep}},
                "e2e": {"value": e2e, "unit": "cell-iters/s", "h2d_bytes_per_step": 5 * 8 * n,
                        "d2h_bytes_per_step": 5 * 8 * n + 40,
                        "api": "jg_step_host per step: the state (rho, rhou, rhoE) from pinned host arrays, "
                               "the state preamble and one step, the state and the residual back; "
                               "host wall clock"},
                "gpu_launches": kernels_per_step * args.steps,
                "roofline": dom, "roofline_other": other,
                "face_loop_ms": face_avg, "relaxation_ms": solve_avg,
                "finite_residual": finite,
                "bicgstab_like_for_like": bicgstab,
                "time_to_converge": conv,
                "hbm_scale": hbm,
                "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line))
    j.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
