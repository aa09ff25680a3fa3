"""Benchmark: grid-point RK steps/s of the LEE time advance on B200.

Workload (one GPU): 3-D curvilinear block of 256^3 points, x = xi + 0.1 sin(2 pi eta/L)
sin(2 pi zeta/L) and cyclic permutations, uniform mean flow Mach 0.5 along x, eight
Gaussian pulses (amplitude 1e-3, half-width 4, centres from numpy seed 2), RK4 at
CFL 0.5, 4th-order central differences and the 8th-order filter. Synthetic data.

The headline form is FP32 with compensated accumulation; the plain FP64 form is timed
in the same run for the mixed-vs-FP64 ratio, and the p' error of the compensated form
against FP64 after 500 steps is measured in the same run.

`python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]`
For N > 1 (torchrun) every rank advances its own replica: the path does not shard
(one GPU holds all blocks; no inter-GPU exchange), so scaling is weak.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from camille_b200 import api, cases  # noqa: E402

METRIC = "grid-point RK steps/s, mixed vs FP64 @<=1e-5 rel L2 p'; adjoint/forward time"
UNIT = "grid-point RK steps/s"
STAGE_PAIR_DRAM_BYTES_PER_POINT = 130.7
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def measured_hbm_gbs() -> tuple[float, str]:
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.TemporaryFile(mode="w+")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def stage_bytes_per_point(info, comp: bool, sponge_field: bool) -> float:
    """Algorithmic HBM bytes per grid point of one fused stage launch, averaged over the
    four RK4 stages: every stage reads its input, y_n and the accumulator once and writes
    the next input and the accumulator once (words per stage: FP64 3,5,5,3 x V;
    compensated 4,5,5,5 x V, or 4,5,5,3 x V when the last stage writes the increment alone),
    plus the non-uniform coefficient fields (J*metrics) and the summed sponge-strength field
    the TMA stage kernels read where sponges exist."""
    V, e = info.state_vars, info.bytes_per_value
    last = 3 if getattr(info, "increment_step", 0) else 5
    words = (4 + 5 + 5 + last) / 4.0 if comp else (3 + 5 + 5 + 3) / 4.0
    return words * V * e + (info.num_coef_fields + (1 if sponge_field else 0)) * e


def filter_bytes_per_point(info, comp: bool, dim: int) -> float:
    """The fused filter reads the pre-filter state once and writes the filtered state once
    (FP64: 2 V words; compensated: y_pre and its rounding error in -- or y_n and the last stage's
    increment -- and y and its error out, 4 V words); the per-direction passes move more."""
    V, e = info.state_vars, info.bytes_per_value
    if info.tma_filter:
        filt = 4 if comp else 2
    elif comp:
        filt = {2: 3 + 6, 3: 3 + 4 + 6}[dim]
    else:
        filt = {2: 2 + 3, 3: 2 + 2 + 3}[dim]
    return filt * V * e


def step_bytes_per_point(info, comp: bool, dim: int, sponge_field: bool) -> float:
    """Algorithmic bytes per grid point per RK4 step as this build schedules it: four stages
    and the filter."""
    return 4 * stage_bytes_per_point(info, comp, sponge_field) + filter_bytes_per_point(info, comp, dim)


def contract_bytes_per_point(info, comp: bool, sponge_field: bool) -> float:
    """The byte contract of a classic RK4 step, independent of this build's schedule: 18 V state
    words (plain FP64) or 20 V (FP32 with a persistent compensation word read and written once
    per step), plus every per-point coefficient field read once per stage."""
    V, e = info.state_vars, info.bytes_per_value
    return (20 if comp else 18) * V * e + 4 * (info.num_coef_fields + (1 if sponge_field else 0)) * e


SPONGE_FRACTION = 16.0 / 256.0  # sponge width per side, relative to the block size
SPONGE_CONSTANT = 1.0


WORKLOADS = {
    "curvi3d": "curvi3d {n}^3 Mach 0.5, 8 Gaussian pulses (seed 2), RK4 CFL 0.5, OA4 central FD + OA8 filter, "
               "plus an added Freund sponge frame n/16 wide (constant 1) that the plain curvilinear workload "
               "does not have",
    "pulse2d": "pulse2d {n}^2 on [-50,50]^2, quiescent, Gaussian p' pulse, RK4 CFL 0.5, OA4 FD + OA8 filter, "
               "20-cell Freund sponges (constant 5)",
    "batch": "batch2d: 64 independent 2-D Cartesian instances, sides round(exp(U[ln 64, ln 512])) (seed 4, "
             "5.2M points), Mach U[0,0.6], monopole omega U[pi/10, pi/3], 20 N/256-cell sponges, RK4 CFL 0.5 per "
             "instance, batched kernels (one launch per stage and per filter for all instances) in step graphs",
    "cylinder": "cylinder2d: background 512^2 on [-40,40]^2 + O-grid 384x96 (first cell 0.005), 4x4 Lagrange "
                "overset, tanh shear layer damped at the wall, monopole (2,0) omega 0.8 pi, RK4 CFL 0.5",
}


def batch_result(args, K: int, W: int, sample_clocks: bool) -> dict:
    """The batch workload: 64 instances of uneven sizes advanced together (lee_advance_blocks,
    FP32-compensated and FP64) and, for comparison, one at a time in plain FP64 (each instance
    in its own context, its own time step). Returns the measured figures."""
    import torch

    case = cases.batch2d(nsteps=K)
    lib = api.product_library()
    npts = case.npoints
    res = {}
    clocks = None
    for form, prec in (("fp32c", api.FP32_COMPENSATED), ("fp64", api.FP64)):
        s = api.Solver(lib, case, precision=prec)
        dts = s.compute_dt_blocks()
        s.advance_blocks(W, dts)
        torch.cuda.synchronize()
        sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) if form == "fp32c" and sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        s.advance_blocks(K, dts)
        st = s.stats()
        if sampler:
            clocks = sampler.stop()
        s.set_timing(True)
        s.advance_blocks(min(K, args.kernel_steps), dts)
        kst = s.stats()
        s.set_timing(False)
        res[form] = {"ms": st.advance_ms, "launches": st.kernel_launches, "kst": kst, "info": s.info(),
                     "state": [s.download(b)[0] for b in range(len(case.blocks))], "dts": dts,
                     "steps_done": W + K + min(K, args.kernel_steps)}
        s.close()
    # the FP32-compensated step in one persistent launch (lee_set_batch_persistent), for each
    # work-item shape it takes: the same steps, timed the same way, and its bits against the
    # per-phase launches
    pers = {}
    for shape in range(5):
        s = api.Solver(lib, case, precision=api.FP32_COMPENSATED)
        s._chk(lib.set_batch_persistent(s.ctx, shape))
        dts = res["fp32c"]["dts"]
        s.advance_blocks(W, dts)
        torch.cuda.synchronize()
        s.advance_blocks(K, dts)
        ms = s.stats().advance_ms
        launches = s.stats().kernel_launches
        s.advance_blocks(min(K, args.kernel_steps), dts)
        same = all(np.array_equal(s.download(b)[0], res["fp32c"]["state"][b]) for b in range(len(case.blocks)))
        pers[shape] = {"ms_per_step": ms / K, "value": npts * K / (ms / 1e3), "launches": int(launches),
                       "same_bits_as_per_phase": bool(same)}
        s.close()
    best_shape = min(pers, key=lambda q: pers[q]["ms_per_step"])
    # one at a time, plain FP64, the same steps
    alone_s, errs = 0.0, []
    n_done = res["fp32c"]["steps_done"]
    for b in range(len(case.blocks)):
        s = api.Solver(lib, cases.instance(case, b), precision=api.FP64)
        dt = float(res["fp64"]["dts"][b])
        s.advance(W, dt)
        s.advance(K, dt)
        alone_s += s.stats().advance_ms / 1e3
        s.advance(n_done - W - K, dt)
        y = s.download(0)[0]
        errs.append(api.rel_l2(res["fp32c"]["state"][b][4], y[4]))
        s.close()
    value = npts * K / (res["fp32c"]["ms"] / 1e3)
    value64 = npts * K / (res["fp64"]["ms"] / 1e3)
    alone = npts * K / alone_s
    kst = res["fp32c"]["kst"]
    peak, peak_kind = measured_hbm_gbs()
    stage_avg = kst.stage_ms / max(kst.stage_launches, 1)
    filt_avg = kst.filter_ms / max(kst.filter_launches, 1)
    info = res["fp32c"]["info"]
    # 2-D FP32-compensated: stage words 4,5,5,5 x V (V = 4) + the sigma field + the J*metrics
    # fields a block keeps (the off-diagonal terms carry rounding noise of 1e-15); filter 4 V words
    stage_b = ((4 + 5 + 5 + 5) / 4.0 * 4 * 4 + 4 + 4 * info.num_coef_fields) * npts
    filt_b = 4 * 4 * 4 * npts
    step_b = 4 * stage_b + filt_b
    achieved = stage_b / (stage_avg / 1e3) / 1e9
    return {
        "workload": WORKLOADS["batch"], "points": npts, "blocks": len(case.blocks), "steps": K,
        "value": value, "ms_per_step": res["fp32c"]["ms"] / K,
        "fp64": {"value": value64, "ms_per_step": res["fp64"]["ms"] / K},
        "mixed_over_fp64": value / value64,
        "one_at_a_time_fp64": {"value": alone, "ms_per_step": alone_s * 1e3 / K, "batched_fp32c_over_it": value / alone},
        "p_rel_l2_vs_fp64_alone": {"max": max(errs), "median": float(np.median(errs)), "steps": n_done},
        "roofline": {"bound": "hbm", "kernel": "batched RK stage (fp32-compensated)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} copy bandwidth", "traffic": None,
                     "avg_launch_ms": stage_avg, "filter_avg_launch_ms": filt_avg,
                     "filter_gbs": filt_b / (filt_avg / 1e3) / 1e9,
                     "step_gbs": step_b * K / (res["fp32c"]["ms"] / 1e3) / 1e9,
                     "step_frac": step_b * K / (res["fp32c"]["ms"] / 1e3) / 1e9 / peak,
                     "stage_strip": list(info.batch_stage_tile), "filter_strip": list(info.batch_filter_tile)},
        "gpu_launches": int(res["fp32c"]["launches"]), "clocks": clocks,
        "persistent": {"note": "every stage and the filter of a step in one cooperative launch with grid barriers "
                               "(lee_set_batch_persistent), FP32-compensated",
                       "best_shape": best_shape, "value": pers[best_shape]["value"],
                       "ms_per_step": pers[best_shape]["ms_per_step"],
                       "over_per_phase": pers[best_shape]["value"] / value,
                       "by_shape": {str(q): v for q, v in pers.items()}},
    }


def small_workload(name: str, K: int, W: int, err_steps: int) -> dict:
    """A configuration that fits in the L2 (the 2-D pulse at 256^2 with 20-cell sponges, the
    two-block cylinder overset layout): the step time of both precisions through lee_advance's
    replayed step graphs (CUDA events, K steps after W), and the p' error of the compensated
    form against FP64 after err_steps steps from the initial state."""
    case = make_case(name, 256, err_steps)
    lib = api.product_library()
    npts = case.npoints
    nblk = len(case.blocks)
    ms, p = {}, {}
    for form, prec in (("fp32c", api.FP32_COMPENSATED), ("fp64", api.FP64)):
        s = api.Solver(lib, case, precision=prec)
        dt = s.compute_dt(case.cfl) if form == "fp32c" else dt
        s.advance(W, dt)
        s.advance(K, dt)
        ms[form] = s.stats().advance_ms / K
        s.close()
        e = api.Solver(lib, case, precision=prec)
        e.advance(err_steps, dt)
        p[form] = np.concatenate([e.download(b)[0][4].ravel() for b in range(nblk)])
        e.close()
    return {"workload": WORKLOADS[name].format(n=256), "points": npts, "steps": K,
            "value": npts / (ms["fp32c"] / 1e3), "ms_per_step": ms["fp32c"],
            "fp64": {"value": npts / (ms["fp64"] / 1e3), "ms_per_step": ms["fp64"]},
            "mixed_over_fp64": ms["fp64"] / ms["fp32c"],
            "p_rel_l2_vs_fp64": {"value": api.rel_l2(p["fp32c"], p["fp64"]), "steps": err_steps}}


def run_batch(args) -> None:
    """`--workload batch`: the batch figures as the bench line."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    r = batch_result(args, args.steps, args.warmup, sample_clocks=True)
    if rank == 0:
        line = {
            "metric": METRIC, "value": r["value"] * world, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32-compensated (fp64 setup)", "data": "synthetic",
            "config": {"workload": r["workload"], "points_per_gpu": r["points"], "blocks": r["blocks"],
                       "l2": f"state {5 * r['points'] * 4 / 1e6:.0f} MB fp32 vs 126 MB L2",
                       "launch": "batched kernels in replayed CUDA step graphs"},
            "fp64": r["fp64"], "mixed_over_fp64": r["mixed_over_fp64"],
            "one_at_a_time_fp64": r["one_at_a_time_fp64"], "p_rel_l2_vs_fp64_alone": r["p_rel_l2_vs_fp64_alone"],
            "roofline": r["roofline"], "e2e": None, "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "cpu_baseline": None, "persistent": r["persistent"],
        }
        print(json.dumps(line))


def make_case(workload: str, n: int, nsteps: int) -> cases.Case:
    if workload == "curvi3d":
        return bench_case(n, nsteps)
    if workload == "pulse2d":
        return cases.pulse2d(n=n, nsteps=nsteps)
    if workload == "cylinder":
        return cases.cylinder2d(nsteps=nsteps)
    raise ValueError(workload)


def bench_case(n: int, nsteps: int) -> cases.Case:
    """The 3-D curvilinear workload with a Freund sponge frame: closure-only boundaries
    with the Mach 0.5 mean flow make the reference's scheme unstable, so the pinned
    workload absorbs outgoing waves in sponges n/16 cells wide (order 2, constant 1)."""
    width = max(4, int(round(SPONGE_FRACTION * n)))
    case = cases.curvi3d(n=n, nsteps=nsteps, sponge=width, sponge_constant=SPONGE_CONSTANT)
    cases.precompute_sponges(case)
    return case


def replica_barrier(world: int, device: str = "cuda") -> None:
    """Barrier of the replicas (each rank runs the whole workload on its own GPU; there is no
    data-path exchange), then the device drained."""
    import torch
    import torch.distributed as dist

    if world > 1:
        dist.barrier()
    if device == "cuda":
        torch.cuda.synchronize()


def replica_max(x: float, world: int, device: str = "cuda") -> float:
    """The maximum over the ranks of a device-timed figure: the slowest replica sets the job's time."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(points: int, steps: int, ms_max: float, world: int) -> float:
    """Whole-job throughput of `world` replicas, each advancing `points` points by `steps` steps,
    timed by the slowest (ms_max)."""
    return world * points * steps / (ms_max / 1e3)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        replica_barrier(world)

    def max_over_ranks(x: float) -> float:
        return replica_max(x, world)

    n = args.n
    case = make_case(args.workload, n, args.error_steps)
    dim = case.num_dim
    nblk = len(case.blocks)
    lib = api.product_library()
    K, W = args.steps, args.warmup
    results = {}
    solvers = {}
    clocks = None
    for form, prec in (("fp32c", api.FP32_COMPENSATED), ("fp64", api.FP64)):
        kinds = {"filter_kernel": args.filter_kernel} if form == "fp32c" or args.filter_kernel in (-1, 0, 2) else {}
        if args.filter_form and (form == "fp32c" or args.filter_form < 3):
            kinds["filter_form"] = args.filter_form
        s = api.Solver(lib, case, precision=prec, device=local, stage_kernel=args.stage_kernel if form == "fp32c" else -1,
                       **kinds)
        solvers[form] = s
        dt = s.compute_dt(case.cfl)
        s.advance(W, dt)
        barrier()
        sampler = ClockSampler(local) if form == "fp32c" else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        # the product path (replayed step graphs), timed by lee_advance's own CUDA events
        s.advance(K, dt)
        st = s.stats()
        barrier()
        if sampler:
            clocks = sampler.stop()
        ms = max_over_ranks(st.advance_ms)
        # per-kernel launch times, for the roofline: the same steps launched one by one with
        # events between the launches
        s.set_timing(True)
        s.advance(min(K, args.kernel_steps), dt)
        kst = s.stats()
        s.set_timing(False)
        info = s.info()
        results[form] = {"ms": ms, "stats": st, "kstats": kst, "info": info, "dt": dt}
    npts = case.npoints

    # accuracy of the compensated form against FP64 at the step count of the workload
    done = W + K + min(K, args.kernel_steps)
    for s in solvers.values():
        if args.error_steps > done:
            s.advance(args.error_steps - done, results["fp64"]["dt"])
    p32 = np.concatenate([solvers["fp32c"].download(b)[0][4].ravel() for b in range(nblk)])
    p64 = np.concatenate([solvers["fp64"].download(b)[0][4].ravel() for b in range(nblk)])
    err = api.rel_l2(p32, p64)
    solvers["fp64"].close()

    # end to end through the C ABI with host buffers: upload from pinned host memory,
    # K steps, download of the state to pinned host memory
    s = solvers["fp32c"]
    pins = []
    for blk in case.blocks:
        host_in = [torch.from_numpy(np.ascontiguousarray(blk.state[v])).pin_memory() for v in range(5)]
        host_out = [torch.empty_like(host_in[v]).pin_memory() for v in range(5)]
        pin_in = (C.POINTER(C.c_double) * 5)(*[C.cast(t.data_ptr(), C.POINTER(C.c_double)) for t in host_in])
        pin_out = (C.POINTER(C.c_double) * 5)(*[C.cast(t.data_ptr(), C.POINTER(C.c_double)) for t in host_out])
        pins.append((host_in, host_out, pin_in, pin_out))
    dt = results["fp32c"]["dt"]
    barrier()
    t0 = time.perf_counter()
    for b, (_, _, pin_in, _) in enumerate(pins):
        s._chk(lib.upload_state(s.ctx, b, pin_in, 0, 0.0))
    s._chk(lib.advance(s.ctx, K, dt))
    stp, tm = C.c_int(), C.c_double()
    for b, (_, _, _, pin_out) in enumerate(pins):
        s._chk(lib.download_state(s.ctx, b, pin_out, C.byref(stp), C.byref(tm)))
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    state_bytes = 5 * npts * 8

    r32, r64 = results["fp32c"], results["fp64"]
    value = replica_value(npts, K, r32["ms"], world)
    value64 = replica_value(npts, K, r64["ms"], world)
    st = r32["kstats"]
    info = r32["info"]
    peak, peak_kind = measured_hbm_gbs()
    stage_avg_ms = st.stage_ms / max(st.stage_launches, 1)
    filt_avg_ms = st.filter_ms / max(st.filter_launches, 1)
    sponge_field = info.tma_stage == 1 and any(bd.kind.startswith("sponge") for bd in case.boundaries)
    stage_b = stage_bytes_per_point(info, True, sponge_field) * npts
    achieved = stage_b / (stage_avg_ms / 1e3) / 1e9
    filt_b = filter_bytes_per_point(info, True, dim) * npts
    filt_gbs = filt_b / (filt_avg_ms / 1e3) / 1e9
    # DRAM bytes of the two-point stage kernel measured by ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum of one step's four launches at 160^3: 130.7 bytes per point on
    # average), scaled to this launch by its points; other kernels and workloads have no capture
    traffic, traffic_src = None, None
    if args.workload == "curvi3d" and info.stage_kernel == 2 and dim == 3:
        traffic = STAGE_PAIR_DRAM_BYTES_PER_POINT * npts
        traffic_src = "ncu at 160^3 (mean of the four stage launches of a step), scaled by points"
    step_b = step_bytes_per_point(info, True, dim, sponge_field) * npts
    step_gbs = step_b * K / (r32["ms"] / 1e3) / 1e9
    contract_gbs = contract_bytes_per_point(info, True, sponge_field) * npts * K / (r32["ms"] / 1e3) / 1e9
    dominant = "stage" if st.stage_ms >= st.filter_ms else "filter"

    adjoint = None
    if args.workload == "curvi3d" and not args.no_adjoint:
        adjoint = run_adjoint(args, lib, barrier, max_over_ranks)

    # the batch workload (64 uneven 2-D instances), FP32-compensated and FP64 batched and FP64
    # one instance at a time, K steps each
    batch = None
    if args.workload == "curvi3d" and not args.no_batch:
        batch = batch_result(args, args.batch_steps, W, sample_clocks=False)

    # the two L2-resident configurations (2-D pulse at 256^2, cylinder overset), both precisions
    small = None
    if args.workload == "curvi3d" and not args.no_small:
        small = {name: small_workload(name, args.small_steps, W, 500) for name in ("pulse2d", "cylinder")}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, lib, local)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": r32["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32-compensated (fp64 setup)", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload].format(n=n),
                       "points_per_gpu": npts, "blocks": nblk, "parallelism": f"replicas x{world} (no sharding)",
                       "l2": (f"state {5 * npts * 4 / 1e6:.0f} MB fp32 / {5 * npts * 8 / 1e6:.0f} MB fp64 vs "
                              "126 MB L2" + (" (inputs larger than L2)" if 5 * npts * 4 > 126e6 else
                                             " (fits in L2: an L2-resident workload)")),
                       "launch": "replayed CUDA step graphs", "dt": dt},
            "fp64": {"value": value64, "ms_per_step": r64["ms"] / K},
            "mixed_over_fp64": value / value64,
            "p_rel_l2_vs_fp64": {"value": err, "steps": max(args.error_steps, W + K)},
            "roofline": {"bound": "hbm", "kernel": "fused RK stage (fp32-compensated)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} copy bandwidth", "traffic": traffic,
                         "traffic_source": traffic_src,
                         "bytes_per_point": stage_bytes_per_point(info, True, sponge_field),
                         "avg_launch_ms": stage_avg_ms, "dominant": dominant,
                         "filter": {"achieved": filt_gbs, "frac": filt_gbs / peak, "avg_launch_ms": filt_avg_ms,
                                    "bytes_per_point": filter_bytes_per_point(info, True, dim)},
                         "step_gbs": step_gbs, "step_frac": step_gbs / peak,
                         "step_bytes_per_point": step_bytes_per_point(info, True, dim, sponge_field),
                         "contract_bytes_per_point": contract_bytes_per_point(info, True, sponge_field),
                         "contract_frac": contract_gbs / peak,
                         "tma_stage": info.tma_stage, "tma_filter": info.tma_filter,
                         "stage_chunk": info.stage_chunk, "filter_chunk": info.filter_chunk,
                         "filter_kernel": info.filter_kernel, "stage_kernel": info.stage_kernel,
                         "filter_rows": info.filter_rows},
            "e2e": {"value": world * npts * K / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": state_bytes / K, "d2h_bytes_per_step": state_bytes / K,
                    "note": "lee_upload_state from pinned host memory, lee_advance(K), lee_download_state"},
            "gpu_launches": int(r32["stats"].kernel_launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "adjoint": adjoint,
            "batch": batch,
            "l2_resident": small,
        }
        print(json.dumps(line))
    solvers["fp32c"].close()
    if world > 1:
        dist.destroy_process_group()


def run_adjoint(args, lib, barrier, max_over_ranks) -> dict:
    """The adjoint workload: 192^3 curvilinear block, Mach 0.5, a 16^3 distributed
    source, 64 microphones, FP32-compensated forward of `adjoint_steps` steps checkpointed every
    100. Times the forward alone (lee_eval_objective) and the gradient (lee_adjoint_gradient)
    with segment recompute and with the first pass's traces; each timed region is bracketed by
    device synchronisation (lee_* calls return after their stream drained)."""
    n, N = args.adjoint_n, args.adjoint_steps
    case = cases.adjoint3d(n=n, nsteps=N, precompute=True)
    s = api.Solver(lib, case, precision=api.FP32_COMPENSATED)
    dt = s.compute_dt()
    s.eval_objective(min(N, 20), dt)  # warm-up: graph capture, traces
    # warm-up of the gradient: as many checkpoint segments as the timed calls (the checkpoint
    # buffers are allocated on first use) and the reverse step's graphs, both modes
    nseg = max(1, -(-N // 100))
    for rec in (True, False):
        s.upload(0, case.blocks[0].state)
        s.adjoint_gradient(min(N, 10 * nseg), dt, checkpoint_every=10, recompute=rec)
    out = {"workload": f"adjoint3d {n}^3 Mach 0.5, 16^3 distributed source (seed 5), 64 microphones, "
                       f"{N} FP32-compensated RK4 steps, checkpoint every 100",
           "steps": N}
    s.upload(0, case.blocks[0].state)
    barrier()
    t0 = time.perf_counter()
    J0 = s.eval_objective(N, dt)
    fwd = max_over_ranks(time.perf_counter() - t0)
    for label, rec in (("recompute", True), ("traces", False)):
        s.upload(0, case.blocks[0].state)
        barrier()
        t0 = time.perf_counter()
        J, g, mism = s.adjoint_gradient(N, dt, checkpoint_every=100, recompute=rec)
        el = max_over_ranks(time.perf_counter() - t0)
        out[label] = {"seconds": el, "adjoint_over_forward": el / fwd, "trace_mismatches": mism,
                      "objective_matches_forward": J == J0}
    out["forward_seconds"] = fwd
    out["forward_ms_per_step"] = fwd * 1e3 / N
    out["gradient_norm"] = float(np.linalg.norm(g))
    s.close()
    return out


def reference_sample(args, workload: str, n: int, steps: int) -> tuple[cases.Case, str]:
    """A bounded sample of the workload for the compiled reference: the 3-D block at a
    smaller n, the 2-D workloads at full size."""
    if workload == "curvi3d":
        return bench_case(n, steps), f"curvi3d {n}^3 (bounded sample of the {args.n}^3 workload)"
    case = make_case(workload, args.n, steps)
    return case, case.name


def reference_ranks(case: cases.Case, requested: int) -> int:
    cores = os.cpu_count() or 1
    nprocs = requested or min(cores, 8)
    return max(nprocs, len(case.blocks))  # one rank per block at least (src/parallel/decomp.cpp:19-30)


def cpu_baseline(args, lib=None, device: int = 0) -> dict:
    """The compiled reference (oracle/_ref) on a bounded sample of the workload, all host cores,
    at the FIX_CFL time step of the sample's first step. With `lib`, the CUDA library advances
    the same sample in both forms and the errors against the reference's own state are
    reported beside the timing."""
    try:
        from oracle import run_ref
        if not run_ref.available():
            return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                    "sample": "oracle/_ref/camille_ref not built"}
        k = args.cpu_steps
        case, desc = reference_sample(args, args.workload, args.cpu_n, k)
        nprocs = reference_ranks(case, args.ref_ranks)
        dt = None
        ours = {}
        if lib is not None:
            for form, prec in (("fp32c", api.FP32_COMPENSATED), ("fp64", api.FP64)):
                s = api.Solver(lib, case, precision=prec, device=device)
                dt = s.compute_dt(case.cfl)
                s.advance(k, dt)
                ours[form] = [s.download(b)[0] for b in range(len(case.blocks))]
                s.close()
        r = run_ref.run(case, mode="run", nsteps=k, dt=dt, nprocs=nprocs, timeout=900)
        sec = r["result"]["seconds"]
        out = {"value": case.npoints * k / sec, "unit": UNIT, "cores": nprocs, "kind": "reference",
               "sample": f"{desc}, {k} RK4 steps ({'FIX_DT at the CFL time step' if dt else 'FIX_CFL'}), "
                         f"solver::solve wall time, {nprocs} MPI ranks (DECOMP_1D), g++ -O3"}
        if ours:
            ref = run_ref.assemble(case, r["ranks"])
            pr = np.concatenate([y[4].ravel() for y in ref])
            out["errors_vs_reference"] = {
                "steps": k,
                "fp32c_p_rel_l2": api.rel_l2(np.concatenate([y[4].ravel() for y in ours["fp32c"]]), pr),
                "fp64_rel_l2": api.rel_l2(np.concatenate([y.ravel() for y in ours["fp64"]]),
                                          np.concatenate([y.ravel() for y in ref]))}
        return out
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}


def run_reference(args) -> None:
    """Reference arm: the camille reference's own FP64 CPU solver on this box's cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import run_ref
    if not run_ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/camille_ref is not built"}))
        return
    steps = args.steps + args.warmup
    case, desc = reference_sample(args, args.workload, args.ref_n, steps)
    nprocs = reference_ranks(case, args.ref_ranks)
    r = run_ref.run(case, mode="run", nsteps=steps, dt=None, nprocs=nprocs, timeout=1800)
    sec = r["result"]["seconds"]
    value = case.npoints * steps / sec
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": steps, "warmup": 0, "ms_per_step": sec * 1e3 / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{desc}: " + WORKLOADS[args.workload].format(n=args.n), "ranks": nprocs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nprocs, "kind": "reference",
                             "sample": f"{desc} x {steps} steps (FIX_CFL), {nprocs} MPI ranks (DECOMP_1D)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--workload", default="curvi3d", choices=list(WORKLOADS))
    ap.add_argument("--kernel-steps", type=int, default=20,
                    help="steps launched one by one with events between launches (roofline)")
    ap.add_argument("--error-steps", type=int, default=500)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing (the 192^3 adjoint workload)")
    ap.add_argument("--adjoint-n", type=int, default=192)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--cpu-n", type=int, default=64)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-batch", action="store_true", help="skip the batch workload's figures in the default line")
    ap.add_argument("--filter-kernel", type=int, default=-1,
                    help="lee_set_filter_kernel for the run (-1: the library's default; 2, 4: the vectorised filter)")
    ap.add_argument("--filter-form", type=int, default=0,
                    help="lee_set_filter_form (0: timed at setup; 1, 2: one or two rows per thread, both runs; "
                         "3: two points per thread, the FP32-compensated run)")
    ap.add_argument("--stage-kernel", type=int, default=-1,
                    help="lee_set_stage_kernel for the FP32-compensated run (-1: the library's default)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--no-small", action="store_true", help="skip the pulse2d 256^2 and cylinder figures")
    ap.add_argument("--small-steps", type=int, default=200)
    ap.add_argument("--ref-n", type=int, default=64)
    ap.add_argument("--ref-ranks", type=int, default=0, help="reference MPI ranks (0: the host's cores, at most 8)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
