"""Coupled-step throughput of ferrox_b200 on one node.

A step is one pass of FerroX's time loop (Source/main.cpp:261-621): the
semiconductor-charge Newton loop with its Poisson multigrid solves, the fused
TDGL update with E from phi, and the steady-state check.  The default workload
is the 64-grain polycrystalline film, 256x256x128 cells (5 nm HZO in 64
seeded Voronoi grains, 70% ferroelectric with random polar axes, on 4 nm
Al2O3), in the mixed-precision form (FP32 stencils and multigrid inside FP64
iterative refinement, FP64 P state), Poisson to 1e-10 relative residual, with
seeded synthetic initial polarization.  The line's "mixed_vs_fp64" times the
plain FP64 step beside it on the same deck and gives every output field's max
relative difference.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload polycrystal|mfism|mfim] [--precision mixed|fp64]
                    [--no-adjoint] [--adjoint-steps-per-leg S] [--adjoint-scale-steps S]

At N = 1 the line also carries "adjoint": the time of fx_backward over
fx_forward_record for the hysteresis loss on the 128x128x48 MFIM stack (800
steps, checkpoints every 50, gradients in alpha, beta, gamma, g11, g44 and
the voltage amplitude), and "adjoint_polycrystal": the same on the 256x256x128
polycrystal with the 64 per-grain alphas, in FP64 and in mixed precision.

The first solve of a step starts from phi extrapolated in time from the last
steps (order 4 by default), so a run's first steps take more V-cycles; the
config names the order and the steps of history at the start of the timed
region.

Multi-GPU runs are independent replicas (one process per GPU, weak scaling):
the path has no data exchange between devices.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "mfism": dict(shape=(128, 128, 144), label="MFISM 5nm HZO/1nm SiO2/30nm p-Si, Newton-coupled"),
    "mfim": dict(shape=(64, 64, 36), label="MFIM 5nm HZO/4nm Al2O3"),
    "polycrystal": dict(shape=(256, 256, 128), label="64-grain polycrystalline HZO on Al2O3"),
}
METRIC = "coupled-step cell-updates/s"
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum, one ncu
# capture, cold cache) of the dominant bandwidth-bound kernel class, by
# (workload, precision, class), with the profile that holds the capture
TRAFFIC = {("mfism", "fp64", "smooth_l0"): (56.72e6, "profiles/k_rbgs_seg_l0_mfism_128x128x144.txt"),
           ("polycrystal", "mixed", "smooth_l0"): (42.64e6, "profiles/k_rbgs_split_l0_polycrystal_mixed.txt")}
FALLBACK_HBM_GBS = 6650.0


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time: every rank takes part in the same MAX
    all-reduce (a no-op on one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells: int, steps: int, world: int, ms_max: float) -> float:
    """Cell updates per second of the whole job: every replica advances its
    own copy of the deck (weak scaling), timed by the slowest rank."""
    return cells * steps * world / (ms_max / 1e3)


def deck(name: str):
    from ferrox_b200 import decks
    nx, ny, nz = WORKLOADS[name]["shape"]
    if name == "mfism":
        return decks.mfism(nx, ny, nz), None
    if name == "mfim":
        return decks.mfim(nx, ny, nz), None
    return decks.polycrystal(nx, ny, nz, ngrains=64, seed=1)


def run_config(args, cells: int) -> dict:
    """The workload the line is quoted on; the same dict on both arms."""
    shape = WORKLOADS[args.workload]["shape"]
    extra = {"settings": list(args.set)} if getattr(args, "set", None) else {}
    return {**extra, "workload": f"{args.workload}-{'x'.join(map(str, shape))}-{args.precision}",
            "description": WORKLOADS[args.workload]["label"], "cells": cells, "mg_rtol": 1e-10,
            "parallelism": "replicas",
            "l2": "inputs larger than L2 (126 MB): every field of the deck is >= 19 MB and the step touches "
                  "hundreds of MB",
            # the run-length dependence: the first solve of a step starts from
            # phi extrapolated in time through the first solves of the last steps
            "phi_extrapolate_order": 4,
            "history_steps_at_timed_start": min(args.warmup, 4)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.idx)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler is live
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:
                time.sleep(0.01)
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(kernel: str, N: int, Nc1: int, sc: bool, scalar: bool, rot: bool, fp: int = 8,
                      planes: bool = False) -> float:
    """Compulsory bytes of one launch: each distinct array read once, each
    output written once; stencil neighbours and ghosts count once.  planes:
    level 0's coefficients depend on z only (a layered stack), so its
    smoother needs no material codes."""
    a = fp if sc else 0
    code = 0 if planes else 1
    if kernel == "smooth_l0":      # one red or black half-sweep: half of a full sweep
        return N * (fp + fp + code + fp + a) / 2.0
    if kernel == "restrict_l0":
        return N * (fp + fp + 1 + a) + Nc1 * fp
    if kernel == "prolong_l0":     # x in and out, the coarse correction, one weight per fine cell
        return N * 2 * fp + Nc1 * fp + N * 4
    if kernel == "tdgl":
        return N * ((3 if scalar else 7) * 8 + 1 + (1 if rot else 0))
    if kernel == "newton":
        return N * (8 * 5 + 4 + 1)
    if kernel == "rho":
        return N * (8 * 3 + 1) + (N * 24 if sc else 0)
    if kernel == "resid64":
        return N * (8 + 8 + 1 + a + 4)
    if kernel == "rhs_p":
        return N * ((1 if scalar else 3) * 8 + 1 + 8)
    if kernel == "steady":
        return N * 8 * 4
    return 0.0


def cpu_baseline(text: str, grains, steps: int) -> dict:
    from ferrox_b200 import decks
    from oracle import inputs as I
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    table = I.parse_table(text)
    p = I.ferrox_params(table)
    if grains is not None:
        tph, ang = decks.grain_fields(grains)
        o = O.Oracle(p, tph, tuple(ang), threads=threads)
    else:
        o = O.Oracle.from_text(text, threads=threads)
    o.step(1)  # warm-up (first Newton pass from the intrinsic charge)
    t0 = time.perf_counter()
    for s in range(2, 2 + steps):
        o.step(s)
    dt = time.perf_counter() - t0
    n = p["n_cell"][0] * p["n_cell"][1] * p["n_cell"][2]
    return {"value": n * steps / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{steps} full coupled steps of the same deck after 1 warm-up step (restated CPU oracle, "
                      f"OpenMP, {threads} threads; the reference build needs AMReX, absent)",
            "seconds": dt}


def precision_compare(stream, workload: str, steps: int, warmup: int) -> dict:
    """The mixed-precision step next to the plain FP64 step on the same seeded
    deck: ms per step of each (CUDA events on the library's stream) and the
    max-norm relative difference of the output fields after warmup + steps
    steps (FP64 taken as the reference)."""
    import numpy as np
    import torch
    from ferrox_b200 import api
    text, grains = deck(workload)
    out, fields = {}, {}
    for prec in ("fp64", "mixed"):
        f = api.FerroX(text, precision=prec)
        if grains is not None:
            f.set_grains(grains["id"], grains["angles"], grains["tphase"])
        f.set_stream(stream.cuda_stream)
        f.step(warmup)
        f.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        out[f"{prec}_ms_per_step"] = e0.elapsed_time(e1) / steps
        f.compute_E()
        names = ["Px", "Py", "Pz", "Phi", "Ex", "Ey", "Ez"] + (["charge", "electrons", "holes"]
                                                              if f.param("contains_sc") == 1.0 else [])
        fields[prec] = {n: f.field(n) for n in names}
        f.close()
    rel = {}
    for n, ref in fields["fp64"].items():
        scale = float(np.abs(ref).max())
        if scale > 0:
            rel[n] = float(np.abs(fields["mixed"][n] - ref).max() / scale)
    out.update({"speedup": out["fp64_ms_per_step"] / out["mixed_ms_per_step"], "steps": warmup + steps,
                "relerr_vs_fp64": rel, "max_relerr": max(rel.values())})
    return out


def adjoint_ratio(stream, precision: str = "fp64", steps_per_leg: int = 400, k: int = 50) -> dict:
    """Gradient of the hysteresis loss on the 128x128x48 MFIM stack (5 nm HZO
    on 4 nm Al2O3) over a triangular sweep -3 V -> +3 V -> -3 V with
    steps_per_leg steps per leg, with respect to alpha, beta, gamma, g11, g44
    and the voltage amplitude; checkpoints every k steps.  Times
    fx_forward_record and fx_backward with CUDA events on the library's
    stream and returns their ratio."""
    import torch
    from ferrox_b200 import api, decks
    v_amp = 3.0
    shape = decks.triangular_sweep(1.0, steps_per_leg)
    target = decks.target_loop(v_amp * shape, seed=7, ps=0.15, vc=1.2)
    text = decks.hysteresis(128, 128, 48, v_amp=v_amp, steps_per_leg=steps_per_leg)
    # the second record of a context is timed, as an optimisation loop (one
    # record and one backward per iteration) sees it: the first pays the
    # module load, the graph captures and the record's allocations
    f = api.FerroX(text, precision=precision)
    f.set_stream(stream.cuda_stream)
    Pz0, phi0 = f.field("Pz"), f.field("Phi")
    f.forward_record(target, v_amp, shape, k)
    f.backward()
    # the timed record starts from the same state as the first
    f.set_initial_P(None, None, Pz0)
    f.set_field("Phi", phi0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    loss = f.forward_record(target, v_amp, shape, k)
    ev[1].record(stream)
    g = f.backward()
    ev[2].record(stream)
    torch.cuda.synchronize()
    fwd, bwd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    T = len(shape)
    out = {"workload": f"hysteresis-128x128x48-{precision}", "steps": T, "checkpoint_every": k,
           "forward_ms": fwd, "backward_ms": bwd, "ratio": bwd / fwd, "loss": loss,
           "grads": dict(zip(api.GRADS, map(float, g))),
           "adjoint_mg_cycles_per_step": f.param("adjoint_mg_cycles") / T,
           "record_bytes": f.param("adjoint_bytes"),
           "note": "backward = segment recompute + adjoint; ratio = backward / forward"}
    f.close()
    return out


def adjoint_scale(stream, steps: int, k: int = 50) -> dict:
    """The adjoint on the 256x256x128 polycrystalline film (64 grains): the
    hysteresis loss over a triangular sweep of `steps` steps, differentiated
    with respect to the 64 per-grain alphas and g11 (and the other
    coefficients), in FP64 and in mixed precision; checkpoints every k steps.
    Reports each precision's forward and backward times and the mixed
    gradient's relative error against the FP64 one."""
    import numpy as np
    import torch
    from ferrox_b200 import api, decks
    text, g = decks.polycrystal(256, 256, 128, ngrains=64, seed=1)
    v_amp = 3.0
    shape = decks.triangular_sweep(1.0, steps // 2)
    target = decks.target_loop(v_amp * shape, seed=7, ps=0.15, vc=1.2)
    out, grads = {}, {}
    for prec in ("fp64", "mixed"):
        f = api.FerroX(text, precision=prec)
        f.set_grains(g["id"], g["angles"], g["tphase"])
        f.set_stream(stream.cuda_stream)
        # the second record of the context is timed (see adjoint_ratio)
        Pz0, phi0 = f.field("Pz"), f.field("Phi")
        f.forward_record(target, v_amp, shape, k)
        f.backward(ngrains=64)
        f.set_initial_P(None, None, Pz0)
        f.set_field("Phi", phi0)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        loss = f.forward_record(target, v_amp, shape, k)
        ev[1].record(stream)
        grads[prec] = f.backward(ngrains=64)
        ev[2].record(stream)
        torch.cuda.synchronize()
        fwd, bwd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
        out[prec] = {"forward_ms": fwd, "backward_ms": bwd, "ratio": bwd / fwd, "loss": loss,
                     "record_bytes": f.param("adjoint_bytes")}
        f.close()
    a, b = grads["mixed"], grads["fp64"]
    grain = [q for q in range(64) if b[6 + q] != 0.0]
    rel = {n: float(abs(a[q] - b[q]) / abs(b[q])) for q, n in enumerate(api.GRADS) if b[q] != 0.0}
    rel["grain_alpha_max"] = float(max(abs(a[6 + q] - b[6 + q]) / abs(b[6 + q]) for q in grain))
    out.update({"workload": "polycrystal-256x256x128, 64 grains", "steps": len(shape), "checkpoint_every": k,
                "mixed_vs_fp64_grad_relerr": rel, "ferroelectric_grains": len(grain)})
    return out


def apply_settings(ctx, args):
    """The --set KEY=VALUE solver settings, applied to a measured context."""
    for kv in args.set:
        key, _, val = kv.partition("=")
        ctx.set_param(key.strip(), float(val))


def e2e_leg(args, api, text, grains, stream, N, world, ke, barrier, torch) -> dict:
    """The metric end to end through the public API: a second context of the
    same deck runs the same W warm-up steps (untimed) and then the same K
    steps as the timed leg, so both legs cover the same stretch of the run
    with the same history of phi.  The state stays resident in HBM, as the
    reference's MultiFabs stay on its device; per step the host sets the
    electrode voltage (fx_set_param, the step's input), runs fx_step(1) and
    reads the mean polarization back (fx_mean_P, the step's result); at the
    end P and phi are read into pinned host buffers (fx_get_field)."""
    g = api.FerroX(text, precision=args.precision)
    if grains is not None:
        g.set_grains(grains["id"], grains["angles"], grains["tphase"])
    if args.host_loop:
        g.set_param("fx.step_graph", 0)
    apply_settings(g, args)
    g.set_stream(stream.cuda_stream)
    g.step(args.warmup)
    g.sync()
    comps = ["Pz"] if g.param("is_polarization_scalar") == 1.0 else ["Px", "Py", "Pz"]
    outs = {n: torch.empty(g.shape, dtype=torch.float64, pin_memory=True).numpy() for n in comps + ["Phi"]}
    barrier()
    torch.cuda.synchronize()
    se0 = g.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        g.set_param("Phi_Bc_hi", g.stats()["Phi_Bc_hi"])
        g.step(1)
        g.mean_P()
    for n, buf in outs.items():
        g.field(n, out=buf)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    se1 = g.stats()
    g.close()
    ems = max_over_ranks(e0.elapsed_time(e1), world)
    return {"value": whole_job_rate(N, ke, world, ems), "unit": "cell-updates/s", "h2d_bytes_per_step": 8.0,
            "d2h_bytes_per_step": (ke * 24 + len(outs) * N * 8) / ke, "steps": ke,
            # a second context: the same warm-up and the same steps as the timed leg
            "after_steps": args.warmup,
            "mg_cycles_per_step": (se1["mg_cycles_total"] - se0["mg_cycles_total"]) / ke}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import inputs as I
    from oracle import oracle as O
    from ferrox_b200 import decks
    text, grains = deck(args.workload)
    threads = os.cpu_count() or 1
    p = I.ferrox_params(I.parse_table(text))
    if grains is not None:
        tph, ang = decks.grain_fields(grains)
        o = O.Oracle(p, tph, tuple(ang), threads=threads)
    else:
        o = O.Oracle.from_text(text, threads=threads)
    step = 0
    for _ in range(args.warmup):
        step += 1
        o.step(step)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step += 1
        o.step(step)
    dt = time.perf_counter() - t0
    n = p["n_cell"][0] * p["n_cell"][1] * p["n_cell"][2]
    v = n * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": run_config(args, n),
            "reference_precision": "fp64 (the reference has no mixed-precision path)",
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full coupled steps after {args.warmup} warm-up steps "
                                       f"(restated CPU oracle in FP64, OpenMP {threads} threads; the reference "
                                       "build needs AMReX, absent)"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="polycrystal", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    # leave out the FP64 side-by-side and the e2e leg (short runs under a profiler)
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    # the same kernels driven by the host loop (a synchronisation per loop
    # test) instead of one graph per step; ncu profiles kernels only there
    ap.add_argument("--host-loop", action="store_true")
    # a solver setting of the measured contexts (fx_set_param), e.g. --set fx.mg_seg=16
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE")
    ap.add_argument("--adjoint-steps-per-leg", type=int, default=400)
    ap.add_argument("--adjoint-scale-steps", type=int, default=400,
                    help="also run the polycrystal adjoint (FP64 and mixed) over this many steps")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    from ferrox_b200 import api

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    text, grains = deck(args.workload)
    f = api.FerroX(text, precision=args.precision)
    if grains is not None:
        f.set_grains(grains["id"], grains["angles"], grains["tphase"])
    if args.host_loop:
        f.set_param("fx.step_graph", 0)
    apply_settings(f, args)
    # a dedicated stream: the library's work and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    f.set_stream(stream.cuda_stream)
    N = f.N
    f.step(args.warmup)
    f.sync()
    st0 = f.stats()

    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    done = f.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    st1 = f.stats()
    graph_ran = f.param("step_graph_ran") == 1.0
    if done != args.steps:
        raise RuntimeError(f"the reference loop ended after {done} of {args.steps} steps")
    ms_max = max_over_ranks(ms, world)
    value = whole_job_rate(N, args.steps, world, ms_max)

    # end to end through the public API: a second context of the same deck
    # runs the same W warm-up steps (untimed) and then the same K steps as the
    # timed leg, so both legs cover the same stretch of the run with the same
    # history of phi.  The state stays resident in HBM, as the reference's
    # MultiFabs stay on its device; per step the host sets the electrode
    # voltage (fx_set_param, the step's input), runs fx_step(1) and reads the
    # mean polarization back (fx_mean_P, the step's result); at the end P and
    # phi are read into pinned host buffers (fx_get_field)
    ke = args.e2e_steps or args.steps
    e2e = None
    if not args.no_e2e:
        e2e = e2e_leg(args, api, text, grains, stream, N, world, ke, barrier, torch)

    # per-launch kernel durations: K more steps with CUDA events around every
    # launch (kept out of the timed region, whose cost they raise)
    f.set_param("fx.profile", 1)
    f.reset_kernel_times()
    f.step(args.steps)
    kt = f.kernel_times()
    f.set_param("fx.profile", 0)

    if rank == 0:
        peak, peak_src = peaks()
        sc = f.param("contains_sc") == 1.0
        rot = f.param("num_variants") > 0
        # dominant kernel class of the timed region among the bandwidth-bound
        # classes (those with an algorithmic byte count); the latency-bound
        # coarse multigrid levels are reported by share in kernel_ms_share
        bw_classes = ["smooth_l0", "restrict_l0", "prolong_l0", "tdgl", "newton", "rho", "resid64", "rhs_p", "steady"]
        dom = max((k for k in bw_classes if kt[k][1]), key=lambda k: kt[k][0])
        dms, dcnt = kt[dom]
        Nc1 = N // 2  # level 1 halves z on these stacks (dz < dx)
        fp = 4 if args.precision == "mixed" and dom in ("smooth_l0", "restrict_l0", "prolong_l0") else 8
        planes = f.param("mg_level0_planes") == 1.0
        per_launch = algorithmic_bytes(dom, N, Nc1, sc, True, rot, fp, planes)
        tkey = (args.workload, args.precision, dom)
        achieved = per_launch / (dms / dcnt / 1e3) / 1e9 if dcnt else None
        total_ms = sum(v[0] for v in kt.values())
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": TRAFFIC[tkey][0] if tkey in TRAFFIC else None,
                "traffic_source": f"ncu dram bytes per launch, {TRAFFIC[tkey][1]}" if tkey in TRAFFIC
                else "no ncu capture of this kernel class on this workload and precision",
                "peak_source": f"{peak_src} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": per_launch, "launches": dcnt, "avg_launch_us": 1e3 * dms / dcnt,
                "kernel_share": dms / total_ms, "top_class": max(kt, key=lambda k: kt[k][0])}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(text, grains, 3)
        adj_scale = None
        if world == 1 and args.adjoint_scale_steps > 0:
            adj_scale = adjoint_scale(stream, args.adjoint_scale_steps)
        prec_cmp = None
        if world == 1 and args.precision == "mixed" and not args.no_compare:
            prec_cmp = precision_compare(stream, args.workload, args.steps, args.warmup)
        adj = None
        if world == 1 and not args.no_adjoint:
            adj = adjoint_ratio(stream, args.precision, args.adjoint_steps_per_leg)
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded initial P, synthetic device stack)",
            "config": run_config(args, N),
            "run": {"device_bytes": f.stats()["device_bytes"],
                    "step": "one CUDA graph per step, loop tests on the device" if graph_ran
                    else "host-driven loop"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(st1["kernel_launches"] - st0["kernel_launches"]),
            "clocks": clocks,
            "kernel_ms_share": {k: round(v[0] / total_ms, 4) for k, v in kt.items() if v[1]},
            "mg_cycles_per_step": (st1["mg_cycles_total"] - st0["mg_cycles_total"]) / args.steps,
            "newton_passes_per_step": (st1["newton_iters_total"] - st0["newton_iters_total"]) / args.steps,
            "adjoint": adj,
            "mixed_vs_fp64": prec_cmp,
            "adjoint_polycrystal": adj_scale,
        }
        print(json.dumps(line), flush=True)
    f.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
