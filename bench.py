"""Benchmark of the sm_100a mPDeC5 time step (one JSON line on rank 0).

Workload: the wave-over-dry-island case on a 2048x2048 periodic grid ([0,10]^2,
Gaussian island b = 1.2 exp(-((x-5)^2+(y-5)^2)/0.5), still water h + b = 1 with
a hump of amplitude 0.3 and width 0.3 at x = 2), CFL 0.4, g = 9.81.  A step is
TimeStep() + one mPDeC5 step (13 RHS evaluations, 13 Patankar solves).

  value        split-precision cell-steps/s with the state resident in HBM
  fp64         the plain FP64 form on the same workload (the metric's baseline)
  e2e          the same metric through the C ABI with host buffers: every step
               copies the ghosted state host->device and back (swm_set_state /
               swm_get_state), as a Fortran driver keeping U on the host would
  roofline     dominant kernel, algorithmic bytes / CUDA-event time
  accuracy     the island case at 256^2 up to t = 0.8 (the hump runs up and over the
               dry island top): split, FP64 and FP64-FMA GPU forms and, with the CPU leg,
               the oracle on the same dt sequence -- L1 (sum |dU| dx dy), relative L1,
               L-inf; the FP64-FMA form's distance from the oracle is the reference's
               reproducibility floor (what a change of rounding alone costs on this run)
  cpu_baseline the CPU restatement (oracle, OpenMP build, all host threads) timed on
               the accuracy leg's run, plus one host core on a bounded sample

Multi-GPU (--gpus N under torchrun): replicas only -- every rank steps its own
copy of the workload on its GPU, no data-path collective; value = N * cells *
steps / (max over ranks of the timed region).

--impl reference times the reference's CPU path (the oracle restatement: the
Fortran reference cannot be compiled in this image) on the same workload (island
2048^2) with all host threads.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sw-mpdec_b200"))

METRIC = "mPDeC5 cell-steps/s at 2048²: split-precision vs FP64 GPU at L1 err ≤1e-6"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the split
# step's kernels, each from one earlier ncu capture at 2048x2048 (4,194,304 cells):
# constants, not measured by this run.  Each names the commit of the capture; a kernel
# changed after it makes the figure stale.  Scaled by cells for other grid sizes (the
# traffic of these kernels grows with the cell count).
NCU_TRAFFIC_2048 = {
    "rhs": (101655552.0 + 91263232.0, "2c446c5"),
    "jacobi": (403459328.0 + 58311680.0, "77d112e"),
}

# Accuracy leg: the island case (stated hump at x = 2) at 256^2 up to t = 0.8, by which
# the hump has run up and over the dry island top (wetting and drying).  The split and
# FP64 forms take the FP64 form's dt sequence; with the CPU leg on, the oracle takes it
# too (that run is also the timed CPU baseline) and both are compared with it.
ACC_N = 256
ACC_T_END = 0.8

# Wall-clock budget of the reference arm's timed steps (host CPU).
REF_BUDGET_S = 150.0

# Algorithmic bytes per cell-step of the whole mPDeC5 step: every phase reads its
# inputs and writes its outputs once (halo re-reads not counted), the Patankar
# matrix is re-read on every Jacobi sweep.  Per step: dt reduction 24, 13 RHS (FP64
# 56 / split 40), 13 combinations (96 / 64), 13 assemblies (112 / 80), and 64 per
# Jacobi sweep summed over the 13 solves.
STEP_BYTES_BASE = {"fp64": 3456.0, "split": 2416.0}
STEP_BYTES_PER_SWEEP = 64.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.first = 0

    def start(self):
        """Start sampling every 25 ms; return once the first sample has arrived, so
        that a short timed region is covered from its beginning."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "25"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.time() + 5.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None

    def mark(self):
        """The timed region starts now: earlier samples are not counted."""
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[3 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_solver(swm, c, precision, solver="stencil", block=4, device=0, source_table=1,
                timescheme=5):
    return swm.Solver(nx=c["nx"], ny=c["ny"], x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                      well_balanced=c["well_balanced"], precision=precision, solver=solver,
                      jacobi_block=block, device=device, source_table=source_table,
                      timescheme=timescheme)


# Timed forms: the split form (the metric's numerator) and the plain FP64 form twice,
# with the bathymetry source from the per-cell gradient table (bit-identical to the
# oracle: the metric's baseline) and from the per-column/row factors (no per-cell
# table; one RHS within 1e-13 of the oracle's source, not bit-identical over a run).
FORMS = {"fp64": ("fp64", 1), "fp64_factored": ("fp64", 0), "split": ("split", 1)}


def timed_steps(s, torch, steps, warmup, on_start=None):
    """W untimed steps, then K steps bracketed by CUDA events on the library stream;
    on_start() is called just before the first timed step."""
    for _ in range(warmup):
        s.step(0.0, s.timestep())
    st = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if on_start:
        on_start()
    e0.record(st)
    iters = 0
    for _ in range(steps):
        s.step(0.0, s.timestep())
        iters += sum(s.stats()["jacobi_iters"])
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), iters


def errors(a, b, c):
    """Per variable (h, hu, hv): the reference's L1 error sum |a - b| dx dy
    (postprocessing.f90:47,51), the relative L1 sum |a - b| / sum |b|, and L-infinity."""
    dx = (c["x1"][0] - c["x0"][0]) / c["nx"]
    dy = (c["x1"][1] - c["x0"][1]) / c["ny"]
    d = np.abs(a - b)
    return {"l1": [float(d[v].sum() * dx * dy) for v in range(3)],
            "rel_l1": [float(d[v].sum() / max(np.abs(b[v]).sum(), 1e-300)) for v in range(3)],
            "linf": [float(d[v].max()) for v in range(3)]}


def accuracy_pass(split_l1, floor_l1, own_l1, bar=1e-6):
    """The split form's bar per variable: L1 <= bar, or, where the reference's
    reproducibility floor is above bar/2, within 1.25 x the floor with its own FP32
    error (distance from the FP64-FMA form) <= max(bar, floor/4)."""
    ok = True
    for v in range(3):
        if floor_l1[v] <= 0.5 * bar:
            ok = ok and split_l1[v] <= bar
        else:
            ok = ok and split_l1[v] <= 1.25 * floor_l1[v] and own_l1[v] <= max(bar, 0.25 * floor_l1[v])
    return bool(ok)


def accuracy_leg(swm, cases, with_cpu, block, device):
    """Split, FP64 and FP64-FMA forms (and, in the CPU leg, the oracle) over a wet-dry
    horizon on the same dt sequence; returns (accuracy, cpu_baseline or None).

    The FP64-FMA form (FP64 throughout, contraction and sum-of-squares smoothness
    indicators: different rounding only) measures the reference's reproducibility
    floor: the reference's expanded smoothness indicators cancel to rounding noise on
    nearly flat stencils, so any arithmetic that is not bit-identical to it drifts
    from it by about that much on this run."""
    c = cases.case("island", n=ACC_N)
    planes = cases.cell_averages(c)
    s64 = make_solver(swm, c, "fp64", block=block, device=device)
    s64.set_planes(planes)
    dts, t = [], 0.0
    while ACC_T_END - t > 1e-12:
        dt = min(s64.timestep(), ACC_T_END - t)
        s64.step(t, dt)
        dts.append(dt)
        t += dt
    p64 = s64.get_planes()
    s64.close()
    other = {}
    for form in ("split", "fp64_fma"):
        so = make_solver(swm, c, form, block=block, device=device)
        so.set_planes(planes)
        for dt in dts:
            so.step(0.0, dt)
        other[form] = so.get_planes()
        so.close()
    p32, pfm = other["split"], other["fp64_fma"]
    dry0 = int((planes[0] <= 1.0001e-6).sum())
    acc = {"workload": f"island {ACC_N}x{ACC_N} (hump at x = 2) to t = {t:.3f}: the hump runs "
                       f"up and over the dry island top", "steps": len(dts), "t_end": t,
           "dry_cells_initial": dry0, "dry_cells_final": int((p64[0] <= 1.0001e-6).sum()),
           "bar": "split-form L1 = sum |U - U_ref| dx dy (postprocessing.f90:47,51) <= 1e-6 "
                  "per variable, U_ref the oracle (FP64); where the reference's own "
                  "reproducibility floor (the FP64-FMA form's L1 from it) is above half the "
                  "bar: split L1 <= 1.25 x floor and split-vs-FP64-FMA L1 <= max(1e-6, floor/4)",
           "split_vs_fp64": errors(p32, p64, c),
           "fp64_fma_vs_fp64": errors(pfm, p64, c),
           "split_vs_fp64_fma": errors(p32, pfm, c),
           "min_h_split": float(p32[0].min())}
    if not with_cpu:
        return acc, None
    # --- CPU leg: the oracle (test infrastructure) is the timed CPU baseline and the
    # accuracy reference of the same run
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    op = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                       bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"])
    o = O.Oracle(op, threaded=True)
    o.set_planes(planes)
    t0 = time.perf_counter()
    for dt in dts:
        o.timestep()
        o.step(0.0, dt)
    el = time.perf_counter() - t0
    po = o.get_planes()
    del o
    acc["split_vs_oracle"] = errors(p32, po, c)
    acc["fp64_fma_vs_oracle"] = errors(pfm, po, c)
    acc["fp64_vs_oracle"] = {"bitwise": bool(np.array_equal(p64, po)),
                             "rel_l1": errors(p64, po, c)["rel_l1"]}
    acc["pass"] = accuracy_pass(acc["split_vs_oracle"]["l1"], acc["fp64_fma_vs_oracle"]["l1"],
                                acc["split_vs_fp64_fma"]["l1"])
    cells = c["nx"] * c["ny"]
    cpu = {"value": cells * len(dts) / el, "unit": "cell-steps/s", "cores": O.threads(True),
           "kind": "port",
           "sample": f"the accuracy leg's run: island {ACC_N}x{ACC_N}, {len(dts)} mPDeC5 steps "
                     f"to t = {t:.3f}, CPU restatement of the Fortran (oracle/swm_oracle.c, "
                     f"OpenMP build, all host threads)"}
    # one host core: the serial build on 2 steps of the island case at 512^2
    n1, k1 = 512, 2
    c1 = cases.case("island", n=n1)
    o1 = O.Oracle(O.make_params(c1["nx"], c1["ny"], c1["x0"], c1["x1"], g=c1["g"], cfl=c1["cfl"],
                                bathy_flag=c1["bathy_flag"], bathy_par=c1["bathy_par"]))
    o1.set_planes(cases.cell_averages(c1))
    t0 = time.perf_counter()
    for _ in range(k1):
        o1.step(0.0, o1.timestep())
    el1 = time.perf_counter() - t0
    cpu["single_core"] = {"value": n1 * n1 * k1 / el1, "unit": "cell-steps/s", "cores": 1,
                          "sample": f"island {n1}x{n1}, {k1} mPDeC5 steps, serial build"}
    return acc, cpu


def reference_arm(args, rank, world):
    """The reference's CPU path on the arm's own workload (island at --n, default
    2048^2): the oracle's OpenMP build on all host threads.  A step at 2048^2 takes
    seconds on the CPU, so at most one warm-up step (page-in) is run."""
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    n = args.n
    warm = min(max(args.warmup, 0), 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import oracle as O
    c = cases.case("island", n=n)
    p = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"])
    o = O.Oracle(p, threaded=True)
    o.set_planes(cases.cell_averages(c))
    t_step = None
    for _ in range(warm):
        t0 = time.perf_counter()
        o.step(0.0, o.timestep())
        t_step = time.perf_counter() - t0
    # a step of the 2048^2 grid takes ~14 s on 16 host threads: time at most as many
    # steps as fit in REF_BUDGET_S, so that the arm ends within a few minutes
    steps = args.steps
    if t_step:
        steps = max(1, min(args.steps, int(REF_BUDGET_S / t_step)))
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(0.0, o.timestep())
    el = time.perf_counter() - t0
    v = c["nx"] * c["ny"] * steps / el
    cores = O.threads(True)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"island {n}x{n} periodic (wave over dry island), mPDeC5, "
                               f"CFL 0.4", "cells": n * n, "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{steps} mPDeC5 steps (of {args.steps} asked, at most "
                                   f"{REF_BUDGET_S:.0f} s of them) of the island case at {n}x{n} "
                                   f"after {warm} warm-up step(s) (at most one: a step takes "
                                   f"seconds on the CPU); the Fortran reference has no "
                                   f"compiler here, so its C restatement (oracle) is timed"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="swm")
    ap.add_argument("--block", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-only", action="store_true")  # profiling runs
    ap.add_argument("--ensemble-island", type=int, default=0)  # profiling: one island N^2
    ap.add_argument("--no-accuracy", action="store_true")  # profiling runs: no wet-dry leg
    ap.add_argument("--n", type=int, default=2048)
    # profiling runs only: a subset of the timed forms, or another time scheme (its
    # kernels under ncu); either prints the per-form step times and nothing else
    ap.add_argument("--forms", default=",".join(FORMS))
    ap.add_argument("--timescheme", type=int, default=5)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    import torch
    import swm
    import cases
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    c = cases.case("island", n=args.n)
    cells = c["nx"] * c["ny"]
    planes = cases.cell_averages(c)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    import replicas

    def max_over_ranks(x):
        return replicas.aggregate(x, 0.0, dist, device="cuda")[0]

    def ensemble_leg():
        # ensemble: 256 problems of uneven size in one batch (split; the step form and the
        # Jacobi sweeps per pass autotuned); under torchrun the problem list is sharded
        # across ranks
        # profiling: a batch holding one island grid (the single-grid workload's systems)
        members = ([cases.case("island", n=args.ensemble_island)] if args.ensemble_island
                   else cases.ensemble(seed=0))
        sizes = [m["nx"] * m["ny"] for m in members]
        mine = replicas.shard(sizes, rank, world)
        plist = [swm.make_params(m["nx"], m["ny"], m["x0"], m["x1"], g=m["g"], cfl=m["cfl"],
                                 bathy_flag=m["bathy_flag"], bathy_par=m["bathy_par"],
                                 precision="split", solver="stencil", jacobi_block=0,
                                 device=local) for m in (members[i] for i in mine)]
        bt = swm.Batch(plist)
        for k, i in enumerate(mine):
            bt.set_planes(k, cases.cell_averages(members[i]))
        for _ in range(max(args.warmup, 1)):  # the first step also picks the schedule
            bt.step()
        st = torch.cuda.ExternalStream(bt.stream())
        # every timed run below starts from this state (the Jacobi sweeps depend on it)
        snap = [bt.get_planes(k) for k in range(len(mine))]

        def restore():
            for k, P in enumerate(snap):
                bt.set_planes(k, P)

        def time_ensemble():
            restore()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(args.steps):
                bt.step()
            e1.record(st)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        ms_ens, cell_steps = replicas.aggregate(time_ensemble(), bt.cells() * args.steps,
                                                dist, device="cuda")
        blk, tot, last = bt.stats()
        launches, ctas = bt.launch_info()
        # both step forms fixed in turn, timed from the same state, for comparison
        forms = {}
        for name, per_phase in (("persistent", False), ("phased", True)):
            bt.set_launches(per_phase)
            bt.step()  # warm the new graph
            ms_f = replicas.aggregate(time_ensemble(), 0.0, dist, device="cuda")[0]
            nl, nc = bt.launch_info()
            forms[name] = {"launches_per_step": nl, "ms_per_step": ms_f / args.steps,
                           "value": cell_steps / (ms_f * 1e-3)}
            if not per_phase:
                forms[name]["ctas"] = nc
            # one more step from the same state with its phases timed (the persistent
            # launch by a global timer inside it, the per-phase form by CUDA events)
            restore()
            forms[name]["phase_ms"] = {k: round(v, 4) for k, v in bt.phase_times().items()}
        ens = {"workload": (f"one island {args.ensemble_island}^2 problem, split precision"
                            if args.ensemble_island else
                            "256 problems, sides log-uniform in [64,512], vortex / dam break / "
                            "Gaussian lake families, seed 0, split precision"),
               "value": cell_steps / (ms_ens * 1e-3), "unit": "cell-steps/s",
               "cells": int(sum(sizes)), "ms_per_step": ms_ens / args.steps,
               "schedule": {"form": "persistent" if launches == 1 else "phased",
                            "jacobi_block": blk, "launches_per_step": launches,
                            "persistent_ctas": ctas, "chosen_by": "autotuner, first step"},
               "jacobi_iters_per_step_max": int(last.sum(axis=0).max()),
               "forms": forms}
        bt.close()
        return ens

    if args.ensemble_only:  # profiling runs: the ensemble leg alone
        ens = ensemble_leg()
        if rank == 0:
            print(json.dumps({"profiling_run": True, "ensemble": ens}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    results = {}
    clocks = None
    forms = args.forms.split(",")
    partial = set(forms) != set(FORMS) or args.timescheme != 5
    for prec in forms:
        form, table = FORMS[prec]
        s = make_solver(swm, c, form, block=args.block, device=local, source_table=table,
                        timescheme=args.timescheme)
        s.set_planes(planes)
        barrier()
        sampler = ClockSampler(local) if prec == "split" else None
        if sampler:
            sampler.start()
        ms, iters = timed_steps(s, torch, args.steps, args.warmup,
                                on_start=sampler.mark if sampler else None)
        if sampler:
            clocks = sampler.stop()
        barrier()
        ms = max_over_ranks(ms)
        prof = s.profile_step(0.0, s.timestep())  # one extra eagerly-launched step
        final = s.get_planes()
        prof_wrapped = None
        if prec == "split" and not partial:  # the RHS with every tile loaded without TMA
            s.set_tma(False)
            prof_wrapped = s.profile_step(0.0, s.timestep())
            s.set_tma(True)
        results[prec] = dict(ms=ms, iters=iters, prof=prof, final=final, prof_wrapped=prof_wrapped)
        s.close()
        del s

    if partial:
        if rank == 0:
            print(json.dumps({"profiling_run": True, "timescheme": args.timescheme,
                              "ms_per_step": {k: v["ms"] / args.steps for k, v in results.items()}}),
                  flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    # the split form against the FP64 form after the timed steps (short horizon); the
    # wet-dry accuracy leg against the oracle runs after the GPU legs
    short = errors(results["split"]["final"], results["fp64"]["final"], c)
    short["steps"] = args.steps + args.warmup + 1  # + the profiled step
    short["bar"] = "split-form L1 <= 1e-6 per variable against the FP64 form, which is " \
                   "bit-identical to the oracle"
    short["pass"] = bool(max(short["l1"]) <= 1e-6)
    short["min_h_split"] = float(results["split"]["final"][0].min())

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        s = make_solver(swm, c, "split", block=args.block, device=local)
        Ug = torch.from_numpy(cases.ghosted(planes)).pin_memory().numpy()
        Uo = torch.empty(Ug.shape, dtype=torch.float64).pin_memory().numpy()
        s.set_state(Ug)
        for _ in range(args.warmup):
            s.set_state(Ug)
            s.step(0.0, s.timestep())
            s.get_state()
        barrier()
        st = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            s.set_state(Ug)
            s.step(0.0, s.timestep())
            s.lib.swm_get_state(s.h, swm._dp(Uo), None)
        e1.record(st)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1))
        nbytes = Ug.nbytes
        e2e = {"value": world * cells * args.steps / (ms_e2e * 1e-3), "unit": "cell-steps/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 16,
               "ms_per_step": ms_e2e / args.steps}
        s.close()

    ens = None if args.no_ensemble else ensemble_leg()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # accuracy over a wet-dry horizon; with the CPU leg, the oracle's run of it is the
    # timed CPU baseline and the accuracy reference (rank 0 only, after all timing)
    acc, cpu = None, None
    try:
        if not args.no_accuracy:
            acc, cpu = accuracy_leg(swm, cases, world == 1 and not args.no_cpu, args.block,
                                    local)
    except Exception as exc:  # a failed side leg must not hide the GPU number
        acc = {"error": str(exc)}

    sp, fp = results["split"], results["fp64"]
    value = world * cells * args.steps / (sp["ms"] * 1e-3)
    value64 = world * cells * args.steps / (fp["ms"] * 1e-3)
    ff = results["fp64_factored"]
    value64f = world * cells * args.steps / (ff["ms"] * 1e-3)
    # the ratio is quoted against the plain FP64 form that meets the FP64 bar
    # (bit-identical to the oracle); the factored-source variant regroups the source's
    # products, so over whole runs it drifts from the oracle like any rounding change
    best64 = value64
    nj = sp["iters"] / args.steps
    pk, src = peaks()
    peak = float(pk["hbm_gbs"])
    # dominant kernel class of the split step (eager profile of one step)
    pr = sp["prof"]
    classes = {"rhs": (pr["rhs_ms"], pr["rhs_launches"]),
               "patankar_assemble": (pr["assemble_ms"], pr["assemble_launches"]),
               "jacobi": (pr["jacobi_ms"], pr["jacobi_launches"])}
    dom = max(classes, key=lambda k: classes[k][0])
    prof_iters = sum(results["split"]["prof"].get("iters", []) or []) or nj
    # algorithmic bytes per launch: Jacobi 64 B/cell/iteration (5 coefficients, rhs,
    # x read, x written); RHS 56 B/cell (U read, momentum RHS and the two mass face
    # fluxes written); combination + assembly 208 B/cell
    if dom == "jacobi":
        alg = 64.0 * cells * prof_iters / max(classes[dom][1], 1)
    elif dom == "rhs":
        alg = 56.0 * cells
    else:
        alg = 208.0 * cells
    t_launch = classes[dom][0] / max(classes[dom][1], 1) * 1e-3
    achieved = alg / t_launch / 1e9
    tb, traffic_commit = NCU_TRAFFIC_2048.get(dom, (None, None))
    traffic = tb * cells / 2048.0**2 if tb else None
    traffic_src = (f"constant from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, "
                   f"one launch at 2048^2) at commit {traffic_commit}, scaled by cells; not "
                   f"measured by this run" if tb else None)
    # whole-step byte model for both forms (N_J = measured Jacobi sweeps per step)
    step_rf = {"unit": "GB/s", "peak": peak, "jacobi_sweeps_per_step": nj,
               "bytes_per_cell_step": {}, "achieved": {}, "frac": {}}
    for form, val, sweeps in (("split", value, nj), ("fp64", best64, fp["iters"] / args.steps)):
        b = STEP_BYTES_BASE[form] + STEP_BYTES_PER_SWEEP * sweeps
        step_rf["bytes_per_cell_step"][form] = b
        step_rf["achieved"][form] = val / world * b / 1e9  # per GPU (replicas)
        step_rf["frac"][form] = val / world * b / 1e9 / peak
    launches = sum(v[1] for v in classes.values()) + 1  # + dt reduction
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sp["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"island {c['nx']}x{c['ny']} periodic (wave over dry island), "
                               f"mPDeC5, CFL 0.4, split precision, stencil Jacobi block {args.block}",
                   "cells": cells, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (~1.5 GB of state and stage arrays per step)"},
        "fp64_factored": {"value": value64f, "ms_per_step": ff["ms"] / args.steps,
                          "jacobi_iters_per_step": ff["iters"] / args.steps,
                          "source": "per-column/row factors of the separable bathymetry "
                                    "gradient (no per-cell table)",
                          "rel_l1_vs_fp64_table": errors(ff["final"], fp["final"], c)["rel_l1"]},
        "fp64": {"value": value64, "ms_per_step": fp["ms"] / args.steps,
                 "source": "bathymetry gradient tabulated at every interior Gauss point",
                 "jacobi_iters_per_step": fp["iters"] / args.steps},
        "split_over_fp64": value / best64,
        "split_over_fp64_form": "fp64 (bit-identical to the oracle)",
        "accuracy": acc,
        "accuracy_timed_steps_split_vs_fp64": short,
        "jacobi_iters_per_step": nj,
        "kernel_ms_per_step": {k: v[0] for k, v in classes.items()},
        "rhs_tile_loads": {
            "tma_us_per_launch": 1e3 * pr["rhs_ms"] / max(pr["rhs_launches"], 1),
            "wrapped_us_per_launch": 1e3 * sp["prof_wrapped"]["rhs_ms"] /
                                     max(sp["prof_wrapped"]["rhs_launches"], 1),
            "note": "split RHS per launch, one eagerly launched step each: interior tiles "
                    "staged by TMA tensor copies vs every tile by wrapped-index loads"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": traffic_src, "alg_bytes_per_launch": alg,
                     "peak_source": src},
        "step_roofline": step_rf,
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
        "e2e": e2e,
        "ensemble": ens,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
