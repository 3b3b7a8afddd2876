"""Benchmark of the B200 time-step backend (LCS.jl hot path).

Default workload "lp512": periodic cube L = 2pi, 512^3 cells, nu = 0.0025
(Re = 400), seeded solenoidal spectral init E(k) ~ k^4 exp(-2 (k/4)^2) with
u_rms = 1, linear-power forcing P = 0.5, HSMAC red-black-fast with time
blocking and overlap, omega 1.7, itrmin 6, itrmax 300, exit at RMS(div) <
1e-8, CFL 0.3, dtmax 0.01, and 2^24 Stokes particles in 3 species (tau_p =
0.02, 0.2, 2.0; density ratio 843; velocity = interpolated fluid velocity).

A step is LCS.timestep! + LCS.evolve! over the whole grid and all particles.
The plain FP64 method is timed first: `value` is its Mcell-steps/s (cells x
steps / device seconds of the timed steps, max over ranks), particle-steps/s
beside it.  The FP32-mixed form then runs the same workload from the same
inputs for the same warm-up and timed steps (`precision_forms`), and its
state is compared with the FP64 state after those steps: relative L2 error
per field, relative error per flow statistic (Flows.stat on the device), per
E(k) shell and per particle species.  Every field is a (n+6)^3 array of
1.1 GB (FP64), so the inputs exceed the 126 MB L2 and no flush is needed
between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload lp512|rc256|lp128|batch64|serve|makeindex|couple256]
                  [--precision fp64|fp32-mixed] [--no-forms] [--no-cpu-baseline]

--impl reference times the CPU restatement of the reference (oracle/, the
port of LCSCPU: the reference is Julia and cannot run here) on the host's
cores, each step a bounded sample of the same workload (below).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lcs.jl_b200"))

import numpy as np  # noqa: E402

from lcs_b200 import config as lcfg  # noqa: E402
from lcs_b200 import inits  # noqa: E402
from lcs_b200.workloads import WORKLOADS, host_inputs, load_engine, make_run_config  # noqa: E402

# workloads with a run function of their own
OTHER_WORKLOADS = ("batch64", "serve", "makeindex", "couple256")

# DRAM bytes (read + write) per interior cell of one launch of the sweep
# kernel, from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum) of
# a D2 sweep (box 0:n+2) at 256^3, one per precision and default tile shape
# (FP64 13-row tiles, FP32 29-row tiles): not measured in the run that
# reports them.
SWEEP_DRAM_BYTES_PER_CELL = {"fp64": 67.8, "fp32-mixed": 35.5}
SWEEP_KERNELS = ("hsmac_rw", "hsmac_fused")
# FP64 operations per interior cell of one rhs!+update! launch (k_rhs, both
# stages alike): smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on
# of an ncu capture of k_rhs at 128^3: 484.4 M adds + 471.9 M multiplies, no
# FMA (the FP64 library is built without contraction), over 128^3 cells.
RHS_FLOPS_PER_CELL = 456.0

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
TWO_PI = 2.0 * math.pi


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.th = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()




def elem_bytes(precision):
    return 4 if precision == "fp32-mixed" else 8


def kernel_table(tot, n, h, T, particles_per_launch, peak):
    """Per-kernel device ms and launches of the profiled steps, with the HBM
    fraction of every kernel that has a byte model (kernel_bytes)."""
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in sorted(tot.items(), key=lambda kv: -kv[1][0])}
    for k, alg in kernel_bytes(n, h, T, particles_per_launch).items():
        if k in kernels and kernels[k]["launches"]:
            ms_l = kernels[k]["ms"] / kernels[k]["launches"]
            gbs = alg / (ms_l / 1e3) / 1e9
            kernels[k].update({"alg_bytes_per_launch": alg, "gbs": round(gbs, 1), "hbm_frac": round(gbs / peak, 3)})
    return kernels


def sweep_roofline(tot, n3, precision, peak, peak_kind):
    """HBM roofline of the dominant kernel, the fused red-black sweep: 8T bytes
    per interior cell (U, V, W, P read and written once) over its average
    CUDA-event launch time."""
    k = max(SWEEP_KERNELS, key=lambda s: tot.get(s, (0.0, 0))[0])
    ms, cnt = tot.get(k, (0.0, 0))
    T = elem_bytes(precision)
    alg = 8 * T * n3
    avg = ms / max(cnt, 1)
    ach = alg / (avg / 1e3) / 1e9 if cnt else None
    return {"kernel": k, "bound": "hbm", "achieved": ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": (ach / peak) if ach else None, "traffic": SWEEP_DRAM_BYTES_PER_CELL[precision] * n3,
            "traffic_source": "not measured in this run: ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                              f"interior cell of a 256^3 capture of the same kernel (a D2 sweep, "
                              f"{SWEEP_DRAM_BYTES_PER_CELL[precision]} B), times n^3",
            "alg_bytes_per_launch": alg, "avg_launch_ms": avg, "launches_profiled": cnt}


def run_form(args, precision, rc_w, flow, parts, world, device, primary):
    """One precision form on the workload: W warm-up steps, K timed steps
    (CUDA-graph replays, device-timed), the state after them downloaded, two
    profiled steps (per-kernel CUDA events) and, for the primary form, the
    end-to-end run through the per-step C-ABI calls with host buffers."""
    import ctypes as C

    from lcs_b200 import Engine

    rc, w = rc_w
    rc.abi.device = device
    rc.abi.use_graphs = 1
    n3 = float(np.prod(rc.dims))
    np_tot = float(sum(w["counts"]))
    eng = Engine(rc.abi)
    load_engine(eng, rc, flow, parts)
    eng.step(args.warmup)  # also builds the step graphs
    eng.synchronize()
    barrier(world)
    with ClockSampler(device) as clk:
        logs, ms = eng.step_timed(args.steps)
    barrier(world)
    ms_max = reduce_max(ms, world)
    res = {"value": world * n3 * args.steps / (ms_max / 1e3) / 1e6, "ms_per_step": ms_max / args.steps,
           "particle_steps_per_s": world * np_tot * args.steps / (ms_max / 1e3), "clocks": clk.summary(),
           "sweeps_per_step": statistics.mean(lg["couple1"]["sweeps"] + lg["couple2"]["sweeps"] for lg in logs),
           "last_log": logs[-1], "after_steps": args.warmup + args.steps}
    # the state after W + K steps, for the error of the FP32-mixed form
    if not args.no_forms:
        res["flow"] = eng.download_flow()
        res["parts"] = [eng.download_particles(s) for s in range(len(parts))]
        res["stat"] = eng.flow_stat()
    res["divergence"] = eng.flow_divergence()

    # per-kernel device times from CUDA events around every launch (same stream)
    eng.profile(True)
    eng.profile_reset()
    prof_steps = 2
    eng.step(prof_steps)
    tot = eng.profile_totals()
    eng.profile(False)
    res["launches_per_step"] = sum(v[1] for v in tot.values()) / prof_steps
    peak, peak_kind = hbm_peak()
    T = elem_bytes(precision)
    res["roofline"] = sweep_roofline(tot, n3, precision, peak, peak_kind)
    res["kernels"] = kernel_table(tot, int(rc.dims[0]), int(rc.abi.halo_size), T, np_tot / max(1, len(rc.species)),
                                  peak)
    if precision == "fp64":
        fp64_peak = C.c_double()
        if eng.lib.lcs_measure_fp64_peak(device, C.byref(fp64_peak)) == 0 and "rhs_update" in tot:
            ms_r, cnt_r = tot["rhs_update"]
            tf = RHS_FLOPS_PER_CELL * n3 / (ms_r / cnt_r / 1e3) / 1e12
            res["fp64"] = {"peak_tflops": round(fp64_peak.value, 2), "peak_kind": "measured (k_fp64_peak, FMA chains)",
                           "rhs_flops_per_cell": RHS_FLOPS_PER_CELL, "rhs_tflops": round(tf, 2),
                           "rhs_frac": round(tf / fp64_peak.value, 3),
                           "note": "rhs has no FMA (no contraction): add/multiply issue at half the FMA rate"}

    if primary:
        # end to end through the public API: pinned host state in, the per-step
        # timestep!/evolve! calls of the Julia shim, state out into pinned memory
        import torch

        def pinned_empty(shape):
            return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

        h2d0, d2h0 = eng.transfer_stats()
        e2e_steps = max(1, min(args.steps, 5))
        out_flow = [pinned_empty(eng.interior_shape) for _ in range(4)]
        out_parts = []
        for si in rc.species:
            ids = torch.empty(si.nvalid, dtype=torch.int64, pin_memory=True).numpy()
            out_parts.append((ids, [pinned_empty(si.nvalid) for _ in range(7)]))
        barrier(world)
        t0 = time.perf_counter()
        load_engine(eng, rc, flow, parts)
        for _ in range(e2e_steps):
            dt = eng.timestep()
            eng.evolve(dt)
        eng._check(eng.lib.lcs_download_flow(eng.handle, *[a.ctypes.data_as(C.POINTER(C.c_double)) for a in out_flow]))
        for s, (out_ids, out_p) in enumerate(out_parts):
            eng._check(eng.lib.lcs_download_particles(eng.handle, s, out_ids.ctypes.data_as(C.POINTER(C.c_int64)),
                                                      *[a.ctypes.data_as(C.POINTER(C.c_double)) for a in out_p]))
        eng.synchronize()
        e2e_s = reduce_max(time.perf_counter() - t0, world)
        h2d1, d2h1 = eng.transfer_stats()
        res["e2e"] = {"value": world * n3 * e2e_steps / e2e_s / 1e6, "unit": "Mcell-steps/s",
                      "h2d_bytes_per_step": (h2d1 - h2d0) / e2e_steps, "d2h_bytes_per_step": (d2h1 - d2h0) / e2e_steps,
                      "steps": e2e_steps,
                      "path": "pinned host state uploaded, per-step lcs_timestep/lcs_evolve, state downloaded into "
                              "pinned memory (host wall clock, max over ranks)"}
    eng.close()
    return res


def precision_errors(a, b, nu):
    """The FP32-mixed state `a` against the FP64 state `b` after the same steps."""
    from lcs_b200 import stats

    def rel(x, y):
        return float(abs(x - y) / abs(y)) if y != 0 else float(abs(x - y))

    def rel_l2(x, y):
        return float(np.linalg.norm((x - y).ravel()) / np.linalg.norm(y.ravel()))

    ek_a = stats.energy_spectrum(*a["flow"][:3])
    ek_b = stats.energy_spectrum(*b["flow"][:3])
    shells = [k for k in range(1, len(ek_b)) if ek_b[k] > 1e-12 * ek_b[1:].max()]
    return {
        "after_steps": b["after_steps"],
        "field_rel_l2": {f: rel_l2(x, y) for f, x, y in zip("UVWP", a["flow"], b["flow"])},
        "stat_rel": {k: rel(a["stat"][k], b["stat"][k]) for k in ("urms", "k", "epsilon", "Re_lambda", "skewness",
                                                                 "flatness")},
        "spectrum_max_rel": max(rel(ek_a[k], ek_b[k]) for k in shells),
        "spectrum_shells": len(shells),
        "particle_rms_velocity_rel": [
            rel(stats.particle_rms_velocity(pa["u"], pa["v"], pa["w"]),
                stats.particle_rms_velocity(pb["u"], pb["v"], pb["w"]))
            for pa, pb in zip(a["parts"], b["parts"])],
        "particle_position_rel_l2": [
            float(np.sqrt(sum(np.sum((pa[k] - pb[k]) ** 2) for k in "xyz") / sum(np.sum(pb[k] ** 2) for k in "xyz")))
            for pa, pb in zip(a["parts"], b["parts"])],
        "fp64_stat": {k: b["stat"][k] for k in ("urms", "epsilon", "Re_lambda", "skewness", "flatness")},
        "note": "statistics: Flows.stat on the device (FP64 reductions) of each form's final state; E(k): "
                "shell sums of 0.5|u_hat|^2; tolerance target for the velocity: rel-L2 <= 1e-4",
    }


# ------------------------------------------------------------------ CPU baseline
class OracleSample:
    """The oracle (C restatement of the reference, OpenMP over all host cores)
    on a bounded sample of the workload.

    A full 512^3 oracle step takes minutes (its 600 HSMAC sweeps dominate), so
    a step is measured in two parts: the step with each couple cut to one
    time-blocked group of 3 sweeps (timestep!, both rhs!/update!, forcing!,
    the particles, 2 x 3 sweeps) and one 3-sweep couple; the step time is the
    first plus (S/3 - 2) times the second, S being the sweeps per step of the
    GPU run of the same workload.  A couple of S/2 sweeps is S/6 such groups
    (halo fill, the overlap sweep with its face phases, two plain sweeps)."""

    def __init__(self, workload, flow, parts):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_engine import OracleEngine, load_oracle

        rc, w = make_run_config(workload, precision="fp64", itrmax=3)
        rc.abi.use_graphs = 0
        self.n3 = float(np.prod(rc.dims))
        self.np_tot = float(sum(w["counts"]))
        self.cores = load_oracle().lcs_oracle_threads()
        self.eng = OracleEngine(rc.abi)
        load_engine(self.eng, rc, flow, parts)

    def capped_step(self):
        t0 = time.perf_counter()
        dt = self.eng.timestep()
        self.eng.evolve(dt)
        self.dt = dt
        return time.perf_counter() - t0

    def group(self):
        t0 = time.perf_counter()
        self.eng.couple(2, self.dt)
        return time.perf_counter() - t0

    def close(self):
        self.eng.close()


def cpu_baseline(workload, flow, parts, sweeps_per_step):
    smp = OracleSample(workload, flow, parts)
    t_step3 = smp.capped_step()
    t_group = smp.group()
    smp.close()
    t = t_step3 + (sweeps_per_step / 3.0 - 2.0) * t_group
    return {"value": smp.n3 / t / 1e6, "unit": "Mcell-steps/s", "cores": smp.cores, "kind": "port",
            "sample": f"one step of the {workload} workload with each couple cut to 3 sweeps ({t_step3:.1f} s) and "
                      f"one 3-sweep couple ({t_group:.2f} s), extrapolated to {sweeps_per_step:.0f} sweeps per step "
                      f"(the GPU run's count): {t:.1f} s per step",
            "particle_steps_per_s": smp.np_tot / t, "seconds_per_step": t}


def run_reference(args):
    """Rank 0 alone times the CPU restatement; other ranks exit without work.
    Warm-up: the capped step (whose non-sweep part is kept) and W 3-sweep
    couples; each timed step: one 3-sweep couple, the step's time assembled as
    in OracleSample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in OTHER_WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU arm for the {args.workload} workload"}))
        return 0
    rc, w = make_run_config(args.workload)
    flow, parts = host_inputs(rc)
    smp = OracleSample(args.workload, flow, parts)
    t_step3 = smp.capped_step()
    groups = [smp.group() for _ in range(max(1, args.warmup))]
    S = float(os.environ.get("LCS_REFERENCE_SWEEPS", "600"))  # both couples run itrmax = 300
    t_rest = t_step3 - 2.0 * groups[0]
    times = [t_rest + S / 3.0 * smp.group() for _ in range(args.steps)]
    smp.close()
    total = sum(times)
    value = smp.n3 * args.steps / total / 1e6
    sample = (f"each step: one 3-sweep HSMAC couple timed, times {S / 3.0:.0f}, plus the non-sweep part of a step "
              f"({t_rest:.1f} s, timed once in warm-up on a step with each couple cut to 3 sweeps)")
    line = {"metric": "Mcell-steps/s", "value": value, "unit": "Mcell-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded spectral field, uniform random particles)",
            "config": {"workload": args.workload, "n": rc.dims[0], "particles": sum(w["counts"]),
                       "species": len(w["counts"]), "precision": "fp64", "parallelism": "replicas"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Mcell-steps/s", "cores": smp.cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "particle_steps_per_s": smp.np_tot * args.steps / total}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    world, rank, local = dist_setup()
    device = local if world > 1 else int(os.environ.get("LCS_DEVICE", "0"))
    rc, w = make_run_config(args.workload, seed=rank, precision=args.precision)
    flow, parts = host_inputs(rc, pinned=True)
    n3 = float(np.prod(rc.dims))
    main = run_form(args, args.precision, (rc, w), flow, parts, world, device, primary=True)

    # the other precision form on the same workload, inputs and step counts
    forms = None
    if not args.no_forms:
        other = "fp32-mixed" if args.precision == "fp64" else "fp64"
        o = run_form(args, other, make_run_config(args.workload, seed=rank, precision=other), flow, parts, world,
                     device, primary=False)
        by = {args.precision: main, other: o}
        forms = {p: {"value": r["value"], "ms_per_step": r["ms_per_step"], "sweeps_per_step": r["sweeps_per_step"],
                     "roofline_frac": r["roofline"]["frac"], "sweep_avg_launch_ms": r["roofline"]["avg_launch_ms"],
                     "clocks": r["clocks"]}
                 for p, r in by.items()}
        forms["fp32-mixed"]["kernels"] = by["fp32-mixed"]["kernels"]
        forms["fp32_mixed_vs_fp64"] = by["fp32-mixed"]["value"] / by["fp64"]["value"]
        forms["errors"] = precision_errors(by["fp32-mixed"], by["fp64"], w["nu"])
        forms["hsmac_epsp"] = ("epsp = 1e-8 * dxmin in both forms (RMS div < 1e-8); the sweep counts per step are "
                               "those above")
        for r in by.values():
            for k in ("flow", "parts"):
                r.pop(k, None)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload in WORKLOADS:
        base = cpu_baseline(args.workload, flow, parts, main["sweeps_per_step"])
    # the batching form beside the headline: the 64-member ensemble, 3 steps
    batching = None
    if not args.no_forms:
        batching = batch_form(3)
    if rank == 0:
        div_rms, div_max = main["divergence"]
        line = {
            "metric": "Mcell-steps/s",
            "value": main["value"],
            "unit": "Mcell-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": main["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 (FP64 residuals, reductions, positions)",
            "data": "synthetic (seeded spectral field, uniform random particles)",
            "config": {"workload": args.workload, "n": rc.dims[0], "particles": int(sum(w["counts"])),
                       "species": len(w["counts"]), "forcing": w["forcing"]["kind"], "hsmac_itrmax": 300,
                       "hsmac_rms_div_tol": 1e-8,
                       "l2": f"inputs larger than L2 ({(rc.dims[0] + 6) ** 3 * elem_bytes(args.precision) / 1e6:.0f} "
                             "MB per field)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "precision": args.precision},
            "particle_steps_per_s": main["particle_steps_per_s"],
            "hsmac_sweeps_per_step": main["sweeps_per_step"],
            "gpu_launches": int(round(main["launches_per_step"] * args.steps)),
            "clocks": main["clocks"],
            "roofline": main["roofline"],
            "kernels": main["kernels"],
            "fp64": main.get("fp64"),
            "divergence": {"rms": div_rms, "max": div_max, "last_couple_residual": main["last_log"]["couple2"]["div"],
                           "note": "of the velocity after the timed steps, HSMAC form, interior cells"},
            "e2e": main["e2e"],
            "cpu_baseline": ({k: base[k] for k in ("value", "unit", "cores", "kind", "sample")} if base else None),
            "precision_forms": forms,
            "batching_form": batching,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    return 0


# ----------------------------------------------------------------- batching form
def ensemble_members(seed=0):
    """The 64-member ensemble: 16 x 32^3, 24 x 48^3, 16 x 64^3, 8 x 96^3 with
    per-member seeds, nu log-uniform in [0.01, 0.05], one species of 8k-128k
    particles with tau_p log-uniform in [0.01, 1], linear-power forcing
    P = 0.5, FP32-mixed."""
    rng = np.random.default_rng(seed)
    sizes = [32] * 16 + [48] * 24 + [64] * 16 + [96] * 8
    members = []
    for i, n in enumerate(sizes):
        nu = float(np.exp(rng.uniform(np.log(0.01), np.log(0.05))))
        taup = float(np.exp(rng.uniform(np.log(0.01), np.log(1.0))))
        count = int(np.exp(rng.uniform(np.log(8192), np.log(131072))))
        d = lcfg.workload(n, nu, {"kind": "linear-power", "params": {"power": 0.5}}, [taup], [count], seed=1000 + i,
                          precision="fp32-mixed")
        members.append(lcfg.from_dict(d))
    return members


def batch_form(steps):
    """The 64-member ensemble stepped together (lcs_batch_step, grouped by
    shape, autotuned), host wall clock around `steps` steps after one warm-up."""
    from lcs_b200 import Batch

    members = ensemble_members()
    for rc in members:
        rc.abi.use_graphs = 1
    cells = float(sum(np.prod(rc.dims) for rc in members))
    t_create = time.perf_counter()
    b = Batch([rc.abi for rc in members])
    create_s = time.perf_counter() - t_create
    for rc, e in zip(members, b.members):
        load_engine(e, rc, *host_inputs(rc))
    b.step(1)
    t0 = time.perf_counter()
    b.step(steps)
    el = time.perf_counter() - t0
    b.close()
    return {"workload": "batch64", "value": cells * steps / el / 1e6, "unit": "Mcell-steps/s",
            "ms_per_step": el * 1e3 / steps, "steps": steps, "members": len(members), "cells": int(cells),
            "autotune_and_create_s": create_s, "precision": "fp32-mixed",
            "timing": "host wall clock around lcs_batch_step"}


def run_batch(args):
    """The batching form: all 64 members stepped together (lcs_batch_step),
    against the same members stepped one after another."""
    from lcs_b200 import Batch, Engine

    members = ensemble_members()
    for rc in members:
        rc.abi.use_graphs = 1
    cells = float(sum(np.prod(rc.dims) for rc in members))
    parts_total = float(sum(sum(si.nvalid for si in rc.species) for rc in members))
    t_create = time.perf_counter()
    b = Batch([rc.abi for rc in members])
    create_s = time.perf_counter() - t_create
    shapes = {}
    for i, rc in enumerate(members):
        shapes.setdefault(f"{rc.dims[0]}^3", b.tuning(i))
    for rc, e in zip(members, b.members):
        load_engine(e, rc, *host_inputs(rc))
    b.step(max(1, args.warmup))
    import ctypes as C

    def launch_total():
        tot = 0
        for e in b.members:
            n = C.c_int64()
            e._check(e.lib.lcs_launch_count(e.handle, C.byref(n)))
            tot += n.value
        return tot

    l0 = launch_total()
    t0 = time.perf_counter()
    logs = b.step(args.steps)
    batch_s = time.perf_counter() - t0
    launches = launch_total() - l0
    sweeps = float(np.mean([lg["couple1"]["sweeps"] + lg["couple2"]["sweeps"] for ml in logs for lg in ml]))
    b.close()
    # the same members one at a time (each on its own handle)
    seq_steps = max(1, min(args.steps, 3))
    seq_s = 0.0
    for rc in members:
        e = Engine(rc.abi)
        load_engine(e, rc, *host_inputs(rc))
        e.step(1)
        e.synchronize()
        t0 = time.perf_counter()
        e.step(seq_steps)
        seq_s += time.perf_counter() - t0
        e.close()
    value = cells * args.steps / batch_s / 1e6
    seq_value = cells * seq_steps / seq_s / 1e6
    print(json.dumps({
        "metric": "Mcell-steps/s", "value": value, "unit": "Mcell-steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": batch_s * 1e3 / args.steps, "higher_is_better": True,
        "dtype": "f32 (FP64 residuals, reductions, positions)", "data": "synthetic (seeded spectral fields)",
        "config": {"workload": "batch64", "members": len(members), "sizes": "16x32^3, 24x48^3, 16x64^3, 8x96^3",
                   "cells": int(cells), "particles": int(parts_total), "precision": "fp32-mixed"},
        "particle_steps_per_s": parts_total * args.steps / batch_s,
        "hsmac_sweeps_per_member_step": sweeps,
        "graph_kernel_nodes_per_step": launches / args.steps,
        "graph_kernel_nodes_note": "kernel launches captured in the step graphs of all members and groups, the "
                                   "body of each HSMAC WHILE loop counted once",
        "groups": len(shapes),
        "sequential": {"value": seq_value, "steps": seq_steps, "note": "the members one after another, each alone"},
        "batch_vs_sequential": value / seq_value,
        "autotune": {"create_s": create_s, "chosen": shapes},
        "timing": "host wall clock around lcs_batch_step (all members enqueued, then all waited for)",
    }), flush=True)
    return 0


# ------------------------------------------------------------------ serving form
def run_serve(args):
    """The serving form: a seeded Poisson stream (--rate per second) of
    --requests requests with N in {32, 48, 64, 96, 128, 192}, 10^4-10^6
    particles with tau_p log-uniform in [0.01, 2], 50-500 steps (times
    --steps-scale), FP32-mixed, admitted under a 150 GB budget."""
    from lcs_b200 import Server, _abi

    rng = np.random.default_rng(2026)
    sizes = [32, 48, 64, 96, 128, 192]
    flows = {}
    for n in sizes:  # one seeded spectral field per size (the inputs are not timed)
        flows[n] = inits.spectral_flow(n, seed=n)
    srv = Server(device=int(os.environ.get("LCS_DEVICE", "0")), max_active=int(os.environ.get("LCS_SERVE_SLOTS", "32")),
                 steps_per_slice=4, hbm_budget_bytes=150 * 10 ** 9)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, args.requests))
    tickets, work = [], 0.0
    t0 = time.perf_counter()
    for r in range(args.requests):
        n = int(rng.choice(sizes))
        count = int(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        taup = float(np.exp(rng.uniform(np.log(0.01), np.log(2.0))))
        steps = max(1, int(round(rng.integers(50, 501) * args.steps_scale)))
        d = lcfg.workload(n, 0.01, {"kind": "linear-power", "params": {"power": 0.5}}, [taup], [count], seed=r,
                          precision="fp32-mixed")
        rc = lcfg.from_dict(d)
        x, y, z = inits.random_positions(count, 7 + r)
        zero = np.zeros(count)
        sp = [{"diam": np.full(count, rc.species[0].diam), "x": x, "y": y, "z": z, "u": zero, "v": zero, "w": zero}]
        delay = arrivals[r] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        tickets.append(srv.submit(rc.abi, *flows[n], species=sp, nsteps=steps, interp_velocity=True))
        work += float(n) ** 3 * steps
    srv.drain(timeout_s=float(os.environ.get("LCS_SERVE_TIMEOUT_S", "3600")))
    makespan = time.perf_counter() - t0
    st = srv.stats()
    lat = []
    for t in tickets:
        state, _ = srv.poll(t)
        if state == _abi.REQ_DONE:
            lat.append(srv.result(t)["latency_s"])
        srv.release(t)
    srv.close()
    print(json.dumps({
        "metric": "served solves/s; p50/p99 time-to-completion", "value": st["completed"] / makespan,
        "unit": "solves/s", "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
        "mean_latency_s": st["mean_latency_s"], "completed": st["completed"], "failed": st["failed"],
        "makespan_s": makespan, "Mcell_steps_per_s": work / makespan / 1e6,
        "peak_bytes_in_use": st["peak_bytes_in_use"], "busy_s": st["busy_s"],
        "config": {"workload": "serve", "requests": args.requests, "rate_per_s": args.rate,
                   "steps_scale": args.steps_scale, "sizes": sizes, "hbm_budget_bytes": 150 * 10 ** 9,
                   "slots": int(os.environ.get("LCS_SERVE_SLOTS", "32")), "precision": "fp32-mixed"},
        "data": "synthetic (one seeded spectral field per size, seeded particles and request stream)",
        "timing": "host wall clock; latency = submit to result ready",
    }), flush=True)
    return 0


# ------------------------------------------------------------ particle cell index
def kernel_bytes(n, h, T, particles_per_launch):
    """Algorithmic DRAM bytes per launch of the step's kernels (n^3 grid, halo
    h, T-byte field elements):
    - hsmac_rw: U, V, W, P read and written once per cell, 8T x n^3;
    - hsmac_faces: the same per cell of the six face slabs of the first
      time-blocked sweep's box -1..n+3 around the core 2..n;
    - synchalo: the couple's fill (radius h, all 26 directions, U, V, W): one
      read and one write per halo cell;
    - rhs_update: stage 1 reads U, V, W, P, writes U2, V2, W2 (7T); stage 2
      also reads U2, V2, W2 (10T): the mean, 8.5T x n^3;
    - particles: 13 FP64 properties read or written a particle, the mean of the
      two stages (104 and 152 B), the fluid gathers being cache traffic;
    - cfl_max: U, V, W read once (3T x n^3)."""
    n3 = float(n) ** 3
    slab = float(n + 5) ** 3 - float(n - 1) ** 3
    halo = float(n + 2 * h) ** 3 - n3
    return {"hsmac_rw": 8 * T * n3, "hsmac_faces": 8 * T * slab, "synchalo": 3 * 2 * T * halo,
            "rhs_update": 8.5 * T * n3, "particles": 128.0 * particles_per_launch, "cfl_max": 3 * T * n3}


def makeindex_bytes(n, H):
    """Algorithmic DRAM bytes of one makeindex of n particles over H cells, as
    this design moves them: positions 24 + keys/indices 8 (cell_hash); the
    stable LSD sort of 32-bit (hash, index) pairs, one histogram read 4 and 3
    passes of 16 for hashes below 2^24 (radix_sort); perm 4 + 17 8-byte
    properties read and written into the spare block (permute) 2 x 17 x 8;
    keys 4 + Int64 hashes 8 (hash_runs); per cell the run-end array zeroed 8,
    scanned 16 and read 8, starts/stops 16."""
    return n * (24 + 8 + 4 + 3 * 16 + 4 + 2 * 17 * 8 + 4 + 8) + (H + 1) * (8 + 16 + 8) + H * 16


def run_makeindex(args):
    """`Particles.makeindex!` of the lp512 particles (512^3 grid, 2^24 particles
    in 3 species, grid_ratio 4 as in the reference's cfgs/N1024-1.lcs-yaml):
    particles indexed per second, on the order a previous index left after one
    time step (the steady case; `value`, device-timed) and on random order (the
    first index).  e2e is the host wall clock around the synchronous calls."""
    from lcs_b200 import Engine

    ratio = 4
    rc, w = make_run_config("lp512", seed=0, precision="fp64")
    rc.abi.use_graphs = 1
    flow, parts = host_inputs(rc)
    eng = Engine(rc.abi)
    load_engine(eng, rc, flow, parts)
    nsp = len(rc.species)
    total = float(sum(si.nvalid for si in rc.species))
    H = (512 // ratio + 2) ** 3
    algo = float(sum(makeindex_bytes(si.nvalid, H) for si in rc.species))

    def index_all():
        for s in range(nsp):
            eng.particles_makeindex(s, 1, ratio)

    def device_ms():
        t = eng.profile_totals()
        return t["makeindex"][0], {k: v[0] for k, v in t.items()}

    def push_ms(reps=3):
        """Device ms of one motion! pass (the fluid gathers) over every species."""
        for s in range(nsp):
            eng.particles_motion(s, 1)
        eng.profile(True)
        eng.profile_reset()
        for _ in range(reps):
            for s in range(nsp):
                eng.particles_motion(s, 1)
        t = eng.profile_totals()["particles"][0] / reps
        eng.profile(False)
        return t

    push_random_ms = push_ms()  # upload order: uniform random positions
    index_all()  # buffers allocated; the random order is restored below
    eng.synchronize()
    reps = max(1, min(args.steps, 3))
    eng.profile(True)
    eng.profile_reset()
    for _ in range(reps):
        for s, (d, x, y, z) in enumerate(parts):
            zero = np.zeros_like(x)
            eng.upload_particles(s, d, x, y, z, zero, zero, zero)
        index_all()
    first_ms = device_ms()[0] / reps
    eng.profile(False)
    for _ in range(args.warmup):
        index_all()
    eng.step(1)
    index_all()
    eng.step(1)  # particles moved one step since their last index
    eng.synchronize()
    eng.profile(True)
    eng.profile_reset()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        index_all()
    wall_s = (time.perf_counter() - t0) / args.steps
    steady_ms, parts_ms = device_ms()
    steady_ms /= args.steps
    eng.profile(False)
    push_sorted_ms = push_ms()  # the order makeindex! left
    hashes, starts, stops = eng.particles_cellindex(0, ratio)
    ok = bool(np.all(np.diff(hashes) >= 0)) and int(np.sum(stops - starts + 1)) == hashes.size
    # Particles.stat of every species with the reference's production settings
    # (cfgs/N1024-1.lcs-yaml: grid_ratio 4, 16 bins from 1.25e-4, search 2
    # cells, contact 0.01, 64 directions up to k = 768), device-timed per kernel
    tau_eta = eng.flow_stat()["tau_eta"]
    for s in range(nsp):  # warm-up (scratch allocation)
        eng.particles_stat(s, tau_eta, max_wavenumber=768)
    eng.profile(True)
    eng.profile_reset()
    t0 = time.perf_counter()
    for s in range(nsp):
        eng.particles_stat(s, tau_eta, max_wavenumber=768)
    stat_wall_ms = (time.perf_counter() - t0) * 1e3
    stat_ms = {k: v[0] for k, v in eng.profile_totals().items()}
    eng.profile(False)

    # the particle kernels (boundary!, motion!, update!, both stages) of one
    # whole step: on the upload order, then with lcs_set_particle_sort(1)
    def step_particles_ms():
        eng.profile(True)
        eng.profile_reset()
        eng.step(1)
        t = eng.profile_totals()["particles"][0]
        eng.profile(False)
        return t

    for s, (d, x, y, z) in enumerate(parts):
        zero = np.zeros_like(x)
        eng.upload_particles(s, d, x, y, z, zero, zero, zero)
    step_random_ms = step_particles_ms()
    eng.set_particle_sort(1, ratio)
    eng.step(1)  # followed by the first sort
    step_sorted_ms = step_particles_ms()
    eng.set_particle_sort(0, ratio)
    launches = eng.launch_count()
    eng.close()
    peak, peak_src = hbm_peak()
    gbs = algo / (steady_ms * 1e-3) / 1e9
    out = {
        "metric": "particles indexed/s", "value": total / (steady_ms * 1e-3), "unit": "particles/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": steady_ms, "higher_is_better": True,
        "dtype": "f64 positions, u32 keys", "data": "synthetic (seeded uniform positions)",
        "config": {"workload": "makeindex", "n": 512, "particles": int(total), "species": nsp, "grid_ratio": ratio,
                   "cells": int(H), "l2": "inputs (2^24 x 17 x 8 B) exceed L2"},
        "e2e": {"value": total / wall_s, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "note": "host wall clock around the synchronous C-ABI calls"},
        "first_index": {"value": total / (first_ms * 1e-3), "ms": first_ms, "note": "random particle order"},
        "per_kernel_ms": {k: v / args.steps for k, v in parts_ms.items() if k != "makeindex"},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "peak_source": peak_src, "algorithmic_bytes": algo},
        "invariants_ok": ok, "gpu_launches_total": launches,
        "particle_push": {"random_order_ms": push_random_ms, "cell_order_ms": push_sorted_ms,
                          "speedup": push_random_ms / push_sorted_ms,
                          "step_random_order_ms": step_random_ms, "step_sorted_every_step_ms": step_sorted_ms,
                          "note": "motion! of all species (interpolation gathers of U, V, W), device ms, on the "
                                  "upload order and on the cell order makeindex! leaves; step_*: the particle kernels "
                                  "of one whole step (both stages), on the upload order and with "
                                  "lcs_set_particle_sort(1, 4)"},
        "particle_stat": {"wall_ms": stat_wall_ms, "device_ms": stat_ms,
                          "note": "Particles.stat of all 3 species (Summary, makeindex!, rdf, spectrum 19 shells x "
                                  "64 directions)"},
        "timing": "CUDA events on the engine stream around each index (profiling spans)",
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_engine import OracleEngine

        o = OracleEngine(rc.abi)
        d, x, y, z = parts[0]
        zero = np.zeros_like(x)
        o.upload_particles(0, d, x, y, z, zero, zero, zero)
        t0 = time.perf_counter()
        o.particles_makeindex(0, 1, ratio)
        el = time.perf_counter() - t0
        o.close()
        out["cpu_baseline"] = {"value": x.size / el, "unit": "particles/s", "cores": 1, "kind": "port",
                               "sample": f"one makeindex of species 0 ({x.size} particles, random order, {el:.1f} s)"}
    print(json.dumps(out), flush=True)
    return 0


def run_couple(args):
    """Two couples (`Flows.couple!`, HSMAC time blocking and overlap) of the
    seeded 256^3 rc256 fields, 30 sweeps each (epsp below any residual), stage
    2 with dtrk 0.003: the first warms up, the second is device-timed per
    kernel.  The k-th sweep launch of the second couple is launch 30 + k."""
    from lcs_b200 import Engine, _abi

    rc, w = make_run_config("rc256", seed=0, precision=args.precision)
    c = rc.abi
    c.mode = _abi.MODE_FLOW
    c.n_species = 0
    c.itrmin, c.itrmax, c.epsp = 6, 30, 1e-30
    c.use_graphs = 0
    flow, _ = host_inputs(rc)
    eng = Engine(c)
    eng.upload_flow(*flow)
    eng.couple(2, 0.003)
    eng.upload_flow(*flow)
    eng.synchronize()
    eng.profile(True)
    eng.profile_reset()
    lg = eng.couple(2, 0.003)
    tot = eng.profile_totals()
    eng.profile(False)
    eng.close()
    ms = sum(v[0] for v in tot.values())
    n3 = float(rc.dims[0]) ** 3
    out = {
        "metric": "HSMAC sweeps/s", "value": lg["sweeps"] / (ms * 1e-3), "unit": "sweeps/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic (seeded spectral fields)",
        "config": {"workload": "couple256", "n": rc.dims[0], "sweeps": lg["sweeps"], "precision": args.precision},
        "kernels_us": {k: v[0] / v[1] * 1e3 for k, v in sorted(tot.items(), key=lambda kv: -kv[1][0])},
        "mcell_sweeps_per_s": n3 * lg["sweeps"] / (ms * 1e-3) / 1e6,
        "timing": "CUDA events on the engine stream around each launch (profiling spans)",
    }
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + list(OTHER_WORKLOADS), default="lp512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "fp32-mixed"], default="fp64")
    ap.add_argument("--no-forms", action="store_true", help="skip the other precision form and its errors")
    ap.add_argument("--requests", type=int, default=1000, help="serve: number of requests")
    ap.add_argument("--steps-scale", type=float, default=1.0, help="serve: scale of the 50-500 step counts")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: mean arrivals per second")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("batch64", "serve"):
        # one hardware work queue per member stream (read at context creation)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if args.workload == "batch64":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "makeindex":
        return run_makeindex(args)
    if args.workload == "couple256":
        return run_couple(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
