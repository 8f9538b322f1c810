"""Benchmark: particle-steps/s of the SPH step on B200.

Default workload (one GPU): the self-gravitating disph Evrard sphere on a
256^3 lattice, N = 8,783,848 particles, Wendland C4, neighborNumber = 128,
time-dependent AV (0.1, 2.0, 0.2), Balsara switch, artificial conductivity,
Barnes-Hut gravity theta = 0.5, gamma = 5/3; seeded synthetic lattice initial
conditions (no dataset involved), built by ics.py for both arms.  A step is
one Solver::integrate (timestep, predict, tree build, PreInteraction,
FluidForce, GravityForce, correct) over all particles.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the plain FP64 form (the drop-in), timed with CUDA events on the
context stream with inputs resident in HBM; `mixed` reports the FP32 form on
the same workload; `e2e` is the same metric through the C ABI with the
particle state copied host -> device and back every step (pinned buffers).
`roofline` is the dominant stage against the FP64 pipe (algorithmic FLOPs
from the device work counters x the per-unit weights of flop_weights.md, over
the stage's CUDA-event time, against a cuBLAS DGEMM measured in the same
run), with its HBM figure beside it.
Multi-GPU: replicas only (each rank integrates its own copy; no data-path
collective); the timed region is bracketed by barriers and the max over ranks
is reported.  `--impl reference` times the reference's own OpenMP CPU build
(oracle/_ref) on the same workload at its full size, on every host core.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sph-code-simulation_b200"))

import numpy as np  # noqa: E402

import ics  # noqa: E402  (numpy initial conditions: no library load)
import sphparams as SP  # noqa: E402

METRIC = "particle-steps/s on 1 B200: FP64 plain vs FP32+learned-Riemann at ≤1e-5 rel err"
UNIT = "particle-steps/s"


class Workload:
    """One benchmark workload: parameters, initial conditions at a target size,
    and a smaller CPU sample of the same workload for the reference arm."""

    def __init__(self, name, desc, cfg, sample, default_n, cpu_n, learned=False, **overrides):
        self.name, self.desc, self.cfg, self.sample = name, desc, cfg, sample
        self.default_n, self.cpu_n, self.learned, self.overrides = default_n, cpu_n, learned, overrides

    def params(self, precision):
        p = SP.config_params(self.cfg, precision=precision, **self.overrides)
        if self.learned:
            p.riemann_guess = SP.GUESS_MLP
        return p

    def fields(self, n):
        return self.sample(n)


def _evrard(n):
    lattice = max(8, int(round((n * 6.0 / 3.14159265) ** (1.0 / 3.0))))
    return ics.evrard(lattice)


def _shear(n):
    return ics.shear_layer((0.1875 / n) ** (1.0 / 3.0))


def _tube(n):
    return ics.shock_tube((0.05 * 0.05 / n) ** (1.0 / 3.0), ly=0.05)


def _blast(n):
    return ics.blast_field(1.0 / round(n ** (1.0 / 3.0)))


WORKLOADS = {
    "evrard_ssph": Workload("evrard_ssph", "ssph Evrard sphere 17K (cubic, K=50, leaf=1, Balsara, BH gravity)",
                            "evrard_ssph", _evrard, 17256, 17256),
    "shear_disph": Workload("shear_disph", "disph periodic shear layer 1.0M (Wendland C4, K=128, AC)",
                            "shear_disph", _shear, 1.0e6, 6.5e4),
    "tube_gsph": Workload("tube_gsph", "gsph shock tube 2.0M (MUSCL, iterative Riemann, cubic, K=50)",
                          "tube_gsph", _tube, 2.0e6, 6.5e4),
    "tube_gsph_mlp": Workload("tube_gsph_mlp", "gsph shock tube 2.0M with the learned Riemann guess",
                              "tube_gsph", _tube, 2.0e6, 6.5e4, learned=True),
    "tube_gdisph": Workload("tube_gdisph", "gdisph shock tube 2.0M (MUSCL + HLL, cubic, K=50, Balsara, TD-AV, AC)",
                            "tube_gdisph", _tube, 2.0e6, 6.5e4),
    # many point blasts: most pairs are strong-shock Riemann problems (plain
    # solver ~3.5 Newton iterations per solve); the learned start against
    # the plain solver at the reference's 1e-6 and at the learned path's 1e-10
    "blast_gsph": Workload("blast_gsph", "gsph many-blast cube 2.0M (MUSCL, iterative Riemann, cubic, K=50)",
                           "blast_gsph", _blast, 2.0e6, 1.3e5),
    "blast_gsph_tol1e-10": Workload("blast_gsph_tol1e-10", "gsph many-blast cube 2.0M, plain solver to 1e-10",
                                    "blast_gsph", _blast, 2.0e6, 1.3e5, riemann_tol=1e-10),
    "blast_gsph_mlp": Workload("blast_gsph_mlp", "gsph many-blast cube 2.0M with the learned Riemann guess",
                               "blast_gsph", _blast, 2.0e6, 1.3e5, learned=True),
    # The disph sphere's centre breaks down at t ~ 0.003 on this resolution
    # (innermost particles reach u < 0 in predict: the scheme, reproduced by
    # the compiled reference); cflSound 0.006 / cflForce 0.003 keep every
    # default run (warm-up + 20 timed steps per form, and 100-step drift
    # runs) well before it, at the same cost per step.
    "evrard_disph": Workload("evrard_disph", "disph + BH gravity Evrard sphere 8.78M (256^3 lattice, Wendland C4, "
                             "K=128, TD-AV, Balsara, AC, theta=0.5; CFL 0.006/0.003)", "evrard_disph", _evrard,
                             8.78e6, 8.78e6, cfl_sound=0.006, cfl_force=0.003),
}
DEFAULT_WORKLOAD = "evrard_disph"

# fields a step reads from / writes back to the caller in the e2e leg
E2E_IN = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "mass", "dens",
          "pres", "ene", "dene", "sml", "sound", "balsara", "alpha", "gradh"]
E2E_OUT = E2E_IN + ["phi", "neighbor"]

# algorithmic bytes per unit: each node's link + geo (+ ksize for the symmetric
# walk) and each particle's position read once, each list entry written once
NODE_BYTES = 16 + 32          # link (int4) + geo (double4) read per node
PAIR_WALK_NODE_BYTES = NODE_BYTES + 8


# FLOPs per unit of work (flop_weights.md: + - x / sqrt exp counted 1 each in
# the formulas of the reference's loops, common subexpressions of one pair
# shared and per-particle factors hoisted); units are the device work counters
FLOP_W = {
    "cand": 8,                     # r_ij and r^2 of one list entry (3 sub, 3 mul, 2 add)
    "newton_kernel": {"cubic": 25, "wendland": 27, "gauss": 12},  # sqrt, W and dW/dh at one r
    "newton_sum": {"ssph": 4, "disph": 2, "gsph": 4, "gdisph": 2},
    "pre_pair": {"ssph": 72, "disph": 79, "gsph": 78, "gdisph": 120},
    "force_pair": {"ssph": 109, "disph": 122, "gsph": 233, "gdisph": 270},
    "riemann_iter": 40,            # one van Leer Newton step of the exact solver
    "grav_node": 10,               # opening test of one node
    "grav_mono": 14,               # monopole term of an accepted node
    "grav_leaf": 80,               # softened particle pair (two f, two g)
}
_SPH = {0: "ssph", 1: "disph", 2: "gsph", 3: "gdisph", 4: "srgsph"}
_KER = {0: "cubic", 1: "wendland", 2: "gauss"}


def stage_flops(stage: str, c: dict, p) -> float:
    """Algorithmic FLOPs of a stage from the work counters of the timed steps
    (None for stages bound by memory traffic, not arithmetic)."""
    sph, ker = _SPH[p.sph_type], _KER[p.kernel]
    if stage == "pre" and sph in FLOP_W["pre_pair"]:
        newton = FLOP_W["newton_kernel"][ker] + FLOP_W["newton_sum"][sph]
        return (c["pre_candidates"] * FLOP_W["cand"] + c["pre_newton_pairs"] * newton
                + c["pre_pairs"] * FLOP_W["pre_pair"][sph])
    if stage == "force" and sph in FLOP_W["force_pair"]:
        return (c["force_candidates"] * FLOP_W["cand"] + c["force_pairs"] * FLOP_W["force_pair"][sph]
                + c["riemann_iterations"] * FLOP_W["riemann_iter"])
    if stage == "gravity":
        return (c["gravity_nodes"] * FLOP_W["grav_node"] + c["gravity_monopoles"] * FLOP_W["grav_mono"]
                + c["gravity_leaf_pairs"] * FLOP_W["grav_leaf"])
    return None


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_fp_peaks():
    """FP64 and FP32 (no TF32) GEMM throughput of this GPU in TFLOP/s: cuBLAS
    through torch, 8192^3 (2 N^3 FLOPs), best of 5 after 2 warm-ups; the
    FP64 / FP32 pipes' measured roofs for the pair and gravity kernels."""
    import torch
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for name, dt, nn in (("fp64", torch.float64, 8192), ("fp32", torch.float32, 8192)):
            a = torch.randn(nn, nn, dtype=dt, device="cuda")
            b = torch.randn(nn, nn, dtype=dt, device="cuda")
            best = 1e30
            for k in range(7):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                e1.synchronize()
                if k >= 2:
                    best = min(best, e0.elapsed_time(e1))
            out[name] = 2.0 * nn ** 3 / (best * 1e-3) / 1e12
            del a, b
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus: int):
    """One process per GPU (torchrun); returns (rank, world, local_rank)."""
    if n_gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0
    import datetime

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), local


def barrier():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.barrier()
    except Exception:
        pass


def max_over_ranks(x: float) -> float:
    """Max of a per-rank scalar (timed-region milliseconds) over all ranks."""
    try:
        import torch
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()):
            return x
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else None
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    except Exception:
        return x


def whole_job_value(units_per_rank: float, world: int, max_ms: float) -> float:
    """Aggregate throughput: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / (max_ms / 1e3)


def _pinned(n: int, names):
    import torch
    return {f: torch.zeros(n, dtype=torch.float64, pin_memory=True) for f in names}


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def run_gpu(args, rank: int, world: int, local: int):
    import sphgpu as G

    if not G.device_ok():
        raise SystemExit("bench: no usable sm_100 device")
    wl = WORKLOADS[args.workload]
    fields = wl.fields(args.particles or wl.default_n)
    n = len(fields["pos_x"])
    hbm, peak_kind = _peaks()

    def timed(precision, acc_tol=0.0):
        log(f"{wl.name} n={n} precision={precision} mixed_acc_tol={acc_tol}: initialize")
        p = wl.params(precision)
        p.mixed_acc_tol = acc_tol
        sim = G.Simulation(p)
        if wl.learned:
            sim.load_riemann_mlp()
        sim.upload(fields)
        sim.initialize()
        log("warm-up")
        for w in range(args.warmup):
            sim.integrate()
            if args.verbose:
                c = sim.counters()
                log(f"warm-up step {w} done: max_gather {c['max_gather']} max_pair {c['max_pair']} "
                    f"cap {c['gather_capacity']} retries {c['retries']} nodes {c['node_count']} "
                    f"split_warps {c['walk_split_warps']} fallbacks {c['walk_fallbacks']} dt {sim.time_dt()[1]:.3e}")
        sim.synchronize()
        sim.reset_counters()
        sim.enable_timing(True)
        log("barrier")
        barrier()
        log("timed region")
        clocks = ClockSampler(local) if (rank == 0 and precision == SP.FP64 and not args.no_clocks) else None
        if clocks:
            clocks.start()
        log("timer start")
        G.lib().sphgpu_timer_start(sim._h)
        for k in range(args.steps):
            sim.integrate()
            if args.verbose:
                c = sim.counters()
                log(f"timed step {k}: max_gather {c['max_gather']} max_pair {c['max_pair']} "
                    f"cap {c['gather_capacity']} retries {c['retries']} nodes {c['node_count']} "
                    f"split_warps {c['walk_split_warps']} fallbacks {c['walk_fallbacks']} dt {sim.time_dt()[1]:.3e}")
        import ctypes
        ms = ctypes.c_double()
        G.lib().sphgpu_timer_stop(sim._h, ctypes.byref(ms))
        log("timer stop")
        clk = clocks.stop() if clocks else None
        barrier()
        log(f"timed {ms.value:.1f} ms for {args.steps} steps")
        launches = int(G.lib().sphgpu_launch_count(sim._h))
        stages = sim.stage_times()
        counters = sim.counters()
        return sim, p, ms.value, clk, launches, stages, counters

    first = SP.MIXED if args.forms == "mixed" else SP.FP64
    sim, p0, ms, clk, launches, stages, counters = timed(first)
    ms_max = max_over_ranks(ms)
    value = whole_job_value(n * args.steps, world, ms_max)
    hbm_note = _hbm_roofline(G, sim, stages, counters, n, args, hbm, peak_kind)
    sim.close()

    # mixed precision form on the same workload
    mixed = None
    mstages, mcounters, pm = None, None, None
    if args.forms == "both":
        msim, pm, mms, _, _, mstages, mcounters = timed(SP.MIXED)
        mms_max = max_over_ranks(mms)
        mixed = {"value": whole_job_value(n * args.steps, world, mms_max), "ms_per_step": mms_max / args.steps,
                 "dtype": "f32 pair/gravity, f64 accumulators and kick-drift",
                 "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in mstages.items()}}
        msim.close()
        # the same with the FP64 re-evaluation of particles whose FP32 force /
        # gravity rounding could exceed 1e-5 of their acceleration
        csim, _, cms, _, _, cstages, ccounters = timed(SP.MIXED, 1e-5)
        cms_max = max_over_ranks(cms)
        mixed["checked_1e-5"] = {
            "value": whole_job_value(n * args.steps, world, cms_max), "ms_per_step": cms_max / args.steps,
            "rechecked_fraction": ccounters["mixed_rechecks"] / float(n * args.steps),
            "recheck_ms_per_step": round(cstages["recheck"][0] / args.steps, 4)}
        csim.close()

    # FLOP rooflines of the arithmetic stages against measured GEMM peaks
    try:
        fpk = measured_fp_peaks()
    except Exception as e:  # noqa: BLE001 - the roofline then says why it has no peak
        log(f"fp peak measurement failed: {e}")
        fpk = {}
    roofline, stage_roofs = _flop_roofline(stages, counters, p0, args, fpk, hbm_note, "fp64")
    if mixed is not None:
        _, mixed["stage_rooflines"] = _flop_roofline(mstages, mcounters, pm, args, fpk, None, "fp32")

    log("end to end")
    # end to end through the C ABI with host buffers
    e2e = None if args.no_e2e else run_e2e(args, G, fields, world, wl)

    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if first == SP.FP64 else "f32/f64",
        "data": "synthetic", "config": bench_config(wl, n, world, args),
        "form": "fp64 plain" if first == SP.FP64 else "mixed",
        "mixed": mixed, "e2e": e2e, "gpu_launches": launches,
        "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in stages.items()},
        "counters": counters, "roofline": roofline, "stage_rooflines": stage_roofs,
        "fp_peaks_tflops": {k: round(v, 2) for k, v in fpk.items()}, "clocks": clk,
    }


def bench_config(wl, n, world, args):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": wl.desc if not args.particles else f"{wl.desc} at N={n}", "n_particles": n,
            "particles_per_gpu": n, "l2": "inputs larger than L2 (state + neighbour lists > 3 GB per step)",
            "parallelism": f"replicas x{world}"}


def _hbm_roofline(G, sim, stages, counters, n, args, hbm, peak_kind):
    """HBM figure of the dominant stage (algorithmic bytes / launch time)."""
    dom = max(stages.items(), key=lambda kv: kv[1][0])[0]
    dom_ms, dom_launches = stages[dom]
    per_launch_ms = dom_ms / max(dom_launches, 1)
    nodes = counters["node_count"]
    if dom in ("gather_walk", "pair_walk"):
        off, _ = sim.neighbor_search(is_ij=(dom == "pair_walk"))
        entries = float(off[-1])
        nb = NODE_BYTES if dom == "gather_walk" else PAIR_WALK_NODE_BYTES
        algo = nodes * nb + n * 32 + entries * 4 + n * 4
        note = "node table + positions read once, list entries written once"
    elif dom == "pre":
        algo = counters["pre_list_entries"] / max(args.steps, 1) * 4 + n * (96 + 72)
        note = "gather list + particle state read once, outputs written once"
    elif dom == "force":
        algo = counters["force_candidates"] / max(args.steps, 1) * 4 + n * (128 + 32)
        note = "pair list + particle state read once, acc written once"
    elif dom == "gravity":
        algo = nodes * 48 + n * (32 + 32 + 40)
        note = "node records once, particle position / sml / acc read and acc / phi written once"
    else:
        algo = n * 64.0
        note = "particle state read and written once"
    per_step = dom_launches / max(args.steps, 1)
    if per_step > 1.0:
        per_launch_ms = dom_ms / max(args.steps, 1)
        note += f"; stage of {per_step:.0f} launches per step, timed as one"
    achieved = algo / (per_launch_ms / 1e3) / 1e9
    out = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
           "frac": round(achieved / hbm, 4), "traffic": None, "peak_source": peak_kind,
           "algorithmic_bytes_per_launch": algo, "launch_ms": round(per_launch_ms, 4), "accounting": note}
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof) and not args.particles:
        try:
            tr = json.load(open(prof)).get(args.workload, {}).get(dom)
            if tr:
                out["traffic"] = tr
        except (OSError, ValueError):
            pass
    return out


def _flop_roofline(stages, counters, p, args, fpk, hbm_note, pipe):
    """The dominant stage's FLOP roofline (FP64 pipe for the plain form, FP32
    for the mixed one) plus one per arithmetic stage."""
    peak = fpk.get(pipe)
    roofs = {}
    for st in ("pre", "force", "gravity"):
        fl = stage_flops(st, counters, p)
        ms, launches = stages.get(st, (0.0, 0))
        if fl is None or ms <= 0 or launches <= 0:
            continue
        per_step = launches / max(args.steps, 1)
        per_launch_ms = ms / launches if per_step <= 1.0 else ms / max(args.steps, 1)
        fl_launch = fl / max(args.steps, 1)
        ach = fl_launch / (per_launch_ms * 1e-3) / 1e12
        roofs[st] = {"achieved": round(ach, 3), "unit": "TFLOP/s", "peak": round(peak, 2) if peak else None,
                     "frac": round(ach / peak, 4) if peak else None, "flops_per_launch": fl_launch,
                     "launch_ms": round(per_launch_ms, 4)}
    if not roofs:
        return hbm_note, roofs
    dom = max(roofs, key=lambda k: stages[k][0])
    r = roofs[dom]
    out = {"kernel": dom, "bound": pipe, "achieved": r["achieved"], "peak": r["peak"], "unit": "TFLOP/s",
           "frac": r["frac"], "traffic": None,
           "peak_source": f"cuBLAS {'DGEMM' if pipe == 'fp64' else 'SGEMM (no TF32)'} 8192^3 measured in this run",
           "flops_per_launch": r["flops_per_launch"], "launch_ms": r["launch_ms"],
           "accounting": "device work counters x per-unit FLOP weights (flop_weights.md)"}
    tr = _traffic(args, dom)
    if tr:
        out["traffic"] = tr
    if hbm_note is not None:
        out["hbm"] = hbm_note
    return out, roofs


def _traffic(args, stage):
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if args.particles or not os.path.exists(prof):
        return None
    try:
        return json.load(open(prof)).get(args.workload, {}).get(stage)
    except (OSError, ValueError):
        return None


def _gpu_local_cpus(local: int):
    """CPUs on the GPU's own NUMA node (sysfs local_cpulist of its PCI device), or None."""
    try:
        import pynvml
        pynvml.nvmlInit()
        bus = pynvml.nvmlDeviceGetPciInfo(pynvml.nvmlDeviceGetHandleByIndex(local)).busId
        bus = (bus.decode() if isinstance(bus, bytes) else bus).lower()
        dom, rest = bus.split(":", 1)
        path = f"/sys/bus/pci/devices/{int(dom, 16):04x}:{rest}/local_cpulist"
        cpus = set()
        for part in open(path).read().strip().split(","):
            a, _, b = part.partition("-")
            cpus.update(range(int(a), int(b or a) + 1))
        return cpus & os.sched_getaffinity(0) or None
    except Exception:
        return None


def run_e2e(args, G, fields, world, wl):
    # pinned buffers and the copy loop on the GPU's own NUMA node (first-touch
    # placement of the host pages); the previous affinity is restored after
    saved = os.sched_getaffinity(0)
    local_cpus = _gpu_local_cpus(int(os.environ.get("LOCAL_RANK", "0")))
    if local_cpus:
        os.sched_setaffinity(0, local_cpus)
    try:
        return _run_e2e(args, G, fields, world, wl)
    finally:
        os.sched_setaffinity(0, saved)


def _run_e2e(args, G, fields, world, wl):
    import ctypes
    n = len(fields["pos_x"])
    p = wl.params(SP.FP64)
    sim = G.Simulation(p)
    if wl.learned:
        sim.load_riemann_mlp()
    sim.upload(fields)
    sim.initialize()
    host_in = _pinned(n, E2E_IN)
    host_out = _pinned(n, E2E_OUT)
    st = sim.download(E2E_IN)
    for f in E2E_IN:
        host_in[f].numpy()[:] = st[f]
    ptr_in = (ctypes.POINTER(ctypes.c_double) * G.NFIELDS)()
    ptr_out = (ctypes.POINTER(ctypes.c_double) * G.NFIELDS)()
    for f, t in host_in.items():
        ptr_in[G.FIELD_INDEX[f]] = ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))
    for f, t in host_out.items():
        ptr_out[G.FIELD_INDEX[f]] = ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))
    L = G.lib()

    phase = [0.0]   # host seconds in the step call

    def step():
        # one call: the step's inputs in from pinned host buffers, the step,
        # its results out (the downloads of fields final early in the step
        # overlap the rest of it)
        t0 = time.perf_counter()
        rc = L.sphgpu_integrate_host(sim._h, ptr_in, ptr_out)
        assert rc >= 0, sim._err()
        phase[0] += time.perf_counter() - t0

    for _ in range(max(1, args.warmup)):
        step()
    phase[:] = [0.0]
    barrier()
    L.sphgpu_timer_start(sim._h)
    for _ in range(args.steps):
        step()
    ms = ctypes.c_double()
    L.sphgpu_timer_stop(sim._h, ctypes.byref(ms))
    barrier()
    ms_max = max_over_ranks(ms.value)
    # the same copies without the step: what the host link gives on this box
    reps = 3
    L.sphgpu_timer_start(sim._h)
    for _ in range(reps):
        rc = L.sphgpu_upload(sim._h, n, ptr_in)
        assert rc >= 0, sim._err()
        rc = L.sphgpu_download(sim._h, ptr_out)
        assert rc >= 0, sim._err()
    cms = ctypes.c_double()
    L.sphgpu_timer_stop(sim._h, ctypes.byref(cms))
    sim.close()
    h2d, d2h = n * 8 * len(E2E_IN), n * 8 * len(E2E_OUT)
    copy_ms = cms.value / reps
    return {"value": whole_job_value(n * args.steps, world, ms_max), "unit": UNIT,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms_max / args.steps, "copy_ms_per_step": copy_ms,
            "copy_gbs": (h2d + d2h) / (copy_ms * 1e-3) / 1e9 if copy_ms > 0 else None,
            "api": "sphgpu_integrate_host",
            "host_ms_per_step": round(1e3 * phase[0] / max(args.steps, 1), 3)}


class _QuietStdout:
    """Send C-level stdout to stderr: the reference's Logger writes its
    Newton non-convergence notices to std::cout, and stdout must carry only
    the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def cpu_reference(steps: int, warmup: int, workload: str, n_target=None, budget_s: float = 0.0):
    """The reference's own OpenMP CPU build (oracle/_ref) on the workload."""
    with _QuietStdout():
        return _cpu_reference(steps, warmup, workload, n_target, budget_s)


def _cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return ""


def _cpu_reference(steps: int, warmup: int, workload: str, n_target, budget_s: float):
    """initialize (untimed), `warmup` untimed steps, then up to `steps` timed
    steps; with budget_s > 0 the timed steps stop once that much wall time
    has gone into them (at least one step runs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if O.have_reference():
        kind, cls = "reference", O.Reference
    else:
        kind, cls = "port", O.Oracle
    wl = WORKLOADS[workload]
    fields = wl.fields(n_target or wl.cpu_n)
    n = len(fields["pos_x"])
    p = wl.params(SP.FP64)
    p.riemann_guess = SP.GUESS_NONE   # the reference has no learned guess
    sim = cls(p, fields, threads=int(os.environ["OMP_NUM_THREADS"])) if kind == "reference" else cls(p, fields)
    t_init = time.perf_counter()
    sim.initialize()
    t_init = time.perf_counter() - t_init
    for _ in range(warmup):
        sim.integrate()
    done, el = 0, 0.0
    while done < steps:
        t0 = time.perf_counter()
        sim.integrate()
        el += time.perf_counter() - t0
        done += 1
        if budget_s > 0 and el >= budget_s:
            break
    return {"value": n * done / el, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
            "ms_per_step": 1e3 * el / done, "steps": done, "n": n,
            "sample": f"N={n}{' (the full workload)' if n >= wl.default_n * 0.99 else ' (a smaller lattice of the same workload)'}, "
                      f"initialize ({t_init:.1f} s, untimed) + {warmup} untimed + "
                      f"{done} timed steps ({el:.1f} s); host {_cpu_model()}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--particles", type=float, default=0.0,
                    help="workload size (default: the workload's own; profiling uses smaller cases)")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--forms", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="reference arm: wall seconds of timed CPU steps before it stops (at least one step)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_setup(args.gpus)
    wl = WORKLOADS[args.workload]

    if args.impl == "reference":
        if rank != 0:
            return
        n_target = args.particles or wl.default_n
        cb = cpu_reference(args.steps, 0, args.workload, n_target, args.ref_budget)
        n = cb["n"]
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": cb["steps"],
                "warmup": 0, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "device": "host cpu cores", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference", "config": bench_config(wl, n, args.gpus, args), "sample": cb["sample"],
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    out = run_gpu(args, rank, world, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            log("cpu baseline")
            # a bounded sample of the same workload: initialize + one step at
            # 1/16 of its size (the reference arm times it at full size)
            out["cpu_baseline"] = cpu_reference(1, 0, args.workload, max(wl.default_n / 16, 2e4), 0.0)
        print(json.dumps(out), flush=True)
    try:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
    except Exception:
        pass


if __name__ == "__main__":
    main()
