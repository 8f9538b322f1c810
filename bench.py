"""Benchmark: particle-steps/s of the SPH step on B200.

Workload (one GPU): the density-independent SPH periodic shear layer —
box [0,1] x [0,1] x [0,0.125], N = 1,016,400 particles, Wendland C4,
neighborNumber = 128, artificial conductivity on, gamma = 5/3, seeded
synthetic lattice initial conditions (no dataset involved).  A step is one
Solver::integrate (timestep, predict, tree build, PreInteraction, FluidForce,
GravityForce (off here), correct) over all particles.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the plain FP64 form (the drop-in), timed with CUDA events on the
context stream with inputs resident in HBM; `mixed` reports the FP32 form on
the same workload; `e2e` is the same metric through the C ABI with the
particle state copied host -> device and back every step (pinned buffers).
Multi-GPU: replicas only (each rank integrates its own copy; no data-path
collective); the timed region is bracketed by barriers and the max over ranks
is reported.  `--impl reference` times the reference's own OpenMP CPU build
(oracle/_ref) on a bounded sample of the same workload.
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

METRIC = "particle-steps/s on 1 B200: FP64 plain vs FP32+learned-Riemann at ≤1e-5 rel err"
UNIT = "particle-steps/s"


class Workload:
    """One benchmark workload: parameters, initial conditions at a target size,
    and a smaller CPU sample of the same workload for the reference arm."""

    def __init__(self, name, desc, cfg, sample, default_n, cpu_n, learned=False, **overrides):
        self.name, self.desc, self.cfg, self.sample = name, desc, cfg, sample
        self.default_n, self.cpu_n, self.learned, self.overrides = default_n, cpu_n, learned, overrides

    def params(self, G, precision):
        p = G.config_params(self.cfg, precision=precision, **self.overrides)
        if self.learned:
            p.riemann_guess = G.GUESS_MLP
        return p

    def fields(self, G, n):
        return self.sample(G, n)


def _evrard(G, n):
    lattice = max(8, int(round((n * 6.0 / 3.14159265) ** (1.0 / 3.0))))
    return G.sample_evrard(lattice)


def _shear(G, n):
    return G.sample_shear_layer((0.1875 / n) ** (1.0 / 3.0))


def _tube(G, n):
    return G.sample_shock_tube((0.05 * 0.05 / n) ** (1.0 / 3.0), ly=0.05)


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
    # The reference's algorithm (bit-exact oracle) turns non-finite near the
    # sphere's centre at t ~ 0.003-0.004 on this resolution whatever the CFL;
    # cflSound 0.05 / cflForce 0.025 keep 3 warm-up + 10 timed steps finite.
    "evrard_disph": Workload("evrard_disph", "disph + BH gravity sphere 8.8M (Wendland C4, K=128, TD-AV, AC; "
                             "CFL 0.05/0.025)", "evrard_disph", _evrard, 8.78e6, 6.5e4, cfl_sound=0.05,
                             cfl_force=0.025),
}
DEFAULT_WORKLOAD = "shear_disph"

# fields a step reads from / writes back to the caller in the e2e leg
E2E_IN = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "mass", "dens",
          "pres", "ene", "dene", "sml", "sound", "balsara", "alpha", "gradh"]
E2E_OUT = E2E_IN + ["phi", "neighbor"]

# algorithmic bytes per unit: each node's link + geo (+ ksize for the symmetric
# walk) and each particle's position read once, each list entry written once
NODE_BYTES = 16 + 32          # link (int4) + geo (double4) read per node
PAIR_WALK_NODE_BYTES = NODE_BYTES + 8


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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
    fields = wl.fields(G, args.particles or wl.default_n)
    n = len(fields["pos_x"])
    hbm, peak_kind = _peaks()

    def timed(precision):
        log(f"{wl.name} n={n} precision={precision}: initialize")
        p = wl.params(G, precision)
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
        clocks = ClockSampler(local) if (rank == 0 and precision == G.FP64 and not args.no_clocks) else None
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
        return sim, ms.value, clk, launches, stages, counters

    first = G.MIXED if args.forms == "mixed" else G.FP64
    sim, ms, clk, launches, stages, counters = timed(first)
    ms_max = max_over_ranks(ms)
    value = whole_job_value(n * args.steps, world, ms_max)

    # roofline for the dominant kernel (its stage = one launch per step)
    dom = max(stages.items(), key=lambda kv: kv[1][0])[0]
    dom_ms, dom_launches = stages[dom]
    per_launch_ms = dom_ms / max(dom_launches, 1)
    nodes = counters["node_count"]
    algo = None
    if dom in ("gather_walk", "pair_walk"):
        # exact list lengths of the last walk of that kind
        off, _ = sim.neighbor_search(is_ij=(dom == "pair_walk"))
        entries = float(off[-1])
        nb = NODE_BYTES if dom == "gather_walk" else PAIR_WALK_NODE_BYTES
        algo = nodes * nb + n * 32 + entries * 4 + n * 4
        unit_note = "node table + positions read once, list entries written once"
    elif dom == "pre":
        off, _ = sim.neighbor_search(is_ij=False)
        entries = float(off[-1])
        algo = entries * 4 + n * (96 + 72)
        unit_note = "gather list + particle state read once, outputs written once"
    elif dom == "force":
        off, _ = sim.neighbor_search(is_ij=True)
        entries = float(off[-1])
        algo = entries * 4 + n * (128 + 32)
        unit_note = "pair list + particle state read once, acc written once"
    else:
        algo = n * 64.0
        unit_note = "particle state read and written once"
    # a stage of several launches per step (the learned force: force pass,
    # network, row sort, completion) is charged as one pass over its bytes in
    # the stage's time per step, not per launch
    per_step = dom_launches / max(args.steps, 1)
    if per_step > 1.0:
        per_launch_ms = dom_ms / max(args.steps, 1)
        unit_note += f"; stage of {per_step:.0f} launches per step, timed as one"
    achieved = algo / (per_launch_ms / 1e3) / 1e9
    roofline = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": None, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": algo, "launch_ms": round(per_launch_ms, 4),
                "accounting": unit_note}
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof) and not args.particles:
        try:
            tr = json.load(open(prof)).get(args.workload, {}).get(dom)
            if tr:
                roofline["traffic"] = tr
        except (OSError, ValueError):
            pass
    sim.close()

    # mixed precision form on the same workload
    mixed = None
    if args.forms == "both":
        msim, mms, _, _, mstages, _ = timed(G.MIXED)
        mms_max = max_over_ranks(mms)
        mixed = {"value": whole_job_value(n * args.steps, world, mms_max), "ms_per_step": mms_max / args.steps,
                 "dtype": "f32 pair/gravity, f64 accumulators and kick-drift",
                 "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in mstages.items()}}
        msim.close()

    log("end to end")
    # end to end through the C ABI with host buffers
    e2e = None if args.no_e2e else run_e2e(args, G, fields, world, wl)

    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if first == G.FP64 else "f32/f64",
        "data": "synthetic",
        "config": {"workload": wl.desc if not args.particles else f"{wl.desc} at N={n}", "n_particles": n,
                   "particles_per_gpu": n, "form": "fp64 plain" if first == G.FP64 else "mixed",
                   "l2": "inputs larger than L2 (state + neighbour lists ~3 GB per step)",
                   "parallelism": f"replicas x{world}"},
        "mixed": mixed, "e2e": e2e, "gpu_launches": launches,
        "stages_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in stages.items()},
        "counters": counters, "roofline": roofline, "clocks": clk,
    }


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
    p = wl.params(G, G.FP64)
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

    phase = [0.0, 0.0, 0.0]   # host seconds: upload, integrate, download

    def step():
        t0 = time.perf_counter()
        rc = L.sphgpu_upload(sim._h, n, ptr_in)
        assert rc >= 0, sim._err()
        t1 = time.perf_counter()
        L.sphgpu_set_initial_smoothing(sim._h, 0)
        rc = L.sphgpu_integrate(sim._h)
        assert rc >= 0, sim._err()
        t2 = time.perf_counter()
        rc = L.sphgpu_download(sim._h, ptr_out)
        assert rc >= 0, sim._err()
        t3 = time.perf_counter()
        phase[0] += t1 - t0
        phase[1] += t2 - t1
        phase[2] += t3 - t2

    for _ in range(max(1, args.warmup)):
        step()
    phase[:] = [0.0, 0.0, 0.0]
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
            "host_ms_per_step": {k: round(1e3 * v / max(args.steps, 1), 3)
                                 for k, v in zip(("upload", "integrate", "download"), phase)}}


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


def cpu_reference(steps: int, warmup: int, workload: str):
    """The reference's own OpenMP CPU build (oracle/_ref) on a bounded sample."""
    with _QuietStdout():
        return _cpu_reference(steps, warmup, workload)


def _cpu_reference(steps: int, warmup: int, workload: str):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import sphgpu as G
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if O.have_reference():
        kind, cls = "reference", O.Reference
    else:
        kind, cls = "port", O.Oracle
    wl = WORKLOADS[workload]
    fields = wl.fields(G, wl.cpu_n)
    n = len(fields["pos_x"])
    p = wl.params(G, G.FP64)
    p.riemann_guess = G.GUESS_NONE   # the reference has no learned guess
    sim = cls(p, fields, threads=int(os.environ["OMP_NUM_THREADS"])) if kind == "reference" else cls(p, fields)
    sim.initialize()
    for _ in range(warmup):
        sim.integrate()
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.integrate()
    el = time.perf_counter() - t0
    cpu_model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                cpu_model = ln.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": n * steps / el, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
            "ms_per_step": 1e3 * el / steps,
            "sample": f"same workload at N={n}, initialize + {warmup} untimed + {steps} timed steps,"
                      f" {el:.2f} s; host {cpu_model}"}


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
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_setup(args.gpus)

    if args.impl == "reference":
        if rank != 0:
            return
        ref_steps = max(1, min(args.steps, 8))
        cb = cpu_reference(ref_steps, 1, args.workload)
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": ref_steps,
                "warmup": 1, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "device": "host cpu cores",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOADS[args.workload].desc, "sample": cb["sample"]},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    out = run_gpu(args, rank, world, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            log("cpu baseline")
            out["cpu_baseline"] = cpu_reference(2, 1, args.workload)
        print(json.dumps(out), flush=True)
    try:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
    except Exception:
        pass


if __name__ == "__main__":
    main()
