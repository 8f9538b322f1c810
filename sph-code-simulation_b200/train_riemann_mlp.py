"""Train the learned initial guess of the GSPH iterative Riemann solver.

    python sph-code-simulation_b200/train_riemann_mlp.py [--harvest 10e6] [--random 10e6]
        [--epochs 30] [--out sph-code-simulation_b200/riemann_mlp_weights.npy] [--report report.json]

1. Harvest pair states from the plain solver's own runs: the gsph shock
   tube (x in [-0.5, 0.5], y, z in [0, 0.05], p_L = 1000, p_R = 0.01,
   rho = 1, gamma = 1.4, cubic spline, neighborNumber = 50, second-order
   MUSCL, iterative solver) at about 2M particles; the FluidForce calls of
   several steps append hash-sampled pairs (sphgpu_harvest_begin / end).
2. Random states: log-uniform p ratio 1e-4..1e4, log-uniform rho ratio
   1e-3..1e3, velocity jump uniform in +-5 c_L, gamma in {1.4, 5/3}, drawn
   from a Philox stream seeded with 12345.
3. Labels: every state solved on the device to a relative change of 1e-13
   (sphgpu_riemann_batch mode 2); states whose solve did not converge or
   that open a vacuum (p_star < 1e-20 p_L) are dropped.
4. Training on the device with the project's tensor-core kernels
   (sphgpu_mlp_train, Adam, mean squared error in log(p_star / p_L)).
5. Evaluation on held-out states: Newton iterations of the reference's
   solver (mode 0), of the plain start taken to the learned path's 1e-10
   target (mode 3) and of the learned start (mode 1), fallback rate, p_star
   error against the labels.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import sphgpu as G  # noqa: E402

WEIGHTS = os.path.join(HERE, "riemann_mlp_weights.npy")


def random_states(n: int, seed: int = 12345) -> np.ndarray:
    rng = np.random.Generator(np.random.Philox(seed))
    g = np.where(rng.random(n) < 0.5, 1.4, 5.0 / 3.0)
    rR = 10.0 ** rng.uniform(-3, 3, n)
    pR = 10.0 ** rng.uniform(-4, 4, n)
    du = rng.uniform(-5, 5, n) * np.sqrt(g)
    return np.stack([np.zeros(n), np.ones(n), np.ones(n), du, rR, pR, g], axis=1)


def harvest(n_target: int, particles: float = 2.0e6, steps: int = 4) -> np.ndarray:
    dx = (0.05 * 0.05 / particles) ** (1.0 / 3.0)
    fields = G.sample_shock_tube(dx, ly=0.05)
    n = len(fields["pos_x"])
    p = G.config_params("tube_gsph")
    out = []
    with G.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        pairs = sim.counters()["max_pair"] * n  # upper bound on pair evaluations per step
        mod = max(1, int(pairs * steps / (2 * n_target)))
        for _ in range(steps):
            sim.harvest_begin(n_target, mod)
            sim.integrate()
            out.append(sim.harvest_end(n_target))
            if sum(len(o) for o in out) >= n_target:
                break
    rec = np.concatenate(out)[:n_target]
    return rec[:, :7]


def label(sim, states: np.ndarray, chunk: int = 4_000_000):
    ps, its = [], []
    for a in range(0, len(states), chunk):
        p, _, it, _ = sim.riemann_batch(states[a:a + chunk], mode=2)
        ps.append(p)
        its.append(it)
    p = np.concatenate(ps)
    it = np.concatenate(its)
    keep = (it < 100) & (p > 1e-20 * states[:, 2]) & np.isfinite(p)
    return p, keep


def evaluate(sim, states, p_ref):
    out = {}
    for mode, name in ((0, "plain_reference_tol1e-6"), (3, "plain_start_tol1e-10"), (1, "learned_start_tol1e-10")):
        t0 = time.perf_counter()
        p, _, it, fb = sim.riemann_batch(states, mode=mode)
        el = time.perf_counter() - t0
        rel = np.abs(p - p_ref) / p_ref
        out[name] = {"mean_iterations": float(it.mean()), "p99_iterations": float(np.quantile(it, 0.99)),
                     "fallback_rate": float(fb.mean()), "median_rel_err": float(np.median(rel)),
                     "p99_rel_err": float(np.quantile(rel, 0.99)), "max_rel_err": float(rel.max()),
                     "host_call_s": el}
        if mode == 1:
            # learned path cost: iterations + the plain solver's after a fallback
            out[name]["mean_iterations_incl_fallback"] = float(it.mean())
    y = sim.mlp_predict(states)
    dy = np.abs(y - np.log(p_ref / states[:, 2]))
    out["guess_abs_err_log_p"] = {"median": float(np.median(dy)), "p90": float(np.quantile(dy, 0.9)),
                                  "p99": float(np.quantile(dy, 0.99))}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harvest", type=float, default=10e6)
    ap.add_argument("--random", type=float, default=10e6)
    ap.add_argument("--particles", type=float, default=2.0e6)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    t0 = time.perf_counter()
    hv = harvest(int(a.harvest), a.particles) if a.harvest > 0 else np.zeros((0, 7))
    t1 = time.perf_counter()
    rnd = random_states(int(a.random), 12345)
    p = G.config_params("tube_gsph")
    with G.Simulation(p) as sim:
        p_h, k_h = label(sim, hv) if len(hv) else (np.zeros(0), np.zeros(0, bool))
        p_r, k_r = label(sim, rnd)
        t2 = time.perf_counter()
        rng = np.random.default_rng(1)
        # hold out 2 % of each source for evaluation
        def split(x, pp, keep):
            x, pp = x[keep], pp[keep]
            idx = rng.permutation(len(x))
            cut = max(1, len(x) // 50)
            return x[idx[cut:]], pp[idx[cut:]], x[idx[:cut]], pp[idx[:cut]]
        tr_h, pt_h, va_h, pv_h = split(hv, p_h, k_h) if len(hv) else (hv, p_h, hv, p_h)
        tr_r, pt_r, va_r, pv_r = split(rnd, p_r, k_r)
        x_tr = np.concatenate([tr_h, tr_r])
        p_tr = np.concatenate([pt_h, pt_r])
        sim.mlp_init(12345)
        hist = sim.mlp_train(x_tr, p_tr, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=12345)
        # a short low-learning-rate polish
        hist2 = sim.mlp_train(x_tr, p_tr, epochs=max(1, a.epochs // 5), batch=a.batch, lr=a.lr * 0.1,
                              seed=54321)
        t3 = time.perf_counter()
        params = sim.mlp_get_params()
        report = {
            "harvested": int(len(hv)), "harvested_kept": int(k_h.sum()), "random": int(len(rnd)),
            "random_kept": int(k_r.sum()), "train_rows": int(len(x_tr)),
            "loss_history": [float(v) for v in hist] + [float(v) for v in hist2],
            "seconds": {"harvest": t1 - t0, "label": t2 - t1, "train": t3 - t2},
            "eval_harvested": evaluate(sim, va_h, pv_h) if len(va_h) else None,
            "eval_random": evaluate(sim, va_r, pv_r),
        }
    np.save(a.out, params.astype(np.float32))
    js = json.dumps(report, indent=1)
    print(js)
    if a.report:
        with open(a.report, "w") as f:
            f.write(js)


if __name__ == "__main__":
    main()
