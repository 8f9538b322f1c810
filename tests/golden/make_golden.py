"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container where the reference sources are mounted (default
a "reference" directory beside the repository, override with REFDIR) after
`make -C oracle`:

    python tests/golden/make_golden.py

What it writes (all produced by the reference's own compiled modules,
oracle/_ref/libsphref*.so, driven by oracle/ref_harness.cpp):

  evrard_t0.npz      The reference's shipped Evrard t=0 snapshot
                     (sample/evrard/results_new/00000.dat, energy.dat row t=0;
                     configuration sample/evrard/evrard.json: N=30 lattice,
                     ssph, Wendland, neighborNumber=32, leafParticleNumber=32,
                     Balsara + time-dependent AV, G=1).  The script recomputes
                     it with the compiled reference and asserts agreement to the
                     printed 6 digits, then stores every 16th particle's printed
                     row, the recomputed full-precision values for the same
                     particles, and W0.
  evrard_energy.json The rows of the reference's shipped
                     sample/evrard/results_new/energy.dat (time, kinetic,
                     thermal, potential, total; same configuration as
                     evrard_t0).  An older build of the reference wrote them,
                     so later rows bound a run (~1e-2), they do not pin it.
  steps_<cfg>.npz    Small instances of the benchmark workloads (and of the
                     gdisph shock tube, first and second order, and of the
                     ssph Evrard sphere with the Gaussian kernel): the
                     full particle state after Solver::initialize and after
                     each of two Solver::integrate steps, plus dt.
  csv_snapshots.npz  Lines of two CSV v1 snapshots the reference ships
                     (sample/sr_sod/results_coarse/snapshot_0000.csv: header
                     and its first 64 particle rows; test/checkpoint_csv_resume/
                     snapshot_0001.csv: header only), the byte-level check of
                     the CSV writer.
  relax_evrard.npz   Three steps of the reference's Lane-Emden relaxation loop
                     on the ssph Evrard sample (N=12 lattice, alpha = 0.3,
                     K = 0.5), with the reference's table
                     data/lane_emden/n1.5_3d.dat (xi, theta, dtheta, xi_1):
                     states after each step and dt_relax.
  sr_tube.npz        SRGSPH (src/srgsph/*.cpp) on a 3-D special-relativistic
                     Sod tube: states after Solver::initialize, after one
                     predict and one correct with a small fixed dt, and the
                     error a full integrate step stops with (the reference's
                     exact SR Riemann solver returns spurious star pressures
                     for nearly equal states, and the primitive recovery then
                     fails), for first / second order and fixed / iterative h.
  steps_edge_<cfg>.npz
                     Edge cases, same layout as steps_<cfg> plus the OpenMP
                     team size the reference ran with: an Evrard sphere moved
                     off the origin (the non-periodic root box covers the
                     origin with more than one thread, not with one:
                     tree_root_origin 1 / 0), three pairs of coincident
                     particles with different energies (r = 0 pairs), and
                     1, 2 and 7 particles (smoothing-length Newton without
                     convergence, a root of one particle).
  sweep_hashes.json  SHA-256 of the reference's full particle state after
                     initialize and each of two integrate steps, plus dt and
                     K, U, W, and of its distance-sorted gather and symmetric
                     lists after initialize, for
                     56 small configurations: ssph / disph / gsph / gdisph x
                     cubic / Wendland / Gaussian x leaf 1 / leaf 4 / tree level
                     cap 3 on an off-origin sphere with gravity, TD-AV and AC;
                     and a periodic shear layer with particles on the box
                     faces and one coincident pair, iterative and fixed h,
                     Balsara off, first-order gsph with the iterative solver.
                     Inputs are rebuilt from the sweep_* functions below.
  evrard_disph_8.78M_reference.json
                     The full 256^3 disph Evrard sphere (8,783,848 particles)
                     at cflSound 0.05 / cflForce 0.025, step by step until the
                     reference's own state turns non-finite: dt, time, K, U, W,
                     the smallest u, and the first bad particles' ids
                     (`python tests/golden/make_golden.py evrard_big`, slow).
  lists_<cfg>.npz    Distance-sorted neighbour lists (CSR) from
                     BHTree::neighbor_search and from exhaustive_search
                     (gather and is_ij) at the state after initialize.
"""
from __future__ import annotations

import itertools
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "sph-code-simulation_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
import sphgpu as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: REFDIR, else a "reference" directory beside the repository
REFDIR = os.environ.get("REFDIR") or os.path.normpath(os.path.join(ROOT, os.pardir, "reference"))

STATE_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "mass",
                "dens", "pres", "ene", "dene", "sml", "sound", "balsara", "alpha", "gradh", "phi", "neighbor",
                "velp_x", "velp_y", "velp_z", "ene_p",
                "grad_d_x", "grad_d_y", "grad_d_z", "grad_p_x", "grad_p_y", "grad_p_z",
                "grad_v0_x", "grad_v0_y", "grad_v0_z", "grad_v1_x", "grad_v1_y", "grad_v1_z",
                "grad_v2_x", "grad_v2_y", "grad_v2_z"]

# small instances of the benchmark workloads (name, params, sample)
SMALL = {
    "evrard_ssph": (lambda: G.config_params("evrard_ssph"), lambda: G.sample_evrard(12)),
    "evrard_disph": (lambda: G.config_params("evrard_disph", neighbor_number=64),
                     lambda: G.sample_evrard(12)),
    "tube_gsph": (lambda: G.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                  lambda: G.sample_shock_tube(0.025, ly=0.1)),
    "tube_gsph_hll": (lambda: G.config_params("tube_gsph", riemann_solver=G.RIEMANN_HLL,
                                              range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                      lambda: G.sample_shock_tube(0.025, ly=0.1)),
    "shear_disph": (lambda: G.config_params("shear_disph", neighbor_number=64),
                    lambda: G.sample_shear_layer(0.05, lz=0.125)),
    "tube_gdisph": (lambda: G.config_params("tube_gdisph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                    lambda: G.sample_shock_tube(0.025, ly=0.1)),
    "evrard_ssph_gauss": (lambda: G.config_params("evrard_ssph", kernel=G.GAUSSIAN), lambda: G.sample_evrard(12)),
    "tube_gdisph_1st": (lambda: G.config_params("tube_gdisph", gsph_2nd_order=0, use_balsara_switch=0,
                                                range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                        lambda: G.sample_shock_tube(0.025, ly=0.1)),
}


def evrard_energy_golden():
    import json
    rows = np.loadtxt(os.path.join(REFDIR, "sample/evrard/results_new/energy.dat"), comments="#")
    with open(os.path.join(OUT, "evrard_energy.json"), "w") as f:
        json.dump({"columns": ["time", "kinetic", "thermal", "potential", "total"],
                   "rows": [[float(x) for x in r] for r in rows]}, f, indent=1)
    print(f"evrard_energy: {len(rows)} rows")


def _edge_shifted(sph, shift=(1.7, -0.4, 2.3), **kw):
    fields = G.sample_evrard(8)
    for k, s in zip(("pos_x", "pos_y", "pos_z"), shift):
        fields[k] = fields[k] + s
    return G.config_params(sph, **kw), fields


def _edge_coincident():
    """Three particles moved onto three others; the moved ones get 1.7x the
    energy, so the coincident pairs differ in pressure and sound speed."""
    fields = G.sample_evrard(8)
    rng = np.random.default_rng(7)
    src = rng.choice(len(fields["pos_x"]), 6, replace=False)
    for a, b in zip(src[:3], src[3:]):
        for k in ("pos_x", "pos_y", "pos_z"):
            fields[k][b] = fields[k][a]
        fields["ene"][b] = fields["ene"][a] * 1.7
    return G.config_params("evrard_ssph"), fields


def _edge_tiny(n, sph):
    fields = G.sample_evrard(8)
    idx = np.random.default_rng(11).choice(len(fields["pos_x"]), n, replace=False)
    return G.config_params(sph), {k: v[idx].copy() for k, v in fields.items()}


# name -> (params and fields, tree_root_origin, reference OpenMP threads)
EDGE = {
    "shifted_ssph": (lambda: _edge_shifted("evrard_ssph"), 1, 8),
    "shifted_ssph_1t": (lambda: _edge_shifted("evrard_ssph"), 0, 1),
    "shifted_disph": (lambda: _edge_shifted("evrard_disph", neighbor_number=32), 1, 8),
    "coincident_ssph": (_edge_coincident, 1, 8),
    "tiny1_ssph": (lambda: _edge_tiny(1, "evrard_ssph"), 1, 8),
    "tiny2_ssph": (lambda: _edge_tiny(2, "evrard_ssph"), 1, 8),
    "tiny7_disph": (lambda: _edge_tiny(7, "evrard_disph"), 1, 8),
}


def sweep_state_hash(st):
    import hashlib
    h = hashlib.sha256()
    for f in STATE_FIELDS:
        h.update(np.ascontiguousarray(st[f], dtype=np.float64).tobytes())
    return h.hexdigest()


def _sweep_sphere():
    fields = G.sample_evrard(8)
    for k, d in zip(("pos_x", "pos_y", "pos_z"), (1.7, -0.4, 2.3)):
        fields[k] = fields[k] + d
    return fields


def _sweep_layer(iterative):
    fields = G.sample_shear_layer(0.1, lz=0.125)
    n = len(fields["pos_x"])
    idx = np.random.default_rng(3).choice(n, 8, replace=False)
    fields["pos_x"][idx[:2]] = 0.0                        # on rangeMin
    fields["pos_y"][idx[2:4]] = 1.0 - 1e-15               # just below rangeMax
    fields["pos_z"][idx[4:6]] = 0.125 * (1 - 2 ** -52)
    for k in ("pos_x", "pos_y", "pos_z"):
        fields[k][idx[6]] = fields[k][idx[7]]             # a coincident pair
    if not iterative:
        fields["sml"] = np.full(n, 0.25)
    return fields


def sweep_cases():
    """name -> (params, fields builder)."""
    out = {}
    types = (("ssph", G.SSPH), ("disph", G.DISPH), ("gsph", G.GSPH), ("gdisph", G.GDISPH))
    for (sph, st), (kern, kn), (leaf, lvl) in itertools.product(
            types, (("cubic", G.CUBIC_SPLINE), ("wendland", G.WENDLAND), ("gauss", G.GAUSSIAN)),
            ((1, 20), (4, 20), (1, 3))):
        p = G.default_params(sph_type=st, kernel=kn, neighbor_number=32, use_gravity=1, g_constant=1.0,
                             leaf_particle_num=leaf, max_tree_level=lvl, use_time_dependent_av=1, use_ac=1,
                             riemann_solver=G.RIEMANN_HLL, gamma=5.0 / 3.0)
        out[f"sphere_{sph}_{kern}_leaf{leaf}_lvl{lvl}"] = (p, _sweep_sphere)
    variants = (("plain", {}), ("tdav", {"use_balsara_switch": 0, "use_time_dependent_av": 1}),
                ("first_iter", {"gsph_2nd_order": 0, "riemann_solver": G.RIEMANN_ITERATIVE}))
    for (sph, st), it, (tag, extra) in itertools.product(types, (1, 0), variants):
        if tag == "first_iter" and st not in (G.GSPH, G.GDISPH):
            continue
        p = G.default_params(sph_type=st, kernel=G.WENDLAND, neighbor_number=32, periodic=1,
                             range_min=(0.0, 0.0, 0.0), range_max=(1.0, 1.0, 0.125), use_ac=1,
                             iterative_sml=it, gamma=5.0 / 3.0, **extra)
        out[f"layer_{sph}_it{it}_{tag}"] = (p, (lambda it=it: _sweep_layer(it)))
    return out


def sweep_lists_hash(sim):
    """SHA-256 of the distance-sorted gather and symmetric lists (CSR)."""
    import hashlib
    out = []
    for ij in (False, True):
        off, ids = sim.neighbor_lists(ij)
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(off, dtype=np.int64).tobytes())
        h.update(np.ascontiguousarray(ids, dtype=np.int32).tobytes())
        out.append(h.hexdigest())
    return out


def sweep_golden(steps=2, threads=8):
    import json
    rows = []
    for name, (p, mk) in sweep_cases().items():
        ref = O.Reference(p, mk(), threads=threads)
        ref.initialize()
        hashes, dts = [sweep_state_hash(ref.download(STATE_FIELDS))], [0.0]
        lists = sweep_lists_hash(ref)
        energies = [list(ref.energies()[:3])]
        for _ in range(steps):
            ref.integrate()
            hashes.append(sweep_state_hash(ref.download(STATE_FIELDS)))
            dts.append(ref.dt)
            energies.append(list(ref.energies()[:3]))
        rows.append({"name": name, "params": bytes(p).hex(), "threads": threads, "hashes": hashes, "dt": dts,
                     "lists": lists, "energies": energies})
    with open(os.path.join(OUT, "sweep_hashes.json"), "w") as f:
        json.dump(rows, f, indent=1)
    print(f"sweep_hashes: {len(rows)} configurations")


def edge_steps(name, steps=2):
    mk, origin, threads = EDGE[name]
    p, fields = mk()
    p.tree_root_origin = origin
    ref = O.Reference(p, fields, threads=threads)
    ref.initialize()
    states = [ref.download(STATE_FIELDS)]
    dts = [0.0]
    for _ in range(steps):
        ref.integrate()
        states.append(ref.download(STATE_FIELDS))
        dts.append(ref.dt)
    out = {"n": len(fields["pos_x"]), "dt": np.array(dts), "params": np.frombuffer(bytes(p), dtype=np.uint8),
           "threads": threads}
    for k in ("pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "mass", "dens", "pres", "ene"):
        out["ic_" + k] = fields[k]
    for s, st in enumerate(states):
        for f, v in st.items():
            out[f"s{s}_{f}"] = v
    np.savez_compressed(os.path.join(OUT, f"steps_edge_{name}.npz"), **out)
    print(f"steps_edge_{name}: n={out['n']} threads={threads} dt={dts}")


def evrard_golden():
    p = G.default_params(sph_type=G.SSPH, kernel=G.WENDLAND, neighbor_number=32, leaf_particle_num=32,
                         use_balsara_switch=1, use_time_dependent_av=1, av_alpha=1.0, use_ac=0,
                         use_gravity=1, g_constant=1.0, gamma=1.66666666666666666667, cfl_sound=0.2,
                         cfl_force=0.1)
    fields = G.sample_evrard(30)
    ref = O.Reference(p, fields)
    ref.initialize()
    st = ref.download()
    k, u, w, _ = ref.energies()
    shipped = np.loadtxt(os.path.join(REFDIR, "sample/evrard/results_new/00000.dat"), comments="#")
    ids = shipped[:, 14].astype(int)
    order = np.argsort(ids)
    shipped = shipped[order]
    assert len(shipped) == len(fields["pos_x"]) == 14328
    cols = {"pos_x": 0, "pos_y": 1, "pos_z": 2, "acc_x": 6, "acc_y": 7, "acc_z": 8, "mass": 9, "dens": 10,
            "pres": 11, "ene": 12, "sml": 13, "neighbor": 15, "alpha": 16, "gradh": 17}
    worst = 0.0
    for f, c in cols.items():
        ref_v = st[f]
        printed = shipped[:, c]
        rel = np.abs(ref_v - printed) / np.maximum(np.abs(printed), 1e-300)
        # 6 significant digits printed; tiny components compared absolutely
        tol = 6e-6 * np.maximum(np.abs(printed), 1e-6 * np.max(np.abs(printed)))
        bad = np.abs(ref_v - printed) > tol
        assert not bad.any(), (f, np.flatnonzero(bad)[:5])
        worst = max(worst, float(np.max(rel[np.abs(printed) > 1e-3 * np.max(np.abs(printed))])))
    energy = np.loadtxt(os.path.join(REFDIR, "sample/evrard/results_new/energy.dat"), comments="#")
    w0_printed = energy[0, 3]
    assert abs(w - w0_printed) < 1e-6, (w, w0_printed)
    sel = np.arange(0, len(shipped), 16)
    np.savez_compressed(
        os.path.join(OUT, "evrard_t0.npz"),
        ids=sel,
        printed=shipped[sel],
        printed_columns=np.array(list(cols.keys())),
        printed_index=np.array(list(cols.values())),
        **{"ref_" + f: st[f][sel] for f in cols},
        ref_phi=st["phi"][sel],
        w0_printed=w0_printed,
        w0_ref=w,
        k0_ref=k,
        u0_ref=u,
    )
    print(f"evrard_t0: 14328 particles match 00000.dat to 6 digits (worst rel {worst:.2e}); W0 {w:.9f}")


def small_steps(name, steps=2):
    mkp, mks = SMALL[name]
    p = mkp()
    fields = mks()
    ref = O.Reference(p, fields)
    ref.initialize()
    states = [ref.download(STATE_FIELDS)]
    dts = [0.0]
    for _ in range(steps):
        ref.integrate()
        states.append(ref.download(STATE_FIELDS))
        dts.append(ref.dt)
    out = {"n": len(fields["pos_x"]), "dt": np.array(dts), "params": np.frombuffer(bytes(p), dtype=np.uint8)}
    for k in ("pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "mass", "dens", "pres", "ene"):
        out["ic_" + k] = fields[k]
    for s, st in enumerate(states):
        for f, v in st.items():
            out[f"s{s}_{f}"] = v
    np.savez_compressed(os.path.join(OUT, f"steps_{name}.npz"), **out)
    print(f"steps_{name}: n={out['n']} dt={dts}")
    return p, fields


def lists(name):
    mkp, mks = SMALL[name]
    p = mkp()
    fields = mks()
    out = {}
    for exh in (False, True):
        ref = O.Reference(p, fields, exhaustive=exh)
        ref.initialize()
        st = ref.download(STATE_FIELDS)
        tag = "exh" if exh else "tree"
        for is_ij in (0, 1):
            off, ids = ref.neighbor_lists(bool(is_ij))
            out[f"{tag}_ij{is_ij}_off"] = off
            out[f"{tag}_ij{is_ij}_ids"] = ids
        if not exh:
            for f, v in st.items():
                out["state_" + f] = v
    np.savez_compressed(os.path.join(OUT, f"lists_{name}.npz"), **out)
    print(f"lists_{name}: {len(out['tree_ij0_ids'])} gather / {len(out['tree_ij1_ids'])} pair entries")


def csv_golden():
    out = {}
    for tag, rel, rows in (("sr_sod", "sample/sr_sod/results_coarse/snapshot_0000.csv", 64),
                           ("resume", "test/checkpoint_csv_resume/snapshot_0001.csv", 0)):
        with open(os.path.join(REFDIR, rel)) as f:
            lines = f.read().split("\n")
        out[tag] = np.array(lines[:51 + rows])
    np.savez_compressed(os.path.join(OUT, "csv_snapshots.npz"), **out)
    print("csv_snapshots:", {k: len(v) for k, v in out.items()})


RELAX_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "dens", "pres",
                "sml", "sound", "phi"]


def relax_golden(steps=3, alpha=0.3, K=0.5):
    path = os.path.join(REFDIR, "data/lane_emden/n1.5_3d.dat")
    tab = np.loadtxt(path, comments="#")
    xi_1 = None
    with open(path) as f:
        for ln in f:
            if ln.startswith("# xi_1"):
                xi_1 = float(ln.split("=")[1])
    p = G.config_params("evrard_ssph")
    fields = G.sample_evrard(12)
    ref = O.Reference(p, fields)
    out = {"params": np.frombuffer(bytes(p), dtype=np.uint8), "xi": tab[:, 0], "theta": tab[:, 1],
           "dtheta": tab[:, 2], "xi_1": xi_1, "alpha": alpha, "K": K}
    for k in ("pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "mass", "dens", "pres", "ene"):
        out["ic_" + k] = fields[k]
    dts = []
    for s in range(steps):
        dts.append(ref.relax_step(REFDIR, alpha, 1.0, K, 1.0, 1.0))
        st = ref.download(RELAX_FIELDS)
        for f, v in st.items():
            out[f"s{s}_{f}"] = v
    out["dt_relax"] = np.array(dts)
    np.savez_compressed(os.path.join(OUT, "relax_evrard.npz"), **out)
    print("relax_evrard: dt_relax", dts)


SR_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "velp_x", "velp_y", "velp_z", "dens", "pres",
             "ene", "ene_p", "sml", "sound", "grad_d_x", "grad_d_y", "grad_d_z", "grad_p_x", "grad_p_y", "grad_p_z",
             "grad_v0_x", "grad_v0_y", "grad_v0_z", "grad_v1_x", "grad_v1_y", "grad_v1_z", "grad_v2_x", "grad_v2_y",
             "grad_v2_z", "sr_S_x", "sr_S_y", "sr_S_z", "sr_e", "sr_N", "sr_nu", "sr_gamma_lor", "sr_enthalpy",
             "sr_dS_x", "sr_dS_y", "sr_dS_z", "sr_de"]


def sr_golden():
    """SRGSPH on a 3-D special-relativistic Sod tube (dx = 0.025, 360 particles,
    eta = 2.3, first / second order, fixed / iterative smoothing length): the
    state after Solver::initialize, after Solver::predict and Solver::correct
    with a dt of 1e-6 e_min / max|rate| (so every primitive recovery
    converges), and the error a full Solver::integrate stops with."""
    out = {}
    for order in (0, 1):
        for it in (0, 1):
            tag = f"o{order}i{it}"
            p = G.config_params("tube_srgsph", sr_2nd_order=order, iterative_sml=it, sr_eta=2.3,
                                range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1))
            fields = G.sample_sr_shock_tube(0.025, ly=0.1)
            ref = O.Reference(p, fields)
            ref.initialize()
            s0 = ref.download(SR_FIELDS)
            big = max(np.abs(s0[k]).max() for k in ("sr_dS_x", "sr_dS_y", "sr_dS_z", "sr_de"))
            dt = 1e-6 * s0["sr_e"].min() / big
            ref.set_dt(dt)
            ref.predict()
            s1 = ref.download(SR_FIELDS)
            ref.correct()
            s2 = ref.download(SR_FIELDS)
            ref2 = O.Reference(p, fields)
            ref2.initialize()
            try:
                ref2.integrate()
                msg = ""
            except RuntimeError as e:
                msg = str(e).split("failed: ", 1)[-1]
            out[tag + "_params"] = np.frombuffer(bytes(p), dtype=np.uint8)
            out[tag + "_dt"] = dt
            out[tag + "_integrate_error"] = msg
            for k, st in enumerate((s0, s1, s2)):
                for f, v in st.items():
                    out[f"{tag}_s{k}_{f}"] = v
            print(f"sr_tube {tag}: dt_check {dt:.3e}; integrate: {msg or 'ok'}")
    fields = G.sample_sr_shock_tube(0.025, ly=0.1)
    for f in ("pos_x", "pos_y", "pos_z", "mass", "dens", "pres", "ene", "sr_e", "sr_N", "sr_nu", "sr_gamma_lor"):
        out["ic_" + f] = fields[f]
    # FluidForce alone on a prescribed two-state tube, where every Riemann
    # problem is well posed: equal states inside each half (exact star state
    # at the first iterate) and a Sod-size jump across the interface (n 1 /
    # 0.125, P 1 / 0.08, so |log10 P_i/P_j| > cContactDiscontinuity and the
    # second-order path falls back to first order there as well)
    st = sr_force_state(fields)
    for order in (0, 1):
        p = G.config_params("tube_srgsph", sr_2nd_order=order, sr_eta=2.3, range_min=(-0.5, 0.0, 0.0),
                            range_max=(0.5, 0.1, 0.1))
        ref = O.Reference(p, st)
        ref.tree_make()
        ref.set_kernel()
        ref.fluid_force()
        r = ref.download(["sr_dS_x", "sr_dS_y", "sr_dS_z", "sr_de"])
        out[f"force_o{order}_params"] = np.frombuffer(bytes(p), dtype=np.uint8)
        for k, v in r.items():
            out[f"force_o{order}_{k}"] = v
        print(f"sr_tube force o{order}: max |dS_x| {np.abs(r['sr_dS_x']).max():.3e}")
    for k, v in st.items():
        out["fst_" + k] = v
    np.savez_compressed(os.path.join(OUT, "sr_tube.npz"), **out)


def sr_force_state(fields, gamma=5.0 / 3.0):
    """Primitive state of the two-state SR tube as the force reads it."""
    left = fields["pos_x"] < 0.0
    n = np.where(left, 1.0, 0.125)
    P = np.where(left, 1.0, 0.08)
    H = 1.0 + gamma * P / ((gamma - 1.0) * n)
    nu = fields["sr_nu"]
    st = {k: fields[k].copy() for k in ("pos_x", "pos_y", "pos_z", "mass", "sr_nu")}
    st.update({"dens": n, "pres": P, "sr_N": n.copy(), "sr_gamma_lor": np.ones_like(n), "sr_enthalpy": H,
               "sound": np.sqrt((gamma - 1.0) * (H - 1.0) / H), "ene": P / ((gamma - 1.0) * n),
               "sml": 2.3 * np.cbrt(nu / n)})
    return st


def main():
    O.build(reference=True)
    if not O.have_reference():
        raise SystemExit("reference libraries not built; is REFDIR mounted?")
    evrard_golden()
    evrard_energy_golden()
    for name in SMALL:
        small_steps(name)
    for name in ("evrard_ssph", "tube_gsph", "shear_disph"):
        lists(name)
    csv_golden()
    relax_golden()
    sr_golden()
    for name in EDGE:
        edge_steps(name)
    sweep_golden()


def evrard_big_reference(steps=20, threads=0):
    """The compiled reference on the full 256^3 disph Evrard sphere
    (8,783,848 particles, the default benchmark workload's physics) at
    cflSound 0.05 / cflForce 0.025, step by step until its state turns
    non-finite: dt, time, K, U, W, the smallest internal energy, and the
    caller ids of the first particles with u <= 0 or a non-finite sound speed
    or position.  Slow: about 4.5 minutes per step on 6 host cores
    (python tests/golden/make_golden.py evrard_big)."""
    import json
    import time
    p = G.config_params("evrard_disph", cfl_sound=0.05, cfl_force=0.025)
    f = G.sample_evrard(256)
    threads = threads or max(2, os.cpu_count() - 2)
    ref = O.Reference(p, f, threads=threads)
    t0 = time.time()
    ref.initialize()
    rec = {"n": len(f["pos_x"]), "cfl": [0.05, 0.025], "threads": threads, "init_s": time.time() - t0,
           "steps": []}
    for s in range(steps):
        t1 = time.time()
        ref.integrate()
        st = ref.download(["ene", "sound", "pos_x", "dens"])
        bad = np.where(~np.isfinite(st["sound"]) | ~np.isfinite(st["pos_x"]) | (st["ene"] <= 0))[0]
        k, u, w, _ = ref.energies()
        rec["steps"].append({"step": s + 1, "time": ref.time, "dt": ref.dt, "K": k, "U": u, "W": w,
                             "umin": float(np.nanmin(st["ene"])), "rhomax": float(np.nanmax(st["dens"])),
                             "nbad": int(bad.size), "bad": bad[:32].tolist(), "sec": time.time() - t1})
        with open(os.path.join(OUT, "evrard_disph_8.78M_reference.json"), "w") as fh:
            json.dump(rec, fh, indent=1)
        if bad.size:
            break


if __name__ == "__main__":
    if sys.argv[1:] == ["evrard_big"]:
        O.build(reference=True)
        evrard_big_reference()
    elif sys.argv[1:] == ["edge"]:
        O.build(reference=True)
        for name in EDGE:
            edge_steps(name)
        sweep_golden()
    else:
        main()
