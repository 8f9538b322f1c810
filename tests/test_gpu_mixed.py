"""The mixed-precision form (FP32 pair sums, kernels and gravity walk; FP64
accumulators, kick-drift and set predicates) against the plain FP64 form and
the FP64 oracle.

The metric is the mixed form's accuracy criterion: the median over particles of the relative
error |a_mixed - a| / |a| of the acceleration (and of the density), from one
state.  Measured on B200 (one FluidForce + GravityForce from the same state):

| workload | density | acceleration |
|---|---|---|
| disph Evrard sphere 137 K (config 4's set-up) | 7e-8 | 1.9e-7 (met) |
| disph shear layer 130 K (config 1) | 8e-8 | 3.0e-3 (missed) |
| gsph shock tube 250 K (config 2) | 1.4e-7 | ill-defined: ahead of the shock |a| is 1e-20 of max|a| |

In the shear layer's pressure-balanced bulk the acceleration is a residue
1e-3 .. 1e-6 of the cancelling pair terms; the FP32 density and pressure the
force reads (errors ~1e-7) already limit it, so even an FP64 re-evaluation of
the force (mixed_acc_tol) leaves 1.1e-3.  Those cases are xfail below, with
the measured level pinned beside them.
* total energy over 100 steps: the FP64 form follows the oracle to <= 1e-12
  of |E0| [2e-14] and the mixed form to <= 1e-6 [5e-8];
* neighbour sets: identical (FP64 predicates in both forms)."""
import numpy as np
import pytest

import ics
import sphparams as SP
from conftest import rel_err

pytestmark = pytest.mark.gpu

CASES = {
    "evrard_ssph": lambda G: (G.config_params("evrard_ssph"), G.sample_evrard(24)),
    "shear_disph": lambda G: (G.config_params("shear_disph"), G.sample_shear_layer(0.02)),
    "tube_gsph": lambda G: (G.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                            G.sample_shock_tube(0.01, ly=0.1)),
    "evrard_disph": lambda G: (G.config_params("evrard_disph"), G.sample_evrard(24)),
    "tube_gdisph": lambda G: (G.config_params("tube_gdisph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                              G.sample_shock_tube(0.01, ly=0.1)),
}
SPHERES = ("evrard_ssph", "evrard_disph")
# the benchmark workloads at >= 130 K particles
SCALE = {
    "evrard_disph_137k": lambda: (SP.config_params("evrard_disph", cfl_sound=0.006, cfl_force=0.003),
                                  ics.evrard(64)),
    "shear_disph_130k": lambda: (SP.config_params("shear_disph"), ics.shear_layer((0.1875 / 130e3) ** (1 / 3))),
    "tube_gsph_250k": lambda: (SP.config_params("tube_gsph"), ics.shock_tube((0.0025 / 250e3) ** (1 / 3))),
}


def _run(G, p, fields, precision, steps):
    p = p.copy()
    p.precision = precision
    with G.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        for _ in range(steps):
            sim.integrate()
        return sim.download(), sim.neighbor_search(is_ij=False)


def _acc(d):
    return np.stack([d["acc_x"], d["acc_y"], d["acc_z"]], axis=1)


def _acc_err(out, ref):
    a, b = _acc(ref), _acc(out)
    return np.linalg.norm(b - a, axis=1) / np.maximum(np.linalg.norm(a, axis=1), 1e-300)


def _one_evaluation(G, p, state, dt, precision, tol=0.0):
    """tree, PreInteraction, FluidForce, GravityForce from `state`."""
    q = p.copy()
    q.precision = precision
    q.mixed_acc_tol = tol
    with G.Simulation(q) as sim:
        sim.upload(state)
        sim.set_initial_smoothing(False)
        sim.set_dt(dt)
        sim.reset_counters()
        sim.tree_make()
        sim.pre_interaction()
        sim.fluid_force()
        sim.gravity_force()
        return sim.download(), sim.counters()


@pytest.fixture(scope="module", params=sorted(SCALE))
def scale_case(request, gpu):
    """The FP64 form's state after initialize + one step, and one evaluation
    from it in the FP64 form, the mixed form, and the mixed form with the
    FP64 re-evaluation at 1e-5."""
    p, f = SCALE[request.param]()
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        sim.integrate()
        st = sim.download()
        dt = sim.time_dt()[1]
    st = {k: v for k, v in st.items() if not k.startswith("sr_")}
    ref, _ = _one_evaluation(gpu, p, st, dt, gpu.FP64)
    mixed, _ = _one_evaluation(gpu, p, st, dt, gpu.MIXED)
    checked, cnt = _one_evaluation(gpu, p, st, dt, gpu.MIXED, tol=1e-5)
    return request.param, ref, mixed, checked, cnt


def test_mixed_density_median_at_scale(scale_case):
    name, ref, mixed, checked, _ = scale_case
    assert np.median(rel_err(mixed["dens"], ref["dens"])) <= 1e-5, name


def test_mixed_acceleration_median_at_scale(request, scale_case):
    """The accuracy bar: median per-particle relative error <= 1e-5."""
    name, ref, mixed, checked, _ = scale_case
    if not name.startswith("evrard"):
        request.applymarker(pytest.mark.xfail(strict=True, reason="missed: acceleration is a residue of cancelling "
                                                                  "pair terms (see the module docstring)"))
    assert np.median(_acc_err(mixed, ref)) <= 1e-5, name


def test_mixed_acceleration_levels_pinned(scale_case):
    """The measured error levels (regression guard for the cases above)."""
    name, ref, mixed, checked, _ = scale_case
    med = np.median(_acc_err(mixed, ref))
    bound = {"evrard_disph_137k": 1e-6, "shear_disph_130k": 1e-2, "tube_gsph_250k": np.inf}[name]
    assert med <= bound, (name, med)


def test_mixed_recheck_bounds_sphere_particles(scale_case):
    """With mixed_acc_tol = 1e-5 the particles whose FP32 force / gravity
    rounding could exceed 1e-5 are re-evaluated in FP64: on the
    self-gravitating sphere no particle's acceleration is then off by more
    than 1e-5 (a few are without it)."""
    name, ref, mixed, checked, cnt = scale_case
    if not name.startswith("evrard"):
        pytest.skip("the FP32 PreInteraction outputs dominate the error here")
    e = _acc_err(checked, ref)
    assert cnt["mixed_rechecks"] > 0
    assert np.max(e) <= 1e-5, np.max(e)
    assert np.median(e) <= np.median(_acc_err(mixed, ref)) * 1.5


@pytest.mark.parametrize("case", sorted(CASES))
def test_mixed_vs_fp64_one_step(gpu, case):
    p, fields = CASES[case](gpu)
    a, la = _run(gpu, p, fields, gpu.FP64, 1)
    b, lb = _run(gpu, p, fields, gpu.MIXED, 1)
    assert np.median(rel_err(b["dens"], a["dens"])) <= 1e-5
    if case in SPHERES:
        assert np.median(_acc_err(b, a)) <= 1e-5
    # FP64 predicates: the gather lists of both forms are the same sets
    # whenever the smoothing lengths that define them agree bit for bit
    if np.array_equal(a["sml"], b["sml"]):
        np.testing.assert_array_equal(la[0], lb[0])
        np.testing.assert_array_equal(la[1], lb[1])


def test_mixed_initial_sets_identical(gpu):
    """From the same uploaded state the FP32 form's neighbour lists equal the
    FP64 form's (the predicates stay FP64)."""
    p, fields = CASES["shear_disph"](gpu)
    out = []
    for prec in (gpu.FP64, gpu.MIXED):
        q = p.copy()
        q.precision = prec
        with gpu.Simulation(q) as sim:
            f = dict(fields)
            f["sml"] = np.full(len(f["pos_x"]), 0.05)
            sim.upload(f)
            sim.tree_make()
            sim.set_kernel()
            out.append((sim.neighbor_search(False), sim.neighbor_search(True)))
    for k in (0, 1):
        np.testing.assert_array_equal(out[0][k][0], out[1][k][0])
        np.testing.assert_array_equal(out[0][k][1], out[1][k][1])


@pytest.mark.parametrize("case", SPHERES)
def test_energy_against_oracle_100_steps(gpu, O, case):
    """K + U + W every 20 steps over 100 steps of a self-gravitating sphere
    (16^3 lattice cut to the unit sphere, 2176 particles), for the oracle,
    the FP64 form and the mixed form.  The reference's own scheme drifts by
    about 2 % over this collapse at this resolution; the claims are about
    following it."""
    p, fields = CASES[case](gpu)[0], gpu.sample_evrard(16)
    o = O.Oracle(p, fields)
    o.initialize()
    k, u, w, _ = o.energies()
    e_or = [k + u + w]
    for s in range(100):
        o.integrate()
        if (s + 1) % 20 == 0:
            k, u, w, _ = o.energies()
            e_or.append(k + u + w)
    t_or = o.time
    e0 = abs(e_or[0])
    for prec, tol in ((gpu.FP64, 1e-12), (gpu.MIXED, 1e-6)):
        q = p.copy()
        q.precision = prec
        with gpu.Simulation(q) as sim:
            sim.upload(fields)
            sim.initialize()
            k, u, w, _ = sim.energies()
            e = [k + u + w]
            for s in range(100):
                sim.integrate()
                if (s + 1) % 20 == 0:
                    k, u, w, _ = sim.energies()
                    e.append(k + u + w)
            t, _ = sim.time_dt()
        assert abs(t - t_or) <= 1e-5 * t_or
        dev = np.abs(np.array(e) - np.array(e_or)) / e0
        assert dev.max() <= tol, (prec, dev)
