"""SRGSPH on the GPU against the reference (tests/golden/sr_tube.npz, made by
the reference's compiled src/srgsph modules through tests/golden/make_golden.py).

Per configuration (first / second order, fixed / iterative smoothing length)
on a 3-D special-relativistic Sod tube of 360 particles:
* the pre-interaction after initialize (smoothing lengths, N, primitives,
  MUSCL gradients): the list sums run in another order than the reference's
  distance-sorted lists and pow is CUDA's, so they agree to rounding
  (tolerance below, relative to each field's largest magnitude);
* predict and correct from the reference's own state: FP64, unfused, the same
  primitive recovery, bit-identical;
* FluidForce on a prescribed two-state tube where every Riemann problem is
  well posed, to rounding.  On the Sod tube itself the reference's exact SR
  solver does not converge for most pairs (it stops after 50 damped Newton
  steps), and its rates change by up to half their magnitude when one
  coordinate moves by one ulp (tests/test_oracle_golden.py), so no other
  summation order can reproduce them; they are not compared there;
* a full integrate step fails as the reference's does: the spurious star
  pressures make the rates explode and the Lorentz-factor solve of the
  primitive recovery does not converge (SPHGPU_ERR_SR_RECOVERY where the
  reference throws)."""
import numpy as np
import pytest

from conftest import golden, params_from_bytes

pytestmark = pytest.mark.gpu

TAGS = ["o0i0", "o0i1", "o1i0", "o1i1"]
RATES = ("sr_dS_x", "sr_dS_y", "sr_dS_z", "sr_de")
TOL_STATE = 1e-12   # relative to the field's largest magnitude
TOL_RATE = 1e-9


def _fields(g):
    return {k[3:]: g[k] for k in g.files if k.startswith("ic_")}


def _compare(st, g, tag, s, skip=(), tol=None):
    for f in g.files:
        if not f.startswith(f"{tag}_s{s}_"):
            continue
        name = f[len(f"{tag}_s{s}_"):]
        if name in skip:
            continue
        ref = g[f]
        scale = max(np.max(np.abs(ref)), 1e-300)
        err = float(np.max(np.abs(st[name] - ref)) / scale)
        assert err <= (TOL_STATE if tol is None else tol), (tag, s, name, err)


@pytest.mark.parametrize("tag", TAGS)
def test_srgsph_pre_interaction_matches_reference(gpu, tag):
    """Smoothing lengths, N, primitives and MUSCL gradients after initialize."""
    g = golden("sr_tube.npz")
    p = params_from_bytes(gpu, g[tag + "_params"])
    with gpu.Simulation(p) as sim:
        sim.upload(_fields(g))
        sim.initialize()
        _compare(sim.download(), g, tag, 0, skip=RATES)


@pytest.mark.parametrize("tag", TAGS)
def test_srgsph_kick_drift_matches_reference(gpu, tag):
    """Solver::predict / correct (primitive recovery included) from the
    reference's own state after initialize."""
    g = golden("sr_tube.npz")
    p = params_from_bytes(gpu, g[tag + "_params"])
    state = {f[len(tag) + 4:]: g[f] for f in g.files if f.startswith(f"{tag}_s0_")}
    state["mass"] = g["ic_mass"]
    with gpu.Simulation(p) as sim:
        sim.upload(state)
        sim.set_dt(float(g[tag + "_dt"]))
        sim.predict()
        _compare(sim.download(), g, tag, 1, tol=0.0)
        sim.correct()
        _compare(sim.download(), g, tag, 2, tol=0.0)


@pytest.mark.parametrize("order", [0, 1])
def test_srgsph_force_matches_reference(gpu, order):
    """FluidForce on the prescribed two-state tube (every Riemann problem well
    posed): dS/dt and de/dt against the reference's."""
    g = golden("sr_tube.npz")
    p = params_from_bytes(gpu, g[f"force_o{order}_params"])
    st = {k[4:]: g[k] for k in g.files if k.startswith("fst_")}
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.set_kernel()
        sim.fluid_force()
        out = sim.download(list(RATES))
    for k in RATES:
        ref = g[f"force_o{order}_{k}"]
        err = float(np.max(np.abs(out[k] - ref)) / np.max(np.abs(ref)))
        assert err <= TOL_RATE, (order, k, err)


@pytest.mark.parametrize("tag", TAGS)
def test_srgsph_integrate_fails_like_reference(gpu, tag):
    g = golden("sr_tube.npz")
    p = params_from_bytes(gpu, g[tag + "_params"])
    msg = str(g[tag + "_integrate_error"])
    assert msg
    with gpu.Simulation(p) as sim:
        sim.upload(_fields(g))
        sim.initialize()
        with pytest.raises(gpu.SPHException, match=msg) as e:
            sim.integrate()
        assert "(-7)" in str(e.value)


def test_srgsph_rejects_mixed_form(gpu):
    p = gpu.config_params("tube_srgsph", precision=gpu.MIXED)
    with pytest.raises(gpu.SPHException):
        gpu.Simulation(p)
