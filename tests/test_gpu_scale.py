"""GPU parity against the oracle at benchmark scale (130 K - 250 K particles
per workload, and the 17,256-particle Evrard sphere of the ssph workload for
its 20 steps).  The oracle (oracle/sph_oracle.cpp) reproduces the compiled
reference bit for bit on every golden fixture, so it stands in for the
reference at sizes whose reference runs would take hours.

Bars, as in test_gpu_parity.py:
  * tree nodes (topology, centre, edge, mass, centre of mass) bit-identical
    on the same state (src/bhtree.cpp:154-247);
  * gather and symmetric neighbour lists equal as sets on the same state
    (src/bhtree.cpp:277-316);
  * gravity on the same tree and inputs bit-identical (src/bhtree.cpp:347-393);
  * initialize + 2 steps from the same initial conditions: density, h,
    pressure and acceleration to rounding (sums run in a different order than
    the reference's distance-sorted loops).
"""
import numpy as np
import pytest

import ics
import sphparams as SP
from test_gpu_parity import _close

pytestmark = pytest.mark.gpu

WORKLOADS = {
    "shear_disph_130k": lambda: (SP.config_params("shear_disph"), ics.shear_layer((0.1875 / 130e3) ** (1 / 3))),
    "tube_gsph_250k": lambda: (SP.config_params("tube_gsph"), ics.shock_tube((0.0025 / 250e3) ** (1 / 3))),
    "tube_gdisph_250k": lambda: (SP.config_params("tube_gdisph"), ics.shock_tube((0.0025 / 250e3) ** (1 / 3))),
    "evrard_disph_137k": lambda: (SP.config_params("evrard_disph", cfl_sound=0.05, cfl_force=0.025), ics.evrard(64)),
}
STATE = [f for f in SP.FIELDS if not f.startswith("sr_")]


def same_sets(off_a, ids_a, off_b, ids_b, what):
    """CSR lists equal row by row as sets."""
    np.testing.assert_array_equal(off_a, off_b, err_msg=f"{what}: list lengths")
    n = len(off_a) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off_a))
    ka = np.sort(rows * n + ids_a.astype(np.int64))
    kb = np.sort(rows * n + ids_b.astype(np.int64))
    bad = np.flatnonzero(ka != kb)
    assert bad.size == 0, f"{what}: rows differ, first at particle {int(ka[bad[0]] // n)}"


@pytest.fixture(scope="module", params=sorted(WORKLOADS))
def run(request, O):
    """The oracle's initialize + 2 steps, and its state after step 1 (the
    state both sides rebuild tree and lists from)."""
    p, f = WORKLOADS[request.param]()
    o = O.Oracle(p, f)
    o.initialize()
    states = [o.download(STATE)]
    dts = [0.0]
    for _ in range(2):
        o.integrate()
        states.append(o.download(STATE))
        dts.append(o.dt)
    return request.param, p, f, states, dts


def test_scale_steps_match_oracle(gpu, run):
    name, p, f, states, dts = run
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        for s in range(3):
            out = sim.download()
            for fld in ("dens", "sml", "pres"):
                _close(out[fld], states[s][fld], f"{name} step {s} {fld}", median=1e-11, p999=1e-8, worst=1e-5)
            amax = max(np.max(np.abs(states[s][f"acc_{a}"])) for a in "xyz")
            for a in "xyz":
                _close(out[f"acc_{a}"], states[s][f"acc_{a}"], f"{name} step {s} acc_{a}", scale=amax,
                       median=1e-11, p999=1e-8, worst=1e-5)
            if s > 0:
                assert sim.time_dt()[1] == pytest.approx(dts[s], rel=1e-9)
            if s < 2:
                sim.integrate()


def test_scale_tree_and_lists_bitexact(gpu, O, run):
    name, p, f, states, dts = run
    st = states[1]
    o = O.Oracle(p, st)
    o.tree_make()
    o.set_kernel()
    oi, od = o.tree_nodes()
    olists = [o.neighbor_lists(ij) for ij in (False, True)]
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.set_kernel()
        gi, gd = sim.tree_nodes()
        glists = [sim.neighbor_search(is_ij=ij) for ij in (False, True)]
    assert gi.shape == oi.shape
    np.testing.assert_array_equal(gi[:, :2], oi[:, :2])
    np.testing.assert_array_equal(gi[1:, 2], oi[1:, 2])
    np.testing.assert_array_equal(gd[:, :9], od[:, :9])
    for ij in (0, 1):
        same_sets(glists[ij][0], glists[ij][1], olists[ij][0], olists[ij][1], f"{name} is_ij={ij}")


def test_scale_gravity_bitexact(gpu, O, run):
    name, p, f, states, dts = run
    if not p.use_gravity:
        pytest.skip("no gravity in this workload")
    st = dict(states[1])
    for k in ("acc_x", "acc_y", "acc_z"):
        st[k] = np.zeros_like(st["pos_x"])
    o = O.Oracle(p, st)
    o.tree_make()
    o.gravity_force()
    ref = o.download(["acc_x", "acc_y", "acc_z", "phi"])
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.gravity_force()
        out = sim.download(["acc_x", "acc_y", "acc_z", "phi"])
    for k in ref:
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)


def test_evrard_ssph_full_size_20_steps(gpu, O):
    """The ssph Evrard workload at its full 17,256 particles for its 20 steps:
    dt sequence and energies follow the oracle, the state stays within
    rounding growth, and the lists of the final state are the same sets."""
    p = SP.config_params("evrard_ssph")
    f = ics.evrard(32)
    o = O.Oracle(p, f)
    o.initialize()
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        for s in range(20):
            o.integrate()
            sim.integrate()
            assert sim.time_dt()[1] == pytest.approx(o.dt, rel=1e-9), f"dt step {s + 1}"
            ke, ue, we, _ = sim.energies()
            ko, uo, wo, _ = o.energies()
            e0 = abs(ko + uo + wo)
            assert abs((ke + ue + we) - (ko + uo + wo)) <= 1e-10 * e0, f"energy step {s + 1}"
        out = sim.download()
        ref = o.download()
        for fld in ("dens", "sml", "pres", "ene"):
            _close(out[fld], ref[fld], f"step 20 {fld}", median=1e-10, p999=1e-7, worst=1e-4)
        amax = max(np.max(np.abs(ref[f"acc_{a}"])) for a in "xyz")
        for a in "xyz":
            _close(out[f"acc_{a}"], ref[f"acc_{a}"], f"step 20 acc_{a}", scale=amax, median=1e-10, p999=1e-7,
                   worst=1e-4)
    st = {k: v for k, v in ref.items() if k in STATE}
    o2 = O.Oracle(p, st)
    o2.tree_make()
    o2.set_kernel()
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.set_kernel()
        for ij in (False, True):
            go, gids = sim.neighbor_search(is_ij=ij)
            oo, oids = o2.neighbor_lists(ij)
            same_sets(go, gids, oo, oids, f"evrard step 20 is_ij={ij}")
