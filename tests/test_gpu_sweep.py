"""The GPU path on the 56 sweep configurations whose oracle runs are pinned
to the compiled reference by SHA-256 (tests/golden/sweep_hashes.json,
tests/test_oracle_golden.py): every sph type x kernel (cubic, Wendland,
Gaussian) x leaf 1 / leaf 4 / tree level cap 3 on an off-origin sphere with
gravity, TD-AV and AC; periodic layers with particles on the box faces and
one coincident pair, iterative and fixed h, Balsara off, first-order gsph
with the iterative solver.

Bars: tree nodes and gravity bit-identical to the oracle on the same state;
gather and symmetric lists equal as sets on the same state; initialize + 2
steps to rounding (test_gpu_parity.py's bars for the golden steps).
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from test_gpu_parity import _close
from test_gpu_scale import STATE, same_sets

pytestmark = pytest.mark.gpu

sys.path.insert(0, GOLDEN)
import make_golden as M  # noqa: E402

CASES = M.sweep_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_sweep_gpu_against_oracle(gpu, O, name):
    p, mk = CASES[name]
    f = mk()
    o = O.Oracle(p, f)
    o.initialize()
    states, dts = [o.download(STATE)], [0.0]
    for _ in range(2):
        o.integrate()
        states.append(o.download(STATE))
        dts.append(o.dt)
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        for s in range(3):
            out = sim.download()
            np.testing.assert_array_equal(out["neighbor"], states[s]["neighbor"], err_msg=f"step {s} neighbor")
            for fld in ("dens", "sml", "pres", "ene"):
                _close(out[fld], states[s][fld], f"step {s} {fld}", median=1e-11, p999=1e-8, worst=1e-5)
            amax = max(np.max(np.abs(states[s][f"acc_{a}"])) for a in "xyz")
            for a in "xyz":
                _close(out[f"acc_{a}"], states[s][f"acc_{a}"], f"step {s} acc_{a}", scale=amax, median=1e-11,
                       p999=1e-8, worst=1e-5)
            if s > 0:
                assert sim.time_dt()[1] == pytest.approx(dts[s], rel=1e-9)
            if s < 2:
                sim.integrate()

    # tree, lists and gravity on one state (the oracle's after step 1)
    st = dict(states[1])
    o1 = O.Oracle(p, st)
    o1.tree_make()
    o1.set_kernel()
    oi, od = o1.tree_nodes()
    olists = [o1.neighbor_lists(ij) for ij in (False, True)]
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.set_kernel()
        gi, gd = sim.tree_nodes()
        glists = [sim.neighbor_search(is_ij=ij) for ij in (False, True)]
    np.testing.assert_array_equal(gi[:, :2], oi[:, :2])
    np.testing.assert_array_equal(gi[1:, 2], oi[1:, 2])
    np.testing.assert_array_equal(gd, od)
    for ij in (0, 1):
        same_sets(glists[ij][0], glists[ij][1], olists[ij][0], olists[ij][1], f"is_ij={ij}")
    if p.use_gravity:
        for k in ("acc_x", "acc_y", "acc_z"):
            st[k] = np.zeros_like(st["pos_x"])
        og = O.Oracle(p, st)
        og.tree_make()
        og.gravity_force()
        ref = og.download(["acc_x", "acc_y", "acc_z", "phi"])
        with gpu.Simulation(p) as sim:
            sim.upload(st)
            sim.tree_make()
            sim.gravity_force()
            out = sim.download(["acc_x", "acc_y", "acc_z", "phi"])
        for k in ref:
            np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
