"""The reference's own Solver sequence (Solver::initialize / integrate as
oracle/ref_harness.cpp drives the reference's modules, src/solver.cpp:941-978)
with the GPU modules of sph-code-simulation_b200/host/gpu_modules.hpp swapped
in for TimeStep, PreInteraction, FluidForce, GravityForce and make_tree,
against the same sequence with the reference's CPU modules, over 2 steps.

MIRROR keeps Solver::predict / correct on the host (one upload after predict
and one download after GravityForce per step); RESIDENT runs them on the
device and downloads only when the host reads the particles.  Both must
reproduce the CPU run to rounding (sums in another order)."""
import os

import numpy as np
import pytest

from conftest import golden, params_from_bytes
from test_gpu_parity import _close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def have_swap(O):
    if not os.path.exists(O.REF_GPU_LIB) or not O.have_reference():
        pytest.fail("oracle/_ref/libsphref_gpu.so is not built (make -C oracle ref)")
    return True


@pytest.mark.parametrize("name", ["evrard_ssph", "evrard_disph", "shear_disph", "tube_gsph", "tube_gdisph"])
@pytest.mark.parametrize("resident", [False, True], ids=["mirror", "resident"])
def test_gpu_modules_in_reference_sequence(gpu, O, have_swap, name, resident):
    g = golden(f"steps_{name}.npz")
    p = params_from_bytes(gpu, g["params"])
    fields = {k[3:]: g[k] for k in g.files if k.startswith("ic_")}
    cpu = O.Reference(p, fields, threads=4)
    swp = O.ReferenceWithGpuModules(p, fields, resident=resident, threads=4)
    cpu.initialize()
    swp.initialize()
    for s in range(3):
        a, b = swp.download(), cpu.download()
        np.testing.assert_array_equal(a["neighbor"], b["neighbor"], err_msg=f"step {s} neighbor")
        for f in ("dens", "sml", "pres", "ene", "vel_x", "pos_y"):
            _close(a[f], b[f], f"step {s} {f}", median=1e-11, p999=1e-8, worst=1e-5,
                   scale=None if f not in ("vel_x", "pos_y") else np.max(np.abs(b[f])) + 1e-300)
        amax = max(np.max(np.abs(b[f"acc_{x}"])) for x in "xyz")
        for x in "xyz":
            _close(a[f"acc_{x}"], b[f"acc_{x}"], f"step {s} acc_{x}", scale=amax, median=1e-11, p999=1e-8,
                   worst=1e-5)
        if s > 0:
            assert swp.dt == pytest.approx(cpu.dt, rel=1e-9)
            assert swp.time == pytest.approx(cpu.time, rel=1e-12)
        if s < 2:
            cpu.integrate()
            swp.integrate()
    ks, us, ws, _ = swp.energies()
    kc, uc, wc, _ = cpu.energies()
    assert ks + us + ws == pytest.approx(kc + uc + wc, rel=1e-10)
