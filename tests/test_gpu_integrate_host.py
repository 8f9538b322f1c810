"""sphgpu_integrate_host: one step on host buffers, with the downloads of
fields that are final early in the step overlapping the rest of it, equals
sphgpu_upload + sphgpu_integrate + sphgpu_download bit for bit, and carries
the simulation time on."""
import numpy as np
import pytest

import ics
import sphparams as SP

pytestmark = pytest.mark.gpu

CASES = {
    "evrard_disph": lambda: (SP.config_params("evrard_disph", cfl_sound=0.05, cfl_force=0.025), ics.evrard(24)),
    "shear_disph": lambda: (SP.config_params("shear_disph"), ics.shear_layer(0.02)),
    "tube_gsph": lambda: (SP.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                          ics.shock_tube(0.01, ly=0.1)),
}

# the fields a host that keeps the particle records moves each step
STEP_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "mass", "dens",
               "pres", "ene", "dene", "sml", "sound", "balsara", "alpha", "gradh"]


@pytest.mark.parametrize("case", sorted(CASES))
def test_integrate_host_equals_upload_integrate_download(gpu, case):
    p, f = CASES[case]()
    names = list(gpu.FIELDS)
    with gpu.Simulation(p) as a, gpu.Simulation(p) as b:
        for sim in (a, b):
            sim.upload(f)
            sim.initialize()
        st_a = a.download(STEP_FIELDS)
        st_b = b.download(STEP_FIELDS)
        t_sum = 0.0
        for s in range(4):
            out_a = a.integrate_host(st_a, names)
            t_sum += a.time_dt()[1]
            b.upload(st_b)
            b.set_initial_smoothing(False)
            b.integrate()
            out_b = b.download(names)
            for k in names:
                np.testing.assert_array_equal(out_a[k], out_b[k], err_msg=f"step {s + 1} {k}")
            st_a = {k: out_a[k] for k in STEP_FIELDS}
            st_b = {k: out_b[k] for k in STEP_FIELDS}
        t, _ = a.time_dt()
        assert t == pytest.approx(t_sum, rel=1e-14)


def test_integrate_host_partial_tables(gpu):
    """NULL entries in either table: only the given fields move."""
    p, f = CASES["evrard_disph"]()
    with gpu.Simulation(p) as a, gpu.Simulation(p) as b:
        for sim in (a, b):
            sim.upload(f)
            sim.initialize()
        st = a.download(STEP_FIELDS)
        out = a.integrate_host(st, ["pos_x", "dens", "acc_z", "phi"])
        b.upload(st)
        b.set_initial_smoothing(False)
        b.integrate()
        ref = b.download(["pos_x", "dens", "acc_z", "phi"])
        for k in ref:
            np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
