"""The allocation-free TimeStep entry point (sphgpu_timestep_noalloc).

It exists for callers that cannot allocate device memory when they need dt:
a host solver that owns the whole device memory budget through its own pool,
or code that must not incur a cudaMalloc / cudaFree synchronisation.  It must
give exactly the dt of the context entry point sphgpu_timestep, on every call
(the shared device scratch keeps the previous call's contents).  This file is
collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(G):
    L = G.lib()
    f = L.sphgpu_timestep_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    return f


def _reference_dt(G, params, fields):
    with G.Simulation(params) as sim:
        sim.upload(fields)
        sim.initialize()
        st = sim.download(["acc_x", "acc_y", "acc_z", "sml"])
        hvs = sim.h_per_v_sig()
        dt = sim.timestep()
    return st, hvs, dt


@pytest.mark.parametrize("N", [12, 20])
def test_noalloc_timestep_matches_context_entry_point(gpu, N):
    import torch
    f = _bind(gpu)
    p = gpu.config_params("evrard_ssph")
    st, hvs, dt_ref = _reference_dt(gpu, p, gpu.sample_evrard(N))
    n = len(st["sml"])
    acc = torch.tensor(np.stack([st["acc_x"], st["acc_y"], st["acc_z"]], axis=1).ravel(), dtype=torch.float64,
                       device="cuda")
    sml = torch.tensor(st["sml"], dtype=torch.float64, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row through the shared scratch
        out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = f(acc.data_ptr(), sml.data_ptr(), n, hvs, p.cfl_sound, p.cfl_force, out.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0
        assert out.item() == dt_ref


def test_noalloc_rejects_oversized_input(gpu):
    import torch
    f = _bind(gpu)
    acc = torch.zeros(3, dtype=torch.float64, device="cuda")
    sml = torch.ones(1, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_many = 1024 * 4096 + 1
    assert f(acc.data_ptr(), sml.data_ptr(), too_many, 1.0, 0.3, 0.125, out.data_ptr(), None) == -1
    assert f(None, sml.data_ptr(), 1, 1.0, 0.3, 0.125, out.data_ptr(), None) == -1
