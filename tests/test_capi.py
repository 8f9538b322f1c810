"""The C-ABI library: loads without a GPU, exports every declared symbol,
mirrors the reference's parameter defaults, fails loudly without a device."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "sphgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(sphgpu_\w+)\s*\(", src))
    return sorted(names)


def test_exports_every_declared_symbol(G):
    lib = G.lib()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_match_reference_defaults(G):
    """Defaults of Solver::read_parameterfile (src/solver.cpp:311-438)."""
    p = G.default_params()
    assert p.neighbor_number == 50 and p.leaf_particle_num == 1 and p.max_tree_level == 20
    assert p.cfl_sound == 0.3 and p.cfl_force == 0.125 and p.av_alpha == 1.0
    assert p.use_balsara_switch == 1 and p.iterative_sml == 1 and p.theta == 0.5
    assert p.gsph_2nd_order == 1 and p.riemann_solver == G.RIEMANN_HLL
    assert p.alpha_max == 2.0 and p.alpha_min == 0.1 and p.epsilon_av == 0.2
    assert p.gamma == pytest.approx(5.0 / 3.0, rel=1e-15)


def test_params_struct_layout(G, tmp_path):
    """The ctypes mirror has the C compiler's offsets for every field."""
    import ctypes
    import subprocess
    assert ctypes.sizeof(G.Params) == 264
    assert G.Params.sr_2nd_order.offset == 192 and G.Params.tree_root_origin.offset == 196
    assert G.Params.sr_c_speed.offset == 200
    names = [f[0] for f in G.Params._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "sphgpu.h"\nint main(void) {\n'
                   + "".join(f'    printf("%zu\\n", offsetof(sphgpu_params, {n}));\n' for n in names)
                   + '    printf("%zu\\n", sizeof(sphgpu_params));\n    return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[:-1] == [getattr(G.Params, n).offset for n in names]
    assert got[-1] == ctypes.sizeof(G.Params)


def test_samples(G):
    ev = G.sample_evrard(32)
    assert len(ev["pos_x"]) == 17256
    r = np.sqrt(ev["pos_x"] ** 2 + ev["pos_y"] ** 2 + ev["pos_z"] ** 2)
    assert r.max() <= 1.0 and np.allclose(ev["mass"].sum(), 1.0)
    sh = G.sample_shear_layer(0.05)
    assert np.all((sh["pos_y"] > 0.25) & (sh["pos_y"] < 0.75) == (sh["dens"] == 2.0))
    tu = G.sample_shock_tube(0.025, ly=0.1)
    assert np.all((tu["pos_x"] < 0) == (tu["pres"] == 1000.0))
    sr = G.sample_sr_shock_tube(0.025, ly=0.1)
    left = sr["pos_x"] < 0
    assert left.sum() == 320 and (~left).sum() == 40
    assert np.all(sr["sr_nu"] == sr["sr_nu"][0]) and np.all(sr["sr_S_x"] == 0.0)
    assert np.all(sr["sr_N"][left] == 1.0) and np.all(sr["sr_N"][~left] == 0.125)


def test_create_without_device_fails_loudly(G):
    if G.device_ok():
        pytest.skip("a device is present")
    with pytest.raises(G.SPHException):
        G.Simulation(G.default_params())


def test_bad_params_rejected(G):
    with pytest.raises(G.SPHException, match="maxTreeLevel"):
        G.Simulation(G.default_params(max_tree_level=30))
    with pytest.raises(G.SPHException, match="kernel"):
        G.Simulation(G.default_params(kernel=7))
    with pytest.raises(G.SPHException, match="tree_root_origin"):
        G.Simulation(G.default_params(tree_root_origin=2))


def test_binding_declares_every_entry_point(G):
    """Every function include/sphgpu.h declares has a ctypes signature in the
    binding (an undeclared one would pass 64-bit handles as C ints)."""
    src = open(os.path.join(ROOT, "include", "sphgpu.h")).read()
    names = set(re.findall(r"\b(sphgpu_\w+)\s*\(", src))
    L = G.lib()
    for name in sorted(names):
        assert getattr(L, name).argtypes is not None, name


def test_particle_count_bounds_checked_first(G):
    """upload rejects counts its int32 node indices cannot address (5 n + 2
    nodes) before it touches a device, so this runs with or without one."""
    import ctypes
    src = open(os.path.join(ROOT, "include", "sphgpu.h")).read()
    limit = int(re.search(r"#define SPHGPU_MAX_PARTICLES (\d+)", src).group(1))
    assert 5 * limit + 2 <= 2 ** 31 - 1 < 5 * (limit + 1) + 2
    L = G.lib()
    p = G.default_params()
    h = ctypes.c_void_p()
    L.sphgpu_create(ctypes.byref(p), ctypes.byref(h))
    assert h
    try:
        for n in (0, -5, limit + 1):
            assert L.sphgpu_upload(h, n, None) == -1, n
            assert b"particle count out of range" in L.sphgpu_last_error(h)
    finally:
        L.sphgpu_destroy(h)
