"""bench.py's reference arm (the reference's own OpenMP CPU build in
oracle/_ref) prints one JSON line with the same metric, unit and config as
the GPU arm and the keys the contract asks for, and maps no product library;
the FLOP accounting of the roofline follows flop_weights.md."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_json_line(O):
    if not O.have_reference():
        pytest.skip("oracle/_ref is not built here")
    sys.path.insert(0, ROOT)
    import bench
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--particles", "2e4"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and 1 <= d["steps"] <= 2
    assert d["config"]["workload"].startswith("disph + BH gravity Evrard sphere")
    n = d["config"]["n_particles"]
    assert n == len(bench.ics.evrard(round((2e4 * 6.0 / 3.14159265) ** (1 / 3)))["pos_x"])

    class A:
        particles = 2e4
    assert d["config"] == bench.bench_config(bench.WORKLOADS[bench.DEFAULT_WORKLOAD], n, 1, A)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and f"N={n}" in cb["sample"]
    assert d["value"] > 0 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_maps_no_product_library(O):
    """The reference arm builds its parameters and initial conditions without
    libsphgpu.so (sphparams.py, ics.py), so only oracle/_ref is mapped."""
    if not O.have_reference():
        pytest.skip("oracle/_ref is not built here")
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "bench.cpu_reference(1, 0, 'evrard_disph', 5e3, 0.0); "
            "m = open('/proc/self/maps').read(); "
            "print('sphgpu' in m, 'libsphref' in m)") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split()[-2:] == ["False", "True"], r.stdout


def test_flop_accounting():
    sys.path.insert(0, ROOT)
    import bench
    import sphparams as SP
    p = SP.config_params("evrard_disph")
    c = {"pre_candidates": 10, "pre_newton_pairs": 3, "pre_pairs": 2, "force_candidates": 5, "force_pairs": 4,
         "riemann_iterations": 0, "gravity_nodes": 7, "gravity_monopoles": 6, "gravity_leaf_pairs": 1}
    W = bench.FLOP_W
    assert bench.stage_flops("pre", c, p) == 10 * 8 + 3 * (W["newton_kernel"]["wendland"] + 2) + 2 * 79
    assert bench.stage_flops("force", c, p) == 5 * 8 + 4 * 122
    assert bench.stage_flops("gravity", c, p) == 7 * 10 + 6 * 14 + 80
    assert bench.stage_flops("gather_walk", c, p) is None
    # every weight in bench.py appears in the committed table
    doc = open(os.path.join(ROOT, "flop_weights.md")).read()
    for k in ("pre_pair", "force_pair"):
        for sph, v in W[k].items():
            assert f"| {sph} | {v} |" in doc or f"| {v} |" in doc, (k, sph, v)
