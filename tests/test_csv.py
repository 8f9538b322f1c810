"""Snapshots in the reference's CSV v1 format.

Byte-level check against two snapshots the reference ships
(tests/golden/csv_snapshots.npz, made by tests/golden/make_golden.py): the
header is rebuilt from the values it prints and every line except the
Timestamp must come out identical; the 64 stored particle rows are rewritten
from their own parsed values and must match character for character.  Then a
write/read round trip (host only) and, on the GPU, a context's snapshot
against its downloaded state."""
import numpy as np
import pytest

from conftest import golden


def _meta_from_header(G, lines):
    kv = {}
    for ln in lines:
        if ln.startswith("# ") and ": " in ln:
            k, v = ln[2:].split(": ", 1)
            kv[k] = v
    m = G.CsvMeta()
    m.step = int(kv["Step"])
    m.time = float(kv["Time (code)"])
    names = {"Standard SPH": G.SSPH, "Density Independent SPH": G.DISPH, "Godunov SPH": G.GSPH}
    m.sph_type = names.get(kv["SPH Type"], 99)
    m.kernel = {"Cubic Spline": G.CUBIC_SPLINE, "Wendland C4": G.WENDLAND}.get(kv["Kernel"], 99)
    m.gamma = float(kv["Gamma"])
    m.g_constant = float(kv["G"])
    m.neighbor_number = int(kv["Neighbor Number"])
    m.use_gravity = kv["Gravity"] == "enabled"
    m.use_balsara = kv["Balsara Switch"] == "enabled"
    m.use_time_dependent_av = kv["Time-Dependent AV"] == "enabled"
    m.kinetic = float(kv["Kinetic"].split(" [")[0])
    m.thermal = float(kv["Thermal"].split(" [")[0])
    m.potential = float(kv["Potential"].split(" [")[0])
    m.precision = 16
    m.timestamp = kv["Timestamp"].encode()
    return m


def _rows_to_fields(G, rows):
    vals = [r.split(",") for r in rows]
    ids = np.array([int(v[0]) for v in vals], dtype=np.int64)
    fields = {}
    for c, name in enumerate(G.CSV_FIELDS):
        col = [v[c + 1] for v in vals]
        fields[name] = np.array([float(x) for x in col])
    return fields, ids


@pytest.mark.parametrize("tag", ["sr_sod", "resume"])
def test_writer_reproduces_reference_snapshot(G, tmp_path, tag):
    lines = [str(x) for x in golden("csv_snapshots.npz")[tag]]
    head, rows = lines[:51], lines[51:]
    meta = _meta_from_header(G, head)
    fields, ids = _rows_to_fields(G, rows) if rows else ({f: np.zeros(0) for f in G.CSV_FIELDS}, None)
    path = str(tmp_path / "snap.csv")
    G.csv_write(path, fields, meta, ids=ids)
    with open(path) as f:
        mine = f.read().split("\n")
    assert len(mine) == len(head) + len(rows) + 1 and mine[-1] == ""
    for k, (a, b) in enumerate(zip(mine[:51], head)):
        if b.startswith("# Particle Count: "):
            assert a == f"# Particle Count: {len(rows)}"
        else:
            assert a == b, (k, a, b)
    for a, b in zip(mine[51:], rows):
        assert a == b


def test_round_trip(G, tmp_path):
    rng = np.random.default_rng(7)
    n = 1000
    fields = {f: rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n) for f in G.CSV_FIELDS}
    fields["neighbor"] = rng.integers(0, 500, n).astype(np.float64)
    meta = G.CsvMeta(step=12, time=0.125, sph_type=G.DISPH, kernel=G.WENDLAND, gamma=5.0 / 3.0, g_constant=1.0,
                     neighbor_number=128, kinetic=1.5, thermal=2.5, potential=-3.0, precision=16)
    path = str(tmp_path / "rt.csv")
    G.csv_write(path, fields, meta)
    back, ids, m2 = G.csv_read(path)
    np.testing.assert_array_equal(ids, np.arange(n))
    for f in G.CSV_FIELDS:
        np.testing.assert_array_equal(back[f], fields[f], err_msg=f)
    assert (m2.step, m2.time, m2.gamma, m2.neighbor_number) == (12, 0.125, 5.0 / 3.0, 128)
    assert (m2.kinetic, m2.thermal, m2.potential) == (1.5, 2.5, -3.0)


@pytest.mark.gpu
def test_context_snapshot(gpu, tmp_path):
    p = gpu.config_params("evrard_ssph")
    with gpu.Simulation(p) as sim:
        sim.upload(gpu.sample_evrard(12))
        sim.initialize()
        sim.integrate()
        path = str(tmp_path / "ctx.csv")
        sim.write_csv(path, step=1)
        st = sim.download(gpu.CSV_FIELDS)
        k, u, w, _ = sim.energies()
        t, _ = sim.time_dt()
    back, ids, meta = gpu.csv_read(path)
    np.testing.assert_array_equal(ids, np.arange(len(st["pos_x"])))
    for f in gpu.CSV_FIELDS:
        np.testing.assert_array_equal(back[f], st[f], err_msg=f)
    assert (meta.step, meta.time) == (1, t)
    assert (meta.kinetic, meta.thermal, meta.potential) == (k, u, w)
    # resume (load_for_resume): same particles and time in a fresh context
    with gpu.Simulation(p) as sim2:
        assert sim2.read_csv(path) == 1
        again = sim2.download(gpu.CSV_FIELDS)
        t2, _ = sim2.time_dt()
    assert t2 == t
    for f in gpu.CSV_FIELDS:
        if f != "neighbor":
            np.testing.assert_array_equal(again[f], st[f], err_msg=f)
