"""Skin (Verlet) gather lists (gather_skin, walk.cu): the lists of one walk at
(1 + skin) times the gather radius are reused, moved to each new tree's
particle order, while every gather sphere stays inside its list's sphere; the
consumers take exactly the reference's list members from them.  The steps
must equal those with a fresh exact walk every step: the same neighbour
counts and states to rounding (sums over the same sets in another order),
and the same tree and gravity bit for bit."""
import numpy as np
import pytest

import ics
import sphparams as SP
from test_gpu_parity import _close

pytestmark = pytest.mark.gpu

CASES = {
    "evrard_disph": lambda: (SP.config_params("evrard_disph", cfl_sound=0.05, cfl_force=0.025), ics.evrard(24)),
    "shear_disph": lambda: (SP.config_params("shear_disph"), ics.shear_layer(0.02)),
    "tube_gsph": lambda: (SP.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                          ics.shock_tube(0.01, ly=0.1)),
    "evrard_ssph_fixed_h": lambda: (SP.config_params("evrard_ssph", iterative_sml=0), ics.evrard(16)),
}


def _run(G, p, f, skin, steps):
    q = p.copy()
    q.gather_skin = skin
    with G.Simulation(q) as sim:
        sim.upload(f)
        sim.initialize()
        sim.reset_counters()
        out = []
        for _ in range(steps):
            sim.integrate()
            out.append(sim.download())
        return out, sim.counters()


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("skin", [0.05, 0.002])
def test_skin_lists_match_exact_walk(gpu, case, skin):
    p, f = CASES[case]()
    ref, c0 = _run(gpu, p, f, 0.0, 6)
    out, c1 = _run(gpu, p, f, skin, 6)
    assert c0["skin_reuses"] == 0
    if skin >= 0.05:
        assert c1["skin_reuses"] >= 1, c1     # the reuse path ran
    else:
        # a skin too thin to be reused widens (2x, then 4x, after two builds
        # in a row that served fewer than two steps); two unused builds at the
        # widest pause it (exact walks)
        assert c1["skin_builds"] <= 5, c1
    assert c1["skin_builds"] + c1["skin_reuses"] <= 6
    for s, (a, b) in enumerate(zip(out, ref)):
        np.testing.assert_array_equal(a["neighbor"], b["neighbor"], err_msg=f"step {s + 1}")
        for fld in ("dens", "sml", "pres", "ene"):
            _close(a[fld], b[fld], f"step {s + 1} {fld}", median=1e-12, p999=1e-9, worst=1e-6)
        amax = max(np.max(np.abs(b[f"acc_{x}"])) for x in "xyz")
        for x in "xyz":
            _close(a[f"acc_{x}"], b[f"acc_{x}"], f"step {s + 1} acc_{x}", scale=amax, median=1e-12, p999=1e-9,
                   worst=1e-6)


def test_skin_lists_export_exact_lists(gpu):
    """sphgpu_neighbor_search still returns the reference's lists (a fresh
    exact walk) after steps that reused skin lists."""
    p, f = CASES["shear_disph"]()
    p.gather_skin = 0.05
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        for _ in range(6):
            sim.integrate()
        assert sim.counters()["skin_reuses"] >= 1
        st = sim.download()
        off, ids = sim.neighbor_search(is_ij=False)
    q = p.copy()
    q.gather_skin = 0.0
    with gpu.Simulation(q) as sim:
        sim.upload({k: v for k, v in st.items() if not k.startswith("sr_")})
        sim.tree_make()
        off2, ids2 = sim.neighbor_search(is_ij=False)
    np.testing.assert_array_equal(off, off2)
    n = len(off) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    np.testing.assert_array_equal(np.sort(rows * n + ids), np.sort(rows * n + ids2))


def test_skin_lists_survive_uploads(gpu):
    """An upload of the same particle count keeps the skin lists (their rows
    follow the particles into caller order at the next tree build); an
    upload that moves particles past the skin forces a rebuild.  Steps with
    an upload before each equal those with exact walks."""
    p, f = CASES["evrard_disph"]()
    runs = []
    for skin in (0.0, 0.05):
        q = p.copy()
        q.gather_skin = skin
        with gpu.Simulation(q) as sim:
            sim.upload(f)
            sim.initialize()
            sim.reset_counters()
            outs = []
            moved = None
            for s in range(6):
                st = {k: v for k, v in sim.download().items() if not k.startswith("sr_")}
                if s == 3:
                    # a few particles moved by about one smoothing length
                    st["pos_x"] = st["pos_x"].copy()
                    st["pos_x"][:40] += 0.1
                    before = sim.counters()["skin_builds"]
                sim.upload(st)
                sim.set_initial_smoothing(False)
                sim.integrate()
                if s == 3:
                    moved = sim.counters()["skin_builds"] - before
                outs.append(sim.download())
            runs.append((outs, sim.counters(), moved))
    (ref, c0, _), (out, c1, moved) = runs
    assert c0["skin_reuses"] == 0
    # initialize built the lists; the steps around the move reuse them
    assert c1["skin_reuses"] >= 3, c1
    assert moved == 1, moved   # the moved particles outran the skin: one rebuild
    for s, (a, b) in enumerate(zip(out, ref)):
        np.testing.assert_array_equal(a["neighbor"], b["neighbor"], err_msg=f"step {s + 1}")
        for fld in ("dens", "sml", "pres", "ene"):
            _close(a[fld], b[fld], f"step {s + 1} {fld}", median=1e-12, p999=1e-9, worst=1e-6)
