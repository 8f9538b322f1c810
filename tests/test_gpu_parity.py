"""GPU parity: the CUDA path (through the C ABI) against the oracle and the
reference's golden fixtures.

Bars (FP64 plain form):
  * octree topology, node geometry, mass and centre of mass: bit-identical;
  * neighbour lists: identical as sets to the reference's tree lists and, for
    the gather search, its exhaustive lists;
  * gravity (same tree, same inputs): bit-identical;
  * predict / correct / timestep on identical inputs: bit-identical;
  * PreInteraction and FluidForce from identical inputs: sums are taken in a
    different order than the reference's distance-sorted loops, so they agree
    to rounding — relative error <= 1e-12 at the median and <= 1e-9 at the
    99.9th percentile (a Newton iteration whose |dh| sits on the 1e-4
    convergence threshold can end one iteration apart; such particles are
    allowed up to 1e-6 and must be fewer than 0.1 %).
"""
import numpy as np
import pytest

from conftest import golden, params_from_bytes, rel_err

pytestmark = pytest.mark.gpu

SMALL = ["evrard_ssph", "evrard_ssph_gauss", "evrard_disph", "tube_gsph", "tube_gsph_hll", "shear_disph", "tube_gdisph",
         "tube_gdisph_1st"]
PRE_FIELDS = ["dens", "pres", "sml", "gradh", "balsara", "alpha"]


def _case(G, name):
    g = golden(f"steps_{name}.npz")
    p = params_from_bytes(G, g["params"])
    fields = {k[3:]: g[k] for k in g.files if k.startswith("ic_")}
    return g, p, fields


def _close(a, b, what, median=1e-12, p999=1e-9, worst=1e-6, scale=None):
    """Rounding-level agreement; `scale` switches to error / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if scale is None:
        nz = np.abs(b) > 0
        e = rel_err(a[nz], b[nz]) if nz.any() else np.zeros(1)
        e = np.concatenate([e, np.abs(a[~nz])])
    else:
        e = np.abs(a - b) / scale
    assert np.median(e) <= median, (what, np.median(e))
    assert np.quantile(e, 0.999) <= p999, (what, np.quantile(e, 0.999))
    assert e.max() <= worst, (what, e.max(), int(np.argmax(e)))


def _state(sim, names=None):
    return sim.download(names)


@pytest.mark.parametrize("name", ["evrard_ssph", "tube_gsph", "shear_disph"])
def test_tree_nodes_bitexact(gpu, O, name):
    g, p, fields = _case(gpu, name)
    o = O.Oracle(p, fields)
    o.tree_make()
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.tree_make()
        gi, gd = sim.tree_nodes()
    oi, od = o.tree_nodes()
    assert gi.shape == oi.shape
    np.testing.assert_array_equal(gi[:, :2], oi[:, :2])
    np.testing.assert_array_equal(gi[1:, 2], oi[1:, 2])      # the reference never counts the root
    np.testing.assert_array_equal(gd[:, :8], od[:, :8])      # centre, edge, mass, centre of mass


def test_tree_nodes_leaf32_evrard(gpu, O):
    """Multi-particle leaves (leafParticleNumber = 32): list order and centre of mass."""
    p = gpu.default_params(sph_type=gpu.SSPH, kernel=gpu.WENDLAND, neighbor_number=32, leaf_particle_num=32,
                           use_gravity=1)
    fields = gpu.sample_evrard(20)
    o = O.Oracle(p, fields)
    o.tree_make()
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.tree_make()
        gi, gd = sim.tree_nodes()
    oi, od = o.tree_nodes()
    np.testing.assert_array_equal(gi[:, :2], oi[:, :2])
    np.testing.assert_array_equal(gd[:, :8], od[:, :8])


@pytest.mark.parametrize("name", ["evrard_ssph", "tube_gsph", "shear_disph"])
def test_neighbor_sets_match_reference(gpu, name):
    """Gather and symmetric lists equal the reference's (golden) lists as sets."""
    g = golden(f"lists_{name}.npz")
    s = golden(f"steps_{name}.npz")
    p = params_from_bytes(gpu, s["params"])
    fields = {k[len("state_"):]: g[k] for k in g.files if k.startswith("state_")}
    n = len(fields["pos_x"])
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.tree_make()
        sim.set_kernel()
        for ij in (0, 1):
            off, ids = sim.neighbor_search(is_ij=bool(ij))
            roff, rids = g[f"tree_ij{ij}_off"], g[f"tree_ij{ij}_ids"]
            np.testing.assert_array_equal(off, roff)
            for i in range(n):
                a = np.sort(ids[off[i]:off[i + 1]])
                b = np.sort(rids[roff[i]:roff[i + 1]])
                np.testing.assert_array_equal(a, b, err_msg=f"particle {i} is_ij={ij}")
        # exhaustive predicate (gather radius): same sets as the tree search
        off, ids = sim.neighbor_search(is_ij=False, exhaustive=True)
        eoff, eids = g["exh_ij0_off"], g["exh_ij0_ids"]
        np.testing.assert_array_equal(off, eoff)
        for i in range(n):
            np.testing.assert_array_equal(np.sort(ids[off[i]:off[i + 1]]), np.sort(eids[eoff[i]:eoff[i + 1]]))
        off1, ids1 = sim.neighbor_search(is_ij=True, exhaustive=True)
        eoff, eids = g["exh_ij1_off"], g["exh_ij1_ids"]
        np.testing.assert_array_equal(off1, eoff)


@pytest.mark.parametrize("name", ["evrard_ssph", "evrard_disph", "shear_disph"])
def test_gravity_and_kick_drift_bitexact(gpu, O, name):
    g, p, fields = _case(gpu, name)
    st = {k[3:]: g[k] for k in g.files if k.startswith("s1_")}
    st = {k: v for k, v in st.items() if k in gpu.FIELD_INDEX}
    st["acc_x"] = np.zeros_like(st["acc_x"])
    st["acc_y"] = np.zeros_like(st["acc_x"])
    st["acc_z"] = np.zeros_like(st["acc_x"])
    o = O.Oracle(p, st)
    o.tree_make()
    o.gravity_force()
    dt = float(g["dt"][2])
    o.set_dt(dt)
    o.predict()
    ref = o.download()
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.gravity_force()
        sim.set_dt(dt)
        sim.predict()
        out = sim.download()
    for f in ("acc_x", "acc_y", "acc_z", "phi", "pos_x", "pos_y", "pos_z", "vel_x", "velp_z", "ene", "ene_p",
              "sound"):
        np.testing.assert_array_equal(out[f], ref[f], err_msg=f)


def test_gravity_direct_bitexact(gpu, O):
    g, p, fields = _case(gpu, "evrard_ssph")
    st = {k[3:]: g[k] for k in g.files if k.startswith("s0_") and k[3:] in gpu.FIELD_INDEX}
    for k in ("acc_x", "acc_y", "acc_z"):
        st[k] = np.zeros_like(st["pos_x"])
    o = O.Oracle(p, st, exhaustive=True)
    o.gravity_force(direct=True)
    ref = o.download()
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.tree_make()
        sim.gravity_force(direct=True)
        out = sim.download()
    for f in ("acc_x", "acc_y", "acc_z", "phi"):
        np.testing.assert_array_equal(out[f], ref[f], err_msg=f)


@pytest.mark.parametrize("name", SMALL)
def test_pre_interaction_from_identical_state(gpu, O, name):
    g, p, fields = _case(gpu, name)
    st = {k[3:]: g[k] for k in g.files if k.startswith("s1_") and k[3:] in gpu.FIELD_INDEX}
    dt = float(g["dt"][2])
    o = O.Oracle(p, st)
    o.set_first(False)
    o.set_dt(dt)
    o.tree_make()
    o.pre_interaction()
    ref = o.download()
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.set_initial_smoothing(False)
        sim.set_dt(dt)
        sim.tree_make()
        sim.pre_interaction()
        out = sim.download()
        hv = sim.h_per_v_sig()
    np.testing.assert_array_equal(out["neighbor"], ref["neighbor"])
    for f in PRE_FIELDS:
        if p.sph_type == gpu.GSPH and f in ("gradh", "balsara", "alpha"):
            continue
        _close(out[f], ref[f], f)
    if p.sph_type in (gpu.GSPH, gpu.GDISPH) and p.gsph_2nd_order:
        for f in [x for x in gpu.FIELDS if x.startswith("grad_")]:
            sc = np.max(np.abs(ref[f])) + 1e-300
            _close(out[f], ref[f], f, scale=sc, median=1e-12, p999=1e-10)
    assert hv == pytest.approx(o.h_per_v_sig(), rel=1e-9)


@pytest.mark.parametrize("name", SMALL)
def test_fluid_force_from_identical_state(gpu, O, name):
    g, p, fields = _case(gpu, name)
    o = O.Oracle(p, fields)
    o.initialize()
    o.integrate()
    st = o.download()          # a post-pre state (dens, pres, gradh, grads from the same call)
    st = {k: v for k, v in st.items() if k in gpu.FIELD_INDEX}
    o.tree_make()
    o.set_kernel()
    o.set_dt(float(g["dt"][1]))
    o.fluid_force()
    ref = o.download()
    with gpu.Simulation(p) as sim:
        sim.upload(st)
        sim.set_dt(float(g["dt"][1]))
        sim.tree_make()
        sim.set_kernel()
        sim.fluid_force()
        out = sim.download()
    amax = max(np.max(np.abs(ref[f])) for f in ("acc_x", "acc_y", "acc_z"))
    for f in ("acc_x", "acc_y", "acc_z"):
        _close(out[f], ref[f], f, scale=amax, median=1e-14, p999=1e-12, worst=1e-10)
    dmax = np.max(np.abs(ref["dene"])) + 1e-300
    _close(out["dene"], ref["dene"], "dene", scale=dmax, median=1e-14, p999=1e-12, worst=1e-10)


@pytest.mark.parametrize("name", SMALL)
def test_steps_against_reference_golden(gpu, name):
    """initialize + 2 integrate steps against the reference's own states."""
    g, p, fields = _case(gpu, name)
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        for s in range(3):
            out = sim.download()
            np.testing.assert_array_equal(out["neighbor"] >= 0, True)
            for f in ("dens", "sml", "pres"):
                _close(out[f], g[f"s{s}_{f}"], f"step {s} {f}", median=1e-11, p999=1e-8, worst=1e-5)
            amax = max(np.max(np.abs(g[f"s{s}_acc_{a}"])) for a in "xyz")
            for a in "xyz":
                _close(out[f"acc_{a}"], g[f"s{s}_acc_{a}"], f"step {s} acc_{a}", scale=amax, median=1e-11,
                       p999=1e-8, worst=1e-5)
            if s > 0:
                _, dt = sim.time_dt()
                assert dt == pytest.approx(float(g["dt"][s]), rel=1e-9)
            if s < 2:
                sim.integrate()


def test_evrard_t0_golden(gpu):
    """The shipped Evrard t=0 snapshot (sample/evrard/results_new/00000.dat)."""
    g = golden("evrard_t0.npz")
    p = gpu.default_params(sph_type=gpu.SSPH, kernel=gpu.WENDLAND, neighbor_number=32, leaf_particle_num=32,
                           use_balsara_switch=1, use_time_dependent_av=1, av_alpha=1.0, use_gravity=1,
                           g_constant=1.0, gamma=1.66666666666666666667, cfl_sound=0.2, cfl_force=0.1)
    with gpu.Simulation(p) as sim:
        sim.upload(gpu.sample_evrard(30))
        sim.initialize()
        st = sim.download()
        k, u, w, _ = sim.energies()
    ids = g["ids"]
    for col, idx in zip(g["printed_columns"], g["printed_index"]):
        col = str(col)
        printed = g["printed"][:, idx]
        tol = 6e-6 * np.maximum(np.abs(printed), 1e-6 * np.max(np.abs(printed)))
        assert np.all(np.abs(st[col][ids] - printed) <= tol), col
    assert w == pytest.approx(float(g["w0_ref"]), rel=1e-12)
    assert abs(w - float(g["w0_printed"])) < 1e-6


def test_energies_match_oracle(gpu, O):
    g, p, fields = _case(gpu, "evrard_ssph")
    o = O.Oracle(p, fields)
    o.initialize()
    ko, uo, wo, mo = o.energies()
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        k, u, w, m = sim.energies()
    assert k == pytest.approx(ko, abs=1e-15) and u == pytest.approx(uo, rel=1e-13)
    assert w == pytest.approx(wo, rel=1e-10)
    np.testing.assert_allclose(m, mo, atol=1e-12)


@pytest.mark.parametrize("leaf", [4, 20, 100])
def test_gravity_bitexact_leaf_sizes(gpu, O, leaf):
    """Leaves of up to 100 particles (queues that fill inside one leaf):
    still bit-identical to the oracle."""
    p = gpu.config_params("evrard_ssph", leaf_particle_num=leaf)
    f = gpu.sample_evrard(16)
    n = len(f["pos_x"])
    f["sml"] = np.full(n, 0.12)
    for k in ("acc_x", "acc_y", "acc_z"):
        f[k] = np.zeros(n)
    o = O.Oracle(p, f)
    o.tree_make()
    o.gravity_force()
    ref = o.download()
    for prec in (gpu.FP64, gpu.MIXED):
        q = p.copy()
        q.precision = prec
        with gpu.Simulation(q) as sim:
            sim.upload(f)
            sim.tree_make()
            sim.gravity_force()
            out = sim.download()
        for k in ("acc_x", "acc_y", "acc_z", "phi"):
            if prec == gpu.FP64:
                np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
            else:
                scale = np.abs(ref[k]).max()
                assert np.median(np.abs(out[k] - ref[k])) <= 1e-6 * scale, k


def test_relaxation_against_reference_golden(gpu):
    """Three Lane-Emden relaxation steps against the reference's own states
    (the equilibrium term uses CUDA's pow, so agreement is to rounding)."""
    g = golden("relax_evrard.npz")
    p = params_from_bytes(gpu, g["params"])
    fields = {k[3:]: g[k] for k in g.files if k.startswith("ic_")}
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        for s in range(len(g["dt_relax"])):
            d = sim.relax_step(g["xi"], g["theta"], g["dtheta"], float(g["xi_1"]), float(g["alpha"]), float(g["K"]),
                               first=(s == 0))
            assert d == pytest.approx(float(g["dt_relax"][s]), rel=1e-10)
            out = sim.download()
            for f in ("pos_x", "pos_y", "pos_z"):
                _close(out[f], g[f"s{s}_{f}"], f"step {s} {f}", median=1e-14, p999=1e-12, worst=1e-10)
            np.testing.assert_array_equal(out["vel_x"], 0.0)
            amax = max(np.max(np.abs(g[f"s{s}_acc_{a}"])) for a in "xyz")
            for a in "xyz":
                _close(out[f"acc_{a}"], g[f"s{s}_acc_{a}"], f"step {s} acc_{a}", scale=amax, median=1e-12,
                       p999=1e-9, worst=1e-7)
