"""FluidForce's pair lists built from the gather lists after PreInteraction
(csrc/flist.cu) against the symmetric tree walk.

The force sums over the pairs with r < max(h_i, h_j); the reference finds them
with its is_ij tree search and the pair test in the force loop.  Here the
lists come from one scan of the gather lists.  The sets must be identical to
the tree walk's lists filtered by that test, with no duplicates, for periodic
and open boxes, one- and 32-particle leaves, iterative and fixed h."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _min_image(d, L):
    """include/periodic.hpp:34-72: the closest of d, d + L, d - L, ties to the earlier."""
    b, c = d + L, d - L
    ad, ab, ac = np.abs(d), np.abs(b), np.abs(c)
    out = np.where((ad <= ab) & (ad <= ac), d, np.where((ab <= ac) & (ab <= ad), b, c))
    return np.where(np.abs(d) <= 0.5 * L, d, out)


def _sets_from_walk(G, p, st, off, ids):
    x = np.stack([st["pos_x"], st["pos_y"], st["pos_z"]], 1)
    h = st["sml"]
    L = np.array(p.range_max[:]) - np.array(p.range_min[:])
    out = []
    for i in range(len(h)):
        js = ids[off[i]:off[i + 1]]
        d = x[i][None, :] - x[js]
        if p.periodic:
            for k in range(3):
                d[:, k] = _min_image(d[:, k], L[k])
        r = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        keep = r < np.maximum(h[i], h[js])
        out.append(set(js[keep].tolist()))
    return out


CASES = {
    "evrard_ssph": lambda G: (G.config_params("evrard_ssph"), G.sample_evrard(14)),
    "evrard_leaf32": lambda G: (G.default_params(sph_type=G.SSPH, kernel=G.WENDLAND, neighbor_number=32,
                                                 leaf_particle_num=32, use_gravity=1), G.sample_evrard(14)),
    "shear_disph": lambda G: (G.config_params("shear_disph", neighbor_number=64), G.sample_shear_layer(0.04)),
    "tube_gsph": lambda G: (G.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1)),
                            G.sample_shock_tube(0.02, ly=0.1)),
    "evrard_fixed_h": lambda G: (G.config_params("evrard_ssph", iterative_sml=0), G.sample_evrard(14)),
}


def test_force_lists_when_gather_radius_too_small(gpu):
    """A density 8x too high makes the gather radius (the guessed h x 1.2) about
    0.6 of the final h; whichever lists FluidForce then takes, built or walked,
    hold exactly the pairs r < max(h_i, h_j)."""
    p = gpu.config_params("evrard_ssph")
    fields = gpu.sample_evrard(14)
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        sim.integrate()
        st = sim.download()
        st["dens"] = st["dens"] * 8.0
        sim.upload(st)
        sim.set_initial_smoothing(False)
        sim.tree_make()
        sim.pre_interaction()
        off, ids = sim.force_pairs()
        pos = sim.download(["pos_x", "pos_y", "pos_z", "sml"])
        woff, wids = sim.neighbor_search(is_ij=True)
    want = _sets_from_walk(gpu, p, pos, woff, wids)
    for i in range(len(pos["sml"])):
        got = ids[off[i]:off[i + 1]]
        assert len(got) == len(set(got.tolist())) and set(got.tolist()) == want[i], i


@pytest.mark.parametrize("case", sorted(CASES))
def test_force_lists_equal_tree_walk_pairs(gpu, case):
    p, fields = CASES[case](gpu)
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        sim.integrate()
        c = sim.counters()
        assert c["force_list_builds"] >= 1, c
        # the state of the last step: its tree, its h; lists built by the pre-interaction
        sim.tree_make()
        sim.pre_interaction()
        before = sim.counters()["force_list_builds"]
        off, ids = sim.force_pairs()
        # two calls (sizes, then ids), both on the built lists, not the walk's
        assert sim.counters()["force_list_builds"] == before + 2
        st = sim.download(["pos_x", "pos_y", "pos_z", "sml"])
        woff, wids = sim.neighbor_search(is_ij=True)
    want = _sets_from_walk(gpu, p, st, woff, wids)
    n = len(st["sml"])
    for i in range(n):
        got = ids[off[i]:off[i + 1]]
        assert len(got) == len(set(got.tolist())), (case, i, "duplicate")
        assert set(got.tolist()) == want[i], (case, i)
