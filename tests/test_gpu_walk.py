"""The group neighbour walk against the per-lane walk (which replays the
reference's recursion test by test): identical sets on every workload type,
including the Evrard sphere with 32-particle leaves and a case with
particles placed exactly on other particles' search radius."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lists(sim, is_ij, mode):
    sim.set_walk_mode(mode)
    off, ids = sim.neighbor_search(is_ij=is_ij)
    return off, ids


def _same_sets(a, b):
    off_a, ids_a = a
    off_b, ids_b = b
    np.testing.assert_array_equal(off_a, off_b)
    for i in range(len(off_a) - 1):
        np.testing.assert_array_equal(np.sort(ids_a[off_a[i]:off_a[i + 1]]), np.sort(ids_b[off_b[i]:off_b[i + 1]]))


@pytest.mark.parametrize("case", ["evrard_ssph", "shear_disph", "tube_gsph", "evrard_leaf32"])
def test_group_walk_equals_per_lane_walk(gpu, case):
    if case == "evrard_leaf32":
        p = gpu.default_params(sph_type=gpu.SSPH, kernel=gpu.WENDLAND, neighbor_number=32, leaf_particle_num=32,
                               use_gravity=1)
        fields = gpu.sample_evrard(20)
    elif case == "shear_disph":
        p = gpu.config_params("shear_disph", neighbor_number=64)
        fields = gpu.sample_shear_layer(0.04)
    elif case == "tube_gsph":
        p = gpu.config_params("tube_gsph", range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.1, 0.1))
        fields = gpu.sample_shock_tube(0.02, ly=0.1)
    else:
        p = gpu.config_params("evrard_ssph")
        fields = gpu.sample_evrard(20)
    with gpu.Simulation(p) as sim:
        sim.upload(fields)
        sim.initialize()
        sim.integrate()
        sim.tree_make()
        sim.set_kernel()
        for ij in (False, True):
            _same_sets(_lists(sim, ij, 0), _lists(sim, ij, 1))


def test_group_walk_on_exact_radius(gpu):
    """Lattice particles whose sml equals a lattice distance: many pairs sit
    exactly on the radius, where the box tests decide."""
    n1 = 12
    g = (np.arange(n1) + 0.5) / n1
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    fields = {"pos_x": x.ravel().copy(), "pos_y": y.ravel().copy(), "pos_z": z.ravel().copy()}
    n = fields["pos_x"].size
    fields["mass"] = np.full(n, 1.0 / n)
    fields["dens"] = np.ones(n)
    fields["ene"] = np.ones(n)
    fields["sml"] = np.full(n, 2.0 / n1)  # exactly two lattice spacings (in FP: close to it)
    for periodic in (0, 1):
        p = gpu.default_params(periodic=periodic, range_min=(0.0, 0.0, 0.0), range_max=(1.0, 1.0, 1.0))
        with gpu.Simulation(p) as sim:
            sim.upload(fields)
            sim.tree_make()
            sim.set_kernel()
            for ij in (False, True):
                _same_sets(_lists(sim, ij, 0), _lists(sim, ij, 1))
