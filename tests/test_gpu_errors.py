"""Failure detection on the device without faulting it: conditions the
reference throws on come back as status codes / SPHException, and list
capacity overflow is recovered by growing the buffer and re-running."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cube(n1, h):
    g = (np.arange(n1) + 0.5) / n1
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    n = n1 ** 3
    return {"pos_x": x.ravel().copy(), "pos_y": y.ravel().copy(), "pos_z": z.ravel().copy(),
            "mass": np.full(n, 1.0 / n), "dens": np.ones(n), "ene": np.ones(n), "sml": np.full(n, h)}


def test_neighbor_overflow_is_fatal(gpu):
    """More than neighborNumber * 1000 neighbours (src/bhtree.cpp:129-135)."""
    f = _cube(13, 0.05)                       # 2197 particles
    f["sml"][0] = 10.0                        # one particle sees them all
    p = gpu.default_params(neighbor_number=1)  # limit 1000
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.tree_make()
        with pytest.raises(gpu.SPHException, match="overflow"):
            sim.neighbor_search(is_ij=False)
        # the context stays usable
        sim.set_walk_mode(0)
        f["sml"][0] = 0.05
        sim.upload(f)
        sim.tree_make()
        off, _ = sim.neighbor_search(is_ij=False)
        assert off[-1] > 0


def test_nonfinite_position_is_reported(gpu):
    f = _cube(8, 0.2)
    f["pos_x"][7] = np.nan
    with gpu.Simulation(gpu.default_params()) as sim:
        sim.upload(f)
        with pytest.raises(gpu.SPHException, match="non-finite"):
            sim.tree_make()
        f["pos_x"][7] = 0.5
        sim.upload(f)
        sim.tree_make()


def test_capacity_grows_and_walk_reruns(gpu):
    """Lists longer than the initial capacity (3 x neighborNumber) are
    counted, the buffer grows and the walk re-runs; the result equals the
    exhaustive lists."""
    f = _cube(12, 0.3)
    p = gpu.default_params(neighbor_number=8)
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.tree_make()
        sim.reset_counters()
        off, ids = sim.neighbor_search(is_ij=False)
        c = sim.counters()
        assert c["retries"] >= 1 and c["gather_capacity"] >= c["max_gather"] > 24
        eoff, eids = sim.neighbor_search(is_ij=False, exhaustive=True)
    np.testing.assert_array_equal(off, eoff)
    for i in range(len(off) - 1):
        np.testing.assert_array_equal(np.sort(ids[off[i]:off[i + 1]]), np.sort(eids[eoff[i]:eoff[i + 1]]))


def test_calls_out_of_order_are_rejected(gpu):
    with gpu.Simulation(gpu.default_params()) as sim:
        with pytest.raises(gpu.SPHException):
            sim.tree_make()                    # nothing uploaded
        sim.upload(_cube(6, 0.3))
        with pytest.raises(gpu.SPHException, match="before tree"):
            sim.fluid_force()


def test_node_pool_error_does_not_outlive_a_new_upload(gpu):
    """Two particles closer than the deepest level can split need a chain of
    more nodes than the 5 N + 2 pool holds: the reference's "There is no free
    node." (src/bhtree.cpp:222-224).  A later valid upload of the same size
    builds its tree."""
    f = {"pos_x": np.array([0.5, 0.5 + 1e-9]), "pos_y": np.full(2, 0.5), "pos_z": np.full(2, 0.5),
         "mass": np.full(2, 0.5), "dens": np.ones(2), "ene": np.ones(2), "sml": np.full(2, 0.1)}
    with gpu.Simulation(gpu.default_params()) as sim:
        sim.upload(f)
        with pytest.raises(gpu.SPHException, match="no free node"):
            sim.tree_make()
        f["pos_x"][1] = -0.5
        sim.upload(f)
        sim.tree_make()
        assert sim.counters()["node_count"] >= 3


@pytest.mark.parametrize("bits,what", [(1, "mass"), (2, "set_kernel"), (4, "gravity walk"),
                                       (8, "mixed gravity walk")])
def test_pass_guard_is_reported_at_the_next_wait(gpu, bits, what):
    """The bottom-up passes and the gravity walks bound their loops and set a
    status bit instead of looping on a corrupt tree; the bit is reported by
    the next call that waits on the stream, and the context stays usable."""
    p = gpu.config_params("evrard_ssph")
    f = gpu.sample_evrard(8)
    with gpu.Simulation(p) as sim:
        sim.upload(f)
        sim.initialize()
        gpu.lib().sphgpu_test_flag_pass_guard(sim._h, bits)
        with pytest.raises(gpu.SPHException, match=what):
            sim.synchronize()
        sim.synchronize()                      # reported once, then cleared
        gpu.lib().sphgpu_test_flag_pass_guard(sim._h, bits)
        with pytest.raises(gpu.SPHException, match="bounded device pass"):
            sim.integrate()                    # tree_make's wait sees it
        sim.upload(f)
        sim.initialize()
        sim.integrate()
