"""The numpy initial conditions of the benchmark workloads (ics.py) agree with
the C generators of the library (host/samples.cpp) to the last bit or two,
and the library-free parameter defaults (sphparams.py) equal the C ones."""
import ctypes

import numpy as np
import pytest


@pytest.mark.parametrize("make", ["evrard", "shear", "tube"])
def test_ics_match_c_generators(G, make):
    import ics
    if make == "evrard":
        a, b = ics.evrard(24), G.sample_evrard(24)
    elif make == "shear":
        dx = (0.1875 / 3e4) ** (1 / 3)
        a, b = ics.shear_layer(dx), G.sample_shear_layer(dx)
    else:
        dx = (0.0025 / 3e4) ** (1 / 3)
        a, b = ics.shock_tube(dx), G.sample_shock_tube(dx)
    assert set(a) == set(b)
    for f in a:
        assert a[f].shape == b[f].shape, f
        scale = np.maximum(np.abs(b[f]), 1e-300)
        assert np.all(np.abs(a[f] - b[f]) <= 4.5e-16 * scale), f


def test_python_defaults_equal_c_defaults(G):
    import sphparams as SP
    a, b = G.default_params(), SP.defaults()
    assert bytes(a) == bytes(b)
    for name in ("evrard_ssph", "shear_disph", "tube_gsph", "tube_gdisph", "evrard_disph"):
        assert ctypes.sizeof(SP.config_params(name)) == ctypes.sizeof(G.Params)
