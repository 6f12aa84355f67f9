"""Host-side parts of the cable fitting API: the region and probe maps, the
default configuration, and argument checks that fail before any device work."""
import ctypes as C

import numpy as np
import pytest

from tests import cable_cases as CC


def test_region_maps_match_the_kernel_rule(native):
    from chaste_b200 import fitting as F

    for n, R in ((1000, 4), (7, 3), (2, 1), (64, 8)):
        nr, er = F.node_regions(n, R), F.element_regions(n, R)
        assert nr.min() == 0 and nr.max() == R - 1 and np.all(np.diff(nr) >= 0)
        assert er.size == n - 1 and er.max() == R - 1 and np.all(np.diff(er) >= 0)
        np.testing.assert_array_equal(nr, CC.node_regions(n, R))
        np.testing.assert_array_equal(er, CC.element_regions(n, R))
    assert np.bincount(F.node_regions(1000, 4)).tolist() == [250, 250, 250, 250]
    p = F.even_probes(1000, 20)
    assert p.size == 20 and p[0] == 0 and p[-1] == 999


def test_default_cable_config(native):
    from chaste_b200 import fitting as F

    c = F.default_cable_config()
    assert (c.n_nodes, c.h, c.time_step, c.n_steps, c.n_regions, c.checkpoint_every) == (1000, 0.01, 0.01, 40000,
                                                                                           4, 200)
    assert (c.conductivity, c.surface_area_to_volume_ratio, c.capacitance) == (1.75, 1400.0, 1.0)
    assert c.n_stimulated_nodes == 2 and c.stimulus_magnitude == -5e5 and c.ksp_tolerance == 1e-8


@pytest.mark.parametrize("field,value", [("n_nodes", 1025), ("n_nodes", 1), ("n_regions", 9), ("n_regions", 0),
                                         ("checkpoint_every", 0), ("time_step", 0.0), ("n_steps", 0),
                                         ("model", 5)])
def test_cable_create_rejects_bad_configs_before_touching_a_device(native, field, value):
    from chaste_b200 import fitting as F

    c = F.default_cable_config()
    setattr(c, field, value)
    probes = np.array([1, 5], dtype=np.int32)
    h = C.c_void_p()
    assert native.lib().cg_cable_create(C.byref(c), native.iptr(probes), 2, 0, C.byref(h)) == 1


def test_cable_create_rejects_bad_probes(native):
    from chaste_b200 import fitting as F

    c = F.default_cable_config()
    h = C.c_void_p()
    for probes in ([1, 1], [-1, 4], [0, 1000]):
        p = np.array(probes, dtype=np.int32)
        assert native.lib().cg_cable_create(C.byref(c), native.iptr(p), p.size, 0, C.byref(h)) == 1
