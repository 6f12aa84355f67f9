"""Host side of the printing-step output: names and tables the GPU maps are filed
under, and the CellProperties restatement the GPU tests compare against."""
import os
import re

import numpy as np

from tests import cellprops as CP

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_state_names_match_the_generated_headers():
    from chaste_b200.codegen import STATE_NAMES

    for model, header in ((0, "lr91.h"), (1, "tt06.h")):
        with open(os.path.join(ROOT, "chaste_b200", "csrc", "models", header)) as f:
            text = f.read()
        names = re.search(r"kStateNames\[\d+\] = \{([^}]*)\}", text).group(1)
        assert [x.strip().strip('"') for x in names.split(",")] == STATE_NAMES[model]


def test_post_processing_dataset_names():
    """PostProcessingWriter::ConvertToHdf5FriendlyString (PostProcessingWriter.cpp:394-416)."""
    from chaste_b200.heart import MonodomainProblem as P

    assert P._hdf5_friendly(-30.0) == "_minus_30"
    assert P._hdf5_friendly(-30.5) == "_minus_30pt50"
    assert P._hdf5_friendly(0.0) == "_0"
    assert P._hdf5_friendly(12.25) == "_12pt25"


def test_heart_config_post_processing_requests():
    from chaste_b200.heart import HeartConfig

    hc = HeartConfig.Instance()
    hc.Reset()
    assert not hc.IsPostProcessingRequested()
    hc.SetApdMaps([(90, -30)])
    assert hc.IsPostProcessingRequested() and hc.apd_maps == [(90.0, -30.0)]
    hc.Reset()
    assert not hc.IsPostProcessingRequested()


def _trace(n_aps, unfinished):
    """A synthetic paced trace: resting -85 mV, upstrokes to +40 mV, 300 ms plateaus."""
    t = np.arange(0.0, 500.0 * n_aps + (150.0 if unfinished else 0.0), 0.5)
    v = np.full(t.size, -85.0)
    for k in range(n_aps + (1 if unfinished else 0)):
        t0 = 10.0 + 500.0 * k
        up = (t >= t0) & (t < t0 + 2.0)
        v[up] = -85.0 + (t[up] - t0) / 2.0 * 125.0
        plat = (t >= t0 + 2.0) & (t < t0 + 300.0)
        v[plat] = 40.0 - (t[plat] - t0 - 2.0) / 298.0 * 60.0
        down = (t >= t0 + 300.0) & (t < t0 + 320.0)
        v[down] = -20.0 - (t[down] - t0 - 300.0) / 20.0 * 65.0
    return t, v


def test_cellprops_restatement_counts_unfinished_action_potentials():
    t, v = _trace(2, unfinished=True)
    p = CP.calculate_properties(t, v)
    assert len(p["onsets"]) == 3 and len(p["max_up"]) == 3 and p["unfinished"]
    apd = CP.action_potential_durations(t, v, p, 90.0)
    assert len(apd) == 2 and np.allclose(apd, apd[0])
    apd_map, up_t, up_v = CP.node_maps(t, np.stack([v, np.full_like(v, -85.0)], axis=1))
    assert len(apd_map[0]) == 2 and apd_map[1] == [0.0] and up_t[1] == [0.0] and up_v[1] == [0.0]
    assert CP.conduction_velocities([1.0, 501.0], [3.0, 503.0, 1003.0], 0.5, False) == [0.25, 0.25]
    assert CP.conduction_velocities([], [3.0], 0.5, False) == [0.0]
