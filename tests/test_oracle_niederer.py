"""The oracle's state-variable interpolation and backward-Euler cells pinned by
Chaste's Niederer et al. 2011 benchmark activation map
(TestNiederer2011BenchmarkSimulation::TestRunOnCoarsestMesh, tolerance 1.5e-3 ms).

The run takes about five minutes on one host core, so it is opt-in:
CHASTE_ORACLE_SLOW=1 python -m pytest tests/test_oracle_niederer.py
(last run: max |act - golden| = 7.8e-4 ms over the 4305 nodes).
"""
import os

import numpy as np
import pytest

from tests import tissue_cases as TC


@pytest.mark.skipif(os.environ.get("CHASTE_ORACLE_SLOW") != "1", reason="opt-in: about five minutes of CPU")
def test_oracle_niederer_activation_map(oracle, golden_dir):
    gold = np.loadtxt(golden_dir / "niederer_activation_h0.05_dt0.01.txt")
    o, xyz = TC.make_oracle(oracle, **TC.NIEDERER)
    assert xyz.shape[0] == gold.size
    act = TC.niederer_activation(o, gold.size)
    assert (act > 0).all()
    assert float(np.abs(act - gold).max()) <= 1.5e-3
