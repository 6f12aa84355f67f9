"""The oracle's cable restatement (forward and discrete adjoint) on the CPU.

Its forward run is pinned to the oracle tissue (the monodomain restatement
checked against Chaste's own known answers) on the same cable, and its adjoint
gradient to central differences of its own loss; the GPU cable kernels are
then checked against it."""
import numpy as np
import pytest

from tests import cable_cases as CC

EPS = 1e-6


@pytest.fixture(scope="module")
def O(oracle):
    return oracle


def test_cable_forward_matches_oracle_tissue(O):
    cfg = CC.PlainCableConfig(n_nodes=90, n_steps=1500, n_regions=3)
    probes = CC.even_probes(cfg.n_nodes, 7)
    rng = np.random.default_rng(2)
    for params in (np.ones((3, 7)), CC.lognormal_params(rng, 1, 3, 7, 0.3)[0]):
        ref = CC.oracle_traces(O, cfg, params, probes)
        got = O.cable_run(CC.oracle_config(O, cfg), params, probes, traces=True)["traces"]
        err = np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= 1e-6, err
        assert ref.max() > 0.0


def test_cable_adjoint_matches_central_differences(O):
    cfg = CC.PlainCableConfig(n_nodes=60, n_steps=1200, n_regions=2, rtol=1e-12)
    probes = CC.even_probes(cfg.n_nodes, 5)
    oc = CC.oracle_config(O, cfg)
    rng = np.random.default_rng(4)
    truth = CC.lognormal_params(rng, 1, 2, 7, 0.3)[0]
    targets = O.cable_run(oc, truth, probes, traces=True)["traces"]
    p0 = np.ones((2, 7))
    res = O.cable_run(oc, p0, probes, targets, gradient=True)
    g = res["grad"]
    fd = np.zeros_like(g)
    for k in range(g.size):
        pp, pm = p0.copy(), p0.copy()
        pp.flat[k] += EPS
        pm.flat[k] -= EPS
        fd.flat[k] = (O.cable_run(oc, pp, probes, targets)["loss"] - O.cable_run(oc, pm, probes, targets)["loss"]) \
            / (2 * EPS)
    scale = np.max(np.abs(fd))
    err = np.abs(g - fd) / np.maximum(np.abs(fd), 1e-3 * scale)
    assert res["loss"] > 0
    assert err.max() <= 1e-4, (err.max(), g, fd)


def test_cable_adjoint_matches_forward_mode(O):
    """The reverse sweep (generated reverse products) against a tangent-linear run per
    parameter (the primal cell-model templates on dual numbers): no finite-difference
    step, so it also holds where a perturbation would move a node across one of
    LR91's discontinuous gate-rate switches at -40 mV."""
    cfg = CC.PlainCableConfig(n_nodes=120, n_steps=2000, n_regions=3, rtol=1e-12, checkpoint_every=128)
    probes = CC.even_probes(cfg.n_nodes, 6)
    oc = CC.oracle_config(O, cfg)
    truth = CC.lognormal_params(np.random.default_rng(8), 1, 3, 7, 0.3)[0]
    targets = O.cable_run(oc, truth, probes, traces=True)["traces"]
    p0 = CC.lognormal_params(np.random.default_rng(9), 1, 3, 7, 0.1)[0]
    g = O.cable_run(oc, p0, probes, targets, gradient=True)["grad"]
    gt = O.cable_tangent_gradient(oc, p0, probes, targets)
    err = np.abs(g - gt) / np.maximum(np.abs(gt), 1e-3 * np.max(np.abs(gt)))
    assert err.max() <= 1e-6, (err.max(), g, gt)
