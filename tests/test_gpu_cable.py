"""Cable fitting on the GPU: forward runs against the oracle tissue, and the
adjoint gradient against central finite differences on the GPU (eps 1e-6, all
sets in one launch) and against the FP64 CPU reference gradient of the oracle.  The gradient checks solve to a tight tolerance (rtol 1e-12)
so the finite differences are not dominated by the CG stopping test."""
import numpy as np
import pytest

from tests import cable_cases as CC

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6    # probe voltages vs the oracle, relative to max(|V|, 1 mV)
GRAD_TOL = 1e-4   # adjoint vs central differences, relative
EPS = 1e-6        # central-difference step on the scale factors


@pytest.fixture(scope="module")
def env(native, oracle):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from chaste_b200 import fitting

    return native, oracle, fitting, torch


def _fd_sets(p0, eps):
    """2 x (R * stride) parameter sets: +eps then -eps on every entry."""
    R, S = p0.shape
    sets = np.repeat(p0[None], 2 * R * S, axis=0)
    for k in range(R * S):
        sets[2 * k].flat[k] += eps
        sets[2 * k + 1].flat[k] -= eps
    return sets


def _rel_err(g, fd):
    scale = max(np.max(np.abs(fd)), 1e-300)
    return np.abs(g - fd) / np.maximum(np.abs(fd), 1e-3 * scale)


def test_cable_forward_matches_oracle(env):
    N, O, F, torch = env
    cfg = CC.cable_config(N, n_nodes=120, n_steps=2500, n_regions=4)
    probes = F.even_probes(cfg.n_nodes, 8)
    rng = np.random.default_rng(7)
    params = np.concatenate([np.ones((1, 4, 7)), CC.lognormal_params(rng, 2, 4, 7, 0.3)])
    cable = F.Cable(cfg, probes)
    out = cable.forward(torch.tensor(params, device="cuda"), traces=True, iterations=True)
    tr = out["traces"].cpu().numpy()
    for s in range(params.shape[0]):
        ref = CC.oracle_traces(O, cfg, params[s], probes)
        err = np.max(np.abs(tr[s] - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= FWD_TOL, (s, err)
        assert ref.max() > 0.0   # the wave reached the probes
    assert int(out["iterations"].min()) > 0


def _gradient_case(F, CC, N, torch, n_nodes, n_steps, R, ckpt, seed=3):
    cfg = CC.cable_config(N, n_nodes=n_nodes, n_steps=n_steps, n_regions=R, checkpoint_every=ckpt, rtol=1e-12)
    probes = F.even_probes(n_nodes, 6)
    cable = F.Cable(cfg, probes)
    rng = np.random.default_rng(seed)
    truth = CC.lognormal_params(rng, 1, R, cable.stride, 0.3)
    targets = cable.forward(torch.tensor(truth, device="cuda"), traces=True)["traces"][0].contiguous()
    p0 = np.ones((1, R, cable.stride))
    return cfg, probes, cable, targets, p0


def test_adjoint_matches_gpu_central_differences(env):
    N, O, F, torch = env
    cfg, probes, cable, targets, p0 = _gradient_case(F, CC, N, torch, n_nodes=200, n_steps=3000, R=4, ckpt=200)
    d0 = torch.tensor(p0, device="cuda")
    out = cable.forward(d0, targets, keep_checkpoints=True)
    g = cable.backward(d0, targets).cpu().numpy()[0]
    sets = torch.tensor(_fd_sets(p0[0], EPS), device="cuda")
    loss = cable.forward(sets, targets)["loss"].cpu().numpy()
    fd = ((loss[0::2] - loss[1::2]) / (2 * EPS)).reshape(g.shape)
    err = _rel_err(g, fd)
    assert np.all(np.isfinite(g))
    assert float(out["loss"][0]) > 0
    assert err.max() <= GRAD_TOL, (err.max(), np.unravel_index(err.argmax(), err.shape), g, fd)


def test_adjoint_matches_oracle_gradient(env):
    """Against the FP64 CPU reference gradient: the oracle's discrete adjoint,
    itself checked against central differences of the oracle's loss on the CPU."""
    N, O, F, torch = env
    cfg, probes, cable, targets, p0 = _gradient_case(F, CC, N, torch, n_nodes=200, n_steps=3000, R=4, ckpt=128,
                                                     seed=11)
    d0 = torch.tensor(p0, device="cuda")
    loss = cable.forward(d0, targets, keep_checkpoints=True)["loss"].item()
    g = cable.backward(d0, targets).cpu().numpy()[0]
    ref = O.cable_run(CC.oracle_config(O, cfg), p0[0], probes, targets.cpu().numpy(), gradient=True)
    assert abs(loss - ref["loss"]) <= 1e-9 * abs(ref["loss"])
    err = _rel_err(g, ref["grad"])
    assert err.max() <= 1e-6, (err.max(), g, ref["grad"])
    # and against forward mode (tangent-linear runs on the CPU, no reverse products)
    gt = O.cable_tangent_gradient(CC.oracle_config(O, cfg), p0[0], probes, targets.cpu().numpy())
    err = _rel_err(g, gt)
    assert err.max() <= 1e-6, (err.max(), g, gt)


def test_autograd_function_and_batched_adjoint(env):
    N, O, F, torch = env
    cfg, probes, cable, targets, p0 = _gradient_case(F, CC, N, torch, n_nodes=64, n_steps=600, R=2, ckpt=50)
    rng = np.random.default_rng(5)
    sets = np.concatenate([p0, CC.lognormal_params(rng, 2, 2, cable.stride, 0.2)])
    params = torch.tensor(sets, device="cuda", requires_grad=True)
    loss = F.cable_mse_loss(params, targets, cable)
    (loss * torch.tensor([1.0, 2.0, 3.0], device="cuda", dtype=torch.float64)).sum().backward()
    for s in range(3):
        one = torch.tensor(sets[s:s + 1], device="cuda")
        cable.forward(one, targets, keep_checkpoints=True)
        g = cable.backward(one, targets)[0]
        assert torch.equal(params.grad[s], g * (s + 1.0)), s


def test_backward_needs_a_checkpointed_forward(env):
    N, O, F, torch = env
    cfg = CC.cable_config(N, n_nodes=32, n_steps=50, n_regions=2, checkpoint_every=10)
    cable = F.Cable(cfg, [3, 20])
    p = torch.ones((1, 2, cable.stride), dtype=torch.float64, device="cuda")
    tg = torch.zeros((50, 2), dtype=torch.float64, device="cuda")
    cable.forward(p, tg)
    with pytest.raises(N.ChasteGpuError) as e:
        cable.backward(p, tg)
    assert e.value.status == 7   # CG_ERR_ORDER
