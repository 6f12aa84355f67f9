"""Bidomain on the GPU (cg_set_bidomain_mesh): the known answers of
heart/test/bidomain/TestBidomainProblem.hpp, and per-node V and phi_e against the
oracle's bidomain restatement every step (1e-6 relative, CG iteration counts within
one) for the singular system with its null space, a pinned phi_e node, and 2D/3D
slabs with anisotropic conductivities."""
import numpy as np
import pytest

from tests import tissue_cases as TC
from tests.test_oracle_bidomain import bidomain_case

pytestmark = pytest.mark.gpu

RTOL = 1e-6


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


def _gpu_1d(N, case, pc=1):
    from oracle import pyoracle as O  # mesh generator only

    xyz, conn, _ = O.slab_mesh(1, case["h"], case["size"], 0.0, 0.0)
    cfg = N.default_config()
    cfg.model, cfg.ode_method = N.MODEL_LR91, N.ODE_FORWARD_EULER
    cfg.ode_time_step = cfg.pde_time_step = 0.01
    cfg.surface_area_to_volume_ratio, cfg.capacitance = case["am"], case["cm"]
    cfg.ksp_preconditioner = pc
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 1, case["abs_tol"]
    t = N.Tissue(cfg)
    t.set_bidomain_mesh(xyz, conn, case["sigma_i"], case["sigma_e"])
    if case["fixed"]:
        t.fix_extracellular_potential(case["fixed"])
    t.set_cells()
    t.set_stimulus(np.where(xyz[:, 0] ** 2 <= 1e-10, 0, -1), [N.stimulus(N.STIM_SIMPLE, -600.0, 0.5, 0.0)])
    return t


def _case(kats, name):
    return next(c for c in kats["bidomain"] if c["name"] == name)


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


@pytest.mark.parametrize("name", ["TestSimpleBidomain1D", "TestBidomainDg01DPinned"])
def test_bidomain_known_answers_and_oracle_parity(N, oracle, kats, name):
    c = _case(kats, name)
    g = _gpu_1d(N, c)
    o, _ = bidomain_case(oracle, dict(c, end=0.0))
    steps = int(round(c["end"] / 0.01))
    worst = 0.0
    for _ in range(steps):
        g.step(1)
        its_o = o.step(1)
        worst = max(worst, _rel(g.voltage(), o.voltage()), _rel(g.extracellular_potential(), o.extracellular()))
        assert abs(g.stats().last_cg_iterations - int(its_o[0])) <= 1
    assert worst <= RTOL, worst
    v, phi = g.voltage(), g.extracellular_potential()
    if "solution" in c:
        u = np.empty(2 * v.size)
        u[0::2], u[1::2] = v, phi
        assert np.abs(u[c["solution_index"]] - np.array(c["solution"])).max() <= c["tolerance"]
        assert abs(phi.mean()) <= 1e-9   # the null space keeps mean(phi_e) at its initial zero
    else:
        assert np.abs(v[c["voltage_nodes"]] - np.array(c["voltage"])).max() <= c["tolerance"]
        assert phi[c["fixed"][0]] == 0.0


def test_bidomain_approaches_monodomain_for_large_extracellular_conductivity(N, kats):
    c = _case(kats, "TestCompareBidomainProblemWithMonodomain")
    b = _gpu_1d(N, c)
    from oracle import pyoracle as O

    xyz, conn, _ = O.slab_mesh(1, c["h"], c["size"], 0.0, 0.0)
    cfg = N.default_config()
    cfg.surface_area_to_volume_ratio, cfg.capacitance = 1.0, 1.0
    cfg.ode_time_step = cfg.pde_time_step = 0.01
    cfg.ksp_preconditioner = 1
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 1, 2e-4
    m = N.Tissue(cfg)
    m.set_mesh(xyz, conn, c["sigma_i"])
    m.set_cells()
    m.set_stimulus(np.where(xyz[:, 0] ** 2 <= 1e-10, 0, -1), [N.stimulus(N.STIM_SIMPLE, -600.0, 0.5, 0.0)])
    steps = int(round(c["end"] / 0.01))
    b.step(steps)
    m.step(steps)
    assert m.voltage()[0] > 0.0
    assert np.abs(m.voltage() - b.voltage()).max() <= c["max_v_difference_from_monodomain"]
    assert np.abs(b.extracellular_potential()).max() <= c["max_abs_phi_e"]


@pytest.mark.parametrize("case_name,pinned", [("LR91_2D", False), ("TT06_3D", False), ("TT06_3D", True)])
def test_bidomain_slabs_against_oracle(N, oracle, case_name, pinned):
    """2D LR91 and 3D TT06 slabs (anisotropic sigma_i, sigma_e = 2.5 sigma_i scaled per axis),
    Vm and phi_e every step against the oracle."""
    case = dict(getattr(TC, case_name))
    case["abs_tol"] = None
    case["rel_tol"] = 1e-9
    dim = case["dim"]
    xyz, conn, _ = oracle.slab_mesh(dim, case["h"], *case["size"])
    si = np.tile(np.asarray(case["sigma"][:dim], float), (conn.shape[0], 1))
    se = si * np.array([2.5, 4.0, 4.0])[:dim]
    cfg = N.default_config()
    cfg.model, cfg.ode_method = case["model"], case["method"]
    cfg.ode_time_step, cfg.pde_time_step = case["dt_ode"], case["dt_pde"]
    cfg.ksp_preconditioner = 1
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, case["rel_tol"]
    g = N.Tissue(cfg)
    g.set_bidomain_mesh(xyz, conn, si, se)
    fixed = [xyz.shape[0] - 1] if pinned else None
    if pinned:
        g.fix_extracellular_potential(fixed)
    g.set_cells()
    sid = TC.slab_stim_ids(xyz, case["box_hi"])
    g.set_stimulus(sid, [N.stimulus(N.STIM_SIMPLE, *case["stim"])])
    o, _ = TC.make_oracle(oracle, **case)
    o.set_bidomain(xyz, conn, si, se, fixed=fixed)
    worst, its_diff = 0.0, 0
    for _ in range(40):
        g.step(1)
        its_o = o.step(1)
        worst = max(worst, _rel(g.voltage(), o.voltage()), _rel(g.extracellular_potential(), o.extracellular()))
        its_diff = max(its_diff, abs(g.stats().last_cg_iterations - int(its_o[0])))
    assert worst <= RTOL, worst
    assert its_diff <= 1
    assert np.ptp(g.voltage()) > 10.0   # the stimulus has started a wave
