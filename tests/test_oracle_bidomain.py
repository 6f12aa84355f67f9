"""The oracle's bidomain restatement (BidomainProblem without a bath) against the
known answers of heart/test/bidomain/TestBidomainProblem.hpp held in
tests/golden/chaste_kats.json: the singular system with the null space of constant
phi_e, a pinned phi_e node, and the large-sigma_e limit that approaches monodomain."""
import numpy as np


def bidomain_case(O, case, pc=1, monodomain=False):
    xyz, conn, _ = O.slab_mesh(1, case["h"], case["size"], 0.0, 0.0)
    cfg = O.Config(O.LR91, O.FE, 0.01, 0.01, case["am"], case["cm"], pc, 1, case["abs_tol"], 0, 10000)
    sid = np.where(xyz[:, 0] ** 2 <= 1e-10, 0, -1).astype(np.int32)
    si = np.full((conn.shape[0], 1), case["sigma_i"])
    t = O.Tissue(cfg, 1, xyz, conn, si, sid, [O.simple(-600.0, 0.5, 0.0)])
    if not monodomain:
        t.set_bidomain(xyz, conn, si, np.full((conn.shape[0], 1), case["sigma_e"]),
                       fixed=case["fixed"] or None)
    its = t.step(int(round(case["end"] / 0.01)))
    return t, its


def _case(kats, name):
    return next(c for c in kats["bidomain"] if c["name"] == name)


def test_simple_bidomain_1d_null_space(oracle, kats):
    c = _case(kats, "TestSimpleBidomain1D")
    t, its = bidomain_case(oracle, c)
    u = np.empty(2 * t.n)
    u[0::2], u[1::2] = t.voltage(), t.extracellular()
    err = np.abs(u[c["solution_index"]] - np.array(c["solution"])).max()
    assert err <= c["tolerance"], err
    assert its.min() > 0
    # the null space keeps the mean of phi_e where the initial condition put it (zero)
    assert abs(t.extracellular().mean()) <= 1e-9


def test_bidomain_with_a_pinned_extracellular_node(oracle, kats):
    c = _case(kats, "TestBidomainDg01DPinned")
    t, _ = bidomain_case(oracle, c)
    v, phi = t.voltage(), t.extracellular()
    assert np.abs(v[c["voltage_nodes"]] - np.array(c["voltage"])).max() <= c["tolerance"]
    assert abs(phi[c["fixed"][0]]) <= 1e-12
    assert np.abs(v[c["rest_from_node"]:] - c["rest"]).max() <= c["rest_tolerance"]


def test_bidomain_approaches_monodomain_for_large_extracellular_conductivity(oracle, kats):
    c = _case(kats, "TestCompareBidomainProblemWithMonodomain")
    b, _ = bidomain_case(oracle, c)
    m, _ = bidomain_case(oracle, c, monodomain=True)
    assert m.voltage()[0] > 0.0
    assert np.abs(m.voltage() - b.voltage()).max() <= c["max_v_difference_from_monodomain"]
    assert np.abs(b.extracellular()).max() <= c["max_abs_phi_e"]
