"""GPU tissue through the C-ABI against the oracle and Chaste's tissue KATs."""
import numpy as np
import pytest

from tests import tissue_cases as TC

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6   # per-node Vm parity target in FP64 (relative to max(|V|, 1 mV))


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


def _cmp(v_gpu, v_orc):
    return np.max(np.abs(v_gpu - v_orc) / np.maximum(np.abs(v_orc), 1.0))


@pytest.mark.parametrize("use_csr,pc", [(False, 1), (True, 1), (False, 2)], ids=["slab_stencil", "csr",
                                                                                  "bjacobi_ilu0"])
def test_chaste_tissue_kats_on_gpu(N, oracle, kats, use_csr, pc):
    """TestMonodomainProblem.hpp KATs through the GPU path (Jacobi on the stencil and CSR
    operators; bjacobi, Chaste's default, as ILU(0) of the whole matrix), and per-node
    parity with the oracle, CG iteration counts within one."""
    for case in kats["tissue"]:
        d = case["dim"]
        kw = dict(model=TC.LR91, method=TC.FE, dt_ode=0.01, dt_pde=0.01, dim=d, h=case["h"],
                  size=tuple(case["size"][:3]), sigma=(case["sigma"],) * 3,
                  stim=(case["stim"], case["stim_duration"], 0.0), box_hi=(1e-5,) + (1e9,) * 2,
                  am=case["am"], cm=case["cm"], pc=pc)
        if "abs_tol" in case:
            kw["abs_tol"] = case["abs_tol"]
        else:
            kw["rel_tol"] = case["rel_tol"]
        g, _ = TC.make_gpu(N, use_csr=use_csr, **kw)
        o, _ = TC.make_oracle(oracle, **kw)
        nsteps = int(round(case["end"] / 0.01))
        g.step(nsteps)
        its_o = o.step(nsteps)
        v = g.voltage()
        assert np.abs(v[case["nodes"]] - np.array(case["V"])).max() <= case["tolerance"], case["name"]
        assert _cmp(v, o.voltage()) <= FP64_RTOL, case["name"]
        its_g = g.iteration_history(nsteps)
        assert np.abs(its_g - its_o).max() <= 1, case["name"]
        assert g.stats().operator_kind == (0 if use_csr or pc == 2 else 1)


def _parity_run(N, oracle, case, t_end, every, precision=0):
    g, xyz = TC.make_gpu(N, precision=precision, **case)
    o, _ = TC.make_oracle(oracle, **case)
    steps = int(round(t_end / case["dt_pde"]))
    per = int(round(every / case["dt_pde"]))
    worst, vmax_err, its_g, its_o = 0.0, 0.0, [], []
    for _ in range(steps // per):
        g.step(per)
        its_o.extend(o.step(per))
        its_g.extend(g.iteration_history(per))
        vg, vo = g.voltage(), o.voltage()
        worst = max(worst, _cmp(vg, vo))
        vmax_err = max(vmax_err, np.abs(vg - vo).max())
    return g, o, worst, vmax_err, np.array(its_g), np.array(its_o)


def test_lr91_2d_forward_euler_parity(N, oracle):
    """Reduced 2D LR91 FE (dt_ode 0.01, dt_pde 0.1, rtol 1e-8): Vm every 1 ms vs the oracle."""
    g, o, worst, vmax, its_g, its_o = _parity_run(N, oracle, TC.LR91_2D, 20.0, 1.0)
    assert worst <= FP64_RTOL, worst
    assert np.abs(its_g - its_o).max() <= 1
    s_g, s_o = g.states(), o.states()
    assert np.max(np.abs(s_g - s_o) / np.maximum(np.abs(s_o), 1e-3)) <= 1e-5
    ig, _ = g.caches()
    io, _ = o.caches()
    assert np.max(np.abs(ig - io)) <= 1e-6 * max(1.0, np.abs(io).max())


@pytest.mark.parametrize("case_name", ["LR91_2D", "TT06_3D", "LR91_SHEET_10201"])
def test_bjacobi_ilu0_parity(N, oracle, case_name):
    """bjacobi (ILU(0) of the whole matrix, level-scheduled on the device) against the
    oracle's ILU(0) on the reduced benchmark slabs and the full 10,201-node LR91 sheet (all
    three take the one-block solve with its vectors in shared memory): Vm every 1 ms
    within 1e-6, CG iteration counts within one, and fewer iterations than Jacobi."""
    case = dict(getattr(TC, case_name), pc=2)
    g, o, worst, vmax, its_g, its_o = _parity_run(N, oracle, case, 5.0, 1.0)
    assert worst <= FP64_RTOL, worst
    assert np.abs(its_g - its_o).max() <= 1
    j, _ = TC.make_gpu(N, **dict(case, pc=1))
    j.step(len(its_g))
    assert its_g.sum() < j.iteration_history(len(its_g)).sum()


def test_tt06_3d_rush_larsen_parity(N, oracle):
    """Reduced 3D TT06 RL slab (anisotropic sigma, corner stimulus): Vm every 1 ms vs the oracle."""
    g, o, worst, vmax, its_g, its_o = _parity_run(N, oracle, TC.TT06_3D, 10.0, 1.0)
    assert worst <= FP64_RTOL, worst
    assert np.abs(its_g - its_o).max() <= 1


@pytest.mark.parametrize("variant", ["slab", "csr", "slab_two_nodes_per_thread", "slab_four_nodes_per_thread",
                                     "slab_jacobi_inner"])
def test_mixed_precision_against_fp64(N, variant):
    """Mixed mode (FP32 states, FP32 inner CG, FP64 refinement) within 0.5 mV of FP64 and activation within 1 ms.

    slab: the pipelined inner solve with one node per thread; csr: the assembled
    operator (two-reduction inner PCG); slab_two_nodes_per_thread: a slab of
    159,681 nodes, more than the co-resident grid has threads, so each thread
    keeps two nodes' inner vectors in registers; slab_four_nodes_per_thread: a slab
    of 473,556 nodes, the largest register-resident case (4 per thread on 148 SMs)."""
    case = dict(TC.TT06_3D)
    pipe = {"slab": 1, "slab_jacobi_inner": 1, "slab_two_nodes_per_thread": 2, "slab_four_nodes_per_thread": 4}
    if variant == "csr":
        case["use_csr"] = True
    elif variant == "slab_two_nodes_per_thread":
        case.update(size=(1.0, 0.5, 0.3), box_hi=(0.1, 0.1, 0.1))
    elif variant == "slab_four_nodes_per_thread":
        case.update(size=(2.0, 0.75, 0.3), box_hi=(0.1, 0.1, 0.1))
    elif variant == "slab_jacobi_inner":
        case["inner_pc"] = 1
    a, _ = TC.make_gpu(N, precision=0, **case)
    b, _ = TC.make_gpu(N, precision=1, **case)
    st = b.stats()
    assert st.pipelined_nodes_per_thread == pipe.get(variant, 0)
    assert st.inner_preconditioner == (N.INNER_PC_LINE if variant in pipe and variant != "slab_jacobi_inner"
                                       else N.INNER_PC_JACOBI)
    worst = 0.0
    for _ in range(20):
        a.step(10)
        b.step(10)
        worst = max(worst, np.abs(a.voltage() - b.voltage()).max())
    assert worst <= 0.5, worst
    ta, tb = a.activation_times(), b.activation_times()
    assert np.all((ta >= 0) == (tb >= 0))
    act = ta >= 0
    assert act.sum() > 0
    assert np.abs(ta[act] - tb[act]).max() <= 1.0


def test_line_preconditioned_inner_solve_takes_fewer_iterations(N):
    """The mixed solve's x-line inner preconditioner against its Jacobi inner solve on
    an anisotropic slab (sigma_x / sigma_y = 9): same FP64 stopping test, same answer
    within the tolerance, fewer inner iterations.  The two contexts also share the
    pipelined kernel with different shared-memory sizes."""
    case = dict(TC.TT06_3D, size=(1.0, 0.5, 0.3), box_hi=(0.1, 0.1, 0.1))
    line, _ = TC.make_gpu(N, precision=1, **case)
    jac, _ = TC.make_gpu(N, precision=1, inner_pc=1, **case)
    ref, _ = TC.make_gpu(N, precision=0, **case)
    for t in (line, jac, ref):
        t.step(40)
    il, ij = line.stats().total_cg_iterations, jac.stats().total_cg_iterations
    assert il <= 0.75 * ij, (il, ij)
    assert np.abs(line.voltage() - ref.voltage()).max() <= 0.5
    assert np.abs(line.voltage() - jac.voltage()).max() <= 0.5


def test_inner_preconditioner_is_symmetric_and_inverts_the_x_lines(N, oracle):
    """The mixed solve's x-line inner preconditioner B, applied on the device: <Bx, y> =
    <x, By> to FP32 rounding, x^T B x > 0, and T B x = x with T the tridiagonal x-part
    of the assembled A restricted to the 32-node segments B works on."""
    case = dict(TC.TT06_3D, size=(0.4, 0.1, 0.05))
    t, _ = TC.make_gpu(N, precision=1, **case)
    o, _ = TC.make_oracle(oracle, **case)
    n = t.n
    seg = t.stats().inner_line_segment
    assert seg == 32
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    bx, by = t.apply_inner_preconditioner(x), t.apply_inner_preconditioner(y)
    assert abs(bx @ y - x @ by) <= 1e-5 * float(np.abs(bx) @ np.abs(y))
    assert x @ bx > 0 and y @ by > 0
    rp, cols, vals = o.matrix(0)
    tbx = np.zeros(n)
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            j = cols[k]
            same_segment = j // seg == i // seg
            if j == i or (abs(j - i) == 1 and same_segment):
                tbx[i] += vals[k] * bx[j]
    assert np.max(np.abs(tbx - x)) <= 1e-4 * np.max(np.abs(x))


@pytest.mark.parametrize("case_name", ["LR91_2D", "TT06_3D"])
def test_operator_splitting_parity(N, oracle, case_name):
    """OperatorSplittingMonodomainSolver on the GPU (FP64) against the oracle's
    restatement: half step of the cells with V, diffusion, second half."""
    case = dict(getattr(TC, case_name))
    case["solver"] = 1
    g, _ = TC.make_gpu(N, **case)
    o, _ = TC.make_oracle(oracle, **case)
    worst = 0.0
    for _ in range(10):
        g.step(5)
        o.step(5)
        vo = o.voltage()
        worst = max(worst, float(np.max(np.abs(g.voltage() - vo) / np.maximum(np.abs(vo), 1.0))))
    assert worst <= FP64_RTOL, worst
    assert o.voltage().max() > -60.0          # the stimulus took
    # mixed precision in the same mode, within 0.5 mV of FP64
    m, _ = TC.make_gpu(N, precision=1, **case)
    m.step(50)
    assert float(np.max(np.abs(m.voltage() - g.voltage()))) <= 0.5


def test_operator_splitting_backward_euler_known_answer_on_gpu(N):
    """TestOperatorSplittingMonodomainSolver.hpp:102-146 through the GPU: 1D slab of
    101 nodes, backward-Euler LR91 cells, ODE/PDE steps 0.005/0.01 ms, 4 ms,
    -1e6 uA/cm^3 for 0.5 ms on x <= 0.02: V at node 30 is 5.0567 (+- 1e-3)."""
    cfg = N.default_config()
    cfg.model, cfg.ode_method = N.MODEL_LR91, N.ODE_BACKWARD_EULER
    cfg.ode_time_step, cfg.pde_time_step = 0.005, 0.01
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 1, 2e-4
    cfg.ksp_preconditioner = N.PC_JACOBI
    cfg.solver = N.SOLVER_OPERATOR_SPLITTING
    t = N.Tissue(cfg)
    t.set_slab_mesh(1, 0.01, 1.0, 0.0, 0.0, sigma=(1.75, 1.75, 1.75))
    t.set_cells()
    x = np.arange(t.n) * 0.01
    t.set_stimulus(np.where(np.abs(x) < 0.02 + 1e-6, 0, -1).astype(np.int32),
                   [N.stimulus(N.STIM_SIMPLE, -1e6, 0.5, 0.0)])
    t.step(400)
    assert abs(t.voltage()[30] - 5.0567) <= 1e-3


@pytest.mark.parametrize("solver,case_name", [(0, "LR91_2D"), (1, "LR91_2D"), (0, "TT06_3D")])
def test_backward_euler_cells_parity(N, oracle, solver, case_name):
    """Backward-Euler cells on the GPU (FP64) against the oracle, with V clamped
    (default solver) and with V (operator splitting)."""
    case = dict(getattr(TC, case_name))
    case.update(method=2, solver=solver)
    g, _ = TC.make_gpu(N, **case)
    o, _ = TC.make_oracle(oracle, **case)
    worst = 0.0
    for _ in range(5):
        g.step(4)
        o.step(4)
        vo = o.voltage()
        worst = max(worst, float(np.max(np.abs(g.voltage() - vo) / np.maximum(np.abs(vo), 1.0))))
    assert worst <= FP64_RTOL, worst
    m, _ = TC.make_gpu(N, precision=1, **case)
    m.step(20)
    assert float(np.max(np.abs(m.voltage() - g.voltage()))) <= 0.5


@pytest.mark.parametrize("method,solver,case_name", [(3, 0, "LR91_2D"), (4, 0, "LR91_2D"), (3, 1, "LR91_2D"),
                                                     (4, 1, "LR91_2D"), (3, 0, "TT06_3D"), (4, 0, "TT06_3D")])
def test_generalised_rush_larsen_cells_parity(N, oracle, method, solver, case_name):
    """Cells whose ODE solver is GRL1 (method 3) or GRL2 (method 4), on the GPU in FP64
    against the oracle, with V clamped (default solver) and with V (operator
    splitting); mixed precision within 0.5 mV of FP64."""
    case = dict(getattr(TC, case_name))
    case.update(method=method, solver=solver)
    g, _ = TC.make_gpu(N, **case)
    o, _ = TC.make_oracle(oracle, **case)
    worst = 0.0
    for _ in range(5):
        g.step(4)
        o.step(4)
        worst = max(worst, _cmp(g.voltage(), o.voltage()))
    assert worst <= FP64_RTOL, worst
    m, _ = TC.make_gpu(N, precision=1, **case)
    m.step(20)
    assert float(np.max(np.abs(m.voltage() - g.voltage()))) <= 0.5


@pytest.mark.parametrize("method,case_name,use_csr", [(1, "TT06_3D", False), (2, "TT06_3D", True),
                                                     (0, "LR91_2D", False)])
def test_state_variable_interpolation_parity(N, oracle, method, case_name, use_csr):
    """SVI correction on the GPU (FP64, stencil and CSR operators) against the oracle,
    and a check that it changes the solution (elements on the wavefront qualify)."""
    case = dict(getattr(TC, case_name))
    case.update(method=method, svi=1)
    g, _ = TC.make_gpu(N, use_csr=use_csr, **case)
    o, _ = TC.make_oracle(oracle, **case)
    plain, _ = TC.make_gpu(N, **dict(case, svi=0))
    worst, moved = 0.0, 0.0
    for _ in range(5):
        g.step(4)
        o.step(4)
        plain.step(4)
        vg, vo = g.voltage(), o.voltage()
        worst = max(worst, _cmp(vg, vo))
        moved = max(moved, float(np.abs(vg - plain.voltage()).max()))
    assert worst <= FP64_RTOL, worst
    assert moved > 1e-3, moved
    m, _ = TC.make_gpu(N, precision=1, **case)
    m.step(20)
    assert float(np.max(np.abs(m.voltage() - g.voltage()))) <= 0.5


def test_state_variable_interpolation_rejects_operator_splitting(N):
    cfg = N.default_config()
    cfg.use_state_variable_interpolation, cfg.solver = 1, N.SOLVER_OPERATOR_SPLITTING
    with pytest.raises(N.ChasteGpuError) as e:
        N.Tissue(cfg)
    assert e.value.status == 10  # CG_ERR_UNSUPPORTED


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_niederer_benchmark_activation_map(N, golden_dir, precision):
    """TestNiederer2011BenchmarkSimulation::TestRunOnCoarsestMesh on the GPU: TT06
    backward-Euler cells with SVI on the h = 0.05 slab for 40 ms; Chaste's activation
    map within its 1.5e-3 ms (FP64), within 0.05 ms in mixed precision."""
    gold = np.loadtxt(golden_dir / "niederer_activation_h0.05_dt0.01.txt")
    t, xyz = TC.make_gpu(N, precision=precision, **TC.NIEDERER)
    assert t.n == gold.size == xyz.shape[0]
    act = TC.niederer_activation(t, t.n)
    assert (act > 0).all()
    err = float(np.abs(act - gold).max())
    assert err <= (1.5e-3 if precision == 0 else 0.05), err


def test_snapshot_restore_is_bitwise(N):
    case = dict(TC.LR91_2D)
    a, _ = TC.make_gpu(N, **case)
    a.step(20)
    blob = a.snapshot()
    a.step(30)
    v1 = a.voltage()
    b, _ = TC.make_gpu(N, **case)
    b.restore(blob)
    b.step(30)
    assert np.array_equal(v1, b.voltage())
    assert b.stats().steps == 50


def test_two_node_caches_match_standalone_cells(N, oracle):
    """TestMonodomainTissue.hpp:133-237: the Iion cache equals a standalone ComputeExceptVoltage."""
    O = oracle
    cfg = N.default_config()
    cfg.pde_time_step = 0.5
    t = N.Tissue(cfg)
    xyz = np.array([[0.0, 0, 0], [1.0, 0, 0]])
    t.set_mesh(xyz, np.array([[0, 1]]), np.array([[1.75]]))
    t.set_cells()
    t.set_stimulus(np.array([0, -1]), [N.stimulus(N.STIM_SIMPLE, -600.0 * 1400.0, 0.5, 0.0)])
    t.step(1)
    iion, _ = t.caches()
    for node, st in ((0, O.simple(-600.0 * 1400.0, 0.5, 0.0)), (1, None)):
        y = O.initial_states(O.LR91)
        ref = O.cell_except_voltage(O.LR91, O.FE, y, 0.0, 0.5, 0.01, st, am=1400.0)
        assert abs(iion[node] - ref) <= 1e-10 * max(1.0, abs(ref))


def test_cg_failure_is_reported_not_faulted(N):
    """KSP_DIVERGED_ITS analogue: a 1-iteration cap returns CG_ERR_CG_MAXIT and stops later steps."""
    case = dict(TC.LR91_2D)
    case["rel_tol"] = 1e-14
    g, _ = TC.make_gpu(N, max_iterations=1, **case)
    with pytest.raises(N.ChasteGpuError) as e:
        g.step(2)
    assert e.value.status == 3
    assert g.stats().steps == 1


def test_nan_voltage_is_reported(N):
    case = dict(TC.LR91_2D)
    g, _ = TC.make_gpu(N, **case)
    v = g.voltage()
    v[5] = np.nan
    g.set_voltage(v)
    with pytest.raises(N.ChasteGpuError) as e:
        g.step(1)
    assert e.value.status == 5


def test_state_out_of_range_is_reported(N):
    """VerifyStateVariables analogue (AbstractCardiacCell.cpp:100-104): a gate above 1
    with range checking on returns CG_ERR_STATE_RANGE."""
    case = dict(TC.LR91_2D)

    def tissue(check):
        cfg = N.default_config()
        cfg.model, cfg.ode_method = case["model"], case["method"]
        cfg.ode_time_step, cfg.pde_time_step = case["dt_ode"], case["dt_pde"]
        cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, 1e-8
        cfg.ksp_preconditioner = N.PC_JACOBI
        cfg.check_state_ranges = check
        t = N.Tissue(cfg)
        t.set_slab_mesh(case["dim"], case["h"], *case["size"], sigma=case["sigma"])
        return t

    ref = tissue(0)
    ref.set_cells()
    init = ref.states().copy()
    # the slow time-dependent K gate X (state 6, rates ~1e-3 /ms) of node 7 outside
    # [0, 1]; a fast gate would be pulled back inside within the step's substeps
    init[7, 6] = 1.5
    t = tissue(1)
    t.set_cells(init_states=init)
    t.set_stimulus(np.full(t.n, -1, np.int32), [N.stimulus(N.STIM_SIMPLE, 0.0, 0.0)])
    with pytest.raises(N.ChasteGpuError) as e:
        t.step(1)
    assert e.value.status == 6


def test_bounded_device_wait_times_out_and_the_device_stays_usable(N):
    """Failure path of the persistent kernels' grid reductions, without a fault: a
    wait for an arrival that never comes ends after its limit with the timeout bit,
    and a tissue step afterwards still matches."""
    import ctypes as C

    bits, waited = C.c_int(0), C.c_double(0.0)
    rc = N.lib().cg_selftest_barrier_timeout(0, 50.0, C.byref(bits), C.byref(waited))
    assert rc == 0
    assert bits.value & 16
    assert 40.0 <= waited.value <= 1000.0, waited.value
    g, _ = TC.make_gpu(N, **dict(TC.LR91_2D))
    g.step(3)
    assert np.all(np.isfinite(g.voltage()))


def test_monodomain_problem_api_on_gpu(N, kats):
    """MonodomainProblem + PlaneStimulusCellFactory (the Chaste-facing API) reproduces TestMonodomainProblem1D."""
    from chaste_b200 import heart as H

    case = [c for c in kats["tissue"] if c["name"] == "TestMonodomainProblem1DWithRelativeTolerance"][0]
    hc = H.HeartConfig.Instance()
    hc.Reset()
    hc.SetIntracellularConductivities(0.0005)
    hc.SetSimulationDuration(2.0)
    hc.SetSurfaceAreaToVolumeRatio(1.0)
    hc.SetCapacitance(1.0)
    hc.SetUseRelativeTolerance(1e-9)
    hc.SetFibreLength(0.1, 0.01)
    p = H.MonodomainProblem(H.PlaneStimulusCellFactory(H.CellLuoRudy1991FromCellML, -600.0, 0.5))
    p.Initialise()
    p.Solve()
    v = p.GetSolution()
    assert np.abs(v[case["nodes"]] - np.array(case["V"])).max() <= case["tolerance"]
    cell = p.GetTissue().GetCardiacCell(3)
    assert abs(cell.GetVoltage() - v[3]) == 0.0
    hc.Reset()


@pytest.mark.parametrize("precision", [0, 1])
def test_host_buffer_steps_match_device_steps(N, precision):
    """cg_step_host (V copied in piece by piece under the first step's ODE, V copied
    out, one synchronisation) reproduces the device-resident steps bit for bit when
    the caller passes back what it got (keep_history), and set_voltage + step when it
    declares the voltage new (no history: the mixed solve's guess is V itself)."""
    case = dict(TC.TT06_3D)
    dev, _ = TC.make_gpu(N, precision=precision, **case)
    host, _ = TC.make_gpu(N, precision=precision, **case)
    dev.step(5)
    host.step(5)
    v = host.voltage()
    out = np.empty_like(v)
    for _ in range(15):
        dev.step(1)
        host.step_host(v, 1, out, keep_history=True)
        v, out = out, v
        assert np.array_equal(v, dev.voltage())
    assert host.stats().steps == dev.stats().steps == 20
    # a voltage declared new: the same as cg_set_voltage followed by cg_step (the two
    # tissues hold bitwise the same states here)
    w = v.copy()
    w[::7] += 0.25
    dev.set_voltage(w)
    dev.step(3)
    host.step_host(w, 3, out, keep_history=False)
    assert np.array_equal(out, dev.voltage())
    # reading back only, and writing only
    host.step_host(None, 2, out)
    assert np.array_equal(out, host.voltage())
    host.step_host(out, 0, None)
    assert np.array_equal(out, host.voltage())


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case_name", ["TT06_3D", "LR91_2D"])
def test_host_buffer_steps_replayed_from_graphs(N, precision, case_name):
    """With page-locked buffers the first step's ODE reads V from the caller's buffer
    through its device mapping and cg_step_host replays each (v_in, v_out) pair's call
    from a graph; two alternating buffer pairs reproduce the device-resident steps bit
    for bit (Rush-Larsen and forward Euler), and a change of the cells (new kernel
    arguments) drops the cached calls."""
    import torch

    case = dict(getattr(TC, case_name))
    dev, _ = TC.make_gpu(N, precision=precision, **case)
    host, _ = TC.make_gpu(N, precision=precision, **case)
    dev.step(3)
    host.step(3)
    a = torch.empty(host.n, dtype=torch.float64, pin_memory=True).numpy()
    b = torch.empty(host.n, dtype=torch.float64, pin_memory=True).numpy()
    host.voltage(out=a)
    for _ in range(12):
        dev.step(1)
        host.step_host(a, 1, b, keep_history=True)
        a, b = b, a
        assert np.array_equal(a, dev.voltage())
    assert host.stats().steps == dev.stats().steps
    # several steps per call: the first call of a (buffers, steps) pair is captured, the
    # next ones replay it
    for _ in range(3):
        dev.step(4)
        host.step_host(a, 4, b, keep_history=True)
        a, b = b, a
        assert np.array_equal(a, dev.voltage())
        assert host.stats().steps == dev.stats().steps
    assert host.stats().host_call_graph == 1
    # new cells: both tissues restart from the same states, the cached calls are rebuilt
    dev.set_cells()
    host.set_cells()
    dev.set_voltage(a)
    for k in range(4):
        dev.step(1)
        host.step_host(a, 1, b, keep_history=k > 0)   # the first call declares V new, as set_voltage does
        a, b = b, a
    assert np.array_equal(a, dev.voltage())
