"""Printing-step output on the device (cg_output_*): frames in Hdf5DataWriter's layout
and the PostProcessingWriter maps, against the oracle and tests/cellprops.py."""
import numpy as np
import pytest

from tests import cellprops as CP
from tests import tissue_cases as TC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


# LR91 sheet paced from its left edge every 500 ms for 1100 ms: two full action
# potentials everywhere, a third still running at the end
PACED = dict(TC.LR91_2D, size=(0.2, 0.1, 0.0))
PERIOD, T_END, EVERY = 500.0, 1100.0, 2


def _paced(N, O, precision=0):
    g, xyz = TC.make_gpu(N, precision=precision, **PACED)
    sid = TC.slab_stim_ids(xyz, PACED["box_hi"])
    stim = PACED["stim"]
    g.set_stimulus(sid, [N.stimulus(N.STIM_REGULAR, stim[0], stim[1], 0.0, PERIOD, 1e300)])
    o = None
    if O is not None:
        xyz_o, conn, _ = O.slab_mesh(2, PACED["h"], *PACED["size"])
        cfg = O.Config(PACED["model"], PACED["method"], PACED["dt_ode"], PACED["dt_pde"], 1400.0, 1.0, O.PC_JACOBI,
                       0, PACED["rel_tol"] if "rel_tol" in PACED else 1e-8, 0, 10000, 0, 0)
        sig = np.tile(np.asarray(PACED["sigma"][:2], float), (conn.shape[0], 1))
        o = O.Tissue(cfg, 2, xyz_o, conn, sig, sid, [O.regular(stim[0], stim[1], PERIOD, 0.0)])
    return g, o, xyz


def test_frames_layout_times_and_capacity(N, oracle):
    """Frame 0 is the initial condition, frame k the state after k printing steps, in
    (frames, nodes, variables) order with V first; a step that would overflow the frame
    buffer is refused before anything runs."""
    g, o, _ = _paced(N, oracle)
    n_states = 8
    g.configure_output(EVERY, 6, state_vars=[1, 7])
    y0 = g.cell_state(0)
    g.step(4 * EVERY)
    f = g.output_frames()
    assert f.shape == (5, g.n, 3)
    assert np.allclose(g.output_times(), np.arange(5) * EVERY * PACED["dt_pde"])
    assert f[0, 0, 0] == y0[0] and f[0, 0, 1] == y0[1] and f[0, 0, 2] == y0[7]
    ref = []
    ref.append(o.voltage())
    for _ in range(4):
        o.step(EVERY)
        ref.append(o.voltage())
    ref = np.array(ref)
    assert np.max(np.abs(f[:, :, 0] - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-6
    assert np.array_equal(f[-1, :, 0], g.voltage())
    st = g.states()
    assert np.array_equal(f[-1, :, 2], st[:, 7])
    with pytest.raises(N.ChasteGpuError) as e:
        g.step(2 * EVERY)            # needs two more frames, one left
    assert e.value.status == 9       # CG_ERR_NOMEM
    assert g.output_frames().shape[0] == 5 and g.stats().steps == 4 * EVERY
    g.step(EVERY)
    assert g.output_frames().shape[0] == 6
    assert n_states == st.shape[1]


@pytest.fixture(scope="module")
def paced_run(N, oracle):
    g, o, xyz = _paced(N, oracle)
    steps = int(round(T_END / PACED["dt_pde"]))
    g.configure_output(EVERY, steps // EVERY + 1)
    g.enable_activation_modifier(-40.0)
    g.step(steps)
    frames = g.output_frames()[:, :, 0]
    times = g.output_times()
    ref = [o.voltage()]
    for _ in range(steps // EVERY):
        o.step(EVERY)
        ref.append(o.voltage())
    return g, frames, times, np.array(ref), xyz


@pytest.mark.parametrize("percentage", [90.0, 50.0])
def test_cell_property_maps_match_the_restatement(N, paced_run, percentage):
    """APD, upstroke-time and max-upstroke-velocity maps of every node from the device
    frames equal CellProperties restated on the same frames (both APD search
    directions: APD90 looks backwards from the onset, APD50 forwards)."""
    g, frames, times, _, _ = paced_run
    m = g.cell_property_maps(percentage=percentage, threshold=-30.0, max_aps=8)
    apd_ref, up_t_ref, up_v_ref = CP.node_maps(times, frames, percentage, -30.0)
    for i in range(g.n):
        assert len(m["apd"][i]) == len(apd_ref[i]) and np.allclose(m["apd"][i], apd_ref[i], rtol=0, atol=1e-9), i
        assert np.allclose(m["upstroke_time"][i], up_t_ref[i], rtol=0, atol=1e-12), i
        assert np.allclose(m["max_upstroke_velocity"][i], up_v_ref[i], rtol=1e-12, atol=1e-12), i
    assert all(len(r) == 2 for r in m["apd"])            # two complete action potentials
    assert all(len(r) == 3 for r in m["upstroke_time"])  # the third is still running
    assert np.all(m["apd_array"][:, 2:] == -999.0)


def test_cell_property_maps_against_the_oracle_frames(N, paced_run):
    """Maps from the device frames against maps of the oracle's voltages."""
    g, frames, times, ref, _ = paced_run
    m = g.cell_property_maps(max_aps=8)
    apd_ref, up_t_ref, _ = CP.node_maps(times, ref)
    worst_apd = max(abs(a - b) for i in range(g.n) for a, b in zip(m["apd"][i], apd_ref[i]))
    assert worst_apd <= 1e-3
    assert all(np.array_equal(m["upstroke_time"][i], up_t_ref[i]) or
               np.abs(np.subtract(m["upstroke_time"][i], up_t_ref[i])).max() <= 0.21 for i in range(g.n))


def test_activation_output_modifier(N, paced_run):
    """ActivationOutputModifier's four columns at the printing times, against its
    restatement on the same frames."""
    g, frames, times, _, _ = paced_run
    got = g.activation_modifier_times()
    ref = -np.ones((g.n, 4))
    for f, t in enumerate(times):
        v = frames[f]
        a = (v > -40.0) & (ref[:, 0] < 0)
        b = ~a & (ref[:, 0] >= 0) & (ref[:, 1] < 0) & (v < -40.0)
        c = ~a & ~b & (ref[:, 1] >= 0) & (ref[:, 2] < 0) & (v > -40.0)
        d = ~a & ~b & ~c & (ref[:, 2] >= 0) & (ref[:, 3] < 0) & (v < -40.0)
        ref[a, 0] = t
        ref[b, 1] = t
        ref[c, 2] = t
        ref[d, 3] = t
    assert np.array_equal(got, ref)
    assert (got > 0).all()


def test_modifiers_without_frames(N):
    g, _ = TC.make_gpu(N, **PACED)
    g.configure_output(5, 0)
    g.enable_activation_modifier(-40.0)
    g.step(200)
    assert g.output_times().size == 0
    act = g.activation_modifier_times()
    assert (act[:, 0] >= 0).all() and (act[:, 1:] < 0).all()
    assert np.all(np.round(act[:, 0] / 0.5, 9) % 1 == 0)   # printing times of 0.5 ms


def test_conduction_velocity_map(N, paced_run):
    g, frames, times, _, xyz = paced_run
    origin = 0
    dist = np.linalg.norm(xyz - xyz[origin], axis=1)
    cv = g.conduction_velocity_map(origin, dist, max_aps=8)
    raw = [CP.calculate_properties(times, frames[:, i])["t_max_up"] for i in range(g.n)]
    for i in range(g.n):
        ref = CP.conduction_velocities(raw[origin], raw[i], dist[i], i == origin)
        assert np.allclose(cv[i], ref, rtol=1e-12, atol=0), i
    far = int(np.argmax(dist))
    assert 0.01 < cv[far][0] < 1.0   # cm/ms


def test_nodes_without_an_action_potential_hold_zero(N):
    """A sheet that is never stimulated: every map row is [0], as PostProcessingWriter
    writes when CellProperties raises."""
    g, _ = TC.make_gpu(N, **dict(PACED, stim=(0.0, 0.5, 0.0)))
    g.configure_output(5, 11)
    g.step(50)
    m = g.cell_property_maps(max_aps=4)
    assert all(r == [0.0] for r in m["apd"]) and all(r == [0.0] for r in m["upstroke_time"])
    assert np.all(m["apd_array"][:, 1:] == -999.0)


def test_heart_api_output_and_post_processing(N, tmp_path):
    """HeartConfig output variables and post-processing requests through
    MonodomainProblem: Data/Time as Hdf5DataWriter lays them out, the maps under
    PostProcessingWriter's dataset names, and the files WriteOutput leaves."""
    from chaste_b200 import heart as H

    hc = H.HeartConfig.Instance()
    hc.Reset()
    hc.SetIntracellularConductivities(1.75)
    hc.SetSurfaceAreaToVolumeRatio(1400.0)
    hc.SetOdePdeAndPrintingTimeSteps(0.01, 0.1, 0.5)
    hc.SetSimulationDuration(420.0)
    hc.SetFibreLength(1.0, 0.01)
    hc.SetOutputVariables(["Cai"])
    hc.SetApdMaps([(90.0, -30.0)])
    hc.SetUpstrokeTimeMaps([-30.0])
    hc.SetMaxUpstrokeVelocityMaps([-30.0])
    hc.SetConductionVelocityMaps([0])
    try:
        p = H.MonodomainProblem(H.PlaneStimulusCellFactory(H.CellLuoRudy1991FromCellML, -3.0e6, 0.5))
        p.Initialise()
        p.Solve()
        out = p.GetOutput()
        assert out["variables"] == ["V", "Cai"]
        assert out["Data"].shape == (841, 101, 2)
        assert np.allclose(out["Time"], np.arange(841) * 0.5)
        assert np.array_equal(out["Data"][-1, :, 0], p.GetSolution())
        maps = p.GetPostProcessingMaps()
        assert set(maps) == {"Apd_90_minus_30_Map", "UpstrokeTimeMap_minus_30", "MaxUpstrokeVelocityMap_minus_30",
                             "ConductionVelocityFromNode0"}
        v = out["Data"][:, :, 0]
        apd_ref, up_t_ref, up_v_ref = CP.node_maps(out["Time"], v)
        for i in range(101):
            assert np.allclose(maps["Apd_90_minus_30_Map"][i], apd_ref[i], rtol=0, atol=1e-9)
            assert np.allclose(maps["UpstrokeTimeMap_minus_30"][i], up_t_ref[i], rtol=0, atol=1e-12)
        apd = np.array([r[0] for r in maps["Apd_90_minus_30_Map"]])
        assert np.all((apd > 300) & (apd < 420))
        cv = np.array([r[0] for r in maps["ConductionVelocityFromNode0"]])
        assert cv[0] == 0.0 and 0.02 < cv[-1] < 0.2
        p.WriteOutput(tmp_path)
        assert np.load(tmp_path / "Data.npy").shape == (841, 101, 2)
        a = np.load(tmp_path / "Apd_90_minus_30_Map.npy")
        assert a.shape == (1, 101) and np.allclose(a[0], apd)
    finally:
        hc.Reset()
