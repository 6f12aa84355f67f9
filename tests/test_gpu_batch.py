"""Batched single-cell populations (cg_batch_*) against the oracle's single-cell Compute."""
import numpy as np
import pytest

from tests import cellprops

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


def population(n, seed=20261203, max_beats=3):
    rng = np.random.default_rng(seed)
    params = np.ones((n, 9))
    params[:, :6] = np.exp(rng.normal(0.0, 0.2, size=(n, 6)))   # g_Na, g_CaL, g_Kr, g_Ks, g_K1, g_to
    beats = rng.integers(1, max_beats + 1, size=n).astype(np.int32)
    return params, beats


@pytest.mark.parametrize("engine", ["autotuned", "per_beat", "persistent"])
def test_population_matches_oracle_cells(N, oracle, engine):
    O = oracle
    n = 64
    params, beats = population(n)
    beats[:2] = 2
    b = N.CellBatch(N.MODEL_TT06, beats, params)
    if engine == "autotuned":
        tpb = b.autotune(steps=500)
        assert tpb in (32, 64, 128, 256)
        assert b.engine() in (N.BATCH_PER_BEAT, N.BATCH_PERSISTENT)
    elif engine == "per_beat":
        b.set_launch_shape(64, 1)
        assert b.engine() == N.BATCH_PER_BEAT
    else:
        b.set_engine(N.BATCH_PERSISTENT)
    b.run()
    r = b.results()
    stim = O.regular(-52.0, 1.0, 1000.0, 50.0)
    for cell in (0, 1):
        y = O.initial_states(O.TT06)
        tr, y = O.cell_compute(O.TT06, O.RL, y, 0.0, 1000.0 * beats[cell], 0.01, 0.0, stim, params=params[cell])
        t = np.arange(tr.shape[0]) * 0.01
        ref = cellprops.apds(t, tr[:, 0], 90.0)
        got = r["apd64"][cell, : r["n_ap64"][cell]]
        assert len(ref) == len(got) == beats[cell]
        assert np.max(np.abs(np.array(ref) - got)) <= 1e-6
        assert np.max(np.abs(r["states64"][cell] - y) / np.maximum(np.abs(y), 1e-3)) <= 1e-6
    # FP32 against FP64: every AP found, APD90 within 1 ms, finite per-beat Vm error
    assert np.array_equal(r["n_ap64"], r["n_ap32"])
    for cell in range(n):
        k = r["n_ap64"][cell]
        assert np.max(np.abs(r["apd64"][cell, :k] - r["apd32"][cell, :k])) <= 1.0
    dv = r["max_dv"][np.arange(n)[:, None], np.arange(b.max_beats)[None, :]]
    assert np.all(np.isfinite(dv))


def test_cells_per_thread_do_not_change_results(N):
    """Two cells per thread (interleaved in one step loop) give bitwise the results of
    one cell per thread, for an odd population that leaves partial groups."""
    params, beats = population(37, seed=7, max_beats=2)
    out = []
    for tpb, cpt in ((64, 1), (32, 2)):
        b = N.CellBatch(N.MODEL_TT06, beats, params)
        b.set_launch_shape(tpb, cpt)
        assert b.launch_shape() == (tpb, cpt)
        b.run()
        out.append(b.results())
    for key in ("apd64", "apd32", "states64", "states32", "max_dv", "n_ap64", "n_ap32"):
        assert np.array_equal(out[0][key], out[1][key]), key


@pytest.mark.parametrize("model", ["TT06", "LR91"])
def test_persistent_engine_equals_per_beat_launches(N, model):
    """The persistent engine (one launch, work queue, each cell split over a gate
    thread and a state thread) gives the states, APDs and per-beat errors of the
    per-beat launches to rounding (the two compile the same terms into different
    functions, so the compiler may fuse their multiply-adds differently), for an odd
    population with uneven beat counts."""
    params, beats = population(45, seed=11, max_beats=3)
    m = getattr(N, f"MODEL_{model}")
    if model == "LR91":
        params = params[:, :6]
    out = []
    for engine in (N.BATCH_PER_BEAT, N.BATCH_PERSISTENT):
        b = N.CellBatch(m, beats, params)
        b.set_engine(engine)
        b.run()
        out.append(b.results())
    for key in ("n_ap64", "n_ap32"):
        assert np.array_equal(out[0][key], out[1][key]), key
    rel = lambda a, b: np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3))
    assert rel(out[1]["states64"], out[0]["states64"]) <= 1e-8
    assert rel(out[1]["states32"], out[0]["states32"]) <= 1e-2
    assert np.max(np.abs(out[1]["apd64"] - out[0]["apd64"])) <= 1e-6
    assert np.max(np.abs(out[1]["apd32"] - out[0]["apd32"])) <= 0.1
    assert np.max(np.abs(out[1]["max_dv"] - out[0]["max_dv"])) <= 0.5
