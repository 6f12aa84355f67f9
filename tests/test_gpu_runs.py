"""Mixed populations (cg_runs_*): uneven single-cell and cable runs with their own
parameters in one persistent launch, each run against the oracle -- single cells
against its Compute (forward Euler and Rush-Larsen), cables against its cable run --
for the autotuned shape and every other launch shape."""
import numpy as np
import pytest

from tests import cable_cases as CC

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-6   # mV, single-cell voltage samples vs the oracle
STATE_TOL = 1e-6   # relative, final states
CABLE_TOL = 1e-6   # probe voltages vs the oracle, relative to max(|V|, 1 mV)


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


def _cell_specs(N, model, rng, n, max_steps):
    P = N.num_params(model)
    specs = []
    for k in range(n):
        method = N.ODE_RUSH_LARSEN if k % 3 else N.ODE_FORWARD_EULER
        # forward Euler needs a shorter step: TT06 diverges at 0.005 ms (so does the oracle)
        dt = 0.01 if method == N.ODE_RUSH_LARSEN else (0.005 if model == N.MODEL_LR91 else 0.002)
        se = int(rng.choice([1, 5, 10]))
        steps = int(rng.integers(1, max_steps // se + 1)) * se
        params = np.exp(rng.normal(0.0, 0.15, size=P))
        if k % 4 == 0:
            stim = N.stimulus(N.STIM_SIMPLE, -25.5, 2.0, float(rng.uniform(0.0, 5.0)))
        else:
            period, start = float(rng.choice([50.0, 80.0])), float(rng.uniform(1.0, 10.0))
            stim = N.stimulus(N.STIM_REGULAR, -52.0, 1.0, start, period)
        specs.append(dict(method=method, dt=dt, se=se, steps=steps, params=params, stim=stim))
    return specs


def _oracle_stim(O, spec):
    g = spec["stim"]
    if g.kind == 1:
        return O.simple(g.magnitude, g.duration, g.start)
    return O.regular(g.magnitude, g.duration, g.period, g.start)


def _cable_specs(N, model, rng, sizes, dt):
    P = N.num_params(model)
    specs = []
    for n, steps, R in sizes:
        cfg = CC.cable_config(N, n_nodes=n, n_steps=steps, n_regions=R, dt=dt)
        cfg.model = model
        params = np.exp(rng.normal(0.0, 0.1, size=(R, P + 1)))
        probes = CC.even_probes(n, 5)
        specs.append(dict(cfg=cfg, params=params, probes=probes, se=int(rng.choice([1, 2]))))
    return specs


def _build(N, model, cells, cables):
    pop = N.RunPopulation(model)
    ids = [pop.add_cell(s["method"], s["steps"], s["dt"], s["se"], s["params"], s["stim"]) for s in cells]
    for s in cables:
        s["cfg"].n_steps -= s["cfg"].n_steps % s["se"]
    cids = [pop.add_cable(s["cfg"], s["params"], s["probes"], s["se"]) for s in cables]
    return pop, ids, cids


def _check_cells(N, O, model, pop, ids, cells):
    worst_v, worst_s = 0.0, 0.0
    for i, s in zip(ids, cells):
        st, tr = pop.result(i)
        y = O.initial_states(model)
        ref, y = O.cell_compute(model, O.RL if s["method"] == N.ODE_RUSH_LARSEN else O.FE, y, 0.0,
                                (s["steps"] // s["se"]) * (s["se"] * s["dt"]), s["dt"], s["se"] * s["dt"],
                                _oracle_stim(O, s), params=s["params"])
        assert tr.shape == (s["steps"] // s["se"] + 1,)
        assert ref.shape[0] == tr.shape[0]
        worst_v = max(worst_v, float(np.max(np.abs(tr - ref[:, 0]))))
        worst_s = max(worst_s, float(np.max(np.abs(st - y) / np.maximum(np.abs(y), 1e-3))))
    assert worst_v <= TRACE_TOL, worst_v
    assert worst_s <= STATE_TOL, worst_s


def _check_cables(O, pop, cids, cables):
    for i, s in zip(cids, cables):
        st, tr, its = pop.result(i)
        cfg = s["cfg"]
        ref = O.cable_run(CC.oracle_config(O, cfg), s["params"], s["probes"], traces=True)["traces"]
        ref = ref[s["se"] - 1::s["se"]]
        assert tr.shape == ref.shape
        err = np.max(np.abs(tr - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= CABLE_TOL, (cfg.n_nodes, err)
        assert its > 0
        assert np.allclose(st[:, 0][s["probes"]], tr[-1], rtol=0, atol=0)


def test_lr91_cells_and_cables_in_one_launch(N, oracle):
    O = oracle
    rng = np.random.default_rng(20261204)
    cells = _cell_specs(N, N.MODEL_LR91, rng, 70, 6000)
    cables = _cable_specs(N, N.MODEL_LR91, rng, [(50, 900, 1), (120, 1600, 2), (333, 600, 3), (700, 1200, 4)], 0.01)
    pop, ids, cids = _build(N, N.MODEL_LR91, cells, cables)
    tpb, cpt = pop.autotune(steps=100)
    assert tpb in (64, 128, 256) and cpt in (1, 2)
    pop.run()
    _check_cells(N, O, N.MODEL_LR91, pop, ids, cells)
    _check_cables(O, pop, cids, cables)


def test_tt06_population_with_a_cable(N, oracle):
    O = oracle
    rng = np.random.default_rng(7)
    cells = _cell_specs(N, N.MODEL_TT06, rng, 40, 20000)
    cables = _cable_specs(N, N.MODEL_TT06, rng, [(40, 1500, 2)], 0.002)
    pop, ids, cids = _build(N, N.MODEL_TT06, cells, cables)
    pop.set_shape(128, 1)
    pop.run()
    _check_cells(N, O, N.MODEL_TT06, pop, ids, cells)
    _check_cables(O, pop, cids, cables)


def test_every_launch_shape_gives_the_same_runs(N):
    rng = np.random.default_rng(11)
    cells = _cell_specs(N, N.MODEL_LR91, rng, 300, 3000)
    cables = _cable_specs(N, N.MODEL_LR91, rng, [(90, 500, 2), (300, 300, 1)], 0.01)
    pop, ids, cids = _build(N, N.MODEL_LR91, cells, cables)
    base = None
    for tpb in (64, 128, 256):
        for cpt in (1, 2):
            pop.set_shape(tpb, cpt)
            assert pop.shape() == (tpb, cpt)
            pop.run()
            got = [pop.result(i) for i in ids] + [pop.result(i)[:2] for i in cids]
            if base is None:
                base = got
                # a second run from the initial states repeats the first bit for bit
                pop.run()
                again = [pop.result(i) for i in ids] + [pop.result(i)[:2] for i in cids]
                for a, b in zip(base, again):
                    assert all(np.array_equal(x, y) for x, y in zip(a, b))
                continue
            for k, (a, b) in enumerate(zip(base, got)):
                if k < len(ids):   # single cells: the same arithmetic in every shape
                    assert all(np.array_equal(x, y) for x, y in zip(a, b)), (tpb, cpt, k)
                else:              # cables: block sums in another order
                    for x, y in zip(a, b):
                        assert np.max(np.abs(x - y) / np.maximum(np.abs(y), 1.0)) <= 1e-9, (tpb, cpt, k)
