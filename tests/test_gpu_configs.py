"""The benchmark configurations at their full size and duration, on the kernels the
benchmark runs: GPU FP64 against the oracle (per-node Vm every 1 ms within 1e-6
relative, CG iteration counts within one, activation maps), and the mixed-precision
path against GPU FP64 (max |dVm| <= 0.5 mV and activation within 1 ms, the target's
acceptance condition), as Chaste compares solutions in
heart/test/monodomain/TestMonodomainProblem.hpp:303-340 and activation maps in
TestNiederer2011BenchmarkSimulation.hpp:182-203.  Each test prints its measured
maxima (run with -s to see them)."""
import os

import numpy as np
import pytest

from tests import tissue_cases as TC

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-6
THRESHOLD = -40.0   # cg_config.activation_threshold default


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.lib().orc_set_threads(os.cpu_count() or 1)
    yield oracle
    oracle.lib().orc_set_threads(1)


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def _mark(act, v, t):
    new = (v > THRESHOLD) & (act < 0)
    act[new] = t


def _activation_diff(ta, tb):
    both = (ta >= 0) & (tb >= 0)
    assert np.array_equal(ta >= 0, tb >= 0), "different sets of activated nodes"
    return float(np.abs(ta[both] - tb[both]).max()) if both.any() else 0.0, int(both.sum())


def _fp64_and_mixed(N, orc, case, t_end, oracle_until, expect_pipe, every=1.0):
    """Steps the GPU FP64 and mixed tissues (and the oracle up to oracle_until ms)
    together, comparing every `every` ms."""
    g64, xyz = TC.make_gpu(N, precision=0, **case)
    g32, _ = TC.make_gpu(N, precision=1, **case)
    o = TC.make_oracle(orc, **case)[0] if oracle_until > 0 else None
    dt = case["dt_pde"]
    per = int(round(every / dt))
    n_cmp = int(round(t_end / every))
    st = g32.stats()
    if expect_pipe is not None:
        assert st.pipelined_nodes_per_thread == expect_pipe, st.pipelined_nodes_per_thread
    assert st.inner_preconditioner == N.INNER_PC_LINE
    act_o = -np.ones(g64.n)
    worst_rel, worst_mv, worst_its = 0.0, 0.0, 0
    for k in range(n_cmp):
        if o is not None and (k + 1) * every <= oracle_until + 1e-9:
            its_o = []
            for s in range(per):
                its_o.extend(o.step(1))
                _mark(act_o, o.voltage(), (k * per + s + 1) * dt)
            g64.step(per)
            its_g = g64.iteration_history(per)
            worst_its = max(worst_its, int(np.abs(np.asarray(its_g) - np.asarray(its_o)).max()))
            worst_rel = max(worst_rel, _rel(g64.voltage(), o.voltage()))
        else:
            if o is not None:
                o = None
            g64.step(per)
        g32.step(per)
        worst_mv = max(worst_mv, float(np.abs(g32.voltage() - g64.voltage()).max()))
    t64, t32 = g64.activation_times(), g32.activation_times()
    act_mixed, n_act = _activation_diff(t32, t64)
    out = dict(n=g64.n, fp64_vs_oracle_rel=worst_rel, fp64_vs_oracle_its=worst_its,
               mixed_vs_fp64_mv=worst_mv, mixed_vs_fp64_activation_ms=act_mixed, activated=n_act,
               mixed_iterations=int(g32.stats().total_cg_iterations), fp64_iterations=int(g64.stats().total_cg_iterations))
    if oracle_until >= t_end - 1e-9:
        act_fp64, _ = _activation_diff(t64, act_o)
        out["fp64_vs_oracle_activation_ms"] = act_fp64
    return out


def test_c1_sheet_full_size_against_oracle(N, orc):
    """LR91 2D sheet, 10,201 nodes, 100 ms: FP64 against the oracle all the way, mixed against FP64."""
    r = _fp64_and_mixed(N, orc, TC.LR91_SHEET_10201, t_end=100.0, oracle_until=100.0, expect_pipe=None)
    print("lr91_sheet_10201", r)
    assert r["fp64_vs_oracle_rel"] <= FP64_RTOL
    assert r["fp64_vs_oracle_its"] <= 1
    assert r["fp64_vs_oracle_activation_ms"] <= TC.LR91_SHEET_10201["dt_pde"] + 1e-12
    assert r["mixed_vs_fp64_mv"] <= 0.5
    assert r["mixed_vs_fp64_activation_ms"] <= 1.0
    assert r["activated"] == r["n"]


def test_c2_slab_full_size_against_oracle(N, orc):
    """TT06 3D slab, 442,401 nodes, 50 ms (the benchmark's configuration): FP64 against
    the oracle over the whole run; mixed (cg_mixed_pipe_kernel with 3 nodes per thread
    and the x-line inner preconditioner) against FP64."""
    r = _fp64_and_mixed(N, orc, TC.TT06_SLAB_442401, t_end=50.0, oracle_until=50.0, expect_pipe=3)
    print("tt06_slab_442401", r)
    assert r["fp64_vs_oracle_rel"] <= FP64_RTOL
    assert r["fp64_vs_oracle_its"] <= 1
    assert r["fp64_vs_oracle_activation_ms"] <= TC.TT06_SLAB_442401["dt_pde"] + 1e-12
    assert r["mixed_vs_fp64_mv"] <= 0.5
    assert r["mixed_vs_fp64_activation_ms"] <= 1.0
    assert r["activated"] > r["n"] // 2


def test_c5_transmural_slab_full_size(N, orc):
    """TT06 3D slab 2 x 2 x 1 cm at h = 0.0125 (2,099,601 nodes) with endo / mid / epi
    layers, 100 ms: mixed (the HBM-resident two-reduction solve with the x-line inner
    preconditioner, no pipelining) against FP64 over the whole run, FP64 against the
    oracle over the first 5 ms."""
    r = _fp64_and_mixed(N, orc, TC.transmural(TC.TT06_SLAB_2099601), t_end=100.0, oracle_until=5.0, expect_pipe=0)
    print("tt06_slab_2099601", r)
    assert r["fp64_vs_oracle_rel"] <= FP64_RTOL
    assert r["fp64_vs_oracle_its"] <= 1
    assert r["mixed_vs_fp64_mv"] <= 0.5
    assert r["mixed_vs_fp64_activation_ms"] <= 1.0
    assert r["activated"] > r["n"] // 4
