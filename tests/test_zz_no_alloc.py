"""cg_slab_solve_noalloc against the regular tissue path.

The allocation-free entry point exists for callers that cannot allocate device
memory themselves (an embedding program whose pool owns every device buffer,
or code running where cudaMalloc is not allowed): they hand in their own
device buffers and the library works inside a fixed array it reserved at load
time.  This test gives it the same right-hand side and initial guess that a
cg_step diffusion solve used, through the C-ABI, and checks that the solution
matches the one cg_step produced, on two calls in a row with different slabs
(so the second call starts from the first call's leftover scratch contents).
It lives in its own file, collected last, so a failing run has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from tests import tissue_cases as TC

pytestmark = pytest.mark.gpu

TOL = 1e-6   # the FP64 parity tolerance of the tissue tests (relative to max(|V|, 1 mV))


@pytest.fixture(scope="module")
def N(native):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return native


def _one_solve_from_tissue(N, case, warm_steps):
    """Run the regular path, then repeat its last diffusion solve through the no-alloc entry point."""
    import torch

    g, _ = TC.make_gpu(N, **case)
    g.step(warm_steps)
    v0 = g.voltage()
    g.step(1)
    v1 = g.voltage()
    its_ref = int(g.iteration_history(1)[0])
    iion, istim = g.caches()
    am, cm, dt = 1400.0, 1.0, case["dt_pde"]
    z = am * cm * v0 * (1.0 / dt) + (-am * iion - istim)   # MonodomainSolver.cpp:92-101
    d_z = torch.tensor(z, dtype=torch.float64, device="cuda")
    d_x = torch.tensor(v0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cfg = N.default_config()
    cfg.pde_time_step = dt
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, case.get("rel_tol", 1e-8)
    cfg.ksp_preconditioner = N.PC_JACOBI
    cfg.use_mass_lumping = 1 if case.get("lump") else 0
    sig = np.ascontiguousarray(np.asarray(case["sigma"], dtype=np.float64)[: case["dim"]])
    its = C.c_int(-1)
    rc = N.lib().cg_slab_solve_noalloc(C.byref(cfg), case["dim"], case["h"], *case["size"], N.dptr(sig),
                                       C.c_void_p(d_z.data_ptr()), C.c_void_p(d_x.data_ptr()), None, C.byref(its))
    assert rc == 0, N.STATUS_NAMES.get(rc, rc)
    x = d_x.cpu().numpy()
    err = np.max(np.abs(x - v1) / np.maximum(np.abs(v1), 1.0))
    return err, its.value, its_ref


def test_noalloc_solve_matches_tissue_solve_twice(N):
    # first call: 2D LR91 sheet; second call: 3D TT06 slab (other shape, reused scratch)
    err1, its1, ref1 = _one_solve_from_tissue(N, dict(TC.LR91_2D), warm_steps=5)
    assert err1 <= TOL, err1
    assert abs(its1 - ref1) <= 1
    err2, its2, ref2 = _one_solve_from_tissue(N, dict(TC.TT06_3D), warm_steps=12)
    assert err2 <= TOL, err2
    assert abs(its2 - ref2) <= 1


@pytest.mark.parametrize("name", ["cable_1d", "sheet_2d_lumped_mass", "slab_3d_at_the_limit"])
def test_noalloc_solve_other_shapes(N, name):
    """A 1D cable (3 offsets), a lumped-mass sheet, and a 3D slab of exactly the
    32,768-node limit (64 blocks of the persistent kernel, 15 offsets)."""
    if name == "cable_1d":
        case = dict(TC.LR91_2D, dim=1, size=(1.0, 0.0, 0.0), box_hi=(0.0199,))
    elif name == "sheet_2d_lumped_mass":
        case = dict(TC.LR91_2D, lump=True)
    else:
        case = dict(TC.TT06_3D, size=(0.31, 0.31, 0.31), box_hi=(0.05, 0.05, 0.05))
    err, its, ref = _one_solve_from_tissue(N, case, warm_steps=6)
    assert err <= TOL, err
    assert abs(its - ref) <= 1


def test_noalloc_rejects_sizes_beyond_its_scratch(N):
    import torch

    cfg = N.default_config()
    sig = np.array([1.75, 1.75, 1.75])
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    # 0.5 x 0.5 x 0.5 cm at h = 0.01 is 132,651 nodes, above the 32,768-node limit
    rc = N.lib().cg_slab_solve_noalloc(C.byref(cfg), 3, 0.01, 0.5, 0.5, 0.5, N.dptr(sig),
                                       C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), None, None)
    assert rc == 1
