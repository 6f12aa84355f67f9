"""The C-ABI library loads without a GPU and exports every symbol of include/chaste_gpu.h."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "chaste_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cg_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("cg_create", "cg_set_mesh", "cg_set_cells", "cg_set_stimulus", "cg_step",
                 "cg_get_voltage", "cg_get_caches", "cg_snapshot", "cg_restore", "cg_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(native):
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(declared_functions()) <= set(native.SIGNATURES)


def test_defaults_and_status_strings(native):
    c = native.default_config()
    assert (c.ode_time_step, c.pde_time_step, c.surface_area_to_volume_ratio, c.capacitance) == (0.01, 0.01, 1400.0, 1.0)
    assert c.use_absolute_tolerance == 1 and c.ksp_tolerance == 2e-4 and c.max_iterations == 10000
    for s in range(11):
        assert native.lib().cg_status_string(s)
    assert native.num_states(native.MODEL_LR91) == 8
    assert native.num_states(native.MODEL_TT06) == 19
    assert native.num_params(native.MODEL_TT06) == 9


def test_invalid_configs_are_rejected_before_touching_a_device(native):
    c = native.default_config()
    c.pde_time_step = 0.0
    with pytest.raises(native.ChasteGpuError) as e:
        native.Tissue(c)
    assert e.value.status == 1
    c = native.default_config()
    c.ksp_preconditioner = native.PC_BJACOBI
    c.precision = native.PRECISION_MIXED   # bjacobi is an FP64 preconditioner here
    with pytest.raises(native.ChasteGpuError) as e:
        native.Tissue(c)
    assert e.value.status == 10


def test_no_cpu_fallback_without_a_device(native):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(native.ChasteGpuError) as e:
        native.Tissue(native.default_config())
    assert e.value.status == 2
