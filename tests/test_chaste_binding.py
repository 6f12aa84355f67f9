"""The Chaste-side binding (chaste_b200/shim/GpuMonodomainProblem.hpp) compiled
against stand-ins of the Chaste classes it uses (tests/cpp/chaste_stubs) and
linked with libchastegpu.so: the host-side translations (stimuli, cell model and
ODE method, HeartConfig), and a MonodomainProblem solve through the binding's
hooks, which must equal the same run made directly through the C-ABI bit for bit."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def binding_exe(native, tmp_path_factory):
    lib_dir = os.path.join(ROOT, "chaste_b200", "lib")
    exe = str(tmp_path_factory.mktemp("binding") / "test_gpu_binding")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wno-unused-variable", "-Wno-unused-parameter",
           "-Wno-unused-but-set-variable",
           "-I", os.path.join(ROOT, "tests", "cpp", "chaste_stubs"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "chaste_b200", "shim"), "-I", os.path.join(ROOT, "chaste_b200", "csrc"),
           os.path.join(ROOT, "tests", "cpp", "test_gpu_binding.cpp"), "-L", lib_dir, "-lchastegpu",
           f"-Wl,-rpath,{lib_dir}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_binding_translations(binding_exe):
    out = subprocess.run([binding_exe, "describe"], check=True, capture_output=True, text=True).stdout.split("\n")
    assert out[0] == "simple 1 -25.5 2 50"                 # SimpleStimulus read through its serialize()
    assert out[1] == "regular 2 -52 1 10 1000 5000"
    assert out[2] == "zero 0"
    assert out[3] == "model 0 method 0"                    # LR91, forward Euler
    assert out[4] == "config pc 2 abs 0 tol 1e-08"         # HeartConfig bjacobi -> CG_PC_BJACOBI
    assert out[5].startswith("hypre rejected")


def test_binding_raises_without_a_device(binding_exe):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    r = subprocess.run([binding_exe, "run", "slab", "jacobi"], capture_output=True, text=True)
    assert r.returncode == 3
    assert "EXCEPTION: cg_create: CUDA runtime error or no CUDA device" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("mesh,pc", [("slab", "jacobi"), ("mesh", "jacobi"), ("slab", "bjacobi")])
def test_binding_solve_equals_direct_calls(binding_exe, mesh, pc):
    r = subprocess.run([binding_exe, "run", mesh, pc], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "max |binding - direct| 0 " in r.stdout
