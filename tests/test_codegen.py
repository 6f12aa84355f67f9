"""The CellML emitter: generated headers are current and compile as plain C++."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CELLML = "/root/reference/heart/src/odes/cellml"


@pytest.mark.skipif(not os.path.isdir(CELLML), reason="CellML sources not mounted")
def test_generated_headers_are_current(tmp_path):
    from chaste_b200.codegen import emit

    emit.generate(CELLML, [str(tmp_path)])
    for name in ("lr91.h", "tt06.h"):
        new = (tmp_path / name).read_text()
        old = open(os.path.join(ROOT, "chaste_b200", "csrc", "models", name)).read()
        assert new == old, f"{name} is stale: re-run python -m chaste_b200.codegen.emit"


def test_headers_compile_as_cpp(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "lr91.h"\n#include "tt06.h"\n'
                   "int main(){double y[19]={0};double p[9]={1,1,1,1,1,1,1,1,1};double dy[19];"
                   "chb::LuoRudy1991::rhs<double>(y,0.0,1.0,p,dy);"
                   "float yf[19]={0},pf[9]={0},df[19];"
                   "chb::TenTusscher2006Epi::rhs<float>(yf,0.f,1.f,pf,df);return 0;}\n")
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I",
                    os.path.join(ROOT, "chaste_b200", "csrc", "models"), str(src)], check=True)


def test_rush_larsen_state_classification():
    txt = open(os.path.join(ROOT, "chaste_b200", "csrc", "models", "lr91.h")).read()
    flags = [s.strip() == "true" for s in re.search(r"kRushLarsen\[8\] = \{([^}]*)\}", txt).group(1).split(",")]
    # V and Cai forward Euler; the six gates Rush-Larsen
    assert flags == [False, True, True, True, True, True, True, False]
    txt = open(os.path.join(ROOT, "chaste_b200", "csrc", "models", "tt06.h")).read()
    names = re.search(r"kStateNames\[19\] = \{([^}]*)\}", txt).group(1).replace('"', "").split(", ")
    flags = [s.strip() == "true" for s in re.search(r"kRushLarsen\[19\] = \{([^}]*)\}", txt).group(1).split(",")]
    rl = {n for n, f in zip(names, flags) if f}
    # the twelve gates plus R_prime (affine in itself); V and the concentrations by forward Euler
    assert rl == {"Xr1", "Xr2", "Xs", "m", "h", "j", "d", "f", "f2", "fCass", "s", "r", "R_prime"}
