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


def test_removable_singularities_are_finite_in_both_precisions(tmp_path):
    """GHK-type 0/0 points (LR91 alpha_m at -47.13 mV and Xi at -77 mV, TT06 i_CaL at 15 mV) give
    finite values in float and double, continuous with their neighbourhood."""
    src = tmp_path / "s.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cmath>
#include "lr91.h"
#include "tt06.h"
template <class M, typename T> double iion_at(double v) {
    T y[M::kNumStates], p[M::kNumParams];
    for (int i = 0; i < M::kNumStates; ++i) y[i] = (T)M::kInitialStates[i];
    for (int i = 0; i < M::kNumParams; ++i) p[i] = T(1);
    y[0] = (T)v;
    T dy[M::kNumStates];
    M::template rhs<T>(y, T(0), T(1), p, dy);
    double s = 0;
    for (int i = 0; i < M::kNumStates; ++i) s += (double)dy[i];
    return s + (double)M::template iionic<T>(y, T(1), p);
}
int main() {
    const double pts[3] = {-47.13, -77.0, 15.0};
    for (double v : pts) {
        double a = iion_at<chb::LuoRudy1991, float>(v), b = iion_at<chb::LuoRudy1991, double>(v);
        double c = iion_at<chb::TenTusscher2006Epi, float>(v), d = iion_at<chb::TenTusscher2006Epi, double>(v);
        double e = iion_at<chb::TenTusscher2006Epi, double>(v + 1e-3);
        std::printf("%.17g %.17g %.17g %.17g %.17g\n", a, b, c, d, e);
    }
}
''')
    exe = tmp_path / "s"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "chaste_b200", "csrc", "models"),
                    str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    import math

    for line in filter(None, out):
        a, b, c, d, e = map(float, line.split())
        assert all(math.isfinite(x) for x in (a, b, c, d, e))
        assert abs(a - b) <= 1e-3 * max(1.0, abs(b))
        assert abs(c - d) <= 1e-3 * max(1.0, abs(d))
        assert abs(d - e) <= 1e-1 * max(1.0, abs(d))
