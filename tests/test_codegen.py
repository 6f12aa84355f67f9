"""The CellML emitter: generated headers are current and compile as plain C++."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the Chaste source tree, when present: $CHASTE_SOURCE_DIR (the CellML files are not vendored)
CELLML = os.path.join(os.environ.get("CHASTE_SOURCE_DIR", ""), "heart", "src", "odes", "cellml")


@pytest.mark.skipif(not os.path.isdir(CELLML), reason="CHASTE_SOURCE_DIR not set or without the CellML sources")
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


def test_generated_vjps_match_finite_differences(tmp_path):
    """The emitted reverse-mode products of the RHS and of GetIIonic against central differences."""
    src = tmp_path / "v.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cmath>
#include <initializer_list>
#include "lr91.h"
#include "tt06.h"
template <class M> double check(double vshift) {
    const int S = M::kNumStates, P = M::kNumParams;
    double y[S], p[P], w[S], gy[S], gp[P], dy1[S], dy2[S], worst = 0;
    for (int i = 0; i < S; ++i) { y[i] = M::kInitialStates[i]; w[i] = std::sin(1.0 + i); }
    y[0] += vshift;
    for (int k = 0; k < P; ++k) p[k] = 1.0 + 0.1 * k;
    for (int i = 0; i < S; ++i) gy[i] = 0;
    for (int k = 0; k < P; ++k) gp[k] = 0;
    M::template vjp_rhs<double>(y, -10.0, 1.0, p, w, gy, gp);
    for (int j = 0; j < S + P; ++j) {
        double* x = j < S ? &y[j] : &p[j - S];
        const double h = 1e-6 * std::fmax(std::fabs(*x), 1e-3), x0 = *x;
        *x = x0 + h; M::template rhs<double>(y, -10.0, 1.0, p, dy1);
        *x = x0 - h; M::template rhs<double>(y, -10.0, 1.0, p, dy2);
        *x = x0;
        double fd = 0;
        for (int i = 0; i < S; ++i) fd += w[i] * (dy1[i] - dy2[i]) / (2 * h);
        const double g = j < S ? gy[j] : gp[j - S];
        worst = std::fmax(worst, std::fabs(g - fd) / std::fmax(1.0, std::fabs(fd)));
    }
    for (int i = 0; i < S; ++i) gy[i] = 0;
    for (int k = 0; k < P; ++k) gp[k] = 0;
    double one = 1.0;
    M::template vjp_iionic<double>(y, 0.0, 1.0, p, &one, gy, gp);
    for (int j = 0; j < S + P; ++j) {
        double* x = j < S ? &y[j] : &p[j - S];
        const double h = 1e-6 * std::fmax(std::fabs(*x), 1e-3), x0 = *x;
        *x = x0 + h; const double a = M::template iionic<double>(y, 1.0, p);
        *x = x0 - h; const double b = M::template iionic<double>(y, 1.0, p);
        *x = x0;
        const double fd = (a - b) / (2 * h), g = j < S ? gy[j] : gp[j - S];
        worst = std::fmax(worst, std::fabs(g - fd) / std::fmax(1.0, std::fabs(fd)));
    }
    return worst;
}
int main() {
    double w = 0;
    for (double dv : {0.0, 30.0, 90.0}) { w = std::fmax(w, check<chb::LuoRudy1991>(dv)); w = std::fmax(w, check<chb::TenTusscher2006Epi>(dv)); }
    std::printf("%.3e\n", w);
}
''')
    exe = tmp_path / "v"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "chaste_b200", "csrc", "models"),
                    str(src), "-o", str(exe)], check=True)
    worst = float(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    assert worst <= 1e-5, worst


def test_hoisted_voltage_terms_reproduce_the_substep_terms(tmp_path):
    """rl_vterms + rl_terms_states_vt (the voltage-only subexpressions evaluated once per
    PDE step) give rl_terms_states' rates and limits for voltages across the action
    potential, the GHK singular points included, in double to 1e-12 relative."""
    src = tmp_path / "h.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cmath>
#include "lr91.h"
#include "tt06.h"
template <class M> double worst() {
    double w = 0.0;
    const double vs[] = {-90.0, -77.0, -47.13, -20.0, 0.0, 15.0, 15.0000001, 40.0};
    for (double v : vs) {
        double y[M::kNumStates], p[M::kNumParams], r1[M::kNumStates], i1[M::kNumStates];
        double r2[M::kNumStates], i2[M::kNumStates], vt[M::kNumVTerms > 0 ? M::kNumVTerms : 1];
        for (int i = 0; i < M::kNumStates; ++i) { y[i] = M::kInitialStates[i]; r1[i] = r2[i] = i1[i] = i2[i] = 0.0; }
        for (int i = 0; i < M::kNumParams; ++i) p[i] = 1.0 + 0.05 * i;
        y[0] = v;
        M::template rl_terms_states<double>(y, -3.0, 1.0, p, r1, i1);
        M::template rl_vterms<double>(y, p, vt);
        M::template rl_terms_states_vt<double>(y, -3.0, 1.0, p, vt, r2, i2);
        for (int i = 0; i < M::kNumStates; ++i) {
            w = std::fmax(w, std::fabs(r1[i] - r2[i]) / std::fmax(std::fabs(r1[i]), 1e-30));
            w = std::fmax(w, std::fabs(i1[i] - i2[i]) / std::fmax(std::fabs(i1[i]), 1e-30));
        }
    }
    return w;
}
int main() { std::printf("%.3e %.3e\n", worst<chb::LuoRudy1991>(), worst<chb::TenTusscher2006Epi>()); return 0; }
''')
    exe = tmp_path / "h"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "chaste_b200", "csrc", "models"),
                    str(src), "-o", str(exe)], check=True)
    lr, tt = (float(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                               text=True).stdout.split())
    assert lr <= 1e-12 and tt <= 1e-12, (lr, tt)
