// Shared definitions for the generated cell-model headers (lr91.h, tt06.h).
//
// The headers are plain C++17 compiled by g++ for the CPU oracle and by nvcc
// for the sm_100a kernels.  Every model is a struct with static member
// templates over the arithmetic type T (double or float):
//   rhs(y, stim, cm, p, dy)          dy/dt of every state (y[0] is V)
//   rl_terms(y, stim, cm, p, rate, inf)
//   iionic(y, cm, p)                 GetIIonic in uA/cm^2
// and constexpr tables (initial states, names, Rush-Larsen flags, ranges).
#pragma once

#include <cmath>
#include <type_traits>

#if defined(__CUDACC__)
#define CHB_HD __host__ __device__ __forceinline__
#define CHB_UNROLL _Pragma("unroll")
#define CHB_NOUNROLL _Pragma("unroll 1")
#else
#define CHB_HD inline
#define CHB_UNROLL
#define CHB_NOUNROLL
#endif

#ifndef NAN
#define NAN (__builtin_nanf(""))
#endif

namespace chb {

// Elementary functions seen by the generated model code (which calls exp/log/
// sqrt as m_exp/m_log/m_sqrt/m_pow).  Double precision always calls the correctly rounded library
// functions; single precision on the device uses the SFU-based fast
// intrinsics (MUFU.EX2/LG2) when CHB_FAST_FP32 is 1 -- the mixed-precision
// path trades their few-ulp error for throughput and is checked against FP64.
#ifndef CHB_FAST_FP32
#define CHB_FAST_FP32 1
#endif
// On the device the double-precision functions are called, not inlined
// (CHB_FP64_CALLS, default 1): a cell model evaluates dozens of them per step, and one
// shared copy of each keeps the straight-line model code small enough for the
// instruction cache -- inlined, the FP64 kernels stalled on instruction fetch.  The
// values are those of the inlined library functions.
#ifndef CHB_FP64_CALLS
#define CHB_FP64_CALLS 1
#endif
#if defined(__CUDA_ARCH__) && CHB_FP64_CALLS
__device__ __noinline__ double m_exp_call(double x) { return ::exp(x); }
__device__ __noinline__ double m_log_call(double x) { return ::log(x); }
__device__ __noinline__ double m_pow_call(double x, double y) { return ::pow(x, y); }
CHB_HD double m_exp(double x) { return m_exp_call(x); }
CHB_HD double m_log(double x) { return m_log_call(x); }
CHB_HD double m_pow(double x, double y) { return m_pow_call(x, y); }
#else
CHB_HD double m_exp(double x) { return ::exp(x); }
CHB_HD double m_log(double x) { return ::log(x); }
CHB_HD double m_pow(double x, double y) { return ::pow(x, y); }
#endif
CHB_HD double m_sqrt(double x) { return ::sqrt(x); }
CHB_HD float m_exp(float x) {
#if defined(__CUDA_ARCH__) && CHB_FAST_FP32
    return __expf(x);
#else
    return ::expf(x);
#endif
}
CHB_HD float m_log(float x) {
#if defined(__CUDA_ARCH__) && CHB_FAST_FP32
    return __logf(x);
#else
    return ::logf(x);
#endif
}
CHB_HD float m_sqrt(float x) { return ::sqrtf(x); }
CHB_HD float m_pow(float x, float y) {
#if defined(__CUDA_ARCH__) && CHB_FAST_FP32
    return __powf(x, y);
#else
    return ::powf(x, y);
#endif
}

// Quotients.  m_div(a, b) is a / b, except in single precision on the device
// (CHB_FAST_FP32) where it is __fdividef (the SFU reciprocal, 2 ulp).
// m_divk(x, k, kinv) divides by the literal k: exactly in double, by
// multiplication with the rounded reciprocal kinv in float.
CHB_HD double m_div(double a, double b) { return a / b; }
CHB_HD double m_divk(double x, double k, double kinv) {
    (void)kinv;
    return x / k;
}
CHB_HD float m_div(float a, float b) {
#if defined(__CUDA_ARCH__) && CHB_FAST_FP32
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
CHB_HD float m_divk(float x, float k, float kinv) {
#if defined(__CUDA_ARCH__) && CHB_FAST_FP32
    (void)k;
    return x * kinv;
#else
    (void)kinv;
    return x / k;
#endif
}

// Half-width, in units of the exponent argument U, of the window around a
// removable singularity of a GHK-type term within which the emitted code
// interpolates linearly (as chaste_codegen's singularity fixes do).  FP32 needs
// a wider window: exp(U) - 1 loses all digits once |U| nears float epsilon.
template <typename T>
CHB_HD constexpr T singularity_offset();
template <>
CHB_HD constexpr double singularity_offset<double>() { return 1e-7; }
template <>
CHB_HD constexpr float singularity_offset<float>() { return 2e-3f; }

// Forward-Euler step of the non-voltage states with V clamped at y[0]
// (AbstractCardiacCell::ComputeExceptVoltage with SetVoltageDerivativeToZero,
// heart/src/odes/AbstractCardiacCell.cpp:90-105, one EulerIvpOdeSolver step,
// ode/src/solver/EulerIvpOdeSolver.cpp:38-57).
template <class Model, typename T>
CHB_HD void fe_step_except_voltage(T* y, T stim, T cm, const T* p, T dt) {
    T dy[Model::kNumStates];
    Model::template rhs<T>(y, stim, cm, p, dy);
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i) y[i] += dt * dy[i];
}

// Rush-Larsen step of the non-voltage states with V clamped at y[0]
// (AbstractRushLarsenCardiacCell::ComputeExceptVoltage,
// heart/src/odes/AbstractRushLarsenCardiacCell.cpp:106-128).
template <class Model, typename T>
CHB_HD void rl_step_except_voltage(T* y, T stim, T cm, const T* p, T dt) {
    T rate[Model::kNumStates];
    T inf[Model::kNumStates];
    Model::template rl_terms<T>(y, stim, cm, p, rate, inf);
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i) {
        if (Model::rush_larsen(i)) {
            y[i] = inf[i] + (y[i] - inf[i]) * m_exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}

// The same Rush-Larsen step over the substeps of one PDE step, with the terms of the
// voltage-only states (Model::rl_voltage_only) taken out of the substep loop: V is
// clamped, so their inf and exp(rate*dt) are the values rl_step_except_voltage would
// recompute at every substep.  rl_freeze_voltage_terms forms them once, together with
// the voltage-only subexpressions of the other states' terms (Model::rl_vterms); each
// substep then evaluates only what depends on the other states.
template <class Model, typename T>
CHB_HD void rl_freeze_voltage_terms(const T* y, const T* p, T dt, T* vinf, T* vfac, T* vt) {
    T rate[Model::kNumStates];
    Model::template rl_terms_voltage<T>(y, p, rate, vinf);
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i)
        if (Model::rl_voltage_only(i)) vfac[i] = m_exp(rate[i] * dt);
    Model::template rl_vterms<T>(y, p, vt);
}

template <class Model, typename T>
CHB_HD void rl_step_except_voltage_frozen(T* y, T stim, T cm, const T* p, T dt, const T* vinf, const T* vfac,
                                          const T* vt) {
    T rate[Model::kNumStates];
    T inf[Model::kNumStates];
    Model::template rl_terms_states_vt<T, const T*>(y, stim, cm, p, vt, rate, inf);
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i) {
        if (Model::rl_voltage_only(i)) {
            y[i] = vinf[i] + (y[i] - vinf[i]) * vfac[i];
        } else if (Model::rush_larsen(i)) {
            y[i] = inf[i] + (y[i] - inf[i]) * m_exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}

// The frozen terms as slots of a per-thread column: the voltage-only states' inf
// (slots [0, NV)), their exp(rate*dt) (slots [NV, 2 NV)) and the voltage-only
// subexpressions (slots [2 NV, 2 NV + kNumVTerms)), NV the number of voltage-only
// states.  Slot k of a thread lives at column[k * STRIDE].
template <class Model>
CHB_HD constexpr int frozen_slot(int i) {
    int c = 0;
    for (int j = 1; j < i; ++j) c += Model::rl_voltage_only(j) ? 1 : 0;
    return c;
}
template <class Model>
struct FrozenSlots {
    static constexpr int kVoltageOnly = frozen_slot<Model>(Model::kNumStates);
    static constexpr int kSlots = 2 * kVoltageOnly + Model::kNumVTerms;
};

#if defined(__CUDACC__)
// Reads slot k of a shared-memory column where the model code uses it: the loads are
// volatile, so the compiler neither hoists them out of the substep loop nor keeps
// the terms in registers across it.
template <typename T, int STRIDE>
struct FrozenColumn {
    const T* base;
    __device__ __forceinline__ T operator[](int k) const { return *(const volatile T*)(base + k * STRIDE); }
};

// rl_freeze_voltage_terms with the terms written to a shared-memory column.
template <class Model, typename T, int STRIDE>
__device__ __forceinline__ void rl_freeze_voltage_terms_column(const T* y, const T* p, T dt, T* column) {
    constexpr int NV = FrozenSlots<Model>::kVoltageOnly;
    T rate[Model::kNumStates], inf[Model::kNumStates];
    T vt[Model::kNumVTerms > 0 ? Model::kNumVTerms : 1];
    Model::template rl_terms_voltage<T>(y, p, rate, inf);
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i)
        if (Model::rl_voltage_only(i)) {
            column[frozen_slot<Model>(i) * STRIDE] = inf[i];
            column[(NV + frozen_slot<Model>(i)) * STRIDE] = m_exp(rate[i] * dt);
        }
    Model::template rl_vterms<T>(y, p, vt);
CHB_UNROLL
    for (int k = 0; k < Model::kNumVTerms; ++k) column[(2 * NV + k) * STRIDE] = vt[k];
}

// rl_step_except_voltage_frozen reading the frozen terms from the column: the same
// arithmetic on the same values.
template <class Model, typename T, int STRIDE>
__device__ __forceinline__ void rl_step_except_voltage_column(T* y, T stim, T cm, const T* p, T dt,
                                                              const T* column) {
    constexpr int NV = FrozenSlots<Model>::kVoltageOnly;
    T rate[Model::kNumStates];
    T inf[Model::kNumStates];
    const FrozenColumn<T, STRIDE> vt{column + 2 * NV * STRIDE};
    Model::template rl_terms_states_vt<T, FrozenColumn<T, STRIDE>>(y, stim, cm, p, vt, rate, inf);
    const FrozenColumn<T, STRIDE> fz{column};
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i) {
        if (Model::rl_voltage_only(i)) {
            const T vinf = fz[frozen_slot<Model>(i)];
            y[i] = vinf + (y[i] - vinf) * fz[NV + frozen_slot<Model>(i)];
        } else if (Model::rush_larsen(i)) {
            y[i] = inf[i] + (y[i] - inf[i]) * m_exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}
#endif

// Full single-cell steps including the voltage (Compute / SolveAndUpdateState).
template <class Model, typename T>
CHB_HD void fe_step(T* y, T stim, T cm, const T* p, T dt) {
    T dy[Model::kNumStates];
    Model::template rhs<T>(y, stim, cm, p, dy);
CHB_UNROLL
    for (int i = 0; i < Model::kNumStates; ++i) y[i] += dt * dy[i];
}

// AbstractRushLarsenCardiacCell::Compute order: EvaluateEquations, then V by
// forward Euler (UpdateTransmembranePotential), then the other states
// (heart/src/odes/AbstractRushLarsenCardiacCell.cpp:86-94, 149-153).
template <class Model, typename T>
CHB_HD void rl_step(T* y, T stim, T cm, const T* p, T dt) {
    T rate[Model::kNumStates];
    T inf[Model::kNumStates];
    Model::template rl_terms<T>(y, stim, cm, p, rate, inf);
    y[0] += dt * rate[0];
CHB_UNROLL
    for (int i = 1; i < Model::kNumStates; ++i) {
        if (Model::rush_larsen(i)) {
            y[i] = inf[i] + (y[i] - inf[i]) * m_exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}

// VerifyStateVariables analogue: true when every gate is in [0,1] and every
// concentration is positive (and nothing is NaN).
// Backward-Euler step (AbstractBackwardEulerCardiacCell, heart/src/odes/
// AbstractBackwardEulerCardiacCell.hpp: ComputeOneStepExceptVoltage, and
// SolveAndUpdateState with V first by UpdateTransmembranePotential).  With
// with_voltage, V takes an explicit Euler step first; then every state whose ODE is
// linear in itself, f = a + b y (the Rush-Larsen states: b = rate, a = -rate * inf),
// takes the exact implicit step y' = (y + dt a) / (1 - dt b) at the (new) V; then the
// remaining states solve the implicit residual R(y') = y' - y - dt f(V, gates', y')
// by Newton's method (CardiacNewtonSolver, heart/src/odes/CardiacNewtonSolver.hpp:
// Gaussian elimination without pivoting), here with a finite-difference Jacobian and
// iterated until the update is below 1e-13 (double) / 1e-6 (float) relative, at most
// 20 times.  Chaste's generated cells (chaste_codegen's backward-Euler option) take
// the same steps with an analytic Jacobian and stop at an update of 1e-6.
template <class Model, typename T>
CHB_HD void be_step(T* y, T stim, T cm, const T* p, T dt, bool with_voltage) {
    constexpr int S = Model::kNumStates;
    T dy[S], rate[S], inf[S], old[S];
    if (with_voltage) {
        Model::template rhs<T>(y, stim, cm, p, dy);
        y[0] += dt * dy[0];
    }
    Model::template rl_terms<T>(y, stim, cm, p, rate, inf);
CHB_UNROLL
    for (int k = 0; k < S; ++k) old[k] = y[k];
CHB_UNROLL
    for (int k = 1; k < S; ++k)
        if (Model::rush_larsen(k)) y[k] = (old[k] - dt * rate[k] * inf[k]) / (T(1) - dt * rate[k]);
    int nl[S];
    int m = 0;
    for (int k = 1; k < S; ++k)
        if (!Model::rush_larsen(k)) nl[m++] = k;
    if (m == 0) return;
    const T tol = sizeof(T) == 8 ? T(1e-13) : T(1e-6);
    const T fd = sizeof(T) == 8 ? T(1e-7) : T(3e-3);
    T r[S], r2[S], J[S][S], upd[S], yy[S];
    for (int it = 0; it < 20; ++it) {
        Model::template rhs<T>(y, stim, cm, p, dy);
        for (int q = 0; q < m; ++q) r[q] = y[nl[q]] - old[nl[q]] - dt * dy[nl[q]];
        for (int c = 0; c < m; ++c) {
            for (int k = 0; k < S; ++k) yy[k] = y[k];
            const T base = y[nl[c]] < T(0) ? -y[nl[c]] : y[nl[c]];
            const T hh = fd * (base > T(1e-8) ? base : T(1e-8));
            yy[nl[c]] += hh;
            Model::template rhs<T>(yy, stim, cm, p, dy);
            for (int q = 0; q < m; ++q) r2[q] = yy[nl[q]] - old[nl[q]] - dt * dy[nl[q]];
            for (int q = 0; q < m; ++q) J[q][c] = (r2[q] - r[q]) / hh;
        }
        for (int i = 0; i < m; ++i)
            for (int ii = i + 1; ii < m; ++ii) {
                const T fact = J[ii][i] / J[i][i];
                for (int j = i; j < m; ++j) J[ii][j] -= fact * J[i][j];
                r[ii] -= fact * r[i];
            }
        bool done = true;
        for (int i = m; i-- > 0;) {
            upd[i] = r[i];
            for (int j = i + 1; j < m; ++j) upd[i] -= J[i][j] * upd[j];
            upd[i] /= J[i][i];
        }
        for (int q = 0; q < m; ++q) {
            y[nl[q]] -= upd[q];
            const T a = upd[q] < T(0) ? -upd[q] : upd[q];
            const T b = y[nl[q]] < T(0) ? -y[nl[q]] : y[nl[q]];
            if (a > tol * (b > T(1) ? b : T(1))) done = false;
        }
        if (done) break;
    }
}

// Generalised Rush-Larsen steps (GRL1IvpOdeSolver::CalculateNextYValue,
// ode/src/solver/GRL1IvpOdeSolver.cpp:47-93; GRL2IvpOdeSolver::CalculateNextYValue,
// ode/src/solver/GRL2IvpOdeSolver.cpp:47-119) of a cell whose ODE solver is GRL1 or
// GRL2: every state is advanced by the exponential step linearised in itself,
//     y_i' = y_i + f_i / a_i (exp(a_i dt) - 1),  a_i = (f_i(y + delta e_i) - f_i(y)) / delta,
// or by forward Euler where |a_i| < delta, with delta = 1e-8.  GRL2 takes a half step
// to the midpoint first, then re-linearises each state at the midpoint with its own
// component held at the start value.  With VOLT false the voltage derivative is zero
// (ComputeExceptVoltage's SetVoltageDerivativeToZero), so V and its partial are skipped.
// In single precision a perturbation of 1e-8 is below the resolution of most states,
// so the float step perturbs by 2^-10 max(|y_i|, 1e-6) and divides by the perturbation.
template <typename T>
CHB_HD T grl_perturbation(T y) {
    if (sizeof(T) == 8) return T(1.0e-8);
    const T a = y < T(0) ? -y : y;
    return T(0.0009765625) * (a > T(1e-6) ? a : T(1e-6));
}

template <typename T>
CHB_HD T grl_update(T y, T f, T a, T dt) {
    const T aa = a < T(0) ? -a : a;
    return aa < T(1.0e-8) ? y + f * dt : y + (f / a) * (m_exp(a * dt) - T(1));
}

// Calls f(std::integral_constant<int, i>) for a runtime i in [I, N): a loop over the
// states that dispatches to straight-line code per state keeps each state's
// perturbed evaluation (pruned by the compiler to what its own derivative needs)
// in a block of its own, so that nothing stays live from one state to the next.
template <int I, int N, class F>
CHB_HD void dispatch_state(int i, F& f) {
    if constexpr (I < N) {
        if (i == I) f(std::integral_constant<int, I>{});
        else dispatch_state<I + 1, N>(i, f);
    }
}

// a_i = (f_i(y + d e_i) - f_i(y)) / d for every integrated state, unrolled: the
// compiler shares what the perturbed evaluations have in common with f(y).
template <class Model, typename T, bool VOLT>
CHB_HD void grl_partials(const T* y, const T* f, T stim, T cm, const T* p, T* a) {
    constexpr int S = Model::kNumStates;
CHB_UNROLL
    for (int i = VOLT ? 0 : 1; i < S; ++i) {
        T yy[S], g[S];
CHB_UNROLL
        for (int k = 0; k < S; ++k) yy[k] = y[k];
        const T d = grl_perturbation<T>(y[i]);
        yy[i] = y[i] + d;
        Model::template rhs<T>(yy, stim, cm, p, g);
        a[i] = (g[i] - f[i]) / d;
    }
}

template <class Model, typename T, bool VOLT>
CHB_HD void grl1_step(T* y, T stim, T cm, const T* p, T dt) {
    constexpr int S = Model::kNumStates;
    T f[S], a[S];
    Model::template rhs<T>(y, stim, cm, p, f);
    grl_partials<Model, T, VOLT>(y, f, stim, cm, p, a);
CHB_UNROLL
    for (int i = VOLT ? 0 : 1; i < S; ++i) y[i] = grl_update<T>(y[i], f[i], a[i], dt);
}

template <class Model, typename T, bool VOLT>
CHB_HD void grl2_step(T* y, T stim, T cm, const T* p, T dt) {
    constexpr int S = Model::kNumStates;
    T y0[S], f[S], a[S];
CHB_UNROLL
    for (int k = 0; k < S; ++k) y0[k] = y[k];
    Model::template rhs<T>(y0, stim, cm, p, f);
    grl_partials<Model, T, VOLT>(y0, f, stim, cm, p, a);
    T ym[S];
    ym[0] = y0[0];
CHB_UNROLL
    for (int i = VOLT ? 0 : 1; i < S; ++i) ym[i] = grl_update<T>(y0[i], f[i], a[i], T(0.5) * dt);
    // each state re-linearised at the midpoint with its own component at the start value
    auto second = [&](auto ic) {
        constexpr int I = decltype(ic)::value;
        T yy[S], g[S], h[S];
CHB_UNROLL
        for (int k = 0; k < S; ++k) yy[k] = ym[k];
        yy[I] = y0[I];
        Model::template rhs<T>(yy, stim, cm, p, g);
        const T d = grl_perturbation<T>(y0[I]);
        yy[I] = y0[I] + d;
        Model::template rhs<T>(yy, stim, cm, p, h);
        f[I] = g[I];
        a[I] = (h[I] - g[I]) / d;
    };
    // in double precision one block per state (unrolled, the midpoint evaluations of
    // all states stay live together and spill); in single precision unrolled
    if (sizeof(T) == 8) {
CHB_NOUNROLL
        for (int i = VOLT ? 0 : 1; i < S; ++i) dispatch_state<0, S>(i, second);
    } else {
CHB_UNROLL
        for (int i = VOLT ? 0 : 1; i < S; ++i) dispatch_state<0, S>(i, second);
    }
CHB_UNROLL
    for (int i = VOLT ? 0 : 1; i < S; ++i) y[i] = grl_update<T>(y0[i], f[i], a[i], dt);
}

template <class Model, typename T>
CHB_HD bool states_in_range(const T* y) {
    bool ok = true;
CHB_UNROLL
    for (int i = 0; i < Model::kNumStates; ++i) {
        const T v = y[i];
        if (Model::range_class(i) == 1) ok = ok && (v >= T(0) && v <= T(1));
        else if (Model::range_class(i) == 2) ok = ok && (v > T(0));
        else ok = ok && (v == v);
    }
    return ok;
}

}  // namespace chb
