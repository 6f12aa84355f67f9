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

#if defined(__CUDACC__)
#define CHB_HD __host__ __device__ __forceinline__
#define CHB_UNROLL _Pragma("unroll")
#else
#define CHB_HD
#define CHB_UNROLL
#endif

#ifndef NAN
#define NAN (__builtin_nanf(""))
#endif

namespace chb {

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
            y[i] = inf[i] + (y[i] - inf[i]) * exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}

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
            y[i] = inf[i] + (y[i] - inf[i]) * exp(rate[i] * dt);
        } else {
            y[i] += dt * rate[i];
        }
    }
}

// VerifyStateVariables analogue: true when every gate is in [0,1] and every
// concentration is positive (and nothing is NaN).
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
