// Ionic ODE update of every tissue node with the voltage clamped
// (AbstractCardiacTissue::SolveCellSystems, heart/src/tissue/AbstractCardiacTissue.cpp:464-567),
// fused with the Iion cache (UpdateCaches, :730-734) and the per-node RHS term
// z = Am*Cm*V/dt - Am*Iion - Istim(t+dt) (MonodomainSolver.cpp:92-101).
//
// Layout: states are structure-of-arrays, row k-1 holds state k (k >= 1) of
// every node, so a warp reads 32 consecutive values of one state (coalesced).
// V is FP64 (it is the CG solution); the states, Iion and z use T.
#pragma once

#include "../models/lr91.h"
#include "../models/tt06.h"
#include "common.cuh"

namespace chb {

template <typename T>
struct OdeArgs {
    int n;
    double* __restrict__ V;             // V^n in; with vprev, the CG initial guess out
    double* __restrict__ vprev;         // V^{n-1} (mixed precision), or null
    T* __restrict__ states;             // (S-1) x n
    T* __restrict__ iion;               // n
    T* __restrict__ zrhs;               // n
    const uint8_t* __restrict__ stim_id;  // n, 0xFF = none
    const DevStimulus* __restrict__ stims;
    const uint8_t* __restrict__ pset;   // n (may be null)
    const T* __restrict__ params;       // nsets x P
    const long long* __restrict__ step; // device step counter
    int* status;
    double dt_ode, dt_pde, am, cm;
    int check_range;
    double* act;                        // first activation time per node (-1: none yet)
    double act_threshold;
    int half;                           // 0: ComputeExceptVoltage over the step; 1, 2: first or second
                                        // half step including V (operator splitting)
    int lo, hi;                         // half 0: the nodes [lo, hi) of this launch
    int reset_history;                  // with vprev: V^n has no predecessor (guess V^n, no extrapolation)
    const double* v_in;                 // ode_kernel<..., HOSTV = true>: V^n read from here (page-locked
                                        // host memory, through its device mapping) and stored into V
};

// First step with V above the threshold (ActivationOutputModifier::ProcessSolutionAtTimeStep,
// heart/src/problem/ActivationOutputModifier.cpp:91-101), checked once per PDE step.
static __global__ void activation_kernel(int n, const double* __restrict__ V, double* __restrict__ act,
                                  double threshold, double t) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (V[i] > threshold && act[i] < 0.0) act[i] = t;
}

// Half a PDE step of every cell including V, for the operator-splitting solver:
// SolveCellSystems(..., updateVoltage = true) (AbstractCardiacTissue.cpp:531-536) --
// SolveAndUpdateState over [t0, t0 + dt/2] or [t0 + dt/2, t1] by forward Euler, GRL1
// or GRL2 (AbstractOneStepIvpOdeSolver::InternalSolve), backward Euler or Rush-Larsen
// (AbstractRushLarsenCardiacCell.cpp:130-147), V written back, then UpdateCaches at
// the end of the half; after the first half z = Am*Cm*V/dt, the diffusion-only
// right-hand side term (OperatorSplittingMonodomainSolver.cpp:86-89).
template <class M, typename T, int METHOD>
__device__ __forceinline__ void ode_half_step(const OdeArgs<T>& a, double t0, double t1) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const double th0 = a.half == 1 ? t0 : t0 + a.dt_pde / 2.0;
    const double th1 = a.half == 1 ? t0 + a.dt_pde / 2.0 : t1;
    const double dtinv = 1.0 / a.dt_pde;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        T y[S];
        const double v = a.V[i];
        if (a.half == 1 && v > a.act_threshold && a.act[i] < 0.0) a.act[i] = t0;
        y[0] = (T)v;
#pragma unroll
        for (int k = 1; k < S; ++k) y[k] = a.states[(size_t)(k - 1) * a.n + i];
        T p[P > 0 ? P : 1];
        if (a.pset) {
            const T* pp = a.params + (size_t)a.pset[i] * P;
#pragma unroll
            for (int k = 0; k < P; ++k) p[k] = pp[k];
        } else {
#pragma unroll
            for (int k = 0; k < P; ++k) p[k] = T(1);
        }
        const int sid = a.stim_id[i];
        DevStimulus st{0, 0, 0, 0, 0, 0};
        if (sid != 0xFF) st = a.stims[sid];
        const T cm = (T)a.cm;
        DevTimeStepper ts(th0, th1, a.dt_ode);
        while (!ts.at_end()) {
            const double sv = stimulus_value(st, ts.time);
            const T s = sv == 0.0 ? T(0) : (T)(sv / a.am);
            if (METHOD == 1) rl_step<M, T>(y, s, cm, p, (T)a.dt_ode);
            else if (METHOD == 2) be_step<M, T>(y, s, cm, p, (T)a.dt_ode, true);
            else if (METHOD == 3) grl1_step<M, T, true>(y, s, cm, p, (T)(ts.next - ts.time));
            else if (METHOD == 4) grl2_step<M, T, true>(y, s, cm, p, (T)(ts.next - ts.time));
            else fe_step<M, T>(y, s, cm, p, (T)(ts.next - ts.time));
            ts.advance();
        }
        const double vn = (double)y[0];
        a.V[i] = vn;
#pragma unroll
        for (int k = 1; k < S; ++k) a.states[(size_t)(k - 1) * a.n + i] = y[k];
        a.iion[i] = M::template iionic<T>(y, cm, p);
        if (a.half == 1) a.zrhs[i] = (T)(a.am * a.cm * vn * dtinv);
        if (!(vn == vn)) atomicOr(a.status, kStatusNaN);
        if (a.check_range && !states_in_range<M, T>(y)) atomicOr(a.status, kStatusStateRange);
    }
}

// Launch shape of ode_kernel.  The FP64 Rush-Larsen step keeps its frozen terms (the
// voltage-only gates' inf and exp(rate*dt), the voltage-only subexpressions) in a
// per-thread column of shared memory instead of registers, and runs 128-thread blocks
// capped at 128 registers, four blocks per SM: 16 resident warps per SM where 250+
// registers left 8 (one step of 442,401 TT06 cells 0.455 -> 0.302 ms, bit for bit the
// same states).  The other steps run 256-thread blocks, two per SM (at most 128
// registers, which they fit without spilling), except the GRL2 steps and the other
// FP64 steps of the larger models (more than 10 states), which keep the compiler's
// register count: capped, they spill hundreds of bytes a thread.
template <class M, typename T, int METHOD>
struct OdeShape {
    static constexpr bool kColumn = METHOD == 1 && sizeof(T) == 8;
    static constexpr int kThreads = kColumn ? 128 : 256;
    static constexpr int kMinBlocks =
        kColumn ? 4 : (METHOD == 4 || (sizeof(T) == 8 && M::kNumStates > 10)) ? 1 : 2;
    static constexpr int kShared = kColumn ? FrozenSlots<M>::kSlots * kThreads : 1;
};

// HOSTV: V^n is read from a.v_in (a separate instantiation, so that the kernel of the
// device-resident steps keeps its code; measured with the choice made at run time in
// one kernel, that kernel took 0.080 instead of 0.063 ms per step of the 442,401-node slab).
template <class M, typename T, int METHOD, bool HOSTV = false>
__global__ void __launch_bounds__(OdeShape<M, T, METHOD>::kThreads, OdeShape<M, T, METHOD>::kMinBlocks)
    ode_kernel(OdeArgs<T> a) {
    using Shape = OdeShape<M, T, METHOD>;
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    // frozen-term columns, slot k of thread t at frozen[k * kThreads + t] (blockDim.x is at
    // most kThreads: the launch bound rejects larger blocks)
    __shared__ T frozen[Shape::kShared];
    if (*(volatile int*)a.status & ~kStatusStateRange) return;   // a failed step stops the run
    const long long step = *a.step;
    const double t0 = (double)step * a.dt_pde;
    const double t1 = (double)(step + 1) * a.dt_pde;
    const double dtinv = 1.0 / a.dt_pde;
    for (int i = a.lo + blockIdx.x * blockDim.x + threadIdx.x; i < a.hi; i += gridDim.x * blockDim.x) {
        T y[S];
        const double v = HOSTV ? a.v_in[i] : a.V[i];
        // mixed precision: the diffusion solve starts from the linear extrapolation
        // 2 V^n - V^{n-1} (FP64 mode keeps Chaste's guess V^n, LinearSystem.cpp:833-837);
        // the right-hand side below still uses V^n
        if (a.vprev) {
            const double vp = a.reset_history ? v : a.vprev[i];
            a.vprev[i] = v;
            a.V[i] = 2.0 * v - vp;
        } else if (HOSTV) {
            a.V[i] = v;
        }
        // activation bookkeeping of the previous step's solution (time t0)
        if (v > a.act_threshold && a.act[i] < 0.0) a.act[i] = t0;
        y[0] = (T)v;
#pragma unroll
        for (int k = 1; k < S; ++k) y[k] = a.states[(size_t)(k - 1) * a.n + i];
        T p[P > 0 ? P : 1];
        if (a.pset) {
            const T* pp = a.params + (size_t)a.pset[i] * P;
#pragma unroll
            for (int k = 0; k < P; ++k) p[k] = pp[k];
        } else {
#pragma unroll
            for (int k = 0; k < P; ++k) p[k] = T(1);
        }
        const int sid = a.stim_id[i];
        DevStimulus st{0, 0, 0, 0, 0, 0};
        if (sid != 0xFF) st = a.stims[sid];
        const T cm = (T)a.cm;
        if (METHOD == 2) {
            // AbstractBackwardEulerCardiacCell::ComputeExceptVoltage: (t1 - t0)/dt + 0.5
            // steps at t0 + i dt, V fixed
            const unsigned n_sub = (unsigned)((t1 - t0) / a.dt_ode + 0.5);
            for (unsigned k = 0; k < n_sub; ++k) {
                const double sv = stimulus_value(st, t0 + k * a.dt_ode);
                const T s = sv == 0.0 ? T(0) : (T)(sv / a.am);
                be_step<M, T>(y, s, cm, p, (T)a.dt_ode, false);
                y[0] = (T)v;
            }
        } else if constexpr (Shape::kColumn) {
            // Rush-Larsen with the frozen terms in this thread's shared-memory column
            T* column = frozen + threadIdx.x;
            rl_freeze_voltage_terms_column<M, T, Shape::kThreads>(y, p, (T)a.dt_ode, column);
            DevTimeStepper ts(t0, t1, a.dt_ode);
            while (!ts.at_end()) {
                const double sv = stimulus_value(st, ts.time);
                const T s = sv == 0.0 ? T(0) : (T)(sv / a.am);
                rl_step_except_voltage_column<M, T, Shape::kThreads>(y, s, cm, p, (T)a.dt_ode, column);
                ts.advance();
            }
        } else {
            // Rush-Larsen: the voltage-only gates' terms once per PDE step (V is clamped)
            T vinf[S], vfac[S], vt[M::kNumVTerms > 0 ? M::kNumVTerms : 1];
            if (METHOD == 1) rl_freeze_voltage_terms<M, T>(y, p, (T)a.dt_ode, vinf, vfac, vt);
            DevTimeStepper ts(t0, t1, a.dt_ode);
            while (!ts.at_end()) {
                // cell stimulus in uA/cm^2 = tissue stimulus / Am (GetIntracellularAreaStimulus);
                // most nodes have none, and 0 / Am = +0 needs no division
                const double sv = stimulus_value(st, ts.time);
                const T s = sv == 0.0 ? T(0) : (T)(sv / a.am);
                if (METHOD == 1) {
                    rl_step_except_voltage_frozen<M, T>(y, s, cm, p, (T)a.dt_ode, vinf, vfac, vt);
                } else if (METHOD == 3) {
                    grl1_step<M, T, false>(y, s, cm, p, (T)(ts.next - ts.time));
                } else if (METHOD == 4) {
                    grl2_step<M, T, false>(y, s, cm, p, (T)(ts.next - ts.time));
                } else {
                    fe_step_except_voltage<M, T>(y, s, cm, p, (T)(ts.next - ts.time));
                }
                ts.advance();
            }
        }
#pragma unroll
        for (int k = 1; k < S; ++k) a.states[(size_t)(k - 1) * a.n + i] = y[k];
        y[0] = (T)v;
        const T ii = M::template iionic<T>(y, cm, p);
        a.iion[i] = ii;
        const double istim = stimulus_value(st, t1);
        const double F = -a.am * (double)ii - istim;
        a.zrhs[i] = (T)(a.am * a.cm * v * dtinv + F);
        if (a.check_range && !states_in_range<M, T>(y)) atomicOr(a.status, kStatusStateRange);
    }
}

// The operator-splitting half steps (a.half = 1 or 2) in a kernel of their own, so that
// their register allocation does not weigh on ode_kernel's.
template <class M, typename T, int METHOD>
__global__ void __launch_bounds__(256) ode_half_kernel(OdeArgs<T> a) {
    if (*(volatile int*)a.status & ~kStatusStateRange) return;   // a failed step stops the run
    // the second half step runs after the diffusion solve has advanced the step counter
    const long long step = *a.step - (a.half == 2 ? 1 : 0);
    const double t0 = (double)step * a.dt_pde;
    const double t1 = (double)(step + 1) * a.dt_pde;
    ode_half_step<M, T, METHOD>(a, t0, t1);
}

}  // namespace chb
