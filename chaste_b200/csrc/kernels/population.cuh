// Batched single-cell populations, persistent form: ONE launch runs every beat of
// every cell, blocks drawing groups of 32 cells from a work queue ordered by
// decreasing beat count (longest jobs first), and each cell is split over two
// threads in two warps so that its Rush-Larsen step
// (AbstractRushLarsenCardiacCell::Compute, heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104)
// runs as two shorter dependency chains:
//
//   the gate thread   -- the terms of the gates that depend on V alone
//                        (Model::rl_terms_voltage: inf, rate, exp(rate*dt)) and their update;
//   the state thread  -- everything else (Model::rl_terms_states: the currents, dV/dt, the
//                        other gates and the concentrations), V by forward Euler, the
//                        CellProperties bookkeeping and the samples.
//
// Both start a step from the same state, as the reference step does (every term from
// the step's start values, then V, then the gates), so the step is the single-thread
// step's arithmetic (to the compiler's choice of fused multiply-adds, which may differ
// between the two code paths).  They meet once per step at a block barrier:
// the state thread publishes V(t+dt), the gate thread the gates at t+dt, in
// double-buffered shared memory.  A block has four warps: FP64 state, FP64 gates,
// FP32 state, FP32 gates -- lane l of each holds cell l of the group -- so the two
// precisions of a cell step in lockstep and the FP64 state thread compares them at
// every sample (the per-beat largest |V32 - V64|) without storing samples.
#pragma once

#include "batch.cuh"

namespace chb {

constexpr int kPopThreads = 128;   // 4 warps: FP64 state, FP64 gates, FP32 state, FP32 gates
constexpr int kMaxPopGates = 16;   // voltage-only gates of a model (TT06 11, LR91 6)

struct PopArgs {
    BatchArgs b;
    const int* order;       // cells by decreasing beat count
    int n_groups;           // ceil(n_cells / 32)
    int* next_group;        // work-queue counter, zero at launch
    float* max_dv;          // n_cells x max_beats
};

template <typename T>
struct PopShared {
    T v[2][32];                  // V published by the state threads, by step parity
    T g[2][kMaxPopGates][32];    // voltage-only gates published by the gate threads
};

template <class M, typename T, bool GATES>
__device__ __forceinline__ void pop_run_group(const PopArgs& pa, int cell, long long my_steps, long long total,
                                              PopShared<T>& sh, const float (*v32)[32], int prec, T* __restrict__ ys) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const BatchArgs& a = pa.b;
    const int lane = threadIdx.x & 31;
    const bool on = cell >= 0;
    const int c = on ? cell : 0;
    T y[S];
    T p[P > 0 ? P : 1];
#pragma unroll
    for (int k = 0; k < S; ++k) y[k] = ys[(size_t)k * a.n_cells + c];
#pragma unroll
    for (int k = 0; k < P; ++k) p[k] = (T)a.params[(size_t)c * P + k];
    const T dt = (T)a.dt, cm = (T)a.cm;
    // gate slots: voltage-only gate j of the model is state gidx[j]
    int gidx[kMaxPopGates];
    {
        int j = 0;
#pragma unroll
        for (int k = 1; k < S; ++k)
            if (M::rl_voltage_only(k)) gidx[j++] = k;
    }
    constexpr int NG = M::kNumVoltageGates;
    static_assert(NG <= kMaxPopGates, "more voltage-only gates than the shared buffers hold");
    if (!GATES) sh.v[0][lane] = y[0];
    __syncthreads();
    if constexpr (GATES) {
        for (long long s = 0; s < total; ++s) {
            const int b = (int)(s & 1);
            if (on && s < my_steps) {
                y[0] = sh.v[b][lane];
                T rate[S], inf[S];
                M::template rl_terms_voltage<T>(y, p, rate, inf);
#pragma unroll
                for (int j = 0; j < NG; ++j) {
                    const int k = gidx[j];
                    y[k] = inf[k] + (y[k] - inf[k]) * m_exp(rate[k] * dt);
                    sh.g[b ^ 1][j][lane] = y[k];
                }
            }
            __syncthreads();
        }
    } else {
        ApdTracker trk = a.trk[(size_t)prec * a.n_cells + c];
        T ring[kApdRing];
        T up[kApdRing];
        double* apd = a.apd + ((size_t)prec * a.n_cells + c) * a.max_aps;
        if (on) apd_init(trk, (double)y[0]);
        ring[0] = y[0];
        float beat_dv = 0.0f;
        for (long long s = 0; s < total; ++s) {
            const int b = (int)(s & 1);
            const bool live = on && s < my_steps;
            const long long in_beat = s % a.steps_per_beat;
            if (live && prec == 0 && in_beat % a.sample_every == 0)
                beat_dv = fmaxf(beat_dv, fabsf((float)y[0] - v32[b][lane]));
            if (live) {
                const T st = (T)stimulus_value(a.stim, (double)s * a.dt);
                T rate[S], inf[S];
                M::template rl_terms_states<T>(y, st, cm, p, rate, inf);
                y[0] += dt * rate[0];
#pragma unroll
                for (int k = 1; k < S; ++k) {
                    if (M::rl_voltage_only(k)) continue;
                    if (M::rush_larsen(k)) y[k] = inf[k] + (y[k] - inf[k]) * m_exp(rate[k] * dt);
                    else y[k] += dt * rate[k];
                }
                sh.v[b ^ 1][lane] = y[0];
            }
            __syncthreads();
            if (live) {
#pragma unroll
                for (int j = 0; j < NG; ++j) y[gidx[j]] = sh.g[b ^ 1][j][lane];
                ring[(s + 1) % kApdRing] = y[0];
                apd_sample<T>(trk, (double)y[0], s + 1, a.dt, ring, up, 0, apd, a.max_aps);
                if (prec == 0 && in_beat == a.steps_per_beat - 1) {
                    const long long beat = s / a.steps_per_beat;
                    if (beat < a.max_beats) pa.max_dv[(size_t)cell * a.max_beats + beat] = beat_dv;
                    beat_dv = 0.0f;
                }
            }
        }
        if (on) {
            if (!(y[0] == y[0])) atomicOr(a.status, kStatusNaN);
            a.trk[(size_t)prec * a.n_cells + cell] = trk;
        }
    }
    if (!GATES && on) {
        // the state thread's copy holds every state, the gates as the gate thread published them
#pragma unroll
        for (int k = 0; k < S; ++k) ys[(size_t)k * a.n_cells + cell] = y[k];
    }
}

template <class M>
__global__ void __launch_bounds__(kPopThreads) population_kernel(PopArgs pa) {
    const BatchArgs& a = pa.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int s_group;
    __shared__ PopShared<double> sh64;
    __shared__ PopShared<float> sh32;
    for (;;) {
        if (threadIdx.x == 0) s_group = atomicAdd(pa.next_group, 1);
        __syncthreads();
        const int g = s_group;
        __syncthreads();
        if (g >= pa.n_groups) break;
        const int idx = g * 32 + lane;
        const int cell = idx < a.n_cells ? pa.order[idx] : -1;
        long long my_steps = cell >= 0 ? (long long)a.beats[cell] * a.steps_per_beat : 0;
        if (a.steps_override > 0 && my_steps > a.steps_override) my_steps = a.steps_override;
        // every warp holds the same 32 cells, so every warp finds the same group length
        long long total = my_steps;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const long long t = __shfl_xor_sync(0xffffffffu, total, o);
            total = t > total ? t : total;
        }
        switch (warp) {
            case 0: pop_run_group<M, double, false>(pa, cell, my_steps, total, sh64, sh32.v, 0, a.y64); break;
            case 1: pop_run_group<M, double, true>(pa, cell, my_steps, total, sh64, sh32.v, 0, a.y64); break;
            case 2: pop_run_group<M, float, false>(pa, cell, my_steps, total, sh32, sh32.v, 1, a.y32); break;
            default: pop_run_group<M, float, true>(pa, cell, my_steps, total, sh32, sh32.v, 1, a.y32); break;
        }
        __syncthreads();
    }
}

}  // namespace chb
