// Batched single-cell populations: every cell integrated in FP64 and in FP32
// in ONE launch (the first half of the blocks take FP64, the second half FP32),
// with AbstractRushLarsenCardiacCell::Compute semantics
// (heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104: step k at time k*dt,
// EvaluateEquations, V by forward Euler, gates by Rush-Larsen) and the
// action-potential measurements of CellProperties computed on the fly
// (heart/src/postprocessing/CellProperties.cpp:55-220, APD at 90% repolarisation).
//
// One launch covers one beat of every cell that still has beats to run; the
// ODE states and the CellProperties bookkeeping are kept in device memory
// between launches.  The voltage is sampled every `sample_every` steps so a
// second kernel can form the largest |V32 - V64| of each beat.
#pragma once

#include "../models/lr91.h"
#include "../models/tt06.h"
#include "common.cuh"

namespace chb {

constexpr int kApdRing = 256;   // samples kept before an onset (2.56 ms at dt = 0.01 ms)

// State of a streaming restatement of CellProperties::CalculateProperties and
// CalculateActionPotentialDurations(90) for one voltage trace.
struct ApdTracker {
    double prev_v, rest, min_vel, rest_ap, onset, peak, target, t_start;
    long long up_first, up_last;   // sample range frozen at the onset
    int phase;        // 0 below threshold, 1 above, 2 looking for the repolarisation crossing
    int flat, n_ap, pad;
};

struct BatchArgs {
    int n_cells;
    int max_aps;
    int max_beats;
    int sample_every;
    int blocks_per_precision;
    long long steps_per_beat;
    double dt, cm;
    DevStimulus stim;
    const int* __restrict__ beats;        // per cell
    const double* __restrict__ params;    // n_cells x P scale factors
    double* y64;                          // S x n_cells (SoA)
    float* y32;                           // S x n_cells
    ApdTracker* trk;                      // 2 x n_cells (FP64 then FP32)
    double* apd;                          // 2 x n_cells x max_aps
    float* vsamp;                         // 2 x n_samples x n_cells (this beat)
    long long* launch;                    // beats completed by every running cell
    long long steps_override;             // > 0: run only this many steps (autotuning)
    int* status;
};

__device__ __forceinline__ void apd_init(ApdTracker& t, double v0) {
    t.prev_v = v0;
    t.rest = DBL_MAX;
    t.min_vel = DBL_MAX;
    t.rest_ap = 0.0;
    t.onset = 0.0;
    t.peak = -DBL_MAX;
    t.target = 0.0;
    t.t_start = 0.0;
    t.up_first = 0;
    t.up_last = -1;
    t.phase = 0;
    t.flat = 0;
    t.n_ap = 0;
    t.pad = 0;
}

// Sample q (voltage v at time q*dt); ring[i % kApdRing] holds sample i for
// i >= ring_first (this launch).  At an onset the ring is frozen into `up`, the
// samples the backward search for the APD start needs once the peak is known.
// Completed APD90s go to apd_out.
template <typename R>
__device__ __forceinline__ void apd_sample(ApdTracker& k, double v, long long q, double dt, const R* ring,
                                           R* up, long long ring_first, double* apd_out, int max_aps) {
    const double thr = -30.0;   // CellProperties default threshold
    const double t = (double)q * dt, prev_t = (double)(q - 1) * dt;
    const double vel = (v - k.prev_v) / (t - prev_t);
    if (k.phase == 0) {
        if (fabs(vel) <= k.min_vel && fabs(vel) <= 1e-2) {
            k.min_vel = fabs(vel);
            k.rest = k.prev_v;
            k.flat = 1;
        } else if (k.prev_v < k.rest && !k.flat) {
            k.rest = k.prev_v;
        }
        if (v > thr && k.prev_v <= thr) {
            k.rest_ap = k.rest;
            k.min_vel = DBL_MAX;
            k.rest = DBL_MAX;
            k.onset = prev_t + (t - prev_t) / (v - k.prev_v) * (thr - k.prev_v);
            k.flat = 0;
            k.phase = 1;
            k.peak = -DBL_MAX;
            for (int i = 0; i < kApdRing; ++i) up[i] = ring[i];
            k.up_last = q;
            k.up_first = q - kApdRing + 1 > ring_first ? q - kApdRing + 1 : ring_first;
        }
    }
    if (k.phase == 1) {
        if (v > k.peak) k.peak = v;
        if (v < thr && k.prev_v >= thr) {
            // target, then the upward crossing of it searched backwards from the
            // last sample before the onset (CellProperties.cpp:236-275)
            k.target = k.rest_ap + 0.01 * (100.0 - 90.0) * (k.peak - k.rest_ap);
            long long s = (long long)floor(k.onset / dt);
            while (s >= 0 && (double)s * dt >= k.onset) s--;
            while ((double)(s + 1) * dt < k.onset) s++;
            k.t_start = NAN;
            if (s + 1 >= k.up_first && s + 1 <= k.up_last) {
                double pv = (double)up[(s + 1) % kApdRing];
                double pt = (double)(s + 1) * dt;
                for (long long i = s; i >= k.up_first; --i) {
                    const double vi = (double)up[i % kApdRing];
                    const double ti = (double)i * dt;
                    if (vi < k.target) {
                        k.t_start = pt + ((k.target - pv) / (vi - pv)) * (ti - pt);
                        break;
                    }
                    pt = ti;
                    pv = vi;
                }
            }
            k.phase = 2;
        }
    } else if (k.phase == 2) {
        // the repolarisation crossing of the target (CellProperties.cpp:297-312)
        if (v < k.target) {
            const double t_end = prev_t + ((k.target - k.prev_v) / (v - k.prev_v)) * (t - prev_t);
            if (k.n_ap < max_aps) apd_out[k.n_ap] = t_end - k.t_start;
            k.n_ap++;
            k.phase = 0;
        }
    }
    k.prev_v = v;
}

// K cells per thread (cells c0, c0 + cstride, ...), advanced together step by step
// so their independent updates interleave; the stimulus is evaluated once per step.
template <class M, typename T, int K>
__device__ __forceinline__ void batch_cells(const BatchArgs& a, int c0, int cstride, int prec, T* __restrict__ ys) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const long long beat = *a.launch;
    const long long s0 = beat * a.steps_per_beat;
    const long long s1 = a.steps_override > 0 ? s0 + a.steps_override : s0 + a.steps_per_beat;
    int cell[K];
    bool on[K];
    bool any = false;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        cell[j] = c0 + j * cstride;
        on[j] = cell[j] < a.n_cells && s0 < (long long)a.beats[cell[j]] * a.steps_per_beat;
        any |= on[j];
    }
    if (!any) return;
    T y[K][S];
    T p[K][P > 0 ? P : 1];
    ApdTracker trk[K];
    T ring[K][kApdRing];
    T up[K][kApdRing];
    double* apd[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int c = on[j] ? cell[j] : c0;
#pragma unroll
        for (int k = 0; k < S; ++k) y[j][k] = ys[(size_t)k * a.n_cells + c];
#pragma unroll
        for (int k = 0; k < P; ++k) p[j][k] = (T)a.params[(size_t)c * P + k];
        trk[j] = a.trk[(size_t)prec * a.n_cells + c];
        if (s0 == 0) apd_init(trk[j], (double)y[j][0]);
        ring[j][s0 % kApdRing] = y[j][0];
        apd[j] = a.apd + ((size_t)prec * a.n_cells + c) * a.max_aps;
    }
    const long long nsamp = (a.steps_per_beat + a.sample_every - 1) / a.sample_every;
    float* vs = a.vsamp + (size_t)prec * nsamp * a.n_cells;
    const T dt = (T)a.dt, cm = (T)a.cm;
    for (long long s = s0; s < s1; ++s) {
        const T st = (T)stimulus_value(a.stim, (double)s * a.dt);
        const bool sample = (s - s0) % a.sample_every == 0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!on[j]) continue;
            if (sample) vs[(size_t)((s - s0) / a.sample_every) * a.n_cells + cell[j]] = (float)y[j][0];
            rl_step<M, T>(y[j], st, cm, p[j], dt);
            ring[j][(s + 1) % kApdRing] = y[j][0];
            apd_sample<T>(trk[j], (double)y[j][0], s + 1, a.dt, ring[j], up[j], s0, apd[j], a.max_aps);
        }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (!on[j]) continue;
        if (!(y[j][0] == y[j][0])) atomicOr(a.status, kStatusNaN);
#pragma unroll
        for (int k = 0; k < S; ++k) ys[(size_t)k * a.n_cells + cell[j]] = y[j][k];
        a.trk[(size_t)prec * a.n_cells + cell[j]] = trk[j];
    }
}

// blocks [0, blocks_per_precision) integrate in FP64, the rest in FP32; thread t of
// a precision handles cells t, t + T, ..., t + (K-1) T (T = blocks_per_precision *
// blockDim), then the next K*T cells (persistent over the population).
template <class M, int K>
__global__ void batch_kernel(BatchArgs a) {
    const bool fp64 = blockIdx.x < (unsigned)a.blocks_per_precision;
    const int b = fp64 ? blockIdx.x : blockIdx.x - a.blocks_per_precision;
    const int T_threads = a.blocks_per_precision * blockDim.x;
    for (int c = b * blockDim.x + threadIdx.x; c < a.n_cells; c += K * T_threads) {
        if (fp64) batch_cells<M, double, K>(a, c, T_threads, 0, a.y64);
        else batch_cells<M, float, K>(a, c, T_threads, 1, a.y32);
    }
}

// Largest |V32 - V64| over this beat's samples, per cell; then the beat counter.
static __global__ void batch_beat_error_kernel(BatchArgs a, float* max_dv) {
    const long long beat = *a.launch;
    const long long nsamp = (a.steps_per_beat + a.sample_every - 1) / a.sample_every;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < a.n_cells; cell += gridDim.x * blockDim.x) {
        if (beat >= a.beats[cell] || beat >= a.max_beats) continue;
        float m = 0.0f;
        for (long long k = 0; k < nsamp; ++k) {
            const float v64 = a.vsamp[(size_t)k * a.n_cells + cell];
            const float v32 = a.vsamp[((size_t)nsamp + k) * a.n_cells + cell];
            m = fmaxf(m, fabsf(v64 - v32));
        }
        max_dv[(size_t)cell * a.max_beats + beat] = m;
    }
}

static __global__ void batch_advance_kernel(long long* launch) { *launch += 1; }

}  // namespace chb
