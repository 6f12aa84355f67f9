// Printing-step output kept on the device, and the per-node maps Chaste's
// PostProcessingWriter derives from it.
//
// frame_kernel: V and selected state variables of every node at a printing time
// (what AbstractCardiacProblem::Solve hands to Hdf5DataWriter at each printing step,
// heart/src/problem/AbstractCardiacProblem.cpp:552-565), stored as frame x variable x
// node so that both the write here and the per-node read below are coalesced.
//
// cellprops_kernel: one thread per node runs CellProperties::CalculateProperties
// (heart/src/postprocessing/CellProperties.cpp:55-220) over the node's voltage frames,
// then CalculateActionPotentialDurations (:222-330) -- including the start and end
// times it carries from one action potential to the next -- and writes the node's
// lists the way PostProcessingWriter writes them (PostProcessingWriter.cpp:226-312,
// PropagationPropertiesCalculator.cpp:98-160): [0] where CellProperties raises, the
// rest of the row -999.
//
// cv_kernel: PropagationPropertiesCalculator::CalculateAllConductionVelocities
// (PropagationPropertiesCalculator.cpp:226-285) from an origin node's upstroke times.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace chb {

template <typename T>
__global__ void __launch_bounds__(256) frame_kernel(int n, const double* __restrict__ V, const T* __restrict__ states,
                                                    const int* __restrict__ vars, int nv, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = V[i];
        for (int k = 1; k < nv; ++k) out[(size_t)k * n + i] = (double)states[(size_t)(vars[k] - 1) * n + i];
    }
}

// ActivationOutputModifier::ProcessSolutionAtTimeStep (heart/src/problem/
// ActivationOutputModifier.cpp:91-119) at a printing time: first activation, first
// recovery, second activation and second recovery per node (4 x n, -1 until seen).
__global__ void __launch_bounds__(256) activation_modifier_kernel(int n, const double* __restrict__ V, double thr,
                                                                  double t, double* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = V[i];
        double* fa = a + i;
        double* fr = a + (size_t)n + i;
        double* sa = a + 2 * (size_t)n + i;
        double* sr = a + 3 * (size_t)n + i;
        if (v > thr && *fa < 0.0) *fa = t;
        else if (*fa >= 0.0 && *fr < 0.0 && v < thr) *fr = t;
        else if (*fr >= 0.0 && *sa < 0.0 && v > thr) *sa = t;
        else if (*sa >= 0.0 && *sr < 0.0 && v < thr) *sr = t;
    }
}

constexpr double kMapPad = -999.0;   // WriteOutputDataToHdf5 pads missing paces with -999

struct CellPropsArgs {
    int n, n_frames, nv, cap;            // cap: action potentials kept per node
    const double* __restrict__ frames;   // n_frames x nv x n, variable 0 = V
    const double* __restrict__ times;    // n_frames
    double threshold, percentage;
    double* onset;                       // cap x n scratch: onsets, resting values, peaks
    double* rest;
    double* peak;
    double* apd;                         // n x cap, padded with kMapPad
    double* up_time;                     // n x cap
    double* up_vel;                      // n x cap
    int* n_apd;                          // n: APD list lengths (may exceed cap)
    int* n_up;                           // n: upstrokes found (0: none, the map holds [0])
};

__global__ void __launch_bounds__(128) cellprops_kernel(CellPropsArgs a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const size_t fs = (size_t)a.nv * a.n;   // frame stride
        const double* v = a.frames + i;
        const double thr = a.threshold;
        double* apd = a.apd + (size_t)i * a.cap;
        double* upt = a.up_time + (size_t)i * a.cap;
        double* upv = a.up_vel + (size_t)i * a.cap;
        for (int k = 0; k < a.cap; ++k) apd[k] = upt[k] = upv[k] = kMapPad;
        // CalculateProperties
        double max_up = -DBL_MAX, t_up = 0.0, cur_rest = DBL_MAX, cur_peak = -DBL_MAX, min_vel = DBL_MAX;
        bool flat = false;
        int phase = 0, n_on = 0, n_pk = 0, n_upr = 0;
        double prev_v = v[0], prev_t = a.times[0];
        for (int f = 1; f < a.n_frames; ++f) {
            const double vi = v[f * fs], ti = a.times[f];
            const double vel = (ti == prev_t) ? 0.0 : (vi - prev_v) / (ti - prev_t);
            if (vel >= max_up) {
                max_up = vel;
                t_up = ti;
            }
            if (phase == 0) {
                if (fabs(vel) <= min_vel && fabs(vel) <= 1e-2) {
                    min_vel = fabs(vel);
                    cur_rest = prev_v;
                    flat = true;
                } else if (prev_v < cur_rest && !flat) {
                    cur_rest = prev_v;
                }
                if (vi > thr && prev_v <= thr) {
                    if (n_on < a.cap) {
                        a.rest[(size_t)n_on * a.n + i] = cur_rest;
                        a.onset[(size_t)n_on * a.n + i] = prev_t + (ti - prev_t) / (vi - prev_v) * (thr - prev_v);
                    }
                    n_on++;
                    min_vel = DBL_MAX;
                    cur_rest = DBL_MAX;
                    flat = false;
                    phase = 1;
                }
            }
            if (phase == 1) {
                if (vi > cur_peak) cur_peak = vi;
                if (vi < thr && prev_v >= thr) {
                    if (n_pk < a.cap) a.peak[(size_t)n_pk * a.n + i] = cur_peak;
                    n_pk++;
                    cur_peak = thr;
                    if (n_upr < a.cap) {
                        upv[n_upr] = max_up;
                        upt[n_upr] = t_up;
                    }
                    n_upr++;
                    max_up = -DBL_MAX;
                    t_up = 0.0;
                    phase = 0;
                }
            }
            prev_v = vi;
            prev_t = ti;
        }
        if (n_on > n_upr) {   // an action potential still running at the last frame
            if (n_pk < a.cap) a.peak[(size_t)n_pk * a.n + i] = cur_peak;
            n_pk++;
            if (n_upr < a.cap) {
                upv[n_upr] = max_up;
                upt[n_upr] = t_up;
            }
            n_upr++;
        }
        if (n_upr == 0) upv[0] = upt[0] = 0.0;   // GetTimesAtMaxUpstrokeVelocity raises: [0]
        a.n_up[i] = n_upr;
        // CalculateActionPotentialDurations
        int n_apd = 0;
        bool have_start = false, have_end = false, have_index = false;
        double start_time = 0.0, end_time = 0.0;
        int start_index = 0;
        const int n_ap = n_pk < a.cap ? n_pk : a.cap;
        for (int k = 0; k < n_ap && n_on > 0; ++k) {
            const double rk = a.rest[(size_t)k * a.n + i], pk = a.peak[(size_t)k * a.n + i];
            const double target = rk + 0.01 * (100.0 - a.percentage) * (pk - rk);
            // lower_bound of the onset in the frame times, minus one
            const double on = a.onset[(size_t)k * a.n + i];
            int lo = 0, hi = a.n_frames;
            while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (a.times[mid] < on) lo = mid + 1;
                else hi = mid;
            }
            // lo >= 1 unless the first frame sits exactly on the threshold, where Chaste's
            // unsigned index wraps; the search then starts at frame 0
            const int sti = lo > 0 ? lo - 1 : 0;
            if (target >= thr) {
                double pv = v[(size_t)sti * fs], pt = a.times[sti];
                for (int f = sti + 1; f < a.n_frames; ++f) {
                    const double vf = v[(size_t)f * fs];
                    if (vf > target) {
                        start_time = pt + ((target - pv) / (vf - pv)) * (a.times[f] - pt);
                        start_index = f;
                        have_start = have_index = true;
                        break;
                    }
                    pt = a.times[f];
                    pv = vf;
                }
            } else {
                double pv = v[(size_t)(sti + 1) * fs], pt = a.times[sti + 1];
                for (int f = sti; f >= 0; --f) {
                    const double vf = v[(size_t)f * fs];
                    if (vf < target) {
                        start_time = pt + ((target - pv) / (vf - pv)) * (a.times[f] - pt);
                        start_index = f + 1;
                        have_start = have_index = true;
                        break;
                    }
                    pt = a.times[f];
                    pv = vf;
                }
            }
            if (have_end && have_start && start_time < end_time) continue;
            if (have_index) {
                double pv = v[(size_t)(start_index - 1) * fs];
                for (int f = start_index; f < a.n_frames; ++f) {
                    const double vf = v[(size_t)f * fs];
                    if (vf < target) {
                        end_time = a.times[f - 1] + ((target - pv) / (vf - pv)) * (a.times[f] - a.times[f - 1]);
                        have_end = true;
                        if (n_apd < a.cap) apd[n_apd] = end_time - start_time;
                        n_apd++;
                        break;
                    }
                    pv = vf;
                }
            }
        }
        if (n_apd == 0) {   // no onset or no full action potential: the map holds [0]
            apd[0] = 0.0;
            n_apd = 1;
        }
        a.n_apd[i] = n_apd;
    }
}

// Conduction velocities from node `origin` to every node (`dist`: distance to it),
// from the upstroke-time lists; [0] where either node has no upstroke.
__global__ void cv_kernel(int n, int cap, int origin, const double* __restrict__ dist,
                          const double* __restrict__ up_time, const int* __restrict__ n_up,
                          double* __restrict__ cv, int* __restrict__ n_cv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double* out = cv + (size_t)i * cap;
        for (int k = 0; k < cap; ++k) out[k] = kMapPad;
        if (n_up[i] == 0 || n_up[origin] == 0) {
            out[0] = 0.0;
            n_cv[i] = 1;
            continue;
        }
        const int m = n_up[i] < n_up[origin] ? n_up[i] : n_up[origin];
        const int mc = m < cap ? m : cap;
        for (int k = 0; k < mc; ++k) {
            if (i == origin) {
                out[k] = 0.0;
            } else {
                const double dt = up_time[(size_t)i * cap + k] - up_time[(size_t)origin * cap + k];
                out[k] = fabs(dt) < 1e-8 ? 0.0 : dist[i] / dt;
            }
        }
        n_cv[i] = m;
    }
}

}  // namespace chb
