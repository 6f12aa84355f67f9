// Mixed run populations: single-cell runs and cable runs of one cell model, each
// with its own length and parameters, in ONE persistent launch.  Blocks draw jobs
// from a work queue ordered by decreasing estimated cost (longest first); a job is
// either a group of single cells of about one length (each thread steps `K` cells
// together) or one whole cable (the block holds the cable's matrices and CG vectors
// in shared memory, each thread owning nodes t, t + blockDim, ...).  FP64 throughout.
//
// Single cells follow AbstractCardiacCell::Compute(0, t_end, tsamp):
//   Rush-Larsen   AbstractRushLarsenCardiacCell::Compute
//                 (heart/src/odes/AbstractRushLarsenCardiacCell.cpp:57-104):
//                 step j of sampling interval i at t = i*tsamp + j*dt, length dt;
//   forward Euler AbstractOneStepIvpOdeSolver::Solve
//                 (ode/src/solver/AbstractOneStepIvpOdeSolver.cpp:41-91): an inner
//                 TimeStepper between consecutive sampling times of the outer one
//                 (global/src/TimeStepper.cpp:43-135), step length NextStep().
// V is recorded at t = 0 and at the end of every sampling interval.
//
// Cables take the step of cable_forward_kernel (cable.cuh): forward Euler with V
// clamped (ComputeExceptVoltage), z = Am Cm V/dt - Am Iion - Istim
// (MonodomainSolver.cpp:92-101), A V' = M z by Jacobi CG with PETSc's stopping test.
#pragma once

#include "batch.cuh"
#include "cable.cuh"

namespace chb {

constexpr int kRunsMaxThreads = 256;
constexpr int kRunsCableArrays = 10;   // Ad Ao Md Mo dinv x p q r z, smem_nodes doubles each

struct RunCell {
    int method;           // 0 forward Euler, 1 Rush-Larsen
    int n_steps;          // a multiple of sample_every
    int sample_every;
    int pad;
    double dt;
    double tsamp;         // sample_every * dt
    double t_end;         // (n_steps / sample_every) * tsamp
    long long trace_off;  // n_steps / sample_every + 1 voltages
    DevStimulus stim;
};

struct RunCable {
    int n, n_steps, R, n_stim, n_probes, maxit, sample_every, pad;
    double h, sigma0, am, cm, dt, rtol, stim_mag, stim_dur;   // stim_dur padded
    long long param_off;  // R x (P + 1) doubles
    long long probe_off;
    long long trace_off;  // (n_steps / sample_every) x n_probes
    long long state_off;  // S x n, state k of node i at k * n + i
};

struct RunJob {
    int kind;    // 0: cells cell_order[first, first + count); 1: cable `first`
    int first;
    int count;
    int pad;
};

struct RunsArgs {
    int n_jobs;
    int smem_nodes;               // length of each cable array in shared memory
    int* next_job;                // work-queue counter, zero at launch
    const RunJob* jobs;
    const RunCell* cells;
    const int* cell_order;
    const double* cell_params;    // n_cells x P
    double* cell_y;               // S x n_cells
    int n_cells;
    int pad;
    const RunCable* cables;
    const double* cable_params;
    const int* probes;
    double* cable_y;
    long long* cable_iters;       // CG iterations per cable, summed over its steps
    double* trace;
    long long steps_override;     // > 0: every run stops after this many steps
    int* status;
};

// Rounded products and sums: the times must be the reference's to the last bit
// (they decide whether a step falls inside a stimulus window), so no contraction.
__device__ __forceinline__ double ts_at(double start, unsigned k, double dt, double end) {
    // TimeStepper::CalculateNextTime: start + k*dt, snapped to the end within epsilon
    const double eps = end > 1.0 ? DBL_EPSILON * end : DBL_EPSILON;
    const double t = __dadd_rn(start, __dmul_rn((double)k, dt));
    return __dadd_rn(end, -t) <= eps ? end : t;
}

// Time of step s of a single-cell run and its length.
__device__ __forceinline__ void run_cell_time(const RunCell& c, long long s, double& t, double& h) {
    const unsigned i = (unsigned)(s / c.sample_every), j = (unsigned)(s % c.sample_every);
    if (c.method == 1) {
        t = __dadd_rn(__dmul_rn((double)i, c.tsamp), __dmul_rn((double)j, c.dt));
        h = c.dt;
        return;
    }
    const double T0 = i == 0 ? 0.0 : ts_at(0.0, i, c.tsamp, c.t_end);
    const double T1 = ts_at(0.0, i + 1, c.tsamp, c.t_end);
    t = j == 0 ? T0 : ts_at(T0, j, c.dt, T1);
    h = __dadd_rn(ts_at(T0, j + 1, c.dt, T1), -t);
}

template <class M, int K>
__device__ void run_cells(const RunsArgs& a, int first, int count) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const int B = blockDim.x, t = threadIdx.x;
    int cell[K];
    long long n[K];
    RunCell d[K];
    double y[K][S];
    double p[K][P > 0 ? P : 1];
    long long smax = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int idx = t + j * B;
        cell[j] = idx < count ? a.cell_order[first + idx] : -1;
        const int c = cell[j] >= 0 ? cell[j] : a.cell_order[first];
        d[j] = a.cells[c];
        n[j] = cell[j] >= 0 ? d[j].n_steps : 0;
        if (a.steps_override > 0 && n[j] > a.steps_override) n[j] = a.steps_override;
        smax = n[j] > smax ? n[j] : smax;
#pragma unroll
        for (int k = 0; k < S; ++k) y[j][k] = a.cell_y[(size_t)k * a.n_cells + c];
#pragma unroll
        for (int k = 0; k < P; ++k) p[j][k] = a.cell_params[(size_t)c * P + k];
        if (cell[j] >= 0) a.trace[d[j].trace_off] = y[j][0];
    }
    for (long long s = 0; s < smax; ++s) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (s >= n[j]) continue;
            double tt, h;
            run_cell_time(d[j], s, tt, h);
            const double st = stimulus_value(d[j].stim, tt);
            if (d[j].method == 1) rl_step<M, double>(y[j], st, 1.0, p[j], h);
            else fe_step<M, double>(y[j], st, 1.0, p[j], h);
            if ((s + 1) % d[j].sample_every == 0) a.trace[d[j].trace_off + (s + 1) / d[j].sample_every] = y[j][0];
        }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (cell[j] < 0) continue;
        if (!(y[j][0] == y[j][0])) atomicOr(a.status, kStatusNaN);
#pragma unroll
        for (int k = 0; k < S; ++k) a.cell_y[(size_t)k * a.n_cells + cell[j]] = y[j][k];
    }
}

// Sums of N values over the block; every thread gets the totals (fixed order).
template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) red[k * 32 + warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = warp_sum(lane < nw ? red[k * 32 + lane] : 0.0);
}

template <class M>
__device__ void run_cable(const RunsArgs& a, int id, double* sm) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    constexpr int stride = P + 1;
    const RunCable c = a.cables[id];
    const int n = c.n, B = blockDim.x, t = threadIdx.x, L = a.smem_nodes;
    double* Ad = sm;
    double* Ao = sm + L;
    double* Md = sm + 2 * L;
    double* Mo = sm + 3 * L;
    double* dinv = sm + 4 * L;
    double* x = sm + 5 * L;
    double* pv = sm + 6 * L;
    double* qv = sm + 7 * L;
    double* rv = sm + 8 * L;
    double* zv = sm + 9 * L;
    double* red = sm + kRunsCableArrays * L;   // 3 x 32
    const double* prm = a.cable_params + c.param_off;
    double* ys = a.cable_y + c.state_off;
    const double ms = c.am * c.cm / c.dt;
    // tridiagonal A and M, rows summed element by element in ascending order
    for (int i = t; i < n; i += B) {
        double ad = 0.0, md = 0.0;
        for (int e = i - 1; e <= i; ++e) {
            if (e < 0 || e >= n - 1) continue;
            const double sig = c.sigma0 * prm[cable_elem_region(e, n, c.R) * stride + stride - 1];
            const double mdiag = c.h * 2.0 / 6.0;
            ad += ms * mdiag + sig / c.h;
            md += mdiag;
        }
        Ad[i] = ad;
        Md[i] = md;
        dinv[i] = 1.0 / ad;
        if (i < n - 1) {
            const double sig = c.sigma0 * prm[cable_elem_region(i, n, c.R) * stride + stride - 1];
            const double moff = c.h * 1.0 / 6.0;
            Ao[i] = ms * moff - sig / c.h;
            Mo[i] = moff;
        } else {
            Ao[i] = 0.0;
            Mo[i] = 0.0;
        }
        x[i] = ys[i];
    }
    __syncthreads();
    long long steps = c.n_steps;
    if (a.steps_override > 0 && steps > a.steps_override) steps = a.steps_override;
    long long iters = 0;
    for (long long step = 0; step < steps; ++step) {
        const double t0 = (double)step * c.dt, t1 = t0 + c.dt;
        // cells: forward Euler with V clamped, then the right-hand side z
        for (int i = t; i < n; i += B) {
            double y[S], p[P > 0 ? P : 1];
#pragma unroll
            for (int k = 1; k < S; ++k) y[k] = ys[(size_t)k * n + i];
            y[0] = x[i];
            const double* pr = prm + cable_node_region(i, n, c.R) * stride;
#pragma unroll
            for (int k = 0; k < P; ++k) p[k] = pr[k];
            const double v = y[0];
            const bool stim_node = i < c.n_stim;
            const double s0 = (stim_node && 0.0 <= t0 && t0 <= c.stim_dur) ? c.stim_mag : 0.0;
            const double s1 = (stim_node && 0.0 <= t1 && t1 <= c.stim_dur) ? c.stim_mag : 0.0;
            fe_step_except_voltage<M, double>(y, s0 / c.am, c.cm, p, c.dt);
            const double ii = M::template iionic<double>(y, c.cm, p);
            zv[i] = c.am * c.cm * v * (1.0 / c.dt) + (-c.am * ii - s1);
#pragma unroll
            for (int k = 1; k < S; ++k) ys[(size_t)k * n + i] = y[k];
        }
        __syncthreads();
        // b = M z, r = b - A x; PETSc KSPCG with Jacobi, the norm of B b as the
        // reference for the relative tolerance (nonzero initial guess)
        double s3[3] = {0.0, 0.0, 0.0};
        for (int i = t; i < n; i += B) {
            const double bi = tri(Md, Mo, zv, i, n);
            const double ri = bi - tri(Ad, Ao, x, i, n);
            rv[i] = ri;
            const double zi = dinv[i] * ri, wb = dinv[i] * bi;
            s3[0] += zi * zi;
            s3[1] += wb * wb;
            s3[2] += zi * ri;
        }
        block_sums<3>(s3, red);
        double dp = sqrt(s3[0]);
        const double ttol = fmax(c.rtol * sqrt(s3[1]), 1e-50);
        int its = 0;
        if (dp > ttol) {
            double beta = s3[2], betaold = 1.0;
            its = -1;
            for (int it = 0; it < c.maxit; ++it) {
                if (beta == 0.0) {
                    its = it;
                    break;
                }
                const double ratio = beta / betaold;
                for (int i = t; i < n; i += B) {
                    const double zi = dinv[i] * rv[i];
                    pv[i] = it == 0 ? zi : zi + ratio * pv[i];
                }
                __syncthreads();
                double s1v[1] = {0.0};
                for (int i = t; i < n; i += B) {
                    const double qi = tri(Ad, Ao, pv, i, n);
                    qv[i] = qi;
                    s1v[0] += pv[i] * qi;
                }
                block_sums<1>(s1v, red);
                const double alpha = beta / s1v[0];
                double s2[2] = {0.0, 0.0};
                for (int i = t; i < n; i += B) {
                    x[i] += alpha * pv[i];
                    const double ri = rv[i] - alpha * qv[i];
                    rv[i] = ri;
                    const double zi = dinv[i] * ri;
                    s2[0] += zi * zi;
                    s2[1] += zi * ri;
                }
                block_sums<2>(s2, red);
                dp = sqrt(s2[0]);
                if (dp <= ttol) {
                    its = it + 1;
                    break;
                }
                betaold = beta;
                beta = s2[1];
            }
        }
        if (its < 0) {
            if (t == 0) atomicOr(a.status, kStatusCgMaxIt);
        } else {
            iters += its;
        }
        __syncthreads();
        if ((step + 1) % c.sample_every == 0) {
            double* tr = a.trace + c.trace_off + ((step + 1) / c.sample_every - 1) * c.n_probes;
            for (int k = t; k < c.n_probes; k += B) tr[k] = x[a.probes[c.probe_off + k]];
        }
    }
    for (int i = t; i < n; i += B) {
        if (!(x[i] == x[i])) atomicOr(a.status, kStatusNaN);
        ys[i] = x[i];
    }
    if (t == 0) a.cable_iters[id] = iters;
}

// One launch runs every job; K single cells per thread.
template <class M, int K>
__global__ void __launch_bounds__(kRunsMaxThreads) runs_kernel(RunsArgs a) {
    extern __shared__ double runs_smem[];
    __shared__ int s_job;
    for (;;) {
        if (threadIdx.x == 0) s_job = atomicAdd(a.next_job, 1);
        __syncthreads();
        const int j = s_job;
        __syncthreads();
        if (j >= a.n_jobs) break;
        const RunJob job = a.jobs[j];
        if (job.kind == 1) run_cable<M>(a, job.first, runs_smem);
        else run_cells<M, K>(a, job.first, job.count);
        __syncthreads();
    }
}

}  // namespace chb
