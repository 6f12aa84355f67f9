// 1D monodomain cable held entirely in one CTA (shared memory), for parameter
// fitting.  The forward kernel runs one parameter set per CTA, so the runs of a
// finite-difference check or of a population go out in one launch; the adjoint
// kernel differentiates one parameter set per CTA from checkpoints.
//
// Forward step n (Chaste's order with the ODE step equal to the PDE step):
//   y' = y + dt f(y; V_n)                (forward Euler, V clamped:
//                                         AbstractCardiacCell::ComputeExceptVoltage)
//   I  = Iion(y'; V_n)                   (AbstractCardiacTissue::UpdateCaches)
//   z  = Am Cm V_n/dt - Am I - Istim(t_{n+1})   (MonodomainSolver.cpp:92-101)
//   A V_{n+1} = M z,  A = Am Cm/dt M + K(sigma) (MonodomainAssembler.cpp:43-66),
// solved by Jacobi CG with PETSc's stopping test.  Loss: mean over steps and
// probes of (V_{n+1}(probe) - target_n)^2.
//
// Parameters of a set: R regions x (P cell scale factors, conductivity scale).
// Node i belongs to region floor(i R / n); element e (nodes e, e+1) to region
// floor(e R / (n-1)) (both clamped to R-1).
//
// Adjoint of step n, given lam = dL/dV_{n+1} and ly = dL/dy_{n+1}:
//   mu = A^{-1} lam                            (A symmetric)
//   dL/dsigma_e -= mu^T (dK/dsigma_e) V_{n+1}
//   lz = M mu ;  dL/dV_n = Am Cm/dt lz + ... ;  dL/dI = -Am lz
//   then the reverse products of Iion and of the Euler step (emitted with the
//   cell model) give dL/dy_n, the rest of dL/dV_n and dL/dp.
#pragma once

#include "../models/lr91.h"
#include "../models/tt06.h"
#include "common.cuh"

namespace chb {

constexpr int kCableMaxNodes = 1024;
constexpr int kCableMaxRegions = 8;

struct CableArgs {
    int n, n_steps, R, n_probes, n_stim, ckpt_every;
    int maxit;
    double h, sigma0, am, cm, dt, rtol, stim_mag, stim_dur;
    const double* params;      // n_sets x R x (P+1)
    const int* probes;         // n_probes distinct node indices
    const double* targets;     // n_steps x n_probes (null: no loss)
    double* loss;              // n_sets (may be null)
    double* traces;            // n_sets x n_steps x n_probes (may be null)
    double* ckpt;              // n_sets x n_ckpt x S x n  (null: none)
    double* seg;               // n_sets x ckpt_every x S x n  (adjoint scratch)
    double* grad;              // n_sets x R x (P+1)
    int* iters;                // n_sets: CG iterations summed over the run (may be null)
    int* status;
    double y0[32];             // the model's initial states
};

// Sum over the CTA; every thread gets the total (fixed reduction order).
__device__ __forceinline__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = lane < nw ? red[lane] : 0.0;
    return warp_sum(s);
}

__device__ __forceinline__ int cable_node_region(int i, int n, int R) { return min(R - 1, i * R / n); }
__device__ __forceinline__ int cable_elem_region(int e, int n, int R) { return min(R - 1, e * R / (n - 1)); }

struct CableShared {
    double Ad[kCableMaxNodes], Ao[kCableMaxNodes], Md[kCableMaxNodes], Mo[kCableMaxNodes];
    double x[kCableMaxNodes], p[kCableMaxNodes], q[kCableMaxNodes];
    double lam[kCableMaxNodes], vn1[kCableMaxNodes];
    double red[32];
};

// Tridiagonal A and M, rows summed element by element in ascending order
// (row i gets element i-1, then element i), consistent P1 mass h/6 [2 1; 1 2].
static __device__ void cable_assemble(const CableArgs& a, const double* prm, int stride, CableShared& s) {
    const int n = a.n, i = threadIdx.x;
    if (i < n) {
        const double ms = a.am * a.cm / a.dt;
        double ad = 0.0, md = 0.0;
        for (int e = i - 1; e <= i; ++e) {
            if (e < 0 || e >= n - 1) continue;
            const double sig = a.sigma0 * prm[cable_elem_region(e, n, a.R) * stride + stride - 1];
            const double mdiag = a.h * 2.0 / 6.0;
            ad += ms * mdiag + sig / a.h;
            md += mdiag;
        }
        s.Ad[i] = ad;
        s.Md[i] = md;
        if (i < n - 1) {
            const double sig = a.sigma0 * prm[cable_elem_region(i, n, a.R) * stride + stride - 1];
            const double moff = a.h * 1.0 / 6.0;
            s.Ao[i] = ms * moff - sig / a.h;
            s.Mo[i] = moff;
        } else {
            s.Ao[i] = 0.0;
            s.Mo[i] = 0.0;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double tri(const double* d, const double* o, const double* v, int i, int n) {
    double acc = 0.0;
    if (i > 0) acc += o[i - 1] * v[i - 1];
    acc += d[i] * v[i];
    if (i < n - 1) acc += o[i] * v[i + 1];
    return acc;
}

// PETSc KSPCG (standard variant, preconditioned norm, KSPConvergedDefault) with
// Jacobi on A x = b inside the CTA; x in s.x holds the guess and receives the
// solution.  b_norm: measure the tolerance against ||B b|| (nonzero initial
// guess) instead of the initial residual.  Returns the iteration count, or -1
// when maxit was reached.
static __device__ int cable_cg(const CableArgs& a, CableShared& s, double bi, bool b_norm) {
    const int n = a.n, i = threadIdx.x;
    const bool on = i < n;
    __syncthreads();
    const double dinv = on ? 1.0 / s.Ad[i] : 0.0;
    double ri = on ? bi - tri(s.Ad, s.Ao, s.x, i, n) : 0.0;
    double zi = dinv * ri;
    double rnorm0;
    double dp = sqrt(block_sum(zi * zi, s.red));
    if (b_norm) {
        const double wb = dinv * bi;
        rnorm0 = sqrt(block_sum(wb * wb, s.red));
    } else {
        rnorm0 = dp;
    }
    const double ttol = fmax(a.rtol * rnorm0, 1e-50);
    if (dp <= ttol) return 0;
    double beta = block_sum(zi * ri, s.red), betaold = 1.0;
    double pi = 0.0;
    for (int it = 0; it < a.maxit; ++it) {
        if (beta == 0.0) return it;
        pi = it == 0 ? zi : zi + (beta / betaold) * pi;
        if (on) s.p[i] = pi;
        __syncthreads();
        const double qi = on ? tri(s.Ad, s.Ao, s.p, i, n) : 0.0;
        const double alpha = beta / block_sum(pi * qi, s.red);
        if (on) s.x[i] += alpha * pi;
        ri -= alpha * qi;
        zi = dinv * ri;
        dp = sqrt(block_sum(zi * zi, s.red));
        if (dp <= ttol) return it + 1;
        betaold = beta;
        beta = block_sum(zi * ri, s.red);
    }
    return -1;
}

__device__ __forceinline__ double cable_stim(const CableArgs& a, int i, double t) {
    // SimpleStimulus starting at 0 (duration padded as SimpleStimulus.cpp:50 does)
    const double dur = a.stim_dur + a.stim_dur * DBL_EPSILON;
    return (i < a.n_stim && 0.0 <= t && t <= dur) ? a.stim_mag : 0.0;
}

// One ODE step of node i and its right-hand side entry z_i; y[0] = V_n.
template <class M>
__device__ __forceinline__ double cable_node_step(const CableArgs& a, int i, double* y, const double* p, int step) {
    const double t0 = (double)step * a.dt, t1 = t0 + a.dt;
    const double v = y[0];
    fe_step_except_voltage<M, double>(y, cable_stim(a, i, t0) / a.am, a.cm, p, a.dt);
    const double ii = M::template iionic<double>(y, a.cm, p);
    return a.am * a.cm * v * (1.0 / a.dt) + (-a.am * ii - cable_stim(a, i, t1));
}

template <class M>
__global__ void __launch_bounds__(kCableMaxNodes, 1) cable_forward_kernel(CableArgs a) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    constexpr int stride = P + 1;
    extern __shared__ double smem_raw[];
    CableShared& s = *reinterpret_cast<CableShared*>(smem_raw);
    const int n = a.n, i = threadIdx.x;
    const bool on = i < n;
    const int set = blockIdx.x;
    const double* prm = a.params + (size_t)set * a.R * stride;
    cable_assemble(a, prm, stride, s);
    const int n_ckpt = a.ckpt_every > 0 ? (a.n_steps + a.ckpt_every - 1) / a.ckpt_every : 0;
    double* ckpt = a.ckpt ? a.ckpt + (size_t)set * n_ckpt * S * n : nullptr;
    double y[S], p[P];
    for (int k = 0; k < S; ++k) y[k] = a.y0[k];
    for (int k = 0; k < P; ++k) p[k] = on ? prm[cable_node_region(i, n, a.R) * stride + k] : 1.0;
    if (on) s.x[i] = y[0];
    double loss = 0.0;
    int iters = 0;
    for (int step = 0; step < a.n_steps; ++step) {
        if (ckpt && step % a.ckpt_every == 0 && on) {
            double* c = ckpt + (size_t)(step / a.ckpt_every) * S * n;
            c[i] = s.x[i];
            for (int k = 1; k < S; ++k) c[(size_t)k * n + i] = y[k];
        }
        if (on) {
            y[0] = s.x[i];
            s.q[i] = cable_node_step<M>(a, i, y, p, step);
        }
        __syncthreads();
        const double bi = on ? tri(s.Md, s.Mo, s.q, i, n) : 0.0;
        const int its = cable_cg(a, s, bi, true);
        if (its < 0) {
            if (i == 0) atomicOr(a.status, kStatusCgMaxIt);
        } else {
            iters += its;
        }
        __syncthreads();
        for (int k = i; k < a.n_probes; k += blockDim.x) {
            const double v = s.x[a.probes[k]];
            if (a.traces) a.traces[((size_t)set * a.n_steps + step) * a.n_probes + k] = v;
            if (a.targets) {
                const double d = v - a.targets[(size_t)step * a.n_probes + k];
                loss += d * d;
            }
        }
    }
    if (on && !(s.x[i] == s.x[i])) atomicOr(a.status, kStatusNaN);
    loss = block_sum(loss, s.red);
    if (i == 0) {
        if (a.loss) a.loss[set] = loss / ((double)a.n_steps * a.n_probes);
        if (a.iters) a.iters[set] = iters;
    }
}

// Gradient of the loss for parameter set blockIdx.x.  The checkpoints must come
// from cable_forward_kernel with the same arguments; each segment is recomputed
// once from its checkpoint (states before every step kept in `seg`) and then
// walked backwards.
template <class M>
__global__ void __launch_bounds__(kCableMaxNodes, 1) cable_adjoint_kernel(CableArgs a) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    constexpr int stride = P + 1;
    extern __shared__ double smem_raw[];
    CableShared& s = *reinterpret_cast<CableShared*>(smem_raw);
    __shared__ double gsh[kCableMaxRegions * stride];
    const int n = a.n, i = threadIdx.x;
    const bool on = i < n;
    const int set = blockIdx.x;
    const double* prm = a.params + (size_t)set * a.R * stride;
    cable_assemble(a, prm, stride, s);
    const int n_ckpt = (a.n_steps + a.ckpt_every - 1) / a.ckpt_every;
    const double* ckpt = a.ckpt + (size_t)set * n_ckpt * S * n;
    double* seg = a.seg + (size_t)set * a.ckpt_every * S * n;
    const int reg = on ? cable_node_region(i, n, a.R) : 0;
    double p[P], gp[P], ly[S];
    for (int k = 0; k < P; ++k) {
        p[k] = on ? prm[reg * stride + k] : 1.0;
        gp[k] = 0.0;
    }
    for (int k = 0; k < S; ++k) ly[k] = 0.0;
    if (on) s.lam[i] = 0.0;
    double gsig = 0.0;   // element (i, i+1)
    const double inv_np = 1.0 / ((double)a.n_steps * a.n_probes);
    for (int c = n_ckpt - 1; c >= 0; --c) {
        const int first = c * a.ckpt_every;
        const int last = min(a.n_steps, first + a.ckpt_every);
        if (on) s.x[i] = ckpt[(size_t)c * S * n + i];
        double y[S];
        for (int k = 1; k < S; ++k) y[k] = on ? ckpt[((size_t)c * S + k) * n + i] : a.y0[k];
        for (int step = first; step < last; ++step) {
            if (on) {
                y[0] = s.x[i];
                double* dst = seg + (size_t)(step - first) * S * n;
                for (int k = 0; k < S; ++k) dst[(size_t)k * n + i] = y[k];
                s.q[i] = cable_node_step<M>(a, i, y, p, step);
            }
            __syncthreads();
            const double bi = on ? tri(s.Md, s.Mo, s.q, i, n) : 0.0;
            cable_cg(a, s, bi, true);
            __syncthreads();
        }
        if (on) s.vn1[i] = s.x[i];
        __syncthreads();
        for (int step = last - 1; step >= first; --step) {
            for (int k = i; k < a.n_probes; k += blockDim.x) {
                const int node = a.probes[k];
                s.lam[node] += 2.0 * (s.vn1[node] - a.targets[(size_t)step * a.n_probes + k]) * inv_np;
            }
            __syncthreads();
            const double li = on ? s.lam[i] : 0.0;
            if (on) s.x[i] = 0.0;
            cable_cg(a, s, li, false);   // mu = A^{-1} lam in s.x
            __syncthreads();
            if (on && i < n - 1)
                gsig -= (a.sigma0 / a.h) * (s.x[i] - s.x[i + 1]) * (s.vn1[i] - s.vn1[i + 1]);
            const double lz = on ? tri(s.Md, s.Mo, s.x, i, n) : 0.0;
            double lv = a.am * a.cm / a.dt * lz;
            double vn = 0.0;
            if (on) {
                double yn[S], y1[S];
                const double* src = seg + (size_t)(step - first) * S * n;
                for (int k = 0; k < S; ++k) yn[k] = y1[k] = src[(size_t)k * n + i];
                vn = yn[0];
                const double st = cable_stim(a, i, (double)step * a.dt) / a.am;
                fe_step_except_voltage<M, double>(y1, st, a.cm, p, a.dt);
                // I = Iion(y'; V_n)
                const double lI = -a.am * lz;
                double gy[S];
                for (int k = 0; k < S; ++k) gy[k] = 0.0;
                M::template vjp_iionic<double>(y1, 0.0, a.cm, p, &lI, gy, gp);
                lv += gy[0];
                for (int k = 1; k < S; ++k) ly[k] += gy[k];
                // y'_k = y_k + dt f_k(y) for k >= 1 (y'_0 = V_n)
                double w[S], gf[S], gpf[P];
                w[0] = 0.0;
                for (int k = 1; k < S; ++k) w[k] = ly[k];
                for (int k = 0; k < S; ++k) gf[k] = 0.0;
                for (int k = 0; k < P; ++k) gpf[k] = 0.0;
                M::template vjp_rhs<double>(yn, st, a.cm, p, w, gf, gpf);
                lv += a.dt * gf[0];
                for (int k = 1; k < S; ++k) ly[k] += a.dt * gf[k];
                for (int k = 0; k < P; ++k) gp[k] += a.dt * gpf[k];
            }
            __syncthreads();
            if (on) {
                s.lam[i] = lv;
                s.vn1[i] = vn;
            }
            __syncthreads();
        }
    }
    // per-region totals: cell parameters by node region, conductivity by element region
    for (int r = 0; r < a.R; ++r) {
        for (int k = 0; k < P; ++k) {
            const double v = block_sum(on && reg == r ? gp[k] : 0.0, s.red);
            if (i == 0) gsh[r * stride + k] = v;
        }
        const double v = block_sum(on && i < n - 1 && cable_elem_region(i, n, a.R) == r ? gsig : 0.0, s.red);
        if (i == 0) gsh[r * stride + P] = v;
    }
    __syncthreads();
    for (int k = i; k < a.R * stride; k += blockDim.x) a.grad[(size_t)set * a.R * stride + k] = gsh[k];
}

}  // namespace chb
