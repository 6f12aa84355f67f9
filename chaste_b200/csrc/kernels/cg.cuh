// Diffusion solve of one PDE step as ONE persistent, cooperatively launched
// kernel: RHS b = M z (MonodomainSolver.cpp:107), then PETSc's CG
// (KSPSolve_CG, standard variant, left preconditioning, preconditioned-norm
// convergence test of KSPConvergedDefault) from the guess V
// (LinearSystem::Solve, linalg/src/LinearSystem.cpp:833-837, 1099).
//
// Per iteration there are two grid-wide reductions (p.Ap, then z.z and z.r),
// done by the bounded GridSync; every block derives the same scalars from the
// deterministic block-order sums, so the loop exits uniformly.  The search
// direction update and the product are fused through the recurrence
//   p' = z + beta p,  A p' = A z + beta A p,
// so each iteration applies the operator once (to the preconditioned residual
// z, which is stored) and phase B touches only node-local values.
#pragma once

#include "common.cuh"
#include "ops.cuh"

namespace chb {

// Shared-memory staging of the pipelined solve's operator input (slab stencils):
// the offsets fall into n_bands contiguous bands (3 planes in 3D, 1 band in 1D
// and 2D); for each 512-node group of a block, band b's window of the input
// vector is copied with aligned float4 loads to stage[group * cap + base[b] ..],
// and offset o of the node with thread index t is then stage[group * cap + t + rel[o]].
constexpr int kMaxBands = 4;
struct StageArgs {
    int n_bands;
    int lo[kMaxBands];      // smallest offset of the band
    int len[kMaxBands];     // floats copied per group (multiple of 4)
    int base[kMaxBands];    // start of the band in the group's stage (multiple of 4)
    int cap;                // floats per group (multiple of 4)
    int halo;               // entries before entry 0 of a haloed vector (multiple of 4)
    long long alloc_len;    // floats of a haloed allocation, rounded down to a multiple of 4
    int rel[kMaxOffsets];
};

struct CgArgs {
    SlabOp slab;
    StageArgs stage;
    CsrOp csr;
    int n;
    double* x;                  // V: initial guess in, solution out (haloed)
    const double* zrhs;         // per-node RHS term z (FP64 path, haloed)
    const float* zrhs32;        // z (mixed path, haloed)
    const uint8_t* cls8;        // slab class per node
    const double* corr;         // state-variable interpolation correction added to b = M z (or null)
    double* r;
    double* zp;                 // preconditioned residual B r (haloed)
    double* p0;                 // search direction
    double* q;                  // A p
    float* r32;                 // mixed path workspace
    float* z32;                 // (haloed)
    float* p32;
    float* q32;
    float* e32;                 // (haloed)
    float* m32a;                // pipelined inner solve: alternating haloed buffers of B w
    float* m32b;
    double* partials;           // gridDim.x * 4
    GridSync* gs;
    int* status;
    long long* step;
    int* iters_ring;
    int ring;
    int* refine_out;
    double rtol, abstol, dtol;
    int maxit;
    int pc;                     // 0 none, 1 jacobi
    int diag_slot;
    int xm_slot, xp_slot;       // stencil slots of the x-neighbours (offsets -1, +1)
    int line_pc;                // mixed slab solve: inner preconditioner on x-line segments
    const float2* line_ad;      // its factors (a_i, 1/d_i) per node
    int max_refine;
};

template <bool SLAB>
__device__ __forceinline__ int class_of(const CgArgs& a, int i) {
    if constexpr (SLAB) return a.cls8[i];
    else return 0;
}

template <bool SLAB>
__device__ __forceinline__ double dinv_of(const CgArgs& a, const SlabShared<double>& sh, int c, int i) {
    if (a.pc == 0) return 1.0;
    if constexpr (SLAB) return sh.dinv[c];
    else return a.csr.dinv[i];
}

// y_i = (A x)_i or (M x)_i for the row of node i (class c)
template <bool SLAB, int NOFF, bool MASS, typename X>
__device__ __forceinline__ double apply_row(const CgArgs& a, const SlabShared<double>& sh, const int* soff,
                                            int c, int i, const X* x) {
    if constexpr (!SLAB) {
        return csr_row<double, double>(a.csr.rowptr, a.csr.cols, MASS ? a.csr.m : a.csr.a, i, x);
    } else if constexpr (NOFF > 0) {
        if (c == a.slab.interior) return slab_row<NOFF, double, double>(MASS ? a.slab.im : a.slab.ia, a.slab.off, NOFF, i, x);
        return slab_row<NOFF, double, double>(MASS ? &sh.m[c * NOFF] : &sh.a[c * NOFF], a.slab.off, NOFF, i, x);
    } else {
        const int no = a.slab.n_off;
        return slab_row<0, double, double>(MASS ? &sh.m[c * no] : &sh.a[c * no], soff, no, i, x);
    }
}

__device__ __forceinline__ void cg_finish(const CgArgs& a, long long step, int its, int bits) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (bits) atomicOr(a.status, bits);
        a.iters_ring[step % a.ring] = its;
        *a.step = step + 1;
    }
}

template <bool SLAB, int NOFF>
__device__ __forceinline__ void cg_fp64_kernel_body(const CgArgs& a, unsigned& round) {
    __shared__ SlabShared<double> sh;
    __shared__ int soff[kMaxOffsets];
    __shared__ double red[32 * 4];
    if constexpr (SLAB) {
        for (int k = threadIdx.x; k < a.slab.n_off; k += blockDim.x) soff[k] = a.slab.off[k];
        slab_load_shared<double>(a.slab, sh, a.diag_slot);
    }
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double* __restrict__ x = a.x;
    double* __restrict__ r = a.r;
    double* __restrict__ zp = a.zp;
    double* __restrict__ q = a.q;
    double res[4];

    // ---- phase 0: r = M z - A x, z = B r, norms of B b and B r
    {
        double v[4] = {0, 0, 0, 0};
        for (int i = t0; i < n; i += stride) {
            const int c = class_of<SLAB>(a, i);
            const double b = apply_row<SLAB, NOFF, true>(a, sh, soff, c, i, a.zrhs) + (a.corr ? a.corr[i] : 0.0);
            const double av = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, x);
            const double rr = b - av;
            const double d = dinv_of<SLAB>(a, sh, c, i);
            const double w = d * b, zz = d * rr;
            v[0] += fabs(b);
            v[1] += w * w;
            v[2] += zz * zz;
            v[3] += rr * zz;
            r[i] = rr;
            zp[i] = zz;
        }
        if (!grid_reduce<4>(v, red, a.gs, a.partials, res, a.status, round)) return;
    }
    double rnorm0 = sqrt(res[1]);
    double dp = sqrt(res[2]);
    double beta = res[3];
    if (res[0] < 1e-15 && res[0] > 0.0) {
        // LinearSystem.cpp:984-994: tiny RHS -> zero initial guess, r = b
        double v[2] = {0, 0};
        for (int i = t0; i < n; i += stride) {
            const int c = class_of<SLAB>(a, i);
            const double b = apply_row<SLAB, NOFF, true>(a, sh, soff, c, i, a.zrhs) + (a.corr ? a.corr[i] : 0.0);
            const double zz = dinv_of<SLAB>(a, sh, c, i) * b;
            x[i] = 0.0;
            r[i] = b;
            zp[i] = zz;
            v[0] += zz * zz;
            v[1] += b * zz;
        }
        double o2[2];
        if (!grid_reduce<2>(v, red, a.gs, a.partials, o2, a.status, round)) return;
        dp = sqrt(o2[0]);
        beta = o2[1];
        rnorm0 = dp;
    }
    if (rnorm0 == 0.0) rnorm0 = dp;
    const double ttol = fmax(a.rtol * rnorm0, a.abstol);
    if (!isfinite(dp)) return cg_finish(a, step, 0, kStatusNaN);
    if (dp <= ttol) return cg_finish(a, step, 0, 0);
    if (dp >= a.dtol * rnorm0) return cg_finish(a, step, 0, kStatusCgDiverged);

    double betaold = 0.0;
    double* __restrict__ p = a.p0;   // p and A p are only read at their own row: updated in place
    int it = 0;
    for (; it < a.maxit; ++it) {
        if (beta == 0.0) return cg_finish(a, step, it + 1, 0);
        const double bc = it == 0 ? 0.0 : beta / betaold;
        const bool first = it == 0;
        // ---- phase A: p = z + bc p ; A p = A z + bc A p ; p . A p
        {
            double v[1] = {0};
            for (int i = t0; i < n; i += stride) {
                const int c = class_of<SLAB>(a, i);
                const double az = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, zp);
                const double qi = first ? az : az + bc * q[i];
                const double pi = first ? zp[i] : zp[i] + bc * p[i];
                q[i] = qi;
                p[i] = pi;
                v[0] += pi * qi;
            }
            if (!grid_reduce<1>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        const double dpi = res[0];
        if (!(dpi > 0.0)) return cg_finish(a, step, it + 1, isfinite(dpi) ? kStatusCgDiverged : kStatusNaN);
        const double alpha = beta / dpi;
        // ---- phase B: x += alpha p ; r -= alpha A p ; z = B r ; z.z, z.r
        {
            // two grid-stride steps per loop trip, every load before the first store
            // (the nodes and the order of the sums are the plain loop's)
            double v[2] = {0, 0};
            for (int i0 = t0; i0 < n; i0 += 2 * stride) {
                double xo[2], po[2], ro[2], qo[2], dv[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = i0 + u * stride;
                    xo[u] = po[u] = ro[u] = qo[u] = dv[u] = 0.0;
                    if (i < n) {
                        dv[u] = dinv_of<SLAB>(a, sh, class_of<SLAB>(a, i), i);
                        xo[u] = x[i];
                        po[u] = p[i];
                        ro[u] = r[i];
                        qo[u] = q[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = i0 + u * stride;
                    if (i >= n) continue;
                    x[i] = xo[u] + alpha * po[u];
                    const double rr = ro[u] - alpha * qo[u];
                    r[i] = rr;
                    const double zz = dv[u] * rr;
                    zp[i] = zz;
                    v[0] += zz * zz;
                    v[1] += zz * rr;
                }
            }
            if (!grid_reduce<2>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        dp = sqrt(res[0]);
        if (!isfinite(dp)) return cg_finish(a, step, it + 1, kStatusNaN);
        if (dp <= ttol) return cg_finish(a, step, it + 1, 0);
        if (dp >= a.dtol * rnorm0) return cg_finish(a, step, it + 1, kStatusCgDiverged);
        betaold = beta;
        beta = res[1];
    }
    cg_finish(a, step, it, kStatusCgMaxIt);
}

template <bool SLAB, int NOFF>
__global__ void __launch_bounds__(512, 2) cg_fp64_kernel(CgArgs a) {
    unsigned round = 0;
    cg_fp64_kernel_body<SLAB, NOFF>(a, round);
    grid_exit(a.gs);
}

}  // namespace chb
