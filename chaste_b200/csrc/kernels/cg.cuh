// Diffusion solve of one PDE step as ONE persistent, cooperatively launched
// kernel: RHS b = M z (MonodomainSolver.cpp:107), then PETSc's CG
// (KSPSolve_CG, standard variant, left preconditioning, preconditioned-norm
// convergence test of KSPConvergedDefault) from the guess V
// (LinearSystem::Solve, linalg/src/LinearSystem.cpp:833-837, 1099).
//
// Per iteration two grid-wide reductions (p.Ap, then z.z and z.r) are done by
// the bounded GridSync; every block derives the same scalars from the
// deterministic block-order sums, so the loop exits uniformly.  Traffic per
// iteration and node (slab operator, FP64): phase A reads r, p_old, class and
// writes p_new (q = A p_new is formed from r and p_old on the fly); phase B
// reads x, p_new, r, class and writes x, r, recomputing q from p_new.
#pragma once

#include "common.cuh"
#include "ops.cuh"

namespace chb {

struct CgArgs {
    SlabOp slab;
    CsrOp csr;
    int n;
    double* x;                  // V: initial guess in, solution out
    const double* zrhs;         // z (FP64 path)
    const float* zrhs32;        // z (mixed path)
    const uint8_t* cls8;        // slab class per node
    double* r;
    double* p0;
    double* p1;
    double* q;                  // CSR only
    float* r32;                 // mixed path workspace
    float* p32a;
    float* p32b;
    float* e32;
    float* q32;
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
    int max_refine;
};

template <bool SLAB>
__device__ __forceinline__ double dinv_of(const CgArgs& a, const SlabShared<double>& sh, int j) {
    if (a.pc == 0) return 1.0;
    if constexpr (SLAB) return sh.dinv[a.cls8[j]];
    else return a.csr.dinv[j];
}

template <bool SLAB>
__device__ __forceinline__ int class_of(const CgArgs& a, int i) {
    if constexpr (SLAB) return a.cls8[i];
    else return 0;
}

template <bool SLAB, class Load>
__device__ __forceinline__ double rowA(const CgArgs& a, const SlabShared<double>& sh, int c, int i, Load ld) {
    if constexpr (SLAB) return slab_row<double, double>(&sh.a[c * a.slab.n_off], sh.off, a.slab.n_off, i, ld);
    else return csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.a, i, ld);
}

template <bool SLAB, class Load>
__device__ __forceinline__ double rowM(const CgArgs& a, const SlabShared<double>& sh, int c, int i, Load ld) {
    if constexpr (SLAB) return slab_row<double, double>(&sh.m[c * a.slab.n_off], sh.off, a.slab.n_off, i, ld);
    else return csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.m, i, ld);
}

__device__ __forceinline__ void cg_finish(const CgArgs& a, long long step, int its, int bits) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (bits) atomicOr(a.status, bits);
        a.iters_ring[step % a.ring] = its;
        *a.step = step + 1;
    }
}

template <bool SLAB>
__global__ void __launch_bounds__(512) cg_fp64_kernel(CgArgs a) {
    __shared__ SlabShared<double> sh;
    __shared__ double red[32 * 4];
    __shared__ double red_out[4];
    if constexpr (SLAB) slab_load_shared<double>(a.slab, sh, a.diag_slot);
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double* __restrict__ z = a.zrhs;
    double* __restrict__ x = a.x;
    double* __restrict__ r = a.r;
    double res[4];

    // ---- phase 0: r = M z - A x, norms of B b and B r
    {
        double v[4] = {0, 0, 0, 0};
        for (int i = t0; i < n; i += stride) {
            const int c = class_of<SLAB>(a, i);
            const double b = rowM<SLAB>(a, sh, c, i, [&](int j) { return z[j]; });
            const double av = rowA<SLAB>(a, sh, c, i, [&](int j) { return x[j]; });
            const double rr = b - av;
            const double d = dinv_of<SLAB>(a, sh, i);
            const double w = d * b, zz = d * rr;
            v[0] += fabs(b);
            v[1] += w * w;
            v[2] += zz * zz;
            v[3] += rr * zz;
            r[i] = rr;
        }
        block_reduce<4>(v, red, red_out);
        if (!grid_reduce<4>(a.gs, a.partials, red_out, res, a.status)) return;
    }
    double rnorm0 = sqrt(res[1]);
    double dp = sqrt(res[2]);
    double beta = res[3];
    if (res[0] < 1e-15 && res[0] > 0.0) {
        // LinearSystem.cpp:984-994: tiny RHS -> zero initial guess, r = b
        double v[2] = {0, 0};
        for (int i = t0; i < n; i += stride) {
            const int c = class_of<SLAB>(a, i);
            const double b = rowM<SLAB>(a, sh, c, i, [&](int j) { return z[j]; });
            const double d = dinv_of<SLAB>(a, sh, i);
            const double zz = d * b;
            x[i] = 0.0;
            r[i] = b;
            v[0] += zz * zz;
            v[1] += b * zz;
        }
        double o2[2];
        block_reduce<2>(v, red, red_out);
        if (!grid_reduce<2>(a.gs, a.partials, red_out, o2, a.status)) return;
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
    double* po = a.p0;
    double* pn = a.p1;
    int it = 0;
    for (; it < a.maxit; ++it) {
        if (beta == 0.0) return cg_finish(a, step, it + 1, 0);
        const double bc = it == 0 ? 0.0 : beta / betaold;
        // ---- phase A: p_new = B r + bc p_old ; q = A p_new ; p_new . q
        {
            double v[1] = {0};
            const double* __restrict__ pold = po;
            const bool first = it == 0;
            auto pl = [&](int j) {
                const double zj = dinv_of<SLAB>(a, sh, j) * r[j];
                return first ? zj : zj + bc * pold[j];
            };
            for (int i = t0; i < n; i += stride) {
                const int c = class_of<SLAB>(a, i);
                const double qi = rowA<SLAB>(a, sh, c, i, pl);
                const double pi = pl(i);
                pn[i] = pi;
                if constexpr (!SLAB) a.q[i] = qi;
                v[0] += pi * qi;
            }
            block_reduce<1>(v, red, red_out);
            if (!grid_reduce<1>(a.gs, a.partials, red_out, res, a.status)) return;
        }
        const double dpi = res[0];
        if (!(dpi > 0.0)) return cg_finish(a, step, it + 1, isfinite(dpi) ? kStatusCgDiverged : kStatusNaN);
        const double alpha = beta / dpi;
        // ---- phase B: x += alpha p ; r -= alpha q ; z = B r ; z.z, z.r
        {
            double v[2] = {0, 0};
            const double* __restrict__ pnew = pn;
            for (int i = t0; i < n; i += stride) {
                const int c = class_of<SLAB>(a, i);
                double qi;
                if constexpr (SLAB) qi = rowA<SLAB>(a, sh, c, i, [&](int j) { return pnew[j]; });
                else qi = a.q[i];
                const double pi = pnew[i];
                x[i] += alpha * pi;
                const double rr = r[i] - alpha * qi;
                r[i] = rr;
                const double zz = dinv_of<SLAB>(a, sh, i) * rr;
                v[0] += zz * zz;
                v[1] += zz * rr;
            }
            block_reduce<2>(v, red, red_out);
            if (!grid_reduce<2>(a.gs, a.partials, red_out, res, a.status)) return;
        }
        dp = sqrt(res[0]);
        if (!isfinite(dp)) return cg_finish(a, step, it + 1, kStatusNaN);
        if (dp <= ttol) return cg_finish(a, step, it + 1, 0);
        if (dp >= a.dtol * rnorm0) return cg_finish(a, step, it + 1, kStatusCgDiverged);
        betaold = beta;
        beta = res[1];
        double* tmp = po;
        po = pn;
        pn = tmp;
    }
    cg_finish(a, step, it, kStatusCgMaxIt);
}

}  // namespace chb
