// Diffusion solve with PETSc's bjacobi preconditioner on one process, which is
// ILU(0) of the whole matrix in natural order (linalg/src/LinearSystem.cpp:780-829
// selects it; Chaste's default, heart/src/problem/HeartConfigDefaults.hpp:83), in one
// persistent cooperative kernel over the assembled CSR operator.
//
// The CG recurrence, the stopping test and the zero-guess rule are those of
// cg_fp64_kernel (KSPSolve_CG, KSPConvergedDefault with rnorm0 = ||B b||).  B r is
// the two triangular solves of the ILU(0) factors, level-scheduled: the host
// sorts the rows of L (and of U) into levels, a row's level being one more than
// the highest level among the rows it depends on, so the rows of a level are
// independent.  Each row is summed in ascending column order, the order of a
// sequential solve, so B r is the same number whichever thread takes the row.
// Levels are separated by a block barrier when the kernel runs as one block and
// by a grid barrier otherwise.
//
// Fused per iteration: the forward sweep also takes x += alpha p and
// r -= alpha A p for its row, and the backward sweep accumulates (z, z) and
// (z, r); the reduction after the last level is the barrier before the next
// operator application.  Barriers per iteration: one reduction (p . A p), one per
// forward and backward level.
#pragma once

#include "cg.cuh"

namespace chb {

// Level schedule and factors of the ILU(0) preconditioner.
struct IluArgs {
    const double* lu;        // factors in A's CSR pattern (L strictly below the diagonal, unit
                             // diagonal implied; U on and above it)
    const int* diag;         // CSR index of each row's diagonal entry
    const int* f_rows;       // rows in forward-level order
    const int* f_ptr;        // f_ptr[l] .. f_ptr[l+1]: the rows of forward level l
    int f_levels;
    const int* b_rows;       // rows in backward-level order (level 0 holds the last rows)
    const int* b_ptr;
    int b_levels;
    double* bvec;            // b = M z (+ correction), n
    double* wvec;            // B b, n
};

// Every thread of every block arrives; returns false when a bounded wait gave up.
// One block: a block barrier.  Several: the arrival counter of grid_reduce (the
// same rounds, so the two interleave), with acquire and release at device scope.
__device__ __forceinline__ bool level_barrier(GridSync* gs, int* status, unsigned& round) {
    __shared__ int s_ok;
    if (gridDim.x == 1) {
        __syncthreads();
        return true;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned target = (round + 1u) * gridDim.x;
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
        cnt.fetch_add(1u, cuda::memory_order_release);
        s_ok = wait_count(&gs->count, target, status) ? 1 : 0;
    }
    round++;
    __syncthreads();
    return s_ok != 0;
}

// Forward solve L y = r for the rows of one level (y overwrites out).
__device__ __forceinline__ double ilu_forward_row(const CgArgs& a, const IluArgs& f, int i, double ri,
                                                  double* out) {
    double s = ri;
    const int d = f.diag[i];
    for (int k = a.csr.rowptr[i]; k < d; ++k) s -= f.lu[k] * out[a.csr.cols[k]];
    out[i] = s;
    return s;
}

// Backward solve U z = y for a row (z overwrites y in out).
__device__ __forceinline__ double ilu_backward_row(const CgArgs& a, const IluArgs& f, int i, double* out) {
    const int d = f.diag[i];
    double s = out[i];
    const int e = a.csr.rowptr[i + 1];
    for (int k = d + 1; k < e; ++k) s -= f.lu[k] * out[a.csr.cols[k]];
    const double z = s / f.lu[d];
    out[i] = z;
    return z;
}

__device__ void cg_ilu_kernel_body(const CgArgs& a, const IluArgs& f, unsigned& round) {
    __shared__ double red[32 * 4];
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double* __restrict__ x = a.x;
    double* __restrict__ r = a.r;
    double* __restrict__ zp = a.zp;
    double* __restrict__ q = a.q;
    double* __restrict__ p = a.p0;
    double res[4];

    // ---- b = M z (+ correction), r = b - A x, sum |b|
    double babs = 0.0;
    for (int i = t0; i < n; i += stride) {
        const double b = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.m, i, a.zrhs) +
                         (a.corr ? a.corr[i] : 0.0);
        const double av = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.a, i, x);
        f.bvec[i] = b;
        r[i] = b - av;
        babs += fabs(b);
    }
    if (!level_barrier(a.gs, a.status, round)) return;
    // ---- B r into zp and B b into w, both sweeps level by level
    for (int l = 0; l < f.f_levels; ++l) {
        const int e = f.f_ptr[l + 1];
        for (int k = f.f_ptr[l] + t0; k < e; k += stride) {
            const int i = f.f_rows[k];
            ilu_forward_row(a, f, i, r[i], zp);
            ilu_forward_row(a, f, i, f.bvec[i], f.wvec);
        }
        if (!level_barrier(a.gs, a.status, round)) return;
    }
    double v[4] = {babs, 0.0, 0.0, 0.0};
    for (int l = 0; l < f.b_levels; ++l) {
        const int e = f.b_ptr[l + 1];
        for (int k = f.b_ptr[l] + t0; k < e; k += stride) {
            const int i = f.b_rows[k];
            const double zz = ilu_backward_row(a, f, i, zp);
            const double ww = ilu_backward_row(a, f, i, f.wvec);
            v[1] += ww * ww;
            v[2] += zz * zz;
            v[3] += r[i] * zz;
        }
        if (l + 1 < f.b_levels && !level_barrier(a.gs, a.status, round)) return;
    }
    if (!grid_reduce<4>(v, red, a.gs, a.partials, res, a.status, round)) return;
    double rnorm0 = sqrt(res[1]);
    double dp = sqrt(res[2]);
    double beta = res[3];
    if (res[0] < 1e-15 && res[0] > 0.0) {
        // LinearSystem.cpp:984-994: tiny RHS -> zero initial guess, r = b, B r = B b
        double v2[2] = {0, 0};
        for (int i = t0; i < n; i += stride) {
            const double b = f.bvec[i], zz = f.wvec[i];
            x[i] = 0.0;
            r[i] = b;
            zp[i] = zz;
            v2[0] += zz * zz;
            v2[1] += b * zz;
        }
        double o2[2];
        if (!grid_reduce<2>(v2, red, a.gs, a.partials, o2, a.status, round)) return;
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
    int it = 0;
    for (; it < a.maxit; ++it) {
        if (beta == 0.0) return cg_finish(a, step, it + 1, 0);
        const double bc = it == 0 ? 0.0 : beta / betaold;
        const bool first = it == 0;
        // ---- p = z + bc p ; A p = A z + bc A p ; p . A p
        {
            double v1[1] = {0};
            for (int i = t0; i < n; i += stride) {
                const double az = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.a, i, zp);
                const double qi = first ? az : az + bc * q[i];
                const double pi = first ? zp[i] : zp[i] + bc * p[i];
                q[i] = qi;
                p[i] = pi;
                v1[0] += pi * qi;
            }
            if (!grid_reduce<1>(v1, red, a.gs, a.partials, res, a.status, round)) return;
        }
        const double dpi = res[0];
        if (!(dpi > 0.0)) return cg_finish(a, step, it + 1, isfinite(dpi) ? kStatusCgDiverged : kStatusNaN);
        const double alpha = beta / dpi;
        // ---- forward sweep with x += alpha p, r -= alpha A p of each row
        for (int l = 0; l < f.f_levels; ++l) {
            const int e = f.f_ptr[l + 1];
            for (int k = f.f_ptr[l] + t0; k < e; k += stride) {
                const int i = f.f_rows[k];
                x[i] += alpha * p[i];
                const double rr = r[i] - alpha * q[i];
                r[i] = rr;
                ilu_forward_row(a, f, i, rr, zp);
            }
            if (!level_barrier(a.gs, a.status, round)) return;
        }
        // ---- backward sweep with (z, z) and (z, r)
        double v2[2] = {0, 0};
        for (int l = 0; l < f.b_levels; ++l) {
            const int e = f.b_ptr[l + 1];
            for (int k = f.b_ptr[l] + t0; k < e; k += stride) {
                const int i = f.b_rows[k];
                const double zz = ilu_backward_row(a, f, i, zp);
                v2[0] += zz * zz;
                v2[1] += zz * r[i];
            }
            if (l + 1 < f.b_levels && !level_barrier(a.gs, a.status, round)) return;
        }
        if (!grid_reduce<2>(v2, red, a.gs, a.partials, res, a.status, round)) return;
        dp = sqrt(res[0]);
        if (!isfinite(dp)) return cg_finish(a, step, it + 1, kStatusNaN);
        if (dp <= ttol) return cg_finish(a, step, it + 1, 0);
        if (dp >= a.dtol * rnorm0) return cg_finish(a, step, it + 1, kStatusCgDiverged);
        betaold = beta;
        beta = res[1];
    }
    cg_finish(a, step, it, kStatusCgMaxIt);
}

static __global__ void __launch_bounds__(1024, 1) cg_ilu_kernel(CgArgs a, IluArgs f) {
    unsigned round = 0;
    cg_ilu_kernel_body(a, f, round);
    grid_exit(a.gs);
}

}  // namespace chb
