// Bidomain diffusion solve without a bath, in one persistent cooperative kernel:
// BidomainSolver::SetupLinearSystem (heart/src/solver/electrics/bidomain/BidomainSolver.cpp:63-190)
// and LinearSystem::Solve on the interleaved unknowns u = (V_0, phi_0, V_1, phi_1, ...):
//
//   B u = (M z, 0),  B = [ Am Cm/dt M + K_i   K_i       ]   per node pair,
//                        [ K_i                K_i + K_e ]
//
// z = Am Cm V/dt - Am Iion - Istim from the ODE kernel (the phi_e rows of the
// right-hand side are zero: BidomainMassMatrixAssembler puts mass in the V-V block
// only).  PETSc CG (standard variant, preconditioned norm, KSPConvergedDefault) with
// Jacobi or no preconditioner.  Without fixed phi_e nodes B is singular and the solve
// carries the null space of constant phi_e (AbstractBidomainSolver::GenerateNullBasis,
// AbstractBidomainSolver.cpp:112-134): as PETSc's KSP_PCApply does, every
// preconditioned vector z has its component along e = (0, 1/sqrt(n), 0, 1/sqrt(n), ...)
// removed, z' = z - c e with c = z.e.  Inside the iteration the kernel keeps z as the
// preconditioner left it and c beside it: the norms follow from sums taken in the same
// grid reduction (z'.z' = z.z - c^2, z'.r = z.r - c (e.r), since e.e = 1), and the next
// operator application and direction update use z' = z - c e entry by entry, so the
// projection costs no extra reduction.
// Fixed phi_e nodes are identity rows and columns of B (zero right-hand side), set on
// the host.  The operator is B's CSR (rows 2i and 2i+1 share node i's pattern).
#pragma once

#include "cg.cuh"

namespace chb {

struct BidoArgs {
    int n2;                          // 2 n rows
    const int* __restrict__ rp;      // B (CSR, sorted columns)
    const int* __restrict__ ci;
    const double* __restrict__ val;
    const double* __restrict__ dinv; // 1 / diag(B), or null: no preconditioner
    double* u;                       // guess in, solution out
    double* r;
    double* z;
    double* p;
    double* q;
    int nullspace;
    double inv_sqrt_n;               // the null-space basis entry 1/sqrt(n)
};

// u's V entries from the voltage the ODE kernel used (the solve's initial guess is the
// current solution, LinearSystem.cpp:833-837).
static __global__ void bido_copy_voltage_kernel(int n, const double* __restrict__ V, double* __restrict__ u) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) u[2 * i] = V[i];
}

__device__ __forceinline__ double bido_pc(const BidoArgs& b, int i, double r) { return b.dinv ? b.dinv[i] * r : r; }

// The solution's V entries back into the tissue voltage, then the step's bookkeeping.
__device__ __forceinline__ void bido_finish(const CgArgs& a, const BidoArgs& b, long long step, int its, int bits) {
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) a.x[i] = b.u[2 * i];
    cg_finish(a, step, its, bits);
}

__device__ void cg_bidomain_body(const CgArgs& a, const BidoArgs& b, unsigned& round) {
    __shared__ double red[32 * 4];
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n2 = b.n2;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double inv = b.inv_sqrt_n;
    double res[4];

    // ---- rhs (kept in q), r = rhs - B u, z = B r, w = B rhs (in p); sums |rhs| and the
    // null-space coefficients of z and w
    {
        double v[3] = {0, 0, 0};
        for (int i = t0; i < n2; i += stride) {
            const double bi = (i & 1) ? 0.0 : csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.m, i >> 1, a.zrhs);
            const double ri = bi - csr_row<double, double>(b.rp, b.ci, b.val, i, b.u);
            const double zi = bido_pc(b, i, ri), wi = bido_pc(b, i, bi);
            b.q[i] = bi;
            b.r[i] = ri;
            b.z[i] = zi;
            b.p[i] = wi;
            v[0] += fabs(bi);
            if (i & 1) {
                v[1] += zi * inv;
                v[2] += wi * inv;
            }
        }
        if (!grid_reduce<3>(v, red, a.gs, a.partials, res, a.status, round)) return;
    }
    // LinearSystem::Solve: a tiny nonzero right-hand side means a zero initial guess
    // (LinearSystem.cpp:984-994)
    const bool guess_zero = res[0] < 1e-15 && res[0] > 0.0;
    const double az = b.nullspace ? res[1] : 0.0, aw = b.nullspace ? res[2] : 0.0;
    {
        double v[3] = {0, 0, 0};
        for (int i = t0; i < n2; i += stride) {
            double ri = b.r[i], zi = b.z[i], wi = b.p[i];
            if (guess_zero) {
                b.u[i] = 0.0;
                ri = b.q[i];
                b.r[i] = ri;
                zi = wi;
            }
            if (i & 1) {
                zi -= (guess_zero ? aw : az) * inv;
                wi -= aw * inv;
            }
            b.z[i] = zi;
            v[0] += zi * zi;
            v[1] += wi * wi;
            v[2] += zi * ri;
        }
        if (!grid_reduce<3>(v, red, a.gs, a.partials, res, a.status, round)) return;
    }
    double dp = sqrt(res[0]);
    double rnorm0 = guess_zero ? dp : sqrt(res[1]);
    if (rnorm0 == 0.0) rnorm0 = dp;
    double beta = res[2];
    const double ttol = fmax(a.rtol * rnorm0, a.abstol);
    if (!isfinite(dp)) return bido_finish(a, b, step, 0, kStatusNaN);
    if (dp <= ttol) return bido_finish(a, b, step, 0, 0);
    if (dp >= a.dtol * rnorm0) return bido_finish(a, b, step, 0, kStatusCgDiverged);

    double betaold = 0.0;
    double c = 0.0;   // null-space coefficient of the stored z (zero: the z above is projected)
    int it = 0;
    for (; it < a.maxit; ++it) {
        if (beta == 0.0) return bido_finish(a, b, step, it + 1, 0);
        const double bc = it == 0 ? 0.0 : beta / betaold;
        const bool first = it == 0;
        const double ce = c * inv;   // z' = z - ce on the phi_e rows
        // ---- p = z' + bc p ; B p = B z' + bc B p ; p . B p
        {
            double v[1] = {0};
            for (int i = t0; i < n2; i += stride) {
                double bz = 0.0;
                const int e = b.rp[i + 1];
                for (int k = b.rp[i]; k < e; ++k) {
                    const int j = b.ci[k];
                    bz += b.val[k] * ((j & 1) ? b.z[j] - ce : b.z[j]);
                }
                const double zi = (i & 1) ? b.z[i] - ce : b.z[i];
                const double qi = first ? bz : bz + bc * b.q[i];
                const double pi = first ? zi : zi + bc * b.p[i];
                b.q[i] = qi;
                b.p[i] = pi;
                v[0] += pi * qi;
            }
            if (!grid_reduce<1>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        const double dpi = res[0];
        if (!(dpi > 0.0)) return bido_finish(a, b, step, it + 1, isfinite(dpi) ? kStatusCgDiverged : kStatusNaN);
        const double alpha = beta / dpi;
        // ---- u += alpha p ; r -= alpha B p ; z = B r; z.z, z.r and the null-space sums
        {
            double v[4] = {0, 0, 0, 0};
            for (int i = t0; i < n2; i += stride) {
                b.u[i] += alpha * b.p[i];
                const double ri = b.r[i] - alpha * b.q[i];
                b.r[i] = ri;
                const double zi = bido_pc(b, i, ri);
                b.z[i] = zi;
                v[0] += zi * zi;
                v[1] += zi * ri;
                if (i & 1) {
                    v[2] += zi * inv;
                    v[3] += ri * inv;
                }
            }
            if (!grid_reduce<4>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        c = b.nullspace ? res[2] : 0.0;
        const double zz = fmax(res[0] - c * c, 0.0);
        const double zr = res[1] - c * (b.nullspace ? res[3] : 0.0);
        dp = sqrt(zz);
        if (!isfinite(dp)) return bido_finish(a, b, step, it + 1, kStatusNaN);
        if (dp <= ttol) return bido_finish(a, b, step, it + 1, 0);
        if (dp >= a.dtol * rnorm0) return bido_finish(a, b, step, it + 1, kStatusCgDiverged);
        betaold = beta;
        beta = zr;
    }
    bido_finish(a, b, step, it, kStatusCgMaxIt);
}

static __global__ void __launch_bounds__(512, 2) cg_bidomain_kernel(CgArgs a, BidoArgs b) {
    unsigned round = 0;
    cg_bidomain_body(a, b, round);
    grid_exit(a.gs);
}

}  // namespace chb
