// Mixed-precision diffusion solve: FP64 outer residual and iterative
// refinement around FP32 Jacobi-PCG inner solves, in one persistent kernel.
//
//   r = b - A x                  (FP64, b = M z)
//   until ||B r|| <= ttol:       (the FP64 PETSc test: ttol = max(rtol*||B b||, atol))
//      solve A e = r in FP32     (PCG, e0 = 0, relative reduction chosen so one
//                                 sweep is expected to reach ttol)
//      x += e ; r = b - A x      (FP64)
// The inner vectors are float (half the bytes of the FP64 path); scalars and
// reductions stay in double.
#pragma once

#include "cg.cuh"

namespace chb {

template <bool SLAB>
__device__ __forceinline__ float dinv32_of(const CgArgs& a, const SlabShared<float>& s32, int j) {
    if (a.pc == 0) return 1.0f;
    if constexpr (SLAB) return s32.dinv[a.cls8[j]];
    else return a.csr.dinv32[j];
}

template <bool SLAB, class Load>
__device__ __forceinline__ float rowA32(const CgArgs& a, const SlabShared<float>& s32, int c, int i, Load ld) {
    if constexpr (SLAB) return slab_row<float, float>(&s32.a[c * a.slab.n_off], s32.off, a.slab.n_off, i, ld);
    else return csr_row<float, float>(a.csr.rowptr, a.csr.cols, a.csr.a32, i, ld);
}

template <bool SLAB>
__global__ void __launch_bounds__(512) cg_mixed_kernel(CgArgs a) {
    __shared__ SlabShared<double> sh;
    __shared__ SlabShared<float> s32;
    __shared__ double red[32 * 4];
    __shared__ double red_out[4];
    if constexpr (SLAB) {
        slab_load_shared<double>(a.slab, sh, a.diag_slot);
        slab_load_shared<float>(a.slab, s32, a.diag_slot);
    }
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const float* __restrict__ z = a.zrhs32;
    double* __restrict__ x = a.x;
    float* __restrict__ r32 = a.r32;
    float* __restrict__ e32 = a.e32;
    double res[4];
    double rnorm0 = 0.0, ttol = 0.0, dp = 0.0, rz = 0.0;
    int total_its = 0;
    int sweeps = 0;

    for (int sweep = 0;; ++sweep) {
        // ---- FP64 residual r = M z - A x; FP32 copy for the inner solve
        {
            double v[4] = {0, 0, 0, 0};
            for (int i = t0; i < n; i += stride) {
                const int c = class_of<SLAB>(a, i);
                const double b = rowM<SLAB>(a, sh, c, i, [&](int j) { return (double)z[j]; });
                const double av = rowA<SLAB>(a, sh, c, i, [&](int j) { return x[j]; });
                const double rr = b - av;
                const double d = dinv_of<SLAB>(a, sh, i);
                const double w = d * b, zz = d * rr;
                v[0] += fabs(b);
                v[1] += w * w;
                v[2] += zz * zz;
                const float rf = (float)rr;
                r32[i] = rf;
                e32[i] = 0.0f;
                v[3] += (double)rf * (double)(dinv32_of<SLAB>(a, s32, i) * rf);
            }
            block_reduce<4>(v, red, red_out);
            if (!grid_reduce<4>(a.gs, a.partials, red_out, res, a.status)) return;
        }
        dp = sqrt(res[2]);
        rz = res[3];
        if (sweep == 0) {
            rnorm0 = sqrt(res[1]);
            if (rnorm0 == 0.0) rnorm0 = dp;
            ttol = fmax(a.rtol * rnorm0, a.abstol);
        }
        if (!isfinite(dp)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
            return cg_finish(a, step, total_its, kStatusNaN);
        }
        if (dp <= ttol) break;
        if (dp >= a.dtol * rnorm0 || sweep >= a.max_refine) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
            return cg_finish(a, step, total_its, dp >= a.dtol * rnorm0 ? kStatusCgDiverged : kStatusCgMaxIt);
        }
        sweeps++;
        // ---- FP32 PCG on A e = r
        const double target = fmin(0.5, fmax(1e-6, 0.3 * ttol / dp));
        const double dp_in0 = dp;
        double beta = rz, betaold = 0.0;
        float* po = a.p32a;
        float* pn = a.p32b;
        int it = 0;
        bool inner_done = false;
        for (; it < a.maxit && !inner_done; ++it) {
            if (beta == 0.0) break;
            const float bc = it == 0 ? 0.0f : (float)(beta / betaold);
            {
                double v[1] = {0};
                const float* __restrict__ pold = po;
                const bool first = it == 0;
                auto pl = [&](int j) {
                    const float zj = dinv32_of<SLAB>(a, s32, j) * r32[j];
                    return first ? zj : zj + bc * pold[j];
                };
                for (int i = t0; i < n; i += stride) {
                    const int c = class_of<SLAB>(a, i);
                    const float qi = rowA32<SLAB>(a, s32, c, i, pl);
                    const float pi = pl(i);
                    pn[i] = pi;
                    if constexpr (!SLAB) a.q32[i] = qi;
                    v[0] += (double)pi * (double)qi;
                }
                block_reduce<1>(v, red, red_out);
                if (!grid_reduce<1>(a.gs, a.partials, red_out, res, a.status)) return;
            }
            const double dpi = res[0];
            if (!(dpi > 0.0)) break;   // the FP64 residual pass decides what happens next
            const float alpha = (float)(beta / dpi);
            {
                double v[2] = {0, 0};
                const float* __restrict__ pnew = pn;
                for (int i = t0; i < n; i += stride) {
                    const int c = class_of<SLAB>(a, i);
                    float qi;
                    if constexpr (SLAB) qi = rowA32<SLAB>(a, s32, c, i, [&](int j) { return pnew[j]; });
                    else qi = a.q32[i];
                    e32[i] += alpha * pnew[i];
                    const float rr = r32[i] - alpha * qi;
                    r32[i] = rr;
                    const float zz = dinv32_of<SLAB>(a, s32, i) * rr;
                    v[0] += (double)zz * (double)zz;
                    v[1] += (double)zz * (double)rr;
                }
                block_reduce<2>(v, red, red_out);
                if (!grid_reduce<2>(a.gs, a.partials, red_out, res, a.status)) return;
            }
            const double dp_in = sqrt(res[0]);
            betaold = beta;
            beta = res[1];
            if (!(dp_in > target * dp_in0)) inner_done = true;
            float* tmp = po;
            po = pn;
            pn = tmp;
        }
        total_its += it;
        // ---- x += e (FP64); the next residual pass needs every x updated
        {
            for (int i = t0; i < n; i += stride) x[i] += (double)e32[i];
            double v[1] = {0};
            block_reduce<1>(v, red, red_out);
            if (!grid_reduce<1>(a.gs, a.partials, red_out, res, a.status)) return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
    cg_finish(a, step, total_its, 0);
}

}  // namespace chb
