// Mixed-precision diffusion solve: FP64 outer residual and iterative
// refinement around FP32 Jacobi-PCG inner solves, in one persistent kernel.
//
//   r = b - A x                  (FP64, b = M z)
//   until ||B r|| <= ttol:       (the FP64 PETSc test: ttol = max(rtol*||B b||, atol))
//      solve A e = r in FP32     (PCG, e0 = 0)
//      x += e ; r -= A e         (FP64, one fused pass; e is read through the stencil)
// The inner vectors are float (half the bytes of the FP64 path); scalars and
// reductions stay in double.  The inner loop uses the same fused recurrence
// as the FP64 kernel (one operator application per iteration).
#pragma once

#include "cg.cuh"

namespace chb {

template <bool SLAB>
__device__ __forceinline__ float dinv32_of(const CgArgs& a, const SlabShared<float>& s32, int c, int i) {
    if (a.pc == 0) return 1.0f;
    if constexpr (SLAB) return s32.dinv[c];
    else return a.csr.dinv32[i];
}

template <bool SLAB, int NOFF>
__device__ __forceinline__ float apply_row32(const CgArgs& a, const SlabShared<float>& s32, const int* soff,
                                             int c, int i, const float* __restrict__ x) {
    if constexpr (!SLAB) {
        return csr_row<float, float>(a.csr.rowptr, a.csr.cols, a.csr.a32, i, x);
    } else if constexpr (NOFF > 0) {
        if (c == a.slab.interior) return slab_row<NOFF, float, float>(a.slab.ia32, a.slab.off, NOFF, i, x);
        return slab_row<NOFF, float, float>(&s32.a[c * NOFF], a.slab.off, NOFF, i, x);
    } else {
        const int no = a.slab.n_off;
        return slab_row<0, float, float>(&s32.a[c * no], soff, no, i, x);
    }
}

template <bool SLAB, int NOFF>
__global__ void __launch_bounds__(512, 2) cg_mixed_kernel(CgArgs a) {
    __shared__ SlabShared<double> sh;
    __shared__ SlabShared<float> s32;
    __shared__ int soff[kMaxOffsets];
    __shared__ double red[32 * 4];
    __shared__ double red_out[4];
    if constexpr (SLAB) {
        for (int k = threadIdx.x; k < a.slab.n_off; k += blockDim.x) soff[k] = a.slab.off[k];
        slab_load_shared<double>(a.slab, sh, a.diag_slot);
        slab_load_shared<float>(a.slab, s32, a.diag_slot);
    }
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double* __restrict__ x = a.x;
    float* __restrict__ r32 = a.r32;
    float* __restrict__ z32 = a.z32;
    float* __restrict__ p32 = a.p32;
    float* __restrict__ q32 = a.q32;
    float* __restrict__ e32 = a.e32;
    double res[4];
    double rnorm0 = 0.0, ttol = 0.0, dp = 0.0, rz = 0.0;
    int total_its = 0;
    int sweeps = 0;

    double* __restrict__ r = a.r;
    // ---- FP64 residual r = M z - A x (stored in FP64), its FP32 copy and B r
    {
        double v[4] = {0, 0, 0, 0};
        for (int i = t0; i < n; i += stride) {
            const int c = class_of<SLAB>(a, i);
            const double b = apply_row<SLAB, NOFF, true>(a, sh, soff, c, i, a.zrhs32);
            const double av = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, x);
            const double rr = b - av;
            const double d = dinv_of<SLAB>(a, sh, c, i);
            const double w = d * b, zz = d * rr;
            v[0] += fabs(b);
            v[1] += w * w;
            v[2] += zz * zz;
            const float rf = (float)rr;
            const float zf = dinv32_of<SLAB>(a, s32, c, i) * rf;
            r[i] = rr;
            r32[i] = rf;
            z32[i] = zf;
            v[3] += (double)rf * (double)zf;
        }
        block_reduce<4>(v, red, red_out);
        if (!grid_reduce<4>(a.gs, a.partials, red_out, res, a.status)) return;
    }
    rnorm0 = sqrt(res[1]);
    dp = sqrt(res[2]);
    rz = res[3];
    if (rnorm0 == 0.0) rnorm0 = dp;
    ttol = fmax(a.rtol * rnorm0, a.abstol);

    for (int sweep = 0;; ++sweep) {
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
        // ---- FP32 PCG on A e = r.  Each sweep reduces the FP64 residual by at most
        // ~1e-5 (the FP32 operator's own rounding), so the inner target is not set
        // below that; the next sweep takes the rest.
        const double target = fmin(0.5, fmax(3e-5, 0.1 * ttol / dp));
        const double dp_in0 = dp;
        double beta = rz, betaold = 0.0;
        int it = 0;
        bool inner_done = false;
        for (; it < a.maxit && !inner_done; ++it) {
            if (beta == 0.0) break;
            const float bc = it == 0 ? 0.0f : (float)(beta / betaold);
            const bool first = it == 0;
            {
                double v[1] = {0};
                for (int i = t0; i < n; i += stride) {
                    const int c = class_of<SLAB>(a, i);
                    const float az = apply_row32<SLAB, NOFF>(a, s32, soff, c, i, z32);
                    const float qi = first ? az : az + bc * q32[i];
                    const float pi = first ? z32[i] : z32[i] + bc * p32[i];
                    q32[i] = qi;
                    p32[i] = pi;
                    v[0] += (double)pi * (double)qi;
                }
                block_reduce<1>(v, red, red_out);
                if (!grid_reduce<1>(a.gs, a.partials, red_out, res, a.status)) return;
            }
            const double dpi = res[0];
            if (!(dpi > 0.0)) break;   // the FP64 residual update decides what happens next
            const float alpha = (float)(beta / dpi);
            {
                double v[2] = {0, 0};
                for (int i = t0; i < n; i += stride) {
                    const int c = class_of<SLAB>(a, i);
                    e32[i] = first ? alpha * p32[i] : e32[i] + alpha * p32[i];
                    const float rr = r32[i] - alpha * q32[i];
                    r32[i] = rr;
                    const float zz = dinv32_of<SLAB>(a, s32, c, i) * rr;
                    z32[i] = zz;
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
        }
        total_its += it;
        if (it == 0) {
            // nothing was added to e: stop rather than loop
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
            return cg_finish(a, step, total_its, kStatusCgDiverged);
        }
        // ---- refinement in FP64: x += e, r -= A e (e of the neighbours is complete)
        {
            double v[2] = {0, 0};
            for (int i = t0; i < n; i += stride) {
                const int c = class_of<SLAB>(a, i);
                const double ae = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, e32);
                x[i] += (double)e32[i];
                const double rr = r[i] - ae;
                r[i] = rr;
                const double zz = dinv_of<SLAB>(a, sh, c, i) * rr;
                const float rf = (float)rr;
                const float zf = dinv32_of<SLAB>(a, s32, c, i) * rf;
                r32[i] = rf;
                z32[i] = zf;
                v[0] += zz * zz;
                v[1] += (double)rf * (double)zf;
            }
            block_reduce<2>(v, red, red_out);
            if (!grid_reduce<2>(a.gs, a.partials, red_out, res, a.status)) return;
        }
        dp = sqrt(res[0]);
        rz = res[1];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
    cg_finish(a, step, total_its, 0);
}

}  // namespace chb
