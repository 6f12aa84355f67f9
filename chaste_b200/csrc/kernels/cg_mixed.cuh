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

// Target of one FP32 inner solve: reduce the residual by max(kInnerFloor,
// kInnerFactor * ttol / ||B r||).  The FP32 operator's rounding stalls the true
// residual near a 1e-5 relative reduction, so a sweep does not aim below that,
// and the last sweep aims just under the FP64 tolerance (the FP64 test decides
// convergence either way).  Measured on the 442,401-node TT06 slab: (1e-5, 0.8)
// took 19.7 inner iterations per solve against 22.4 for (3e-5, 0.1), both in 2
// sweeps, at the same 0.004 mV difference from the FP64 solve.
// The pipelined solve runs one block of 1024 threads per SM when the slab fills every
// SM with such blocks: the same threads (and registers) as two blocks of 512, with
// half the arrivals and partial sums per grid reduction (measured 2.6 us per
// reduction against 2.9 us for 296 x 512).  Smaller slabs use blocks of 512.
constexpr int kPipeThreads = 1024;

constexpr double kInnerFloor = 1e-5;
constexpr double kInnerFactor = 0.8;

template <bool SLAB>
__device__ __forceinline__ float dinv32_of(const CgArgs& a, const SlabShared<float>& s32, int c, int i) {
    if (a.pc == 0) return 1.0f;
    if constexpr (SLAB) return s32.dinv[c];
    else return a.csr.dinv32[i];
}

template <bool SLAB, int NOFF>
__device__ __forceinline__ float apply_row32(const CgArgs& a, const SlabShared<float>& s32, const int* soff,
                                             int c, int i, const float* x) {
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

// Inner preconditioner of the mixed solve on the slab stencil: T^-1 d, where T is the
// tridiagonal part of A along x (the direction of the largest conductivity)
// restricted to the 32 consecutive nodes a warp holds (rows cut at the warp's ends
// and, through the stencil, at the ends of each x-line).  T is a principal
// block-diagonal part of the SPD matrix A, so it is SPD.
//
// T = L D L^T with L unit lower bidiagonal (l_i = T_{i,i-1} / d_{i-1},
// d_i = T_ii - l_i T_{i,i-1}), so T^-1 = F^T D^-1 F with F = L^-1.  F applies the
// recurrence y_i = v_i + a_i y_{i-1} (a_i = -l_i, a_0 = 0) as a Hillis-Steele scan
// over the warp: five levels s = 1, 2, 4, 8, 16 of y_i += A^(s)_i y_{i-s}, where
// A^(s)_i is the product of the s coefficients a_{i-s+1..i} (zero for i < s, since
// a_0 = 0).  The application is B d = F^T (D^-1 (F d)): the scan, a scaling, then the
// transposed levels in reverse order (z_i += A^(s)_{i+s} z_{i+s}).  B is therefore
// symmetric for the stored coefficients whatever their rounding, and positive
// definite while every d_i > 0: a fixed SPD operator, as CG needs.  The pivots depend
// on A only: the host computes (a_i, 1/d_i) per node once, in FP64 rounded to FP32
// (CgArgs::line_ad, segments of 32 nodes aligned on multiples of 32, which are the
// nodes one warp holds in one register slot or grid-stride step).  A solve forms the
// five A^(s) from a_i by four shuffle levels (warp_line_levels); an application is
// then 10 shuffles and 11 multiply-adds.  Every lane of the warp takes part; the rows
// of nodes past n are the identity (a = 0, 1/d = 1).
constexpr int kLineCoef = 6;   // A^(1), A^(2), A^(4), A^(8), A^(16), 1 / d

__device__ __forceinline__ void warp_line_levels(float a, float (&A)[5]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    A[0] = lane >= 1 ? a : 0.0f;   // nothing before lane 0 within the warp
#pragma unroll
    for (int j = 1; j < 5; ++j) {
        const int s = 1 << (j - 1);
        const float Am = __shfl_up_sync(full, A[j - 1], s);
        A[j] = lane >= s ? A[j - 1] * Am : 0.0f;
    }
}

__device__ __forceinline__ float warp_line_solve(const float (&A)[5], float dinv, float v) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // y = F v
#pragma unroll
    for (int j = 0; j < 5; ++j) v += A[j] * __shfl_up_sync(full, v, 1 << j);
    // z = F^T D^-1 y
    float z = v * dinv;
#pragma unroll
    for (int j = 4; j >= 0; --j) {
        const int s = 1 << j;
        const float t = __shfl_down_sync(full, A[j] * z, s);
        if (lane + s < 32) z += t;
    }
    return z;
}

// Per-slot factors kept in shared memory by the pipelined solve.
__device__ __forceinline__ void warp_line_setup(float2 ad, float* cf, int ld) {
    float A[5];
    warp_line_levels(ad.x, A);
#pragma unroll
    for (int j = 0; j < 5; ++j) cf[j * ld] = A[j];
    cf[5 * ld] = ad.y;
}

__device__ __forceinline__ float warp_line_apply(const float* cf, int ld, float v) {
    float A[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) A[j] = cf[j * ld];
    return warp_line_solve(A, cf[5 * ld], v);
}

// (a_i, 1/d_i) of node i, identity for nodes past n.
__device__ __forceinline__ float2 line_factors(const CgArgs& a, bool on, int i) {
    return on ? __ldg(a.line_ad + i) : make_float2(0.0f, 1.0f);
}

// y = B x with the x-line inner preconditioner alone (cg_apply_inner_preconditioner):
// the same segments and factors the mixed solves use.
static __global__ void line_pc_apply_kernel(int n, const float2* __restrict__ ad, const float* __restrict__ x,
                                     float* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + threadIdx.x - lane; base < n; base += stride) {
        const int i = base + lane;
        const bool on = i < n;
        const float2 f = on ? ad[i] : make_float2(0.0f, 1.0f);
        float A[5];
        warp_line_levels(f.x, A);
        const float z = warp_line_solve(A, f.y, on ? x[i] : 0.0f);
        if (on) y[i] = z;
    }
}

// The inner preconditioner of this kernel at node i (warp-synchronous: every lane of
// the warp calls it, `on` false past n): the x-line solve on slab stencils when
// a.line_pc is set, else Jacobi.
template <bool SLAB>
__device__ __forceinline__ float inner_pc32(const CgArgs& a, const SlabShared<float>& s32, int c, int i, bool on,
                                            float r) {
    if constexpr (SLAB) {
        if (a.line_pc) {
            float A[5];
            const float2 ad = line_factors(a, on, i);
            warp_line_levels(ad.x, A);
            return warp_line_solve(A, ad.y, on ? r : 0.0f);
        }
    }
    return on ? dinv32_of<SLAB>(a, s32, c, i) * r : 0.0f;
}

// The same in two parts, so a loop can load the x-line factors together with its
// other operands: inner_pc_factors (a load, or the identity when there is no line
// solve), then inner_pc32_with.
template <bool SLAB>
__device__ __forceinline__ float2 inner_pc_factors(const CgArgs& a, bool on, int i) {
    if constexpr (SLAB) {
        if (a.line_pc) return line_factors(a, on, i);
    }
    return make_float2(0.0f, 1.0f);
}

template <bool SLAB>
__device__ __forceinline__ float inner_pc32_with(const CgArgs& a, const SlabShared<float>& s32, int c, int i,
                                                 bool on, float r, float2 ad) {
    if constexpr (SLAB) {
        if (a.line_pc) {
            float A[5];
            warp_line_levels(ad.x, A);
            return warp_line_solve(A, ad.y, on ? r : 0.0f);
        }
    }
    return on ? dinv32_of<SLAB>(a, s32, c, i) * r : 0.0f;
}

// Grid-stride steps of the HBM-resident inner loops taken per loop trip (loads of all
// of them issued before the first store).
constexpr int kInnerUnroll = 2;
constexpr int kStencilUnroll = 1;

template <bool SLAB, int NOFF>
__device__ __forceinline__ void cg_mixed_kernel_body(const CgArgs& a, unsigned& round) {
    __shared__ SlabShared<double> sh;
    __shared__ SlabShared<float> s32;
    __shared__ int soff[kMaxOffsets];
    __shared__ double red[32 * 4];
    if constexpr (SLAB) {
        for (int k = threadIdx.x; k < a.slab.n_off; k += blockDim.x) soff[k] = a.slab.off[k];
        slab_load_shared<double>(a.slab, sh, a.diag_slot);
        slab_load_shared<float>(a.slab, s32, a.diag_slot);
    }
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    // warp-uniform grid-stride loops: a warp visits the 32 consecutive nodes
    // base .. base + 31 together (the x-line preconditioner's segment)
    const int lane = threadIdx.x & 31;
    const int w0 = blockIdx.x * blockDim.x + threadIdx.x - lane;
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
        for (int base = w0; base < n; base += stride) {
            const int i = base + lane;
            const bool on = i < n;
            const int c = on ? class_of<SLAB>(a, i) : 0;
            float rf = 0.0f;
            if (on) {
                const double b =
                    apply_row<SLAB, NOFF, true>(a, sh, soff, c, i, a.zrhs32) + (a.corr ? a.corr[i] : 0.0);
                const double av = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, x);
                const double rr = b - av;
                const double d = dinv_of<SLAB>(a, sh, c, i);
                const double w = d * b, zz = d * rr;
                v[0] += fabs(b);
                v[1] += w * w;
                v[2] += zz * zz;
                rf = (float)rr;
                r[i] = rr;
                r32[i] = rf;
            }
            const float zf = inner_pc32<SLAB>(a, s32, c, i, on, rf);
            if (on) z32[i] = zf;
            v[3] += (double)rf * (double)zf;
        }
        if (!grid_reduce<4>(v, red, a.gs, a.partials, res, a.status, round)) return;
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
        const double target = fmin(0.5, fmax(kInnerFloor, kInnerFactor * ttol / dp));
        const double dp_in0 = dp;
        double beta = rz, betaold = 0.0;
        int it = 0;
        bool inner_done = false;
        for (; it < a.maxit && !inner_done; ++it) {
            if (beta == 0.0) break;
            const float bc = it == 0 ? 0.0f : (float)(beta / betaold);
            const bool first = it == 0;
            {
                // kInnerUnroll grid-stride steps per loop trip: every load of the group
                // is issued before any store, so their latencies overlap (the nodes and
                // the order of the sums are those of the plain grid-stride loop)
                double v[1] = {0};
                for (int base = w0; base < n; base += kStencilUnroll * stride) {
                    float az[kStencilUnroll], zo[kStencilUnroll], qo[kStencilUnroll], po[kStencilUnroll];
#pragma unroll
                    for (int u = 0; u < kStencilUnroll; ++u) {
                        const int i = base + u * stride + lane;
                        az[u] = zo[u] = qo[u] = po[u] = 0.0f;
                        if (i < n) {
                            const int c = class_of<SLAB>(a, i);
                            az[u] = apply_row32<SLAB, NOFF>(a, s32, soff, c, i, z32);
                            zo[u] = z32[i];
                            if (!first) {
                                qo[u] = q32[i];
                                po[u] = p32[i];
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kStencilUnroll; ++u) {
                        const int i = base + u * stride + lane;
                        if (i >= n) continue;
                        const float qi = first ? az[u] : az[u] + bc * qo[u];
                        const float pi = first ? zo[u] : zo[u] + bc * po[u];
                        q32[i] = qi;
                        p32[i] = pi;
                        v[0] += (double)pi * (double)qi;
                    }
                }
                if (!grid_reduce<1>(v, red, a.gs, a.partials, res, a.status, round)) return;
            }
            const double dpi = res[0];
            if (!(dpi > 0.0)) break;   // the FP64 residual update decides what happens next
            const float alpha = (float)(beta / dpi);
            {
                double v[2] = {0, 0};
                for (int base = w0; base < n; base += kInnerUnroll * stride) {
                    float pv[kInnerUnroll], qv[kInnerUnroll], rv[kInnerUnroll], eo[kInnerUnroll];
                    int cl[kInnerUnroll];
                    float2 ad[kInnerUnroll];
#pragma unroll
                    for (int u = 0; u < kInnerUnroll; ++u) {
                        const int i = base + u * stride + lane;
                        const bool on = i < n;
                        pv[u] = qv[u] = rv[u] = eo[u] = 0.0f;
                        cl[u] = on ? class_of<SLAB>(a, i) : 0;
                        ad[u] = inner_pc_factors<SLAB>(a, on, i);
                        if (on) {
                            pv[u] = p32[i];
                            qv[u] = q32[i];
                            rv[u] = r32[i];
                            if (!first) eo[u] = e32[i];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kInnerUnroll; ++u) {
                        const int i = base + u * stride + lane;
                        const bool on = i < n;
                        float rr = 0.0f;
                        if (on) {
                            e32[i] = first ? alpha * pv[u] : eo[u] + alpha * pv[u];
                            rr = rv[u] - alpha * qv[u];
                            r32[i] = rr;
                        }
                        const float zz = inner_pc32_with<SLAB>(a, s32, cl[u], i, on, rr, ad[u]);
                        if (on) z32[i] = zz;
                        v[0] += (double)zz * (double)zz;
                        v[1] += (double)zz * (double)rr;
                    }
                }
                if (!grid_reduce<2>(v, red, a.gs, a.partials, res, a.status, round)) return;
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
            for (int base = w0; base < n; base += stride) {
                const int i = base + lane;
                const bool on = i < n;
                const int c = on ? class_of<SLAB>(a, i) : 0;
                float rf = 0.0f;
                if (on) {
                    const double ae = apply_row<SLAB, NOFF, false>(a, sh, soff, c, i, e32);
                    x[i] += (double)e32[i];
                    const double rr = r[i] - ae;
                    r[i] = rr;
                    const double zz = dinv_of<SLAB>(a, sh, c, i) * rr;
                    rf = (float)rr;
                    r32[i] = rf;
                    v[0] += zz * zz;
                }
                const float zf = inner_pc32<SLAB>(a, s32, c, i, on, rf);
                if (on) z32[i] = zf;
                v[1] += (double)rf * (double)zf;
            }
            if (!grid_reduce<2>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        dp = sqrt(res[0]);
        rz = res[1];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
    cg_finish(a, step, total_its, 0);
}

template <bool SLAB, int NOFF>
__global__ void __launch_bounds__(512, 2) cg_mixed_kernel(CgArgs a) {
    unsigned round = 0;
    cg_mixed_kernel_body<SLAB, NOFF>(a, round);
    grid_exit(a.gs);
}

// ---------------------------------------------------------------------------
// Slab-stencil variant with a pipelined inner solve (Ghysels & Vanroose,
// "Hiding global synchronization latency in the preconditioned Conjugate
// Gradient algorithm", Parallel Computing 40, 2014): the two inner products of
// an iteration, (r,u) and (w,u), are reduced together, and the vector the next
// operator application needs, m = B w, is published before that one grid-wide
// reduction, which therefore doubles as the halo barrier.  m alternates
// between two haloed buffers, so a block may publish iteration i+1 while its
// neighbours still read iteration i.  Every thread keeps the inner vectors of
// its KMAX nodes (t0 + k * stride) in registers; only m and, at the end of a
// sweep, the correction e go through memory.  One grid-wide synchronisation
// per inner iteration instead of two.
//
// The FP64 residual passes and the outer stopping test are those of
// cg_mixed_kernel; the inner iteration stops on the preconditioned norm
// sqrt((r, B r)) reaching `target` of its start value.
// Stencil row over a vector that other blocks of this launch have written: the
// loads go to L2 (ld.global.cg), never to a possibly stale L1 or read-only line.
template <int NOFF, typename Acc, typename T, typename X>
__device__ __forceinline__ Acc slab_row_l2(const T* coef, const int* off, int i, const X* x) {
    Acc acc = Acc(0);
#pragma unroll
    for (int o = 0; o < NOFF; ++o) acc += (Acc)coef[o] * (Acc)__ldcg(x + i + off[o]);
    return acc;
}

template <int NOFF>
__device__ __forceinline__ float apply_a32_l2(const CgArgs& a, const SlabShared<float>& s32, int c, int i,
                                              const float* x) {
    if (c == a.slab.interior) return slab_row_l2<NOFF, float>(a.slab.ia32, a.slab.off, i, x);
    return slab_row_l2<NOFF, float>(&s32.a[c * NOFF], a.slab.off, i, x);
}

template <int NOFF>
__device__ __forceinline__ double apply_a64_l2(const CgArgs& a, const SlabShared<double>& sh, int c, int i,
                                               const float* x) {
    if (c == a.slab.interior) return slab_row_l2<NOFF, double>(a.slab.ia, a.slab.off, i, x);
    return slab_row_l2<NOFF, double>(&sh.a[c * NOFF], a.slab.off, i, x);
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Every thread of the block copies its share of the band windows of x (a haloed
// vector that other blocks published before the grid reduction this block has just
// passed) from L2 to the block's stage with 16-byte cp.async (.cg: through L2, no
// registers held), so the copies are in flight while the updates that do not need
// A m run; stage_windows_wait then completes them and the block barrier makes them
// visible.  The windows start 16-byte aligned (plan_stage rounds each band's start
// down to 4 floats) and the stage holds, for register slot k and band b,
// stage[k * cap + base[b] ..] = x[window start ..].  Measured on the 442,401-node slab against one
// thread issuing 1D TMA bulk copies on an mbarrier (which needs proxy fences on its
// critical path): 0.169 vs 0.176 ms per solve.
template <int KMAX>
__device__ __forceinline__ void stage_windows_start(const CgArgs& a, const float* x, float* stage) {
    const StageArgs& g = a.stage;
    const float* xa = x - g.halo;   // allocation start, 256-byte aligned
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cap4 = g.cap / 4;
    const int total4 = KMAX * cap4;
    for (int f4 = threadIdx.x; f4 < total4; f4 += blockDim.x) {
        const int k = f4 / cap4, rem = f4 - k * cap4;
        int b = 0;
        while (b + 1 < g.n_bands && rem * 4 >= g.base[b + 1]) ++b;
        const long long gb = (long long)blockIdx.x * blockDim.x + k * stride;
        const int delta = (g.lo[b] + g.halo) & 3;
        const long long src = gb + g.lo[b] + g.halo - delta + (4LL * rem - g.base[b]);
        if (gb < a.n && src + 4 <= g.alloc_len)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(stage + 4 * f4)), "l"(xa + src)
                         : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void stage_windows_wait() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
}

template <int NOFF>
__device__ __forceinline__ float apply_a32_staged(const CgArgs& a, const SlabShared<float>& s32, int c,
                                                  const float* st) {
    float acc = 0.0f;
    if (c == a.slab.interior) {
#pragma unroll
        for (int o = 0; o < NOFF; ++o) acc += a.slab.ia32[o] * st[a.stage.rel[o]];
    } else {
        const float* coef = &s32.a[c * NOFF];
#pragma unroll
        for (int o = 0; o < NOFF; ++o) acc += coef[o] * st[a.stage.rel[o]];
    }
    return acc;
}

// B d for register slot k: the x-line solve (a.line_pc) or Jacobi.
__device__ __forceinline__ float apply_inner_pc(const CgArgs& a, const float* cf, int ld, bool on, float dinv,
                                                float d) {
    if (!a.line_pc) return dinv * d;
    return warp_line_apply(cf, ld, on ? d : 0.0f);
}

template <int NOFF, int KMAX>
__device__ __forceinline__ void cg_mixed_pipe_kernel_body(const CgArgs& a, unsigned& round) {
    __shared__ SlabShared<double> sh;
    __shared__ SlabShared<float> s32;
    __shared__ double red[32 * 4];
    extern __shared__ float4 stage4[];
    float* stage = reinterpret_cast<float*>(stage4);
    // x-line factors after the staged windows: slot k, word j of thread t at
    // line_cf[(k * kLineCoef + j) * blockDim.x + t]
    float* line_cf = stage + KMAX * a.stage.cap;
    const int ld = blockDim.x;
    slab_load_shared<double>(a.slab, sh, a.diag_slot);
    slab_load_shared<float>(a.slab, s32, a.diag_slot);
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int n = a.n;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double* __restrict__ x = a.x;
    double* __restrict__ r64 = a.r;
    float* z32 = a.z32;
    float* e32 = a.e32;
    int node[KMAX], cls[KMAX];
    float dinv[KMAX];
    bool on[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        node[k] = t0 + k * stride;
        on[k] = node[k] < n;
        cls[k] = on[k] ? (int)a.cls8[node[k]] : 0;
        dinv[k] = on[k] ? (a.pc ? s32.dinv[cls[k]] : 1.0f) : 0.0f;
    }
    if (a.line_pc) {
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
            warp_line_setup(line_factors(a, on[k], node[k]), line_cf + k * kLineCoef * ld + threadIdx.x, ld);
    }
    float r[KMAX], u[KMAX], w[KMAX], m[KMAX], zq[KMAX], q[KMAX], sv[KMAX], p[KMAX], e[KMAX];
    double res[4];

    // ---- FP64 residual r = M z - A x; its FP32 copy r and u = B r (published in z32)
    {
        double v[4] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            r[k] = 0.0f;
            if (on[k]) {
                const int i = node[k], c = cls[k];
                const double b =
                    apply_row<true, NOFF, true>(a, sh, nullptr, c, i, a.zrhs32) + (a.corr ? a.corr[i] : 0.0);
                const double av = apply_row<true, NOFF, false>(a, sh, nullptr, c, i, x);
                const double rr = b - av;
                const double d = dinv_of<true>(a, sh, c, i);
                const double wb = d * b, zz = d * rr;
                v[0] += fabs(b);
                v[1] += wb * wb;
                v[2] += zz * zz;
                r64[i] = rr;
                r[k] = (float)rr;
            }
            u[k] = apply_inner_pc(a, line_cf + k * kLineCoef * ld + threadIdx.x, ld, on[k], dinv[k], r[k]);
            if (on[k]) z32[node[k]] = u[k];
        }
        if (!grid_reduce<4>(v, red, a.gs, a.partials, res, a.status, round)) return;
    }
    double rnorm0 = sqrt(res[1]);
    double dp = sqrt(res[2]);
    if (rnorm0 == 0.0) rnorm0 = dp;
    const double ttol = fmax(a.rtol * rnorm0, a.abstol);
    int total_its = 0, sweeps = 0;

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
        const double target = fmin(0.5, fmax(kInnerFloor, kInnerFactor * ttol / dp));
        // w = A u (u was published before the last grid-wide reduction)
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            w[k] = on[k] ? apply_a32_l2<NOFF>(a, s32, cls[k], node[k], z32) : 0.0f;
            zq[k] = q[k] = sv[k] = p[k] = e[k] = 0.0f;
        }
        double gamma_old = 1.0, alpha_old = 1.0, g0 = 0.0;
        int it = 0;
        for (;; ++it) {
            float* mb = (it & 1) ? a.m32b : a.m32a;
            double v[2] = {0, 0};
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                v[0] += (double)r[k] * (double)u[k];
                v[1] += (double)w[k] * (double)u[k];
                m[k] = apply_inner_pc(a, line_cf + k * kLineCoef * ld + threadIdx.x, ld, on[k], dinv[k], w[k]);
                if (on[k]) mb[node[k]] = m[k];
            }
            if (!grid_reduce<2>(v, red, a.gs, a.partials, res, a.status, round)) return;
            const double gamma = res[0], delta = res[1];
            if (it == 0) g0 = gamma;
            if (!(gamma > 0.0) || !(gamma > target * target * g0) || it >= a.maxit) break;
            const double beta = it == 0 ? 0.0 : gamma / gamma_old;
            const double denom = it == 0 ? delta : delta - beta * gamma / alpha_old;
            if (!(denom > 0.0)) break;   // breakdown: the FP64 residual update decides what follows
            const double alpha = gamma / denom;
            const float af = (float)alpha, bf = (float)beta;
            stage_windows_start<KMAX>(a, mb, stage);
            // the updates that do not need A m run while the windows are in flight
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                q[k] = m[k] + bf * q[k];
                sv[k] = w[k] + bf * sv[k];
                p[k] = u[k] + bf * p[k];
                e[k] += af * p[k];
                r[k] -= af * sv[k];
                u[k] -= af * q[k];
                // published every iteration: the reduction that ends the sweep is then
                // also the barrier the FP64 refinement pass needs
                if (on[k]) e32[node[k]] = e[k];
            }
            stage_windows_wait();
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                const float nk =
                    on[k] ? apply_a32_staged<NOFF>(a, s32, cls[k], stage + k * a.stage.cap + threadIdx.x) : 0.0f;
                zq[k] = nk + bf * zq[k];
                w[k] -= af * zq[k];
            }
            gamma_old = gamma;
            alpha_old = alpha;
        }
        total_its += it;
        if (it == 0) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
            return cg_finish(a, step, total_its, kStatusCgDiverged);
        }
        // ---- x += e and r -= A e in FP64 (e of every node was published before the
        // reduction that ended the sweep)
        {
            double v[1] = {0};
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                r[k] = 0.0f;
                if (on[k]) {
                    const int i = node[k], c = cls[k];
                    const double ae = apply_a64_l2<NOFF>(a, sh, c, i, e32);
                    x[i] += (double)e[k];
                    const double rr = r64[i] - ae;
                    r64[i] = rr;
                    const double zz = dinv_of<true>(a, sh, c, i) * rr;
                    v[0] += zz * zz;
                    r[k] = (float)rr;
                }
                u[k] = apply_inner_pc(a, line_cf + k * kLineCoef * ld + threadIdx.x, ld, on[k], dinv[k], r[k]);
                if (on[k]) z32[node[k]] = u[k];
            }
            if (!grid_reduce<1>(v, red, a.gs, a.partials, res, a.status, round)) return;
        }
        dp = sqrt(res[0]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.refine_out = sweeps;
    cg_finish(a, step, total_its, 0);
}

template <int NOFF, int KMAX>
__global__ void __launch_bounds__(kPipeThreads, 1) cg_mixed_pipe_kernel(CgArgs a) {
    unsigned round = 0;
    cg_mixed_pipe_kernel_body<NOFF, KMAX>(a, round);
    grid_exit(a.gs);
}

}  // namespace chb
