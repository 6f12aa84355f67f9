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
    // Packed rows for the one-block solve with its vectors in shared memory (cg_ilu_smem_kernel):
    // position k of the forward (backward) level order holds row fk_row[k] (bk_row[k]), its
    // count of entries left (right) of the diagonal and those entries' columns and factors in
    // ascending column order, pack_e slots per position (4 or kIluPackE); bk_dg: the row's
    // diagonal factor.
    const int* fk_cnt;
    const int* fk_col;
    const double* fk_val;
    const int* bk_cnt;
    const int* bk_col;
    const double* bk_val;
    const double* bk_dg;
    int pack_e;
    int f_warps, b_warps;    // warps covering the widest forward / backward level
};

// Entries per row of the packed triangular factors (2D meshes of triangles have 3 on either
// side of the diagonal, the Kuhn tetrahedra 7).
constexpr int kIluPackE = 8;

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

// ---------------------------------------------------------------------------
// Small meshes (at most kIluSmemNodes nodes): one block of kIluSmemThreads threads whose
// triangular solves run in place on vectors held in shared memory.  Per level a thread
// takes position ptr[l] + t (levels of at most kIluSmemThreads rows); the packed rows of
// the next levels (row, columns, factors, diagonal) are loaded while this level computes,
// so after each block barrier only shared-memory reads remain on the critical path.
// The rows, their entry order and the arithmetic of each row are those of
// cg_ilu_kernel; the inner products are summed over the nodes in natural order after the
// sweeps instead of in level order.
constexpr int kIluSmemThreads = 512;
constexpr int kIluSmemNodes = 12800;
constexpr int kIluSmemLevels = 2048;

// E: entries per packed row (the slot stride of the packed arrays, 4 or kIluPackE).
template <int E>
struct PackedRow {
    int i;   // -1: no row
    int cnt;
    int col[E];
    double val[E];
    double dg;
};

template <int E>
__device__ __forceinline__ void load_packed_row(PackedRow<E>& r, int k, int end, const int* rows, const int* cnt,
                                                const int* col, const double* val, const double* dg) {
    if (k >= end) {
        r.i = -1;
        r.cnt = 0;
        r.dg = 1.0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            r.col[e] = 0;
            r.val[e] = 0.0;
        }
        return;
    }
    r.i = rows[k];
    r.cnt = cnt[k];
    r.dg = dg ? dg[k] : 1.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        r.col[e] = col[(size_t)k * E + e];
        r.val[e] = val[(size_t)k * E + e];
    }
}

template <int NV, bool BACK, int E>
__device__ __forceinline__ void packed_levels(const int* lptr, int levels, const int* rows, const int* cnt,
                                              const int* col, const double* val, const double* dg, double* z0,
                                              double* z1, int nthreads) {
    // rows loaded AHEAD levels ahead (two for the narrow rows of 2D meshes; one for the
    // 3D rows, whose registers would otherwise spill)
    constexpr int AHEAD = E <= 4 ? 2 : 1;
    const int t = threadIdx.x;
    PackedRow<E> cur, nx1, nx2;
    nx1.i = nx2.i = -1;
    nx1.cnt = nx2.cnt = 0;
    load_packed_row(cur, lptr[0] + t, lptr[1], rows, cnt, col, val, dg);
    if (AHEAD == 2 && levels > 1) load_packed_row(nx1, lptr[1] + t, lptr[2], rows, cnt, col, val, dg);
    for (int l = 0; l < levels; ++l) {
        if (l + AHEAD < levels)
            load_packed_row(AHEAD == 2 ? nx2 : nx1, lptr[l + AHEAD] + t, lptr[l + AHEAD + 1], rows, cnt, col, val,
                            dg);
        if (cur.i >= 0) {
            double s0 = z0[cur.i], s1 = NV > 1 ? z1[cur.i] : 0.0;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (e < cur.cnt) {
                    s0 -= cur.val[e] * z0[cur.col[e]];
                    if (NV > 1) s1 -= cur.val[e] * z1[cur.col[e]];
                }
            }
            if (BACK) {
                s0 = s0 / cur.dg;
                if (NV > 1) s1 = s1 / cur.dg;
            }
            z0[cur.i] = s0;
            if (NV > 1) z1[cur.i] = s1;
        }
        asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
        cur = nx1;
        if (AHEAD == 2) nx1 = nx2;
    }
}

// In-place triangular solve of NV shared-memory vectors (z1 ignored when NV == 1).  Only
// the first `warps` warps (those the widest level needs) take part, synchronising the
// levels on named barrier 1 among themselves; the block meets again at the end.
template <int NV, bool BACK, int E>
__device__ __forceinline__ void packed_sweep(const int* lptr, int levels, const int* rows, const int* cnt,
                                             const int* col, const double* val, const double* dg, double* z0,
                                             double* z1, int warps) {
    if ((int)(threadIdx.x >> 5) < warps) packed_levels<NV, BACK, E>(lptr, levels, rows, cnt, col, val, dg, z0, z1,
                                                                     warps * 32);
    __syncthreads();
}

// The solve of cg_ilu_kernel_body on one block with B r in shared memory (z0) and, in
// phase 0, B b beside it (z1); the level pointers are copied to shared memory first.
template <int E>
__device__ void cg_ilu_smem_body(const CgArgs& a, const IluArgs& f, unsigned& round) {
    __shared__ double red[32 * 4];
    extern __shared__ double dyn[];
    const int n = a.n;
    double* z0 = dyn;
    double* z1 = dyn + n;
    int* fptr = reinterpret_cast<int*>(dyn + 2 * (size_t)n);
    int* bptr = fptr + (f.f_levels + 1);
    for (int l = threadIdx.x; l <= f.f_levels; l += blockDim.x) fptr[l] = f.f_ptr[l];
    for (int l = threadIdx.x; l <= f.b_levels; l += blockDim.x) bptr[l] = f.b_ptr[l];
    if (*(volatile int*)a.status & ~kStatusStateRange) return;
    const long long step = *a.step;
    const int t0 = threadIdx.x, stride = blockDim.x;
    double* __restrict__ x = a.x;
    double* __restrict__ r = a.r;
    double* __restrict__ q = a.q;
    double* __restrict__ p = a.p0;
    double res[4];

    // ---- b = M z (+ correction), r = b - A x; the sweeps' right-hand sides r and b
    double babs = 0.0;
    for (int i = t0; i < n; i += stride) {
        const double b = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.m, i, a.zrhs) +
                         (a.corr ? a.corr[i] : 0.0);
        const double av = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.a, i, x);
        const double rr = b - av;
        f.bvec[i] = b;
        r[i] = rr;
        z0[i] = rr;
        z1[i] = b;
        babs += fabs(b);
    }
    __syncthreads();
    packed_sweep<2, false, E>(fptr, f.f_levels, f.f_rows, f.fk_cnt, f.fk_col, f.fk_val, nullptr, z0, z1, f.f_warps);
    packed_sweep<2, true, E>(bptr, f.b_levels, f.b_rows, f.bk_cnt, f.bk_col, f.bk_val, f.bk_dg, z0, z1, f.b_warps);
    double v[4] = {babs, 0.0, 0.0, 0.0};
    for (int i = t0; i < n; i += stride) {
        const double zz = z0[i], ww = z1[i];
        v[1] += ww * ww;
        v[2] += zz * zz;
        v[3] += r[i] * zz;
    }
    block_reduce<4>(v, red, res, round);
    double rnorm0 = sqrt(res[1]);
    double dp = sqrt(res[2]);
    double beta = res[3];
    if (res[0] < 1e-15 && res[0] > 0.0) {
        // LinearSystem.cpp:984-994: tiny RHS -> zero initial guess, r = b, B r = B b
        double v2[2] = {0, 0};
        for (int i = t0; i < n; i += stride) {
            const double b = f.bvec[i], zz = z1[i];
            x[i] = 0.0;
            r[i] = b;
            z0[i] = zz;
            v2[0] += zz * zz;
            v2[1] += b * zz;
        }
        double o2[2];
        block_reduce<2>(v2, red, o2, round);
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
                const double az = csr_row<double, double>(a.csr.rowptr, a.csr.cols, a.csr.a, i, z0);
                const double qi = first ? az : az + bc * q[i];
                const double pi = first ? z0[i] : z0[i] + bc * p[i];
                q[i] = qi;
                p[i] = pi;
                v1[0] += pi * qi;
            }
            block_reduce<1>(v1, red, res, round);
        }
        const double dpi = res[0];
        if (!(dpi > 0.0)) return cg_finish(a, step, it + 1, isfinite(dpi) ? kStatusCgDiverged : kStatusNaN);
        const double alpha = beta / dpi;
        // ---- x += alpha p, r -= alpha A p; then z = B r in place
        for (int i = t0; i < n; i += stride) {
            x[i] += alpha * p[i];
            const double rr = r[i] - alpha * q[i];
            r[i] = rr;
            z0[i] = rr;
        }
        __syncthreads();
        packed_sweep<1, false, E>(fptr, f.f_levels, f.f_rows, f.fk_cnt, f.fk_col, f.fk_val, nullptr, z0, nullptr, f.f_warps);
        packed_sweep<1, true, E>(bptr, f.b_levels, f.b_rows, f.bk_cnt, f.bk_col, f.bk_val, f.bk_dg, z0, nullptr, f.b_warps);
        double v2[2] = {0, 0};
        for (int i = t0; i < n; i += stride) {
            const double zz = z0[i];
            v2[0] += zz * zz;
            v2[1] += zz * r[i];
        }
        block_reduce<2>(v2, red, res, round);
        dp = sqrt(res[0]);
        if (!isfinite(dp)) return cg_finish(a, step, it + 1, kStatusNaN);
        if (dp <= ttol) return cg_finish(a, step, it + 1, 0);
        if (dp >= a.dtol * rnorm0) return cg_finish(a, step, it + 1, kStatusCgDiverged);
        betaold = beta;
        beta = res[1];
    }
    cg_finish(a, step, it, kStatusCgMaxIt);
}

template <int E>
__global__ void __launch_bounds__(kIluSmemThreads, 1) cg_ilu_smem_kernel(CgArgs a, IluArgs f) {
    unsigned round = 0;
    cg_ilu_smem_body<E>(a, f, round);
    grid_exit(a.gs);
}

}  // namespace chb
