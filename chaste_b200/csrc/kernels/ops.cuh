// Sparse operators of the diffusion solve: the assembled CSR (any mesh) and the
// matrix-free slab stencil (ConstructRegularSlabMesh meshes with uniform sigma).
#pragma once

#include "common.cuh"

namespace chb {

constexpr int kMaxOffsets = 27;
constexpr int kMaxClasses = 27;

// Matrix-free operator of a regular slab: the row of node i is the row of its
// boundary class (3 per axis; x2 for the stagger parity in 2D) in a small
// coefficient table, so a product streams only the vector and a 1-byte class
// per node.  Offsets are in ascending column order, the order a sorted CSR row
// sums in.  Vectors read through the stencil carry a zero halo of `halo`
// entries on both sides, so every i + off[o] of a node i is a valid address and
// the row needs no bounds test (outside neighbours have coefficient 0).
struct SlabOp {
    int n_off, n_cls;
    int interior;          // the most frequent class
    int off[kMaxOffsets];
    // the interior class row, passed by value so unrolled loops read it as
    // constant-bank operands (no registers, no shared-memory loads)
    double ia[kMaxOffsets];
    double im[kMaxOffsets];
    float ia32[kMaxOffsets];
    const double* a_tab;   // [cls][off]
    const double* m_tab;
    const float* a_tab32;
    const float* m_tab32;
};

// Shared-memory copy of the slab tables, filled at kernel start.
template <typename T>
struct SlabShared {
    T a[kMaxClasses * kMaxOffsets];
    T m[kMaxClasses * kMaxOffsets];
    T dinv[kMaxClasses];
};

template <typename T>
__device__ void slab_load_shared(const SlabOp& op, SlabShared<T>& sh, int diag_slot) {
    const T* at;
    const T* mt;
    if constexpr (sizeof(T) == 8) {
        at = reinterpret_cast<const T*>(op.a_tab);
        mt = reinterpret_cast<const T*>(op.m_tab);
    } else {
        at = reinterpret_cast<const T*>(op.a_tab32);
        mt = reinterpret_cast<const T*>(op.m_tab32);
    }
    const int tot = op.n_cls * op.n_off;
    for (int k = threadIdx.x; k < tot; k += blockDim.x) {
        sh.a[k] = at[k];
        sh.m[k] = mt[k];
    }
    __syncthreads();
    for (int c = threadIdx.x; c < op.n_cls; c += blockDim.x) {
        const T d = sh.a[c * op.n_off + diag_slot];
        sh.dinv[c] = d != T(0) ? T(1) / d : T(0);
    }
    __syncthreads();
}

// sum_o coef[o] * x[i + off[o]]; NOFF > 0 unrolls a fixed offset count, 0 loops n_off.
// x is not declared __restrict__: the persistent solves apply the operator to vectors
// that other blocks of the same launch write between grid reductions, so its loads must
// be ordinary coherent loads (ordered by the reductions' acquire), never the read-only
// path a restrict-qualified const pointer allows the compiler to choose.
template <int NOFF, typename T, typename Acc, typename X>
__device__ __forceinline__ Acc slab_row(const T* coef, const int* __restrict__ off, int n_off, int i,
                                        const X* x) {
    Acc acc = Acc(0);
    if constexpr (NOFF > 0) {
#pragma unroll
        for (int o = 0; o < NOFF; ++o) acc += (Acc)coef[o] * (Acc)x[i + off[o]];
    } else {
        for (int o = 0; o < n_off; ++o) acc += (Acc)coef[o] * (Acc)x[i + off[o]];
    }
    return acc;
}

// Assembled operator: A and M share one sorted CSR pattern.
struct CsrOp {
    const int* __restrict__ rowptr;
    const int* __restrict__ cols;
    const double* __restrict__ a;
    const double* __restrict__ m;
    const double* __restrict__ dinv;     // 1 / diag(A)
    const float* __restrict__ a32;
    const float* __restrict__ dinv32;
};

template <typename T, typename Acc, typename X>
__device__ __forceinline__ Acc csr_row(const int* __restrict__ rp, const int* __restrict__ ci,
                                       const T* __restrict__ v, int i, const X* x) {
    Acc acc = Acc(0);
    const int e = rp[i + 1];
    for (int k = rp[i]; k < e; ++k) acc += (Acc)v[k] * (Acc)x[ci[k]];
    return acc;
}

}  // namespace chb
