// State-variable interpolation (SVI): the correction the monodomain RHS gets when
// the ionic current is evaluated at quadrature points from interpolated state
// variables instead of interpolated nodal currents --
// MonodomainCorrectionTermAssembler::ComputeVectorTerm
// (heart/src/solver/electrics/monodomain/MonodomainCorrectionTermAssembler.cpp:47-66)
// on the elements AbstractCorrectionTermAssembler::ElementAssemblyCriterion selects
// (heart/src/solver/electrics/AbstractCorrectionTermAssembler.cpp:109-146: largest
// |Iion_a - Iion_b| over the element's nodes above 1), with the order-2 Gaussian
// rule of AbstractFeVolumeIntegralAssembler (pde/src/solver/GaussianQuadratureRule.cpp).
//
// Two passes, both deterministic (no atomics):
//  svi_element_kernel -- one thread per element: the criterion, and for a selected
//    element its nodal contributions at every quadrature point q (one node has
//    basis value A, the others B):
//        be_j += phi_j(q) * (-Am) * (Iion(sum_k phi_k y_k) - sum_k phi_k Iion_k) * wJ_e
//    written to ebuf[4e + j] with flag[e] = 1 (flag[e] = 0 otherwise);
//  svi_gather_kernel -- one thread per node: the sum over its elements in ascending
//    element order, from a padded column-major (ELL) list of 4e + j entries.
#pragma once

#include "../models/lr91.h"
#include "../models/tt06.h"
#include "common.cuh"

namespace chb {

template <typename T>
struct SviArgs {
    int n, dim, n_elems;
    const double* __restrict__ V;        // V^n
    const T* __restrict__ states;        // (S-1) x n, after the ODE step
    const T* __restrict__ iion;          // nodal Iion cache
    const uint8_t* __restrict__ pset;    // may be null
    const T* __restrict__ params;
    const int* __restrict__ econn;       // n_elems x (dim+1)
    const double* __restrict__ ewj;      // |det J| x reference weight, per element
    uint8_t* __restrict__ flag;          // n_elems
    double* __restrict__ ebuf;           // 4 x n_elems
    const int* __restrict__ ell;         // width x n, entries 4e + j ascending in e, -1 padded
    int ell_width;
    double* __restrict__ corr;           // n
    double am, cm;
    double qa, qb;                       // basis values at a quadrature point: its node, the others
    int big[4];                          // node of each quadrature point with basis value qa
};

template <class M, typename T>
__global__ void __launch_bounds__(256) svi_element_kernel(SviArgs<T> a) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const int nb = a.dim + 1;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < a.n_elems; e += gridDim.x * blockDim.x) {
        int nd[4];
        T ion[4];
        for (int j = 0; j < nb; ++j) {
            nd[j] = a.econn[(size_t)e * nb + j];
            ion[j] = a.iion[nd[j]];
        }
        double di = 0.0;
        for (int x = 0; x < nb; ++x)
            for (int y = x + 1; y < nb; ++y) di = fmax(di, fabs((double)ion[x] - (double)ion[y]));
        const bool active = di > 1.0;
        a.flag[e] = active ? 1 : 0;
        if (!active) continue;
        T p[P > 0 ? P : 1];
        if (a.pset) {
            const T* pp = a.params + (size_t)a.pset[nd[0]] * P;
            for (int m = 0; m < P; ++m) p[m] = pp[m];
        } else {
            for (int m = 0; m < P; ++m) p[m] = T(1);
        }
        const double wj = a.ewj[e];
        double be[4] = {0.0, 0.0, 0.0, 0.0};
        for (int q = 0; q < nb; ++q) {
            T y[S];
            T iint = T(0);
            for (int m = 0; m < S; ++m) y[m] = T(0);
            for (int j = 0; j < nb; ++j) {
                const T phi = (T)(j == a.big[q] ? a.qa : a.qb);
                iint += phi * ion[j];
                y[0] += phi * (T)a.V[nd[j]];
                for (int m = 1; m < S; ++m) y[m] += phi * a.states[(size_t)(m - 1) * a.n + nd[j]];
            }
            const double d = (double)M::template iionic<T>(y, (T)a.cm, p) - (double)iint;
            for (int j = 0; j < nb; ++j) be[j] += (j == a.big[q] ? a.qa : a.qb) * (-a.am) * d * wj;
        }
        for (int j = 0; j < nb; ++j) a.ebuf[(size_t)e * 4 + j] = be[j];
    }
}

__global__ void __launch_bounds__(256) svi_gather_kernel(const int n, const int width, const int* __restrict__ ell,
                                                         const uint8_t* __restrict__ flag,
                                                         const double* __restrict__ ebuf, double* __restrict__ corr) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < width; ++k) {
            const int ent = ell[(size_t)k * n + i];
            if (ent < 0) break;
            if (flag[ent >> 2]) acc += ebuf[ent];
        }
        corr[i] = acc;
    }
}

}  // namespace chb
