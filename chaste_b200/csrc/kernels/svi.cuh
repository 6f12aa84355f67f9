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
// One thread per node gathers the contributions of its elements in ascending
// element order (deterministic, no atomics): for element e and quadrature point q,
// where one node has basis value A and the others B,
//     c_i += phi_i(q) * (-Am) * (Iion(sum_j phi_j y_j) - sum_j phi_j Iion_j) * wJ_e.
#pragma once

#include "../models/lr91.h"
#include "../models/tt06.h"
#include "common.cuh"

namespace chb {

template <typename T>
struct SviArgs {
    int n, dim;
    const double* __restrict__ V;        // V^n
    const T* __restrict__ states;        // (S-1) x n, after the ODE step
    const T* __restrict__ iion;          // nodal Iion cache
    const uint8_t* __restrict__ pset;    // may be null
    const T* __restrict__ params;
    const int* __restrict__ econn;       // n_elems x (dim+1)
    const double* __restrict__ ewj;      // |det J| x reference weight, per element
    const int* __restrict__ nptr;        // node -> elements (ascending), CSR
    const int* __restrict__ nel;
    double* __restrict__ corr;           // n
    double am, cm;
    double qa, qb;                       // basis values at a quadrature point: its node, the others
    int big[4];                          // node of each quadrature point with basis value qa
};

template <class M, typename T>
__global__ void __launch_bounds__(256) svi_kernel(SviArgs<T> a) {
    constexpr int S = M::kNumStates;
    constexpr int P = M::kNumParams;
    const int nb = a.dim + 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int k = a.nptr[i]; k < a.nptr[i + 1]; ++k) {
            const int e = a.nel[k];
            int nd[4], me = 0;
            T ion[4];
            for (int j = 0; j < nb; ++j) {
                nd[j] = a.econn[e * nb + j];
                ion[j] = a.iion[nd[j]];
                if (nd[j] == i) me = j;
            }
            double di = 0.0;
            for (int x = 0; x < nb; ++x)
                for (int y = x + 1; y < nb; ++y) di = fmax(di, fabs((double)ion[x] - (double)ion[y]));
            if (!(di > 1.0)) continue;
            T p[P > 0 ? P : 1];
            if (a.pset) {
                const T* pp = a.params + (size_t)a.pset[nd[0]] * P;
                for (int m = 0; m < P; ++m) p[m] = pp[m];
            } else {
                for (int m = 0; m < P; ++m) p[m] = T(1);
            }
            const double wj = a.ewj[e];
            double be = 0.0;
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
                const T isv = M::template iionic<T>(y, (T)a.cm, p);
                const double phi_me = me == a.big[q] ? a.qa : a.qb;
                be += phi_me * (-a.am) * ((double)isv - (double)iint) * wj;
            }
            acc += be;
        }
        a.corr[i] = acc;
    }
}

}  // namespace chb
