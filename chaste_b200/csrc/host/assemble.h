// Host-side finite-element assembly for the GPU tissue (runs once per mesh).
#pragma once

#include <cstdint>
#include <vector>

namespace chb {

// CSR sharing one pattern between A = Am*Cm/dt*M + K and M.
struct HostCsr {
    int n = 0;
    std::vector<int> rowptr, cols;
    std::vector<double> a, m;
    int find(int i, int j) const;
};

// P1 element matrices of a simplex (closed forms of the order-2 Gauss rule
// the reference uses, exact for P1):
//   M_e = |J| vol_ref (1 + delta_ij) / ((d+1)(d+2))   MassMatrixAssembler.hpp:76-104
//   K_e = |J| vol_ref grad(phi)^T sigma grad(phi)      MonodomainStiffnessMatrixAssembler.hpp:68-84
// Returns false for a degenerate element.
bool element_matrices(int dim, const double* X /*(dim+1) x 3*/, const double* sigma_diag,
                      bool lump, double* Me, double* Ke);

// Assemble A and M in CSR with sorted columns (AbstractFeVolumeIntegralAssembler::DoAssemble,
// pde/src/solver/AbstractFeVolumeIntegralAssembler.hpp:257-324).  Returns false on a bad element.
bool assemble(int dim, int n_nodes, const double* xyz, int n_elems, const int* conn,
              const double* sigma, double mass_scale, bool lump, HostCsr& out);

// Regular slab (ConstructRegularSlabMesh, mesh/src/common/AbstractTetrahedralMesh.cpp:569-614).
struct SlabGrid {
    int dim = 0;
    int nx = 0, ny = 0, nz = 0;   // elements per axis
    double h = 0;
    int NX() const { return nx + 1; }
    int NY() const { return dim > 1 ? ny + 1 : 1; }
    int NZ() const { return dim > 2 ? nz + 1 : 1; }
    long long nodes() const { return (long long)NX() * NY() * NZ(); }
};
bool slab_grid(int dim, double h, double w, double hh, double dd, SlabGrid& g);
void slab_mesh(const SlabGrid& g, std::vector<double>& xyz, std::vector<int>& conn);

// Matrix-free slab stencil: every row of A (and M) equals the row of its
// boundary class up to rounding; the table holds the coefficients per (class, offset).
struct SlabStencil {
    int n_offsets = 0;
    int offsets[27];            // linear index offsets, ascending
    int doff[27][3];            // (di, dj, dk)
    int n_classes = 0;          // 3^dim (x 2 stagger parities in 2D)
    std::vector<double> a, m;   // [class][offset]
};
int slab_class(const SlabGrid& g, int i, int j, int k);
// Builds the table from the assembled CSR (the first row of each class) and checks
// that every row agrees with its class row to 1e-12 relative.
bool build_slab_stencil(const SlabGrid& g, const HostCsr& csr, SlabStencil& st);

}  // namespace chb
