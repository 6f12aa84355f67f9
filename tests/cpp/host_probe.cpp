// Test-only C entry points over the library's host assembly (chaste_b200/csrc/host),
// compiled by tests/test_host_assembly.py with g++ so the host logic is checked without a GPU.
#include <cstring>
#include <vector>

#include "../../chaste_b200/csrc/host/assemble.h"

using namespace chb;

extern "C" int probe_slab(int dim, double h, double w, double hh, double dd, const double* sigma,
                          double mass_scale, int* n_nodes, int* nnz, int* rowptr, int* cols,
                          double* a, double* m, int* stencil_ok, int* n_off, int* n_cls,
                          int* offsets, double* atab, double* mtab, int* cls) {
    SlabGrid g;
    if (!slab_grid(dim, h, w, hh, dd, g)) return -1;
    std::vector<double> xyz;
    std::vector<int> conn;
    slab_mesh(g, xyz, conn);
    const int ne = (int)(conn.size() / (dim + 1));
    std::vector<double> sig((size_t)ne * dim);
    for (int e = 0; e < ne; ++e)
        for (int s = 0; s < dim; ++s) sig[(size_t)e * dim + s] = sigma[s];
    HostCsr csr;
    if (!assemble(dim, (int)g.nodes(), xyz.data(), ne, conn.data(), sig.data(), mass_scale, false, csr)) return -2;
    *n_nodes = (int)g.nodes();
    *nnz = (int)csr.cols.size();
    if (rowptr) {
        std::memcpy(rowptr, csr.rowptr.data(), sizeof(int) * csr.rowptr.size());
        std::memcpy(cols, csr.cols.data(), sizeof(int) * csr.cols.size());
        std::memcpy(a, csr.a.data(), sizeof(double) * csr.a.size());
        std::memcpy(m, csr.m.data(), sizeof(double) * csr.m.size());
        SlabStencil st;
        *stencil_ok = build_slab_stencil(g, csr, st) ? 1 : 0;
        if (*stencil_ok) {
            *n_off = st.n_offsets;
            *n_cls = st.n_classes;
            std::memcpy(offsets, st.offsets, sizeof(int) * st.n_offsets);
            std::memcpy(atab, st.a.data(), sizeof(double) * st.a.size());
            std::memcpy(mtab, st.m.data(), sizeof(double) * st.m.size());
            for (int k = 0; k < g.NZ(); ++k)
                for (int j = 0; j < g.NY(); ++j)
                    for (int i = 0; i < g.NX(); ++i) cls[((size_t)k * g.NY() + j) * g.NX() + i] = slab_class(g, i, j, k);
        }
    }
    return 0;
}
