// Host-side finite-element assembly for the GPU tissue.  See assemble.h.
#include "assemble.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

namespace chb {

int HostCsr::find(int i, int j) const {
    int lo = rowptr[i], hi = rowptr[i + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] == j) return mid;
        if (cols[mid] < j) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

bool element_matrices(int dim, const double* X, const double* sigma, bool lump, double* Me,
                      double* Ke) {
    const int nb = dim + 1;
    // Jacobian columns are the edge vectors from node 0 (the reference map of
    // TetrahedralMesh::GetInverseJacobianForElement).
    double J[3][3] = {{0}}, Ji[3][3] = {{0}};
    for (int c = 0; c < dim; ++c)
        for (int r = 0; r < dim; ++r) J[r][c] = X[(c + 1) * 3 + r] - X[r];
    double det;
    if (dim == 1) {
        det = J[0][0];
        Ji[0][0] = 1.0 / det;
    } else if (dim == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        Ji[0][0] = J[1][1] / det;
        Ji[0][1] = -J[0][1] / det;
        Ji[1][0] = -J[1][0] / det;
        Ji[1][1] = J[0][0] / det;
    } else {
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][0] * J[2][2] - J[1][2] * J[2][0];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        det = J[0][0] * c00 - J[0][1] * c01 + J[0][2] * c02;
        Ji[0][0] = c00 / det;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        Ji[1][0] = -c01 / det;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        Ji[2][0] = c02 / det;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    if (det == 0.0 || !std::isfinite(det)) return false;
    const double vol = std::fabs(det) * (dim == 1 ? 1.0 : (dim == 2 ? 0.5 : 1.0 / 6.0));
    // physical gradients of the barycentric basis: grad(phi_k) = J^{-T} e_k,
    // grad(phi_0) = -sum_k grad(phi_k)
    double G[4][3] = {{0}};
    for (int k = 1; k < nb; ++k)
        for (int s = 0; s < dim; ++s) G[k][s] = Ji[k - 1][s];
    for (int s = 0; s < dim; ++s) {
        double acc = 0.0;
        for (int k = 1; k < nb; ++k) acc -= Ji[k - 1][s];
        G[0][s] = acc;
    }
    const double mdiag = vol * 2.0 / ((dim + 1) * (dim + 2));
    const double moff = vol * 1.0 / ((dim + 1) * (dim + 2));
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            double k = 0.0;
            for (int s = 0; s < dim; ++s) k += G[i][s] * sigma[s] * G[j][s];
            Ke[i * nb + j] = vol * k;
            Me[i * nb + j] = (i == j) ? mdiag : moff;
        }
    if (lump) {
        // MassMatrixAssembler.hpp:88-100: row sums onto the diagonal
        for (int i = 0; i < nb; ++i) {
            double s = Me[i * nb + i];
            for (int j = 0; j < nb; ++j)
                if (j != i) s += Me[i * nb + j];
            for (int j = 0; j < nb; ++j) Me[i * nb + j] = (i == j) ? s : 0.0;
        }
    }
    return true;
}

template <class F>
static void parallel_rows(int n, F f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > 32) nt = 32;
    if (n < 4096) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t)
        th.emplace_back([&, t] { f((int)((long long)n * t / nt), (int)((long long)n * (t + 1) / nt)); });
    f(0, (int)((long long)n / nt));
    for (auto& x : th) x.join();
}

bool assemble(int dim, int n_nodes, const double* xyz, int n_elems, const int* conn,
              const double* sigma, double mass_scale, bool lump, HostCsr& out) {
    const int nb = dim + 1;
    // node -> incident elements (ascending element index)
    std::vector<int> cnt(n_nodes + 1, 0);
    for (long long e = 0; e < n_elems; ++e)
        for (int a = 0; a < nb; ++a) {
            const int v = conn[e * nb + a];
            if (v < 0 || v >= n_nodes) return false;
            cnt[v + 1]++;
        }
    for (int i = 0; i < n_nodes; ++i) cnt[i + 1] += cnt[i];
    std::vector<int> inc(cnt[n_nodes]);
    {
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int e = 0; e < n_elems; ++e)
            for (int a = 0; a < nb; ++a) inc[fill[conn[(long long)e * nb + a]]++] = e;
    }
    out.n = n_nodes;
    out.rowptr.assign(n_nodes + 1, 0);
    std::vector<int> rowlen(n_nodes, 0);
    parallel_rows(n_nodes, [&](int b, int e) {
        std::vector<int> nb_list;
        for (int i = b; i < e; ++i) {
            nb_list.clear();
            for (int q = cnt[i]; q < cnt[i + 1]; ++q)
                for (int a = 0; a < nb; ++a) nb_list.push_back(conn[(long long)inc[q] * nb + a]);
            std::sort(nb_list.begin(), nb_list.end());
            rowlen[i] = (int)(std::unique(nb_list.begin(), nb_list.end()) - nb_list.begin());
        }
    });
    for (int i = 0; i < n_nodes; ++i) out.rowptr[i + 1] = out.rowptr[i] + rowlen[i];
    out.cols.assign(out.rowptr[n_nodes], 0);
    out.a.assign(out.cols.size(), 0.0);
    out.m.assign(out.cols.size(), 0.0);
    bool ok = true;
    parallel_rows(n_nodes, [&](int b, int e) {
        std::vector<int> nb_list;
        double X[12], Me[16], Ke[16];
        for (int i = b; i < e; ++i) {
            nb_list.clear();
            for (int q = cnt[i]; q < cnt[i + 1]; ++q)
                for (int a = 0; a < nb; ++a) nb_list.push_back(conn[(long long)inc[q] * nb + a]);
            std::sort(nb_list.begin(), nb_list.end());
            nb_list.erase(std::unique(nb_list.begin(), nb_list.end()), nb_list.end());
            std::copy(nb_list.begin(), nb_list.end(), out.cols.begin() + out.rowptr[i]);
            // row i gathers the contributions of its elements in ascending element
            // order, the order an element-by-element scatter adds them in
            for (int q = cnt[i]; q < cnt[i + 1]; ++q) {
                const long long el = inc[q];
                int li = -1;
                for (int a = 0; a < nb; ++a) {
                    const int v = conn[el * nb + a];
                    if (v == i) li = a;
                    for (int s = 0; s < 3; ++s) X[a * 3 + s] = xyz[(long long)v * 3 + s];
                }
                if (!element_matrices(dim, X, sigma + el * dim, lump, Me, Ke)) {
                    ok = false;
                    return;
                }
                for (int c = 0; c < nb; ++c) {
                    const int j = conn[el * nb + c];
                    const int k = out.rowptr[i] +
                                  (int)(std::lower_bound(nb_list.begin(), nb_list.end(), j) - nb_list.begin());
                    out.a[k] += mass_scale * Me[li * nb + c] + Ke[li * nb + c];
                    out.m[k] += Me[li * nb + c];
                }
            }
        }
    });
    return ok;
}

bool slab_grid(int dim, double h, double w, double hh, double dd, SlabGrid& g) {
    if (!(h > 0) || !(w > 0) || dim < 1 || dim > 3) return false;
    g.dim = dim;
    g.h = h;
    g.nx = (int)(unsigned)((w + 0.5 * h) / h);
    g.ny = dim > 1 ? (int)(unsigned)((hh + 0.5 * h) / h) : 0;
    g.nz = dim > 2 ? (int)(unsigned)((dd + 0.5 * h) / h) : 0;
    if (std::fabs(g.nx * h - w) > DBL_EPSILON * w) return false;
    if (dim > 1 && (hh <= 0 || std::fabs(g.ny * h - hh) > DBL_EPSILON * hh)) return false;
    if (dim > 2 && (dd <= 0 || std::fabs(g.nz * h - dd) > DBL_EPSILON * dd)) return false;
    return g.nx > 0 && (dim < 2 || g.ny > 0) && (dim < 3 || g.nz > 0);
}

void slab_mesh(const SlabGrid& g, std::vector<double>& xyz, std::vector<int>& conn) {
    const int NX = g.NX(), NY = g.NY(), NZ = g.NZ();
    xyz.assign((size_t)g.nodes() * 3, 0.0);
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                const size_t idx = ((size_t)k * NY + j) * NX + i;
                xyz[idx * 3 + 0] = i * g.h;
                xyz[idx * 3 + 1] = j * g.h;
                xyz[idx * 3 + 2] = k * g.h;
            }
    conn.clear();
    if (g.dim == 1) {
        for (int e = 0; e < g.nx; ++e) {
            conn.push_back(e);
            conn.push_back(e + 1);
        }
    } else if (g.dim == 2) {
        // staggered triangles (AbstractTetrahedralMesh.cpp:349-376)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                const int parity = (i + (g.ny - j)) % 2;
                const int nw = (j + 1) * NX + i, sw = j * NX + i;
                conn.insert(conn.end(), {nw, nw + 1, parity == 1 ? sw + 1 : sw});
                conn.insert(conn.end(), {sw + 1, sw, parity == 1 ? nw : nw + 1});
            }
    } else {
        // six tetrahedra per cube around the 0-7 diagonal (:420-422)
        static const int en[6][4] = {{0, 1, 5, 7}, {0, 1, 3, 7}, {0, 2, 3, 7},
                                     {0, 2, 6, 7}, {0, 4, 6, 7}, {0, 4, 5, 7}};
        conn.reserve((size_t)6 * 4 * g.nx * g.ny * g.nz);
        for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
                for (int i = 0; i < g.nx; ++i) {
                    int gi[8], l = 0;
                    for (int z = 0; z < 2; ++z)
                        for (int y = 0; y < 2; ++y)
                            for (int x = 0; x < 2; ++x) gi[l++] = i + x + NX * (j + y + NY * (k + z));
                    for (int m = 0; m < 6; ++m)
                        for (int q = 0; q < 4; ++q) conn.push_back(gi[en[m][q]]);
                }
    }
}

int slab_class(const SlabGrid& g, int i, int j, int k) {
    const int cx = i == 0 ? 0 : (i == g.nx ? 2 : 1);
    if (g.dim == 1) return cx;
    const int cy = j == 0 ? 0 : (j == g.ny ? 2 : 1);
    if (g.dim == 2) return cx + 3 * cy + 9 * ((i + g.ny - j) & 1);
    const int cz = k == 0 ? 0 : (k == g.nz ? 2 : 1);
    return cx + 3 * cy + 9 * cz;
}

// Largest relative difference accepted between a row and its class row.
constexpr double kSlabRowTolerance = 1e-12;

bool build_slab_stencil(const SlabGrid& g, const HostCsr& csr, SlabStencil& st) {
    const int NX = g.NX(), NY = g.NY(), NZ = g.NZ();
    st.n_classes = g.dim == 1 ? 3 : (g.dim == 2 ? 18 : 27);
    st.n_offsets = 0;
    const int rz = g.dim > 2 ? 1 : 0, ry = g.dim > 1 ? 1 : 0;
    for (int dk = -rz; dk <= rz; ++dk)
        for (int dj = -ry; dj <= ry; ++dj)
            for (int di = -1; di <= 1; ++di) {
                st.doff[st.n_offsets][0] = di;
                st.doff[st.n_offsets][1] = dj;
                st.doff[st.n_offsets][2] = dk;
                st.offsets[st.n_offsets] = di + NX * (dj + NY * dk);
                st.n_offsets++;
            }
    const int no = st.n_offsets;
    std::vector<double> a((size_t)st.n_classes * no, 0.0), m((size_t)st.n_classes * no, 0.0);
    std::vector<char> seen(st.n_classes, 0), used(no, 0);
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                const int row = (k * NY + j) * NX + i;
                const int c = slab_class(g, i, j, k);
                double ra[27], rm[27];
                int found = 0;
                for (int o = 0; o < no; ++o) {
                    const int ii = i + st.doff[o][0], jj = j + st.doff[o][1], kk = k + st.doff[o][2];
                    ra[o] = rm[o] = 0.0;
                    if (ii < 0 || ii >= NX || jj < 0 || jj >= NY || kk < 0 || kk >= NZ) continue;
                    const int q = csr.find(row, row + st.offsets[o]);
                    if (q < 0) continue;
                    ra[o] = csr.a[q];
                    rm[o] = csr.m[q];
                    found++;
                }
                if (found != csr.rowptr[row + 1] - csr.rowptr[row]) return false;
                if (!seen[c]) {
                    seen[c] = 1;
                    for (int o = 0; o < no; ++o) {
                        a[(size_t)c * no + o] = ra[o];
                        m[(size_t)c * no + o] = rm[o];
                    }
                } else {
                    // node coordinates are i*h, so element edges (i+1)*h - i*h differ from
                    // h in the last bit: rows of one class agree to rounding, not bitwise
                    const double* ca = &a[(size_t)c * no];
                    const double* cm = &m[(size_t)c * no];
                    double sa = 0.0, sm = 0.0;
                    for (int o = 0; o < no; ++o) {
                        sa = std::max(sa, std::fabs(ca[o]));
                        sm = std::max(sm, std::fabs(cm[o]));
                    }
                    for (int o = 0; o < no; ++o) {
                        if ((ra[o] == 0.0) != (ca[o] == 0.0) || (rm[o] == 0.0) != (cm[o] == 0.0)) return false;
                        if (std::fabs(ra[o] - ca[o]) > kSlabRowTolerance * sa) return false;
                        if (std::fabs(rm[o] - cm[o]) > kSlabRowTolerance * sm) return false;
                    }
                }
                for (int o = 0; o < no; ++o)
                    if (ra[o] != 0.0 || rm[o] != 0.0) used[o] = 1;
            }
    SlabStencil out;
    out.n_classes = st.n_classes;
    for (int o = 0; o < no; ++o)
        if (used[o]) {
            out.offsets[out.n_offsets] = st.offsets[o];
            for (int s = 0; s < 3; ++s) out.doff[out.n_offsets][s] = st.doff[o][s];
            out.n_offsets++;
        }
    out.a.assign((size_t)out.n_classes * out.n_offsets, 0.0);
    out.m.assign((size_t)out.n_classes * out.n_offsets, 0.0);
    for (int c = 0; c < out.n_classes; ++c) {
        int q = 0;
        for (int o = 0; o < no; ++o)
            if (used[o]) {
                out.a[(size_t)c * out.n_offsets + q] = a[(size_t)c * no + o];
                out.m[(size_t)c * out.n_offsets + q] = m[(size_t)c * no + o];
                q++;
            }
    }
    st = out;
    return true;
}

}  // namespace chb
