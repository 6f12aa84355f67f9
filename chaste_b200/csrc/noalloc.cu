// cg_slab_solve_noalloc: the diffusion solve of one monodomain PDE step on a
// regular slab, for callers that must not allocate device memory.
//
// Who needs this: code that runs where cudaMalloc is not allowed or not
// wanted -- a host application that owns all device memory through its own
// pool (a PETSc-style vector layer handing us its buffers), code called back
// from inside an allocator-free region, or a solver embedded in a larger
// program that forbids allocation after start-up.  Such a caller passes its own
// device buffers for the input (z) and the input/output (x); every other device
// word the solve needs lives in one fixed array defined below.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library reserves it until the process exits, and every call shares it, so
// calls that overlap on the GPU race with each other (serialise them, e.g. on
// one stream).  The array keeps the previous call's contents; each call
// clears the parts that must start at zero (the grid barrier, the status word,
// the halos) before it launches.
//
// In host code the array's name is only a host-side stand-in, not a device
// address.  The first call on each device therefore resolves the real address
// with cudaGetSymbolAddress, with that device current, and caches it; make that
// first call before any stream capture.  The cached address belongs to the
// device's primary context: a cudaDeviceReset after the first call on a device
// is not supported (the module may then load at another address).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "../../include/chaste_gpu.h"
#include "host/assemble.h"
#include "kernels/cg.cuh"

using namespace chb;

namespace {

// Largest slab (in nodes) the static scratch serves.
constexpr int kNoAllocMaxNodes = 32768;
constexpr int kNoAllocMaxBlocks = 256;
static_assert(kNoAllocMaxBlocks <= kMaxGridBlocks, "grid larger than the reduction supports");

// Layout of the scratch array, in bytes.  x, z and B r are read through the
// stencil, so each has a zero halo of up to kNoAllocMaxNodes entries per side.
constexpr size_t kHaloed = 3 * (size_t)kNoAllocMaxNodes * sizeof(double);
constexpr size_t kPlain = (size_t)kNoAllocMaxNodes * sizeof(double);
constexpr size_t kOffX = 0;
constexpr size_t kOffZ = kOffX + kHaloed;
constexpr size_t kOffZp = kOffZ + kHaloed;
constexpr size_t kOffR = kOffZp + kHaloed;
constexpr size_t kOffP = kOffR + kPlain;
constexpr size_t kOffQ = kOffP + kPlain;
constexpr size_t kOffPartials = kOffQ + kPlain;
constexpr size_t kOffTabA = kOffPartials + 2 * kNoAllocMaxBlocks * kPartialStride * sizeof(double);
constexpr size_t kOffTabM = kOffTabA + kMaxClasses * kMaxOffsets * sizeof(double);
constexpr size_t kOffSync = kOffTabM + kMaxClasses * kMaxOffsets * sizeof(double);
constexpr size_t kOffWords = kOffSync + 256;              // status, refine, ring[1], step
constexpr size_t kOffCls = kOffWords + 256;
constexpr size_t kScratchBytes = kOffCls + (size_t)kNoAllocMaxNodes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_addr[64] = {nullptr};

// Device address of the scratch array on the current device (resolved once per device).
int scratch_address(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return CG_OK;
}

// Rows of A and M for every boundary class of the slab, computed from the
// element matrices around one representative node per class, without any
// allocation.  Offsets are the 3^dim neighbourhood in ascending order.
bool class_rows(const SlabGrid& g, const double* sigma, double mass_scale, bool lump, int* n_off,
                int* offsets, double* a, double* m, int* n_cls) {
    const int dim = g.dim, NX = g.NX(), NY = g.NY();
    const int rz = dim > 2 ? 1 : 0, ry = dim > 1 ? 1 : 0;
    int no = 0;
    int doff[27][3];
    for (int dk = -rz; dk <= rz; ++dk)
        for (int dj = -ry; dj <= ry; ++dj)
            for (int di = -1; di <= 1; ++di) {
                doff[no][0] = di;
                doff[no][1] = dj;
                doff[no][2] = dk;
                offsets[no++] = di + NX * (dj + NY * dk);
            }
    *n_off = no;
    *n_cls = dim == 1 ? 3 : (dim == 2 ? 18 : 27);
    std::memset(a, 0, sizeof(double) * (*n_cls) * no);
    std::memset(m, 0, sizeof(double) * (*n_cls) * no);
    static const int en[6][4] = {{0, 1, 5, 7}, {0, 1, 3, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 6, 7}, {0, 4, 5, 7}};
    bool done[kMaxClasses] = {false};
    double tra[kMaxOffsets], trm[kMaxOffsets];
    // candidate coordinates per axis: both ends and the first two interior
    // positions, which together reach every class (both stagger parities in 2D)
    int cand[3][4], nc[3] = {0, 0, 0};
    const int ext[3] = {g.nx, dim > 1 ? g.ny : 0, dim > 2 ? g.nz : 0};
    for (int ax = 0; ax < 3; ++ax)
        for (int v : {0, 1, 2, ext[ax]})
            if (v <= ext[ax] && std::find(cand[ax], cand[ax] + nc[ax], v) == cand[ax] + nc[ax]) cand[ax][nc[ax]++] = v;
    for (int ck = 0; ck < nc[2]; ++ck)
        for (int cj = 0; cj < nc[1]; ++cj)
            for (int ci = 0; ci < nc[0]; ++ci) {
                    const int i = cand[0][ci], j = cand[1][cj], k = cand[2][ck];
                    const int cls = slab_class(g, i, j, k);
                    const int node = i + NX * (j + NY * k);
                    // the row is formed in temporaries; a class met again at another
                    // candidate node must give the same row (to 1e-12 relative)
                    double* ra = tra;
                    double* rm = trm;
                    std::fill(tra, tra + no, 0.0);
                    std::fill(trm, trm + no, 0.0);
                    double X[12], Me[16], Ke[16];
                    auto add = [&](const int* v, int nb, int li, const double* sig) {
                        for (int b = 0; b < nb; ++b) {
                            const int vb = v[b];
                            const int bi = vb % NX, bj = (vb / NX) % NY, bk = vb / (NX * NY);
                            for (int s = 0; s < 3; ++s) X[b * 3 + s] = (s == 0 ? bi : (s == 1 ? bj : bk)) * g.h;
                        }
                        if (!element_matrices(dim, X, sig, lump, Me, Ke)) return false;
                        for (int b = 0; b < nb; ++b) {
                            const int vb = v[b];
                            const int di = vb % NX - i, dj = (vb / NX) % NY - j, dk = vb / (NX * NY) - k;
                            for (int o = 0; o < no; ++o)
                                if (doff[o][0] == di && doff[o][1] == dj && doff[o][2] == dk) {
                                    ra[o] += mass_scale * Me[li * nb + b] + Ke[li * nb + b];
                                    rm[o] += Me[li * nb + b];
                                }
                        }
                        return true;
                    };
                    // incident elements in ascending element index (the assembly order)
                    if (dim == 1) {
                        for (int e = i - 1; e <= i; ++e) {
                            if (e < 0 || e >= g.nx) continue;
                            const int v[2] = {e, e + 1};
                            if (!add(v, 2, e == i ? 0 : 1, sigma)) return false;
                        }
                    } else if (dim == 2) {
                        for (int sj = j - 1; sj <= j; ++sj)
                            for (int si = i - 1; si <= i; ++si) {
                                if (si < 0 || si >= g.nx || sj < 0 || sj >= g.ny) continue;
                                const int parity = (si + (g.ny - sj)) % 2;
                                const int nw = (sj + 1) * NX + si, sw = sj * NX + si;
                                const int up[3] = {nw, nw + 1, parity == 1 ? sw + 1 : sw};
                                const int lo[3] = {sw + 1, sw, parity == 1 ? nw : nw + 1};
                                for (const int* v : {up, lo})
                                    for (int li = 0; li < 3; ++li)
                                        if (v[li] == node && !add(v, 3, li, sigma)) return false;
                            }
                    } else {
                        for (int ck = k - 1; ck <= k; ++ck)
                            for (int cj = j - 1; cj <= j; ++cj)
                                for (int ci = i - 1; ci <= i; ++ci) {
                                    if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny || ck < 0 || ck >= g.nz) continue;
                                    int gi[8], l = 0;
                                    for (int zz = 0; zz < 2; ++zz)
                                        for (int yy = 0; yy < 2; ++yy)
                                            for (int xx = 0; xx < 2; ++xx) gi[l++] = ci + xx + NX * (cj + yy + NY * (ck + zz));
                                    for (int t = 0; t < 6; ++t) {
                                        const int v[4] = {gi[en[t][0]], gi[en[t][1]], gi[en[t][2]], gi[en[t][3]]};
                                        for (int li = 0; li < 4; ++li)
                                            if (v[li] == node && !add(v, 4, li, sigma)) return false;
                                    }
                                }
                    }
                    double* ca = a + (size_t)cls * no;
                    double* cm = m + (size_t)cls * no;
                    if (!done[cls]) {
                        std::copy(tra, tra + no, ca);
                        std::copy(trm, trm + no, cm);
                        done[cls] = true;
                        continue;
                    }
                    double scale = 0.0;
                    for (int o = 0; o < no; ++o) scale = std::max({scale, std::fabs(ca[o]), std::fabs(cm[o])});
                    for (int o = 0; o < no; ++o)
                        if (std::fabs(tra[o] - ca[o]) > 1e-12 * scale || std::fabs(trm[o] - cm[o]) > 1e-12 * scale)
                            return false;
                }
    return true;
}

}  // namespace

extern "C" int cg_slab_solve_noalloc(const cg_config* cfg, int dim, double h, double width, double height,
                                     double depth, const double* sigma, const double* d_z, double* d_x,
                                     void* stream, int* iterations) {
    if (!cfg || !sigma || !d_z || !d_x) return CG_ERR_ARG;
    if (!(cfg->pde_time_step > 0) || !(cfg->surface_area_to_volume_ratio > 0) || !(cfg->capacitance > 0) ||
        !(cfg->ksp_tolerance > 0))
        return CG_ERR_ARG;
    if (cfg->ksp_preconditioner != CG_PC_NONE && cfg->ksp_preconditioner != CG_PC_JACOBI) return CG_ERR_UNSUPPORTED;
    SlabGrid g;
    if (!slab_grid(dim, h, width, height, depth, g)) return CG_ERR_ARG;
    const long long n = g.nodes();
    const long long halo = (long long)g.NX() * g.NY() + g.NX() + 1;
    // sizes beyond the static scratch are rejected, never truncated
    if (n > kNoAllocMaxNodes || halo > kNoAllocMaxNodes) return CG_ERR_ARG;
    unsigned char* base = nullptr;
    int rc = scratch_address(&base);
    if (rc != CG_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // operator tables (host stack memory only)
    const double mass_scale = cfg->surface_area_to_volume_ratio * cfg->capacitance / cfg->pde_time_step;
    int no = 0, ncls = 0, offs[27];
    double ta[kMaxClasses * kMaxOffsets], tm[kMaxClasses * kMaxOffsets];
    if (!class_rows(g, sigma, mass_scale, cfg->use_mass_lumping != 0, &no, offs, ta, tm, &ncls)) return CG_ERR_ARG;
    // drop the offsets whose coefficients vanish in every class (12 of the 27 in 3D,
    // where the 6-tet cubes leave 15 neighbours), keeping ascending order
    {
        int kept = 0;
        for (int o = 0; o < no; ++o) {
            bool used = offs[o] == 0;
            for (int c = 0; c < ncls && !used; ++c)
                used = ta[(size_t)c * no + o] != 0.0 || tm[(size_t)c * no + o] != 0.0;
            if (!used) continue;
            for (int c = 0; c < ncls; ++c) {
                ta[(size_t)c * no + kept] = ta[(size_t)c * no + o];
                tm[(size_t)c * no + kept] = tm[(size_t)c * no + o];
            }
            offs[kept++] = offs[o];
        }
        // re-pack the rows from stride no to stride kept
        for (int c = 1; c < ncls; ++c)
            for (int o = 0; o < kept; ++o) {
                ta[(size_t)c * kept + o] = ta[(size_t)c * no + o];
                tm[(size_t)c * kept + o] = tm[(size_t)c * no + o];
            }
        no = kept;
    }
    int diag = -1;
    for (int o = 0; o < no; ++o)
        if (offs[o] == 0) diag = o;
    static thread_local uint8_t cls[kNoAllocMaxNodes];
    long long count[kMaxClasses] = {0};
    for (int k = 0; k < g.NZ(); ++k)
        for (int j = 0; j < g.NY(); ++j)
            for (int i = 0; i < g.NX(); ++i) {
                const int c = slab_class(g, i, j, k);
                cls[(k * g.NY() + j) * g.NX() + i] = (uint8_t)c;
                count[c]++;
            }
    const int interior = (int)(std::max_element(count, count + ncls) - count);

    double* x = reinterpret_cast<double*>(base + kOffX) + kNoAllocMaxNodes;
    double* z = reinterpret_cast<double*>(base + kOffZ) + kNoAllocMaxNodes;
    double* zp = reinterpret_cast<double*>(base + kOffZp) + kNoAllocMaxNodes;
    GridSync* gs = reinterpret_cast<GridSync*>(base + kOffSync);
    int* words = reinterpret_cast<int*>(base + kOffWords);   // [0] status, [1] refine, [2] ring
    long long* step = reinterpret_cast<long long*>(base + kOffWords + 64);

    CgArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = (int)n;
    a.slab.n_off = no;
    a.slab.n_cls = ncls;
    a.slab.interior = interior;
    for (int o = 0; o < no; ++o) {
        a.slab.off[o] = offs[o];
        a.slab.ia[o] = ta[(size_t)interior * no + o];
        a.slab.im[o] = tm[(size_t)interior * no + o];
        a.slab.ia32[o] = (float)a.slab.ia[o];
    }
    a.slab.a_tab = reinterpret_cast<const double*>(base + kOffTabA);
    a.slab.m_tab = reinterpret_cast<const double*>(base + kOffTabM);
    a.x = x;
    a.zrhs = z;
    a.cls8 = base + kOffCls;
    a.r = reinterpret_cast<double*>(base + kOffR);
    a.zp = zp;
    a.p0 = reinterpret_cast<double*>(base + kOffP);
    a.q = reinterpret_cast<double*>(base + kOffQ);
    a.partials = reinterpret_cast<double*>(base + kOffPartials);
    a.gs = gs;
    a.status = words;
    a.refine_out = words + 1;
    a.iters_ring = words + 2;
    a.ring = 1;
    a.step = step;
    a.rtol = cfg->use_absolute_tolerance ? DBL_EPSILON : cfg->ksp_tolerance;
    a.abstol = cfg->use_absolute_tolerance ? cfg->ksp_tolerance : 1e-50;
    a.dtol = 1e5;
    a.maxit = cfg->max_iterations > 0 ? cfg->max_iterations : 10000;
    a.pc = cfg->ksp_preconditioner == CG_PC_JACOBI ? 1 : 0;
    a.diag_slot = diag;

    // the offset count unrolled at compile time where the main path has that instance
    void (*kernel)(CgArgs) = no == 3    ? cg_fp64_kernel<true, 3>
                             : no == 7  ? cg_fp64_kernel<true, 7>
                             : no == 9  ? cg_fp64_kernel<true, 9>
                             : no == 15 ? cg_fp64_kernel<true, 15>
                                        : cg_fp64_kernel<true, 0>;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 512, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    const int blocks = (int)std::max(1LL, std::min<long long>({(n + 511) / 512, (long long)per_sm * sms,
                                                               (long long)kNoAllocMaxBlocks}));

    // clear what must start at zero, then stage the caller's vectors
    const size_t nb = (size_t)n * sizeof(double);
    bool ok = cudaMemsetAsync(base + kOffSync, 0, 512, s) == cudaSuccess &&
              cudaMemsetAsync(base + kOffX, 0, kHaloed, s) == cudaSuccess &&
              cudaMemsetAsync(base + kOffZ, 0, kHaloed, s) == cudaSuccess &&
              cudaMemsetAsync(base + kOffZp, 0, kHaloed, s) == cudaSuccess &&
              cudaMemcpyAsync(base + kOffTabA, ta, sizeof(double) * ncls * no, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(base + kOffTabM, tm, sizeof(double) * ncls * no, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(base + kOffCls, cls, (size_t)n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(z, d_z, nb, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(x, d_x, nb, cudaMemcpyDeviceToDevice, s) == cudaSuccess;
    if (ok) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(blocks);
        lc.blockDim = dim3(512);
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        ok = cudaLaunchKernelEx(&lc, kernel, a) == cudaSuccess &&
             cudaMemcpyAsync(d_x, x, nb, cudaMemcpyDeviceToDevice, s) == cudaSuccess;
    }
    int host_words[3] = {0, 0, 0};
    ok = ok && cudaMemcpyAsync(host_words, words, sizeof(host_words), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (iterations) *iterations = host_words[2];
    const int bits = host_words[0];
    if (bits & kStatusBarrierTimeout) return CG_ERR_TIMEOUT;
    if (bits & kStatusNaN) return CG_ERR_NAN;
    if (bits & kStatusCgDiverged) return CG_ERR_CG_DIVERGED;
    if (bits & kStatusCgMaxIt) return CG_ERR_CG_MAXIT;
    return CG_OK;
}
