// cg_part_*: one rank's share of a slab monodomain tissue for a multi-GPU run, one
// process per GPU.  Rows (nodes) are owned in contiguous ranges as PETSc's
// PETSC_DECIDE split gives them to Chaste's DistributedVectorFactory
// (global/src/parallel/DistributedVectorFactory.cpp:44-64; local size
// n/world + (rank < n % world)).  With ConstructRegularSlabMesh's numbering
// ((k*NY + j)*NX + i) a contiguous range is a block of z-planes, and every stencil
// neighbour of an owned row lies within H = NX*NY + NX + 1 rows, so a rank keeps its
// vectors with H halo rows on each side and exchanges, before each operator
// application, the H rows next to each neighbour.
//
// The ODE step is local.  The diffusion solve is PETSc's CG with Jacobi as
// cg_fp64_kernel runs it, split at its reductions into phases the caller sequences:
// each phase kernel returns this rank's partial sums, the caller all-reduces them
// across ranks (NCCL between GPUs, gloo in host tests) and passes the scalars to the
// next phase; halos move through cg_part_halo_pack / _unpack (device or host
// buffers; the copies use the unified address space).  The host driver is
// chaste_b200/partition.py.  FP64 and Jacobi / no preconditioner only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/chaste_gpu.h"
#include "host/assemble.h"
#include "kernels/cg.cuh"
#include "kernels/ode.cuh"

using namespace chb;

namespace {

constexpr int kPartThreads = 256;

struct PartArgs {
    SlabOp slab;
    int nloc;          // owned rows
    int lo;            // first owned global row
    int halo;          // H
    const uint8_t* cls;   // class of each owned row
    double* x;         // haloed: entry H + i is owned row i
    double* z;         // haloed RHS term (ODE output)
    double* zp;        // haloed preconditioned residual
    double* r;
    double* p;
    double* q;
    double* b;
    double* partials;  // blocks x 4
    int pc;            // 1 Jacobi
    int diag_slot;
};

__device__ __forceinline__ double part_row(const PartArgs& a, const SlabShared<double>& sh, int c, int i,
                                           const double* x, bool mass) {
    const double* coef = mass ? (c == a.slab.interior ? a.slab.im : &sh.m[c * a.slab.n_off])
                              : (c == a.slab.interior ? a.slab.ia : &sh.a[c * a.slab.n_off]);
    double acc = 0.0;
    for (int o = 0; o < a.slab.n_off; ++o) acc += coef[o] * x[a.halo + i + a.slab.off[o]];
    return acc;
}

// Block sums of up to 4 values into partials[blockIdx][0..3] (fixed order).
__device__ __forceinline__ void block_sums(double (&v)[4], double* partials) {
    __shared__ double s[kPartThreads / 32][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) s[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int j = 0; j < kPartThreads / 32; ++j) t += s[j][threadIdx.x];
        partials[blockIdx.x * 4 + threadIdx.x] = t;
    }
}

// phase 0: b = M z, r = b - A x, zp = B r; sums |b|, |B b|^2, |B r|^2, (r, B r)
// phase 1: zero guess (tiny right-hand side): x = 0, r = b, zp = B b; sums |B b|^2, (b, B b)
// phase 2: q = A zp + bc q, p = zp + bc p (bc = s[0], s[1] != 0 on the first iteration); sum (p, q)
// phase 3: x += alpha p, r -= alpha q, zp = B r (alpha = s[0]); sums |zp|^2, (zp, r)
__global__ void __launch_bounds__(kPartThreads) part_phase_kernel(PartArgs a, int phase, double s0, double s1) {
    __shared__ SlabShared<double> sh;
    slab_load_shared<double>(a.slab, sh, a.diag_slot);
    double v[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nloc; i += gridDim.x * blockDim.x) {
        const int c = a.cls[i];
        const double d = a.pc ? sh.dinv[c] : 1.0;
        const int h = a.halo + i;
        if (phase == 0) {
            const double b = part_row(a, sh, c, i, a.z, true);
            const double rr = b - part_row(a, sh, c, i, a.x, false);
            const double w = d * b, zz = d * rr;
            a.b[i] = b;
            a.r[i] = rr;
            a.zp[h] = zz;
            v[0] += fabs(b);
            v[1] += w * w;
            v[2] += zz * zz;
            v[3] += rr * zz;
        } else if (phase == 1) {
            const double b = a.b[i], zz = d * b;
            a.x[h] = 0.0;
            a.r[i] = b;
            a.zp[h] = zz;
            v[0] += zz * zz;
            v[1] += b * zz;
        } else if (phase == 2) {
            const double az = part_row(a, sh, c, i, a.zp, false);
            const bool first = s1 != 0.0;
            const double qi = first ? az : az + s0 * a.q[i];
            const double pi = first ? a.zp[h] : a.zp[h] + s0 * a.p[i];
            a.q[i] = qi;
            a.p[i] = pi;
            v[0] += pi * qi;
        } else {
            a.x[h] += s0 * a.p[i];
            const double rr = a.r[i] - s0 * a.q[i];
            a.r[i] = rr;
            const double zz = d * rr;
            a.zp[h] = zz;
            v[0] += zz * zz;
            v[1] += zz * rr;
        }
    }
    block_sums(v, a.partials);
}

// Sum of the block partials in block order (one block; thread k sums value k).
__global__ void part_sum_kernel(const double* partials, int blocks, double* out) {
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int j = 0; j < blocks; ++j) t += partials[j * 4 + threadIdx.x];
        out[threadIdx.x] = t;
    }
}

}  // namespace

struct cg_part {
    cg_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    SlabGrid grid;
    SlabStencil st;
    int n = 0, lo = 0, hi = 0, halo = 0, nloc = 0;
    int interior = 0, diag_slot = -1, blocks = 1, ode_blocks = 1;
    int n_states = 0, n_params = 0;
    std::vector<void*> owned;
    double *x = nullptr, *z = nullptr, *zp = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *b = nullptr;
    double *partials = nullptr, *sums = nullptr, *act = nullptr, *atab = nullptr, *mtab = nullptr;
    uint8_t *cls = nullptr, *stim_id = nullptr, *pset = nullptr;
    void* states = nullptr;
    double* iion = nullptr;
    double* params = nullptr;
    DevStimulus* stims = nullptr;
    long long* step = nullptr;
    int* status = nullptr;
    bool have_cells = false;
    ~cg_part() {
        for (void* v : owned) cudaFree(v);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

template <typename P>
int palloc(cg_part* c, P** p, size_t bytes) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(bytes, 16)) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_NOMEM;
    }
    c->owned.push_back(q);
    if (cudaMemset(q, 0, std::max<size_t>(bytes, 16)) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    *p = reinterpret_cast<P*>(q);
    return CG_OK;
}

#define PART_TRY(x)                   \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != CG_OK) return rc_; \
    } while (0)
#define PART_CUDA(call)                  \
    do {                                 \
        if ((call) != cudaSuccess) {     \
            cudaGetLastError();          \
            return CG_ERR_CUDA;          \
        }                                \
    } while (0)

PartArgs part_args(const cg_part* c) {
    PartArgs a;
    std::memset(&a, 0, sizeof(a));
    const SlabStencil& st = c->st;
    a.slab.n_off = st.n_offsets;
    a.slab.n_cls = st.n_classes;
    a.slab.interior = c->interior;
    for (int o = 0; o < st.n_offsets; ++o) {
        a.slab.off[o] = st.offsets[o];
        a.slab.ia[o] = st.a[(size_t)c->interior * st.n_offsets + o];
        a.slab.im[o] = st.m[(size_t)c->interior * st.n_offsets + o];
    }
    a.slab.a_tab = c->atab;
    a.slab.m_tab = c->mtab;
    a.slab.a_tab32 = nullptr;
    a.slab.m_tab32 = nullptr;
    a.nloc = c->nloc;
    a.lo = c->lo;
    a.halo = c->halo;
    a.cls = c->cls;
    a.x = c->x;
    a.z = c->z;
    a.zp = c->zp;
    a.r = c->r;
    a.p = c->p;
    a.q = c->q;
    a.b = c->b;
    a.partials = c->partials;
    a.pc = c->cfg.ksp_preconditioner == CG_PC_JACOBI ? 1 : 0;
    a.diag_slot = c->diag_slot;
    return a;
}

double* haloed(cg_part* c, int which) {
    return which == 0 ? c->x : (which == 1 ? c->z : (which == 2 ? c->zp : nullptr));
}

}  // namespace

extern "C" {

int cg_part_create(const cg_config* cfg, int dim, double h, double width, double height, double depth,
                   const double* sigma, int rank, int world, cg_part** out) {
    if (!cfg || !sigma || !out || world < 1 || rank < 0 || rank >= world) return CG_ERR_ARG;
    *out = nullptr;
    if (cfg->precision != CG_PRECISION_FP64) return CG_ERR_UNSUPPORTED;
    if (cfg->ksp_preconditioner != CG_PC_JACOBI && cfg->ksp_preconditioner != CG_PC_NONE) return CG_ERR_UNSUPPORTED;
    if (cfg->solver != CG_SOLVER_MONODOMAIN || cfg->use_state_variable_interpolation) return CG_ERR_UNSUPPORTED;
    if (cfg->model != CG_MODEL_LR91 && cfg->model != CG_MODEL_TT06) return CG_ERR_ARG;
    if (cfg->ode_method < CG_ODE_FORWARD_EULER || cfg->ode_method > CG_ODE_GRL2) return CG_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return CG_ERR_ARG;
    cg_part* c = new (std::nothrow) cg_part();
    if (!c) return CG_ERR_NOMEM;
    c->cfg = *cfg;
    if (c->cfg.max_iterations <= 0) c->cfg.max_iterations = 10000;
    c->device = cfg->device;
    auto fail = [&](int rc) {
        delete c;
        return rc;
    };
    if (!slab_grid(dim, h, width, height, depth, c->grid) || c->grid.nodes() > (1LL << 31) - 1) return fail(CG_ERR_ARG);
    if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return fail(CG_ERR_CUDA);
    }
    // the global operator's class rows (every rank assembles the same global slab)
    std::vector<double> xyz;
    std::vector<int> conn;
    slab_mesh(c->grid, xyz, conn);
    const int ne = (int)(conn.size() / (dim + 1));
    std::vector<double> sig((size_t)ne * dim);
    for (int e = 0; e < ne; ++e)
        for (int s = 0; s < dim; ++s) sig[(size_t)e * dim + s] = sigma[s];
    c->n = (int)c->grid.nodes();
    HostCsr csr;
    const double mass_scale = cfg->surface_area_to_volume_ratio * cfg->capacitance / cfg->pde_time_step;
    if (!assemble(dim, c->n, xyz.data(), ne, conn.data(), sig.data(), mass_scale, cfg->use_mass_lumping != 0, csr) ||
        !build_slab_stencil(c->grid, csr, c->st))
        return fail(CG_ERR_ARG);
    // PETSc's PETSC_DECIDE split of n rows over world ranks
    const int base = c->n / world, extra = c->n % world;
    c->lo = rank * base + std::min(rank, extra);
    c->hi = c->lo + base + (rank < extra ? 1 : 0);
    c->nloc = c->hi - c->lo;
    int far = 0;
    for (int o = 0; o < c->st.n_offsets; ++o) far = std::max(far, std::abs(c->st.offsets[o]));
    c->halo = far;
    if (world > 1 && c->nloc < c->halo) return fail(CG_ERR_UNSUPPORTED);   // a neighbour's rows within reach only
    std::vector<uint8_t> cls(c->nloc);
    std::vector<long long> count(c->st.n_classes, 0);
    const int NX = c->grid.NX(), NY = c->grid.NY();
    for (int g = 0; g < c->n; ++g) {
        const int i = g % NX, j = (g / NX) % NY, k = g / (NX * NY);
        const int cl = slab_class(c->grid, i, j, k);
        count[cl]++;
        if (g >= c->lo && g < c->hi) cls[g - c->lo] = (uint8_t)cl;
    }
    c->interior = (int)(std::max_element(count.begin(), count.end()) - count.begin());
    for (int o = 0; o < c->st.n_offsets; ++o)
        if (c->st.offsets[o] == 0) c->diag_slot = o;
    if (c->diag_slot < 0) return fail(CG_ERR_ARG);
    const size_t nh = (size_t)c->nloc + 2 * (size_t)c->halo;
    const size_t tab = (size_t)c->st.n_classes * c->st.n_offsets;
    int rc = CG_OK;
    if ((rc = palloc(c, &c->x, nh * 8)) || (rc = palloc(c, &c->z, nh * 8)) || (rc = palloc(c, &c->zp, nh * 8)) ||
        (rc = palloc(c, &c->r, (size_t)c->nloc * 8)) || (rc = palloc(c, &c->p, (size_t)c->nloc * 8)) ||
        (rc = palloc(c, &c->q, (size_t)c->nloc * 8)) || (rc = palloc(c, &c->b, (size_t)c->nloc * 8)) ||
        (rc = palloc(c, &c->atab, tab * 8)) || (rc = palloc(c, &c->mtab, tab * 8)) ||
        (rc = palloc(c, &c->cls, (size_t)c->nloc)) || (rc = palloc(c, &c->sums, 4 * 8)) ||
        (rc = palloc(c, &c->step, sizeof(long long))) || (rc = palloc(c, &c->status, sizeof(int))))
        return fail(rc);
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    c->blocks = (int)std::max(1LL, std::min(((long long)c->nloc + kPartThreads - 1) / kPartThreads, (long long)sms * 8));
    c->ode_blocks = (int)std::max(1LL, std::min(((long long)c->nloc + 255) / 256, (long long)sms * 16));
    if ((rc = palloc(c, &c->partials, (size_t)c->blocks * 4 * 8))) return fail(rc);
    if (cudaMemcpy(c->atab, c->st.a.data(), tab * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->mtab, c->st.m.data(), tab * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->cls, cls.data(), cls.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return fail(CG_ERR_CUDA);
    }
    c->n_states = cfg->model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumStates : LuoRudy1991::kNumStates;
    c->n_params = cfg->model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumParams : LuoRudy1991::kNumParams;
    *out = c;
    return CG_OK;
}

int cg_part_rows(const cg_part* c, int* lo, int* hi, int* halo, int* n_global) {
    if (!c) return CG_ERR_ARG;
    if (lo) *lo = c->lo;
    if (hi) *hi = c->hi;
    if (halo) *halo = c->halo;
    if (n_global) *n_global = c->n;
    return CG_OK;
}

int cg_part_set_cells(cg_part* c, const double* init_states, const int* param_set, const double* param_table,
                      int n_param_sets) {
    if (!c) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    const int S = c->n_states, P = c->n_params, nl = c->nloc;
    const double* y0 = c->cfg.model == CG_MODEL_TT06 ? TenTusscher2006Epi::kInitialStates : LuoRudy1991::kInitialStates;
    if (!c->states) {
        double* s = nullptr;
        PART_TRY(palloc(c, &s, (size_t)(S - 1) * nl * 8));
        c->states = s;
        PART_TRY(palloc(c, &c->iion, (size_t)nl * 8));
        PART_TRY(palloc(c, &c->act, (size_t)nl * 8));
        PART_TRY(palloc(c, &c->stim_id, (size_t)nl));
        PART_TRY(palloc(c, &c->stims, 256 * sizeof(DevStimulus)));
        PART_CUDA(cudaMemset(c->stim_id, 0xFF, (size_t)nl));
    }
    std::vector<double> soa((size_t)(S - 1) * nl), v(nl), act(nl, -1.0);
    for (int i = 0; i < nl; ++i) {
        const double* y = init_states ? init_states + (size_t)(c->lo + i) * S : y0;
        v[i] = y[0];
        for (int k = 1; k < S; ++k) soa[(size_t)(k - 1) * nl + i] = y[k];
    }
    PART_CUDA(cudaMemcpy(c->states, soa.data(), soa.size() * 8, cudaMemcpyHostToDevice));
    PART_CUDA(cudaMemcpy(c->x + c->halo, v.data(), (size_t)nl * 8, cudaMemcpyHostToDevice));
    PART_CUDA(cudaMemcpy(c->act, act.data(), (size_t)nl * 8, cudaMemcpyHostToDevice));
    if (param_set && param_table && n_param_sets > 0) {
        if (n_param_sets > 255) return CG_ERR_ARG;
        std::vector<uint8_t> ps(nl);
        for (int i = 0; i < nl; ++i) {
            const int s = param_set[c->lo + i];
            if (s < 0 || s >= n_param_sets) return CG_ERR_ARG;
            ps[i] = (uint8_t)s;
        }
        if (!c->pset) PART_TRY(palloc(c, &c->pset, (size_t)nl));
        double* tabp = nullptr;
        PART_TRY(palloc(c, &tabp, (size_t)n_param_sets * P * 8));
        c->params = tabp;
        PART_CUDA(cudaMemcpy(c->pset, ps.data(), (size_t)nl, cudaMemcpyHostToDevice));
        PART_CUDA(cudaMemcpy(c->params, param_table, (size_t)n_param_sets * P * 8, cudaMemcpyHostToDevice));
    } else {
        c->pset = nullptr;
        c->params = nullptr;
    }
    PART_CUDA(cudaMemset(c->step, 0, sizeof(long long)));
    PART_CUDA(cudaMemset(c->status, 0, sizeof(int)));
    c->have_cells = true;
    return CG_OK;
}

int cg_part_set_stimulus(cg_part* c, const int* stim_id, const cg_stimulus* stims, int n_stims) {
    if (!c || n_stims < 0 || n_stims > 255 || (n_stims > 0 && (!stims || !stim_id))) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    PART_CUDA(cudaSetDevice(c->device));
    std::vector<uint8_t> ids(c->nloc, 0xFF);
    for (int i = 0; i < c->nloc && stim_id; ++i) {
        const int s = stim_id[c->lo + i];
        if (s >= n_stims) return CG_ERR_ARG;
        if (s >= 0) ids[i] = (uint8_t)s;
    }
    std::vector<DevStimulus> d(std::max(1, n_stims));
    for (int k = 0; k < n_stims; ++k) {
        const cg_stimulus& s = stims[k];
        if (s.kind < CG_STIM_NONE || s.kind > CG_STIM_REGULAR || (s.kind == CG_STIM_REGULAR && !(s.period > 0)))
            return CG_ERR_ARG;
        // duration padding of the reference constructors (SimpleStimulus.cpp:50, RegularStimulus.cpp:55)
        d[k] = DevStimulus{s.kind, s.magnitude,
                           s.kind == CG_STIM_SIMPLE ? s.duration + (s.duration + s.start) * DBL_EPSILON
                                                    : (s.kind == CG_STIM_REGULAR ? s.duration + s.period * DBL_EPSILON : 0.0),
                           s.start, s.period, s.stop};
    }
    PART_CUDA(cudaMemcpy(c->stim_id, ids.data(), ids.size(), cudaMemcpyHostToDevice));
    PART_CUDA(cudaMemcpy(c->stims, d.data(), d.size() * sizeof(DevStimulus), cudaMemcpyHostToDevice));
    return CG_OK;
}

int cg_part_ode(cg_part* c) {
    if (!c) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    PART_CUDA(cudaSetDevice(c->device));
    OdeArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.n = c->nloc;
    a.lo = 0;
    a.hi = c->nloc;
    a.V = c->x + c->halo;
    a.vprev = nullptr;
    a.half = 0;
    a.v_in = nullptr;
    a.states = (double*)c->states;
    a.iion = c->iion;
    a.zrhs = c->z + c->halo;
    a.stim_id = c->stim_id;
    a.stims = c->stims;
    a.pset = c->pset;
    a.params = c->params;
    a.step = c->step;
    a.status = c->status;
    a.dt_ode = c->cfg.ode_time_step;
    a.dt_pde = c->cfg.pde_time_step;
    a.am = c->cfg.surface_area_to_volume_ratio;
    a.cm = c->cfg.capacitance;
    a.check_range = c->cfg.check_state_ranges;
    a.act = c->act;
    a.act_threshold = c->cfg.activation_threshold;
    const bool tt = c->cfg.model == CG_MODEL_TT06;
    const int m = c->cfg.ode_method;
// c->ode_blocks counts 256-thread blocks; the kernel's own block shape keeps that thread budget
#define PART_ODE(M, METHOD)                                                                    \
    ode_kernel<M, double, METHOD><<<c->ode_blocks * 256 / OdeShape<M, double, METHOD>::kThreads, \
                                    OdeShape<M, double, METHOD>::kThreads, 0, c->stream>>>(a)
    if (tt) {
        if (m == CG_ODE_RUSH_LARSEN) PART_ODE(TenTusscher2006Epi, 1);
        else if (m == CG_ODE_BACKWARD_EULER) PART_ODE(TenTusscher2006Epi, 2);
        else if (m == CG_ODE_GRL1) PART_ODE(TenTusscher2006Epi, 3);
        else if (m == CG_ODE_GRL2) PART_ODE(TenTusscher2006Epi, 4);
        else PART_ODE(TenTusscher2006Epi, 0);
    } else {
        if (m == CG_ODE_RUSH_LARSEN) PART_ODE(LuoRudy1991, 1);
        else if (m == CG_ODE_BACKWARD_EULER) PART_ODE(LuoRudy1991, 2);
        else if (m == CG_ODE_GRL1) PART_ODE(LuoRudy1991, 3);
        else if (m == CG_ODE_GRL2) PART_ODE(LuoRudy1991, 4);
        else PART_ODE(LuoRudy1991, 0);
    }
#undef PART_ODE
    PART_CUDA(cudaGetLastError());
    PART_CUDA(cudaStreamSynchronize(c->stream));
    int bits = 0;
    PART_CUDA(cudaMemcpy(&bits, c->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (bits & kStatusNaN) return CG_ERR_NAN;
    if (bits & kStatusStateRange) return CG_ERR_STATE_RANGE;
    return CG_OK;
}

int cg_part_halo_pack(cg_part* c, int which, void* lo_out, void* hi_out) {
    if (!c) return CG_ERR_ARG;
    double* v = haloed(c, which);
    if (!v) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->halo * 8;
    if (lo_out) PART_CUDA(cudaMemcpyAsync(lo_out, v + c->halo, bytes, cudaMemcpyDefault, c->stream));
    if (hi_out) PART_CUDA(cudaMemcpyAsync(hi_out, v + c->nloc, bytes, cudaMemcpyDefault, c->stream));
    PART_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

int cg_part_halo_unpack(cg_part* c, int which, const void* lo_in, const void* hi_in) {
    if (!c) return CG_ERR_ARG;
    double* v = haloed(c, which);
    if (!v) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->halo * 8;
    if (lo_in) PART_CUDA(cudaMemcpyAsync(v, lo_in, bytes, cudaMemcpyDefault, c->stream));
    if (hi_in) PART_CUDA(cudaMemcpyAsync(v + c->halo + c->nloc, hi_in, bytes, cudaMemcpyDefault, c->stream));
    PART_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

int cg_part_cg_phase(cg_part* c, int phase, const double* scalars, double* sums) {
    if (!c || phase < 0 || phase > 3 || !sums) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    const PartArgs a = part_args(c);
    const double s0 = scalars ? scalars[0] : 0.0, s1 = scalars ? scalars[1] : 0.0;
    part_phase_kernel<<<c->blocks, kPartThreads, 0, c->stream>>>(a, phase, s0, s1);
    part_sum_kernel<<<1, 32, 0, c->stream>>>(c->partials, c->blocks, c->sums);
    PART_CUDA(cudaGetLastError());
    PART_CUDA(cudaMemcpyAsync(sums, c->sums, 4 * 8, cudaMemcpyDeviceToHost, c->stream));
    PART_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

int cg_part_finish_step(cg_part* c) {
    if (!c) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    long long s = 0;
    PART_CUDA(cudaMemcpy(&s, c->step, sizeof(long long), cudaMemcpyDeviceToHost));
    s++;
    PART_CUDA(cudaMemcpy(c->step, &s, sizeof(long long), cudaMemcpyHostToDevice));
    return CG_OK;
}

int cg_part_get_voltage(cg_part* c, double* v) {
    if (!c || !v) return CG_ERR_ARG;
    PART_CUDA(cudaSetDevice(c->device));
    PART_CUDA(cudaMemcpy(v, c->x + c->halo, (size_t)c->nloc * 8, cudaMemcpyDeviceToHost));
    return CG_OK;
}

int cg_part_config(const cg_part* c, cg_config* cfg) {
    if (!c || !cfg) return CG_ERR_ARG;
    *cfg = c->cfg;
    return CG_OK;
}

int cg_part_destroy(cg_part* c) {
    if (!c) return CG_ERR_ARG;
    cudaSetDevice(c->device);
    delete c;
    return CG_OK;
}

}  // extern "C"
