// libchastegpu: the C-ABI of include/chaste_gpu.h.  Owns device memory,
// launches the ODE and CG kernels and captures one PDE step as a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <climits>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/chaste_gpu.h"
#include "host/assemble.h"
#include "kernels/cg.cuh"
#include "kernels/cg_bidomain.cuh"
#include "kernels/cg_ilu.cuh"
#include "kernels/cg_mixed.cuh"
#include "kernels/ode.cuh"
#include "kernels/svi.cuh"
#include "kernels/output.cuh"

using namespace chb;

namespace {

constexpr int kRing = 4096;   // iteration-count history per context
constexpr int kHostChunks = 8;   // cg_step_host: pieces of V copied in while the ODE runs on the earlier ones

constexpr int kHostGraphs = 4;   // cg_step_host calls kept as graphs (distinct buffer pairs)

// One cg_step_host call captured as a graph: its host buffers are part of it.
struct HostGraph {
    const double* in;
    double* out;
    int n_steps;
    bool keep;
    cudaGraphExec_t exec;
};

// Status word, step counter and iteration ring read back after each call, copied
// together into page-locked memory so one synchronisation covers them.
struct HostControl {
    int status;
    int pad;
    long long step;
    int ring[kRing];
};
// bjacobi solves of meshes up to this size run as one block (block barriers between
// the levels of the triangular solves); larger ones on the co-resident grid
constexpr int kIluOneBlockNodes = 65536;

struct DeviceBuffers {
    std::vector<void*> owned;
    ~DeviceBuffers() { release(); }
    void release() {
        for (void* p : owned) cudaFree(p);
        owned.clear();
    }
};

}  // namespace

struct cg_ctx {
    cg_config cfg{};
    int n_states = 0, n_params = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_dirty = true;
    DeviceBuffers mem;
    // mesh / operator
    int n = 0, dim = 0;
    bool have_mesh = false, have_cells = false;
    bool slab = false;
    SlabGrid grid;
    SlabStencil stencil;
    HostCsr csr;
    // device arrays
    double* d_V = nullptr;
    double* d_Vprev = nullptr;    // mixed precision: V of the previous step (extrapolated CG guess)
    // state-variable interpolation: element nodes, weights, node -> elements, correction
    int* d_econn = nullptr;
    double* d_ewj = nullptr;
    uint8_t* d_eflag = nullptr;
    double* d_ebuf = nullptr;
    int* d_ell = nullptr;
    double* d_corr = nullptr;
    int n_elems = 0, ell_width = 0;
    bool svi = false;
    // printing-step output: frames of V and chosen state variables (cg_output_*)
    int out_every = 0, out_max = 0, out_count = 0, out_nv = 0;
    long long out_origin = 0;
    double* d_frames = nullptr;      // out_max x out_nv x n
    int* d_out_vars = nullptr;       // out_nv (entry 0 = V)
    std::vector<double> out_times;
    double* d_act4 = nullptr;        // ActivationOutputModifier times, 4 x n
    double act4_threshold = 0.0;
    void* d_states = nullptr;     // (S-1) x n of T
    void* d_iion = nullptr;
    void* d_z = nullptr;
    double* d_act = nullptr;
    uint8_t* d_stim_id = nullptr;
    DevStimulus* d_stims = nullptr;
    uint8_t* d_pset = nullptr;
    void* d_params = nullptr;
    uint8_t* d_cls8 = nullptr;
    double *d_r = nullptr, *d_zp = nullptr, *d_p = nullptr, *d_q = nullptr;
    float *d_r32 = nullptr, *d_z32 = nullptr, *d_p32 = nullptr, *d_q32 = nullptr, *d_e32 = nullptr;
    float *d_m32a = nullptr, *d_m32b = nullptr;
    long long halo = 0;           // zero entries on both sides of stencil-read vectors
    int interior_cls = 0;
    double* d_partials = nullptr;
    GridSync* d_gs = nullptr;
    // status word, step counter and iteration ring in one device block laid out as
    // HostControl, so that one copy reads them all; d_status, d_step, d_ring point into it
    HostControl* d_ctl = nullptr;
    int* d_status = nullptr;
    long long* d_step = nullptr;
    int* d_ring = nullptr;
    int* d_refine = nullptr;
    double *d_atab = nullptr, *d_mtab = nullptr;
    float *d_atab32 = nullptr, *d_mtab32 = nullptr;
    int *d_rowptr = nullptr, *d_cols = nullptr;
    double *d_aval = nullptr, *d_mval = nullptr, *d_dinv = nullptr;
    float *d_aval32 = nullptr, *d_dinv32 = nullptr;
    // host mirrors
    std::vector<int> stim_id_host;
    std::vector<cg_stimulus> stims_host;
    // launch shapes
    int ode_blocks = 0;
    int sms = 0;            // multiprocessors of the device
    int cg_blocks = 0;
    int cg_threads = 512;   // threads per block of the persistent CG kernel
    int pipe_nodes = 0;   // > 0: mixed slab solve by cg_mixed_pipe_kernel with this many nodes per thread
    StageArgs stage{};    // its shared-memory staging of the operator input
    size_t pipe_smem = 0; // dynamic shared memory of that launch
    int diag_slot = 0;
    int xm_slot = -1, xp_slot = -1;   // stencil slots of offsets -1 and +1
    bool line_pc = false;             // the mixed slab solve uses the x-line inner preconditioner
    float2* d_line_ad = nullptr;      // its factors (a_i, 1/d_i) per node
    bool want_line = false;           // mixed slab solve asked for the x-line preconditioner
    int line_segment = 0;             // nodes per x-line segment of the factors (32 or a block)
    std::vector<uint8_t> cls_host;    // slab class of every node (kept for the factors)
    // bjacobi (ILU(0) of the whole matrix): factors, level schedules, b and B b
    bool ilu = false;
    IluArgs ilu_args{};
    size_t ilu_smem = 0;   // > 0: cg_ilu_smem_kernel with this much dynamic shared memory
    // bidomain (cg_set_bidomain_mesh): the interleaved (V, phi_e) operator B, on the host
    // for fixing phi_e nodes and on the device, and the solve's vectors
    bool bido = false;
    bool bido_nullspace = true;
    std::vector<int> b_rp, b_ci;
    std::vector<double> b_val;
    int* d_brp = nullptr;
    int* d_bci = nullptr;
    double* d_bval = nullptr;
    double* d_bdinv = nullptr;
    double* d_u = nullptr;
    double* d_bvec[4] = {};   // r, z, p, q
    int bido_blocks = 0;
    // stats
    long long steps = 0;
    long long total_iters = 0;
    int max_iters = 0;
    double ms_last = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // cg_step_host: a copy stream, one event per chunk of V, and page-locked control words
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t chunk_ev[kHostChunks] = {};
    cudaEvent_t fork_ev = nullptr;
    HostControl* h_ctl = nullptr;
    HostGraph host_graphs[kHostGraphs] = {};   // replayable calls, by their host buffers
    int host_graph_next = 0;
    bool host_call_graph = false;   // the last cg_step_host call was a graph replay
    int capture_error = 0;          // cudaError_t of the last failed capture

    bool mixed() const { return cfg.precision == CG_PRECISION_MIXED; }
    size_t real_size() const { return mixed() ? sizeof(float) : sizeof(double); }
};

namespace {

// The CUDA error behind the calling thread's last CG_ERR_CUDA (for cg_stats).
inline cudaError_t& last_cuda_error() {
    static thread_local cudaError_t e = cudaSuccess;
    return e;
}

#define CG_CUDA(call)                                 \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) {                      \
            last_cuda_error() = e_;                   \
            cudaGetLastError();                       \
            return CG_ERR_CUDA;                       \
        }                                             \
    } while (0)

#define CG_TRY(x)                     \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != CG_OK) return rc_; \
    } while (0)

template <typename P>
int dalloc(cg_ctx* c, P** p, size_t bytes);

// Allocate n entries with c->halo zeroed entries before and after; *p points at entry 0.
template <typename P>
int dalloc_haloed(cg_ctx* c, P** p, size_t n) {
    P* base = nullptr;
    const size_t tot = n + 2 * (size_t)c->halo;
    int rc = dalloc(c, &base, tot * sizeof(P));
    if (rc != 0) return rc;
    if (cudaMemset(base, 0, tot * sizeof(P)) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    *p = base + c->halo;
    return 0;
}

template <typename P>
int dalloc(cg_ctx* c, P** p, size_t bytes) {
    void* q = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&q, bytes) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_NOMEM;
    }
    c->mem.owned.push_back(q);
    *p = reinterpret_cast<P*>(q);
    return CG_OK;
}

int states_of(int model) { return model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumStates : LuoRudy1991::kNumStates; }
int params_of(int model) { return model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumParams : LuoRudy1991::kNumParams; }
const double* init_of(int model) {
    return model == CG_MODEL_TT06 ? TenTusscher2006Epi::kInitialStates : LuoRudy1991::kInitialStates;
}

int status_from_bits(int bits) {
    if (bits & kStatusBarrierTimeout) return CG_ERR_TIMEOUT;
    if (bits & kStatusNaN) return CG_ERR_NAN;
    if (bits & kStatusCgDiverged) return CG_ERR_CG_DIVERGED;
    if (bits & kStatusCgMaxIt) return CG_ERR_CG_MAXIT;
    if (bits & kStatusStateRange) return CG_ERR_STATE_RANGE;
    return CG_OK;
}

DevStimulus to_dev(const cg_stimulus& s) {
    // duration padding exactly as the reference constructors do
    DevStimulus d{};
    d.kind = s.kind;
    d.magnitude = s.magnitude;
    d.start = s.start;
    d.period = s.period;
    d.stop = s.stop;
    if (s.kind == CG_STIM_SIMPLE) d.duration = s.duration + (s.duration + s.start) * DBL_EPSILON;
    else if (s.kind == CG_STIM_REGULAR) d.duration = s.duration + s.period * DBL_EPSILON;
    else d.duration = 0.0;
    return d;
}

double host_stim(const cg_stimulus& s, double t) {
    const DevStimulus d = to_dev(s);
    if (d.kind == 1) return (d.start <= t && t <= d.duration + d.start) ? d.magnitude : 0.0;
    if (d.kind == 2) {
        if (t < d.start) return 0.0;
        const double beat = std::fmod(t - d.start, d.period);
        return (beat >= 0 && beat <= d.duration && t <= d.stop) ? d.magnitude : 0.0;
    }
    return 0.0;
}

}  // namespace

extern "C" {

void cg_default_config(cg_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->model = CG_MODEL_LR91;
    c->ode_method = CG_ODE_FORWARD_EULER;
    c->ode_time_step = 0.01;
    c->pde_time_step = 0.01;
    c->surface_area_to_volume_ratio = 1400.0;
    c->capacitance = 1.0;
    c->ksp_preconditioner = CG_PC_JACOBI;
    c->use_absolute_tolerance = 1;
    c->ksp_tolerance = 2e-4;
    c->use_mass_lumping = 0;
    c->max_iterations = 10000;
    c->precision = CG_PRECISION_FP64;
    c->device = 0;
    c->check_state_ranges = 0;
    c->activation_threshold = -40.0;
    c->mixed_inner_preconditioner = CG_INNER_PC_LINE;
}

const char* cg_status_string(int s) {
    switch (s) {
        case CG_OK: return "ok";
        case CG_ERR_ARG: return "invalid argument";
        case CG_ERR_CUDA: return "CUDA runtime error or no CUDA device";
        case CG_ERR_CG_MAXIT: return "CG reached the maximum number of iterations (KSP_DIVERGED_ITS)";
        case CG_ERR_CG_DIVERGED: return "CG diverged (KSP_DIVERGED_DTOL or indefinite matrix)";
        case CG_ERR_NAN: return "NaN or Inf in the linear solve (KSP_DIVERGED_NANORINF)";
        case CG_ERR_STATE_RANGE: return "a cell state variable left its valid range";
        case CG_ERR_ORDER: return "calls made in the wrong order";
        case CG_ERR_TIMEOUT: return "a device-side barrier timed out";
        case CG_ERR_NOMEM: return "device allocation failed";
        case CG_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

int cg_slab_mesh(int dim, double h, double width, double height, double depth, int* n_nodes, int* n_elems,
                 double* xyz, int* conn) {
    if (!n_nodes || !n_elems || dim < 1 || dim > 3) return CG_ERR_ARG;
    SlabGrid g;
    if (!slab_grid(dim, h, width, height, depth, g) || g.nodes() > INT_MAX) return CG_ERR_ARG;
    const long long ne = dim == 1 ? g.nx : (dim == 2 ? 2LL * g.nx * g.ny : 6LL * g.nx * g.ny * g.nz);
    if (ne > INT_MAX) return CG_ERR_ARG;
    *n_nodes = (int)g.nodes();
    *n_elems = (int)ne;
    if (!xyz && !conn) return CG_OK;
    std::vector<double> x;
    std::vector<int> cn;
    slab_mesh(g, x, cn);
    if (xyz) std::memcpy(xyz, x.data(), x.size() * sizeof(double));
    if (conn) std::memcpy(conn, cn.data(), cn.size() * sizeof(int));
    return CG_OK;
}

int cg_num_states(int model, int* n) {
    if (!n || (model != CG_MODEL_LR91 && model != CG_MODEL_TT06)) return CG_ERR_ARG;
    *n = states_of(model);
    return CG_OK;
}

int cg_num_params(int model, int* n) {
    if (!n || (model != CG_MODEL_LR91 && model != CG_MODEL_TT06)) return CG_ERR_ARG;
    *n = params_of(model);
    return CG_OK;
}

int cg_create(const cg_config* cfg, cg_ctx** out) {
    if (!cfg || !out) return CG_ERR_ARG;
    *out = nullptr;
    if (cfg->model != CG_MODEL_LR91 && cfg->model != CG_MODEL_TT06) return CG_ERR_ARG;
    if (cfg->ode_method < CG_ODE_FORWARD_EULER || cfg->ode_method > CG_ODE_GRL2)
        return CG_ERR_ARG;
    if (!(cfg->ode_time_step > 0) || !(cfg->pde_time_step > 0)) return CG_ERR_ARG;
    if (!(cfg->surface_area_to_volume_ratio > 0) || !(cfg->capacitance > 0)) return CG_ERR_ARG;
    if (!(cfg->ksp_tolerance > 0)) return CG_ERR_ARG;
    if (cfg->ksp_preconditioner != CG_PC_NONE && cfg->ksp_preconditioner != CG_PC_JACOBI &&
        cfg->ksp_preconditioner != CG_PC_BJACOBI)
        return CG_ERR_ARG;
    // bjacobi runs in the FP64 solve only (the mixed solve's outer test is Jacobi-preconditioned)
    if (cfg->ksp_preconditioner == CG_PC_BJACOBI && cfg->precision != CG_PRECISION_FP64) return CG_ERR_UNSUPPORTED;
    if (cfg->precision != CG_PRECISION_FP64 && cfg->precision != CG_PRECISION_MIXED) return CG_ERR_ARG;
    if (cfg->solver != CG_SOLVER_MONODOMAIN && cfg->solver != CG_SOLVER_OPERATOR_SPLITTING) return CG_ERR_ARG;
    if (cfg->use_state_variable_interpolation != 0 && cfg->use_state_variable_interpolation != 1) return CG_ERR_ARG;
    if (cfg->mixed_inner_preconditioner != CG_INNER_PC_LINE && cfg->mixed_inner_preconditioner != CG_INNER_PC_JACOBI)
        return CG_ERR_ARG;
    // Chaste's operator-splitting solver has no correction-term assembler
    if (cfg->use_state_variable_interpolation && cfg->solver == CG_SOLVER_OPERATOR_SPLITTING)
        return CG_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return CG_ERR_ARG;
    cg_ctx* c = new (std::nothrow) cg_ctx();
    if (!c) return CG_ERR_NOMEM;
    c->cfg = *cfg;
    if (c->cfg.max_iterations <= 0) c->cfg.max_iterations = 10000;
    c->n_states = states_of(cfg->model);
    c->n_params = params_of(cfg->model);
    c->device = cfg->device;
    if (cudaSetDevice(c->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return CG_ERR_CUDA;
    }
    *out = c;
    return CG_OK;
}

int cg_destroy(cg_ctx* c) {
    if (!c) return CG_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->d_frames) cudaFree(c->d_frames);
    if (c->d_out_vars) cudaFree(c->d_out_vars);
    if (c->d_act4) cudaFree(c->d_act4);
    c->mem.release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (cudaEvent_t e : c->chunk_ev)
        if (e) cudaEventDestroy(e);
    for (HostGraph& g : c->host_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- mesh --
namespace {

using CgKernel = void (*)(CgArgs);

// The CG kernel instance for this context: CSR, or the slab stencil with the
// offset count unrolled at compile time (3 in 1D, 9 in 2D, 15 in 3D).
template <bool MIXED>
CgKernel pick_cg_kernel_t(const cg_ctx* c) {
    if (!c->slab) return MIXED ? cg_mixed_kernel<false, 0> : cg_fp64_kernel<false, 0>;
    switch (c->stencil.n_offsets) {
        case 3: return MIXED ? cg_mixed_kernel<true, 3> : cg_fp64_kernel<true, 3>;
        case 7: return MIXED ? cg_mixed_kernel<true, 7> : cg_fp64_kernel<true, 7>;
        case 9: return MIXED ? cg_mixed_kernel<true, 9> : cg_fp64_kernel<true, 9>;
        case 15: return MIXED ? cg_mixed_kernel<true, 15> : cg_fp64_kernel<true, 15>;
        default: return MIXED ? cg_mixed_kernel<true, 0> : cg_fp64_kernel<true, 0>;
    }
}

template <int NOFF>
CgKernel pick_pipe_kernel(int k) {
    switch (k) {
        case 1: return cg_mixed_pipe_kernel<NOFF, 1>;
        case 2: return cg_mixed_pipe_kernel<NOFF, 2>;
        case 3: return cg_mixed_pipe_kernel<NOFF, 3>;
        default: return cg_mixed_pipe_kernel<NOFF, 4>;
    }
}

// The pipelined mixed solve, for slabs with an unrolled offset count whose
// nodes fit in registers (at most 4 per thread of the co-resident grid).
CgKernel pick_pipe(const cg_ctx* c, int k) {
    switch (c->stencil.n_offsets) {
        case 3: return pick_pipe_kernel<3>(k);
        case 7: return pick_pipe_kernel<7>(k);
        case 9: return pick_pipe_kernel<9>(k);
        case 15: return pick_pipe_kernel<15>(k);
        default: return nullptr;
    }
}

CgKernel pick_cg_kernel(const cg_ctx* c) {
    if (c->pipe_nodes > 0) return pick_pipe(c, c->pipe_nodes);
    return c->mixed() ? pick_cg_kernel_t<true>(c) : pick_cg_kernel_t<false>(c);
}

// Bands of the slab offsets for the pipelined solve's window copies: offsets
// closer than 1024 share a band (3D: one band per z plane).  False when the
// offsets need more than kMaxBands bands.
int allow_max_dynamic_smem(CgKernel k, int device) {
    int optin = 0;
    CG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    CG_CUDA(cudaFuncGetAttributes(&fa, k));
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (dyn > fa.maxDynamicSharedSizeBytes)
        CG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return CG_OK;
}

bool plan_stage(cg_ctx* c, int threads) {
    StageArgs& g = c->stage;
    g = StageArgs{};
    const SlabStencil& st = c->stencil;
    std::vector<int> offs(st.offsets, st.offsets + st.n_offsets);
    std::sort(offs.begin(), offs.end());
    int lo[kMaxBands], hi[kMaxBands], nb = 0;
    for (size_t i = 0; i < offs.size(); ++i) {
        if (nb == 0 || offs[i] - hi[nb - 1] > 1024) {
            if (nb == kMaxBands) return false;
            lo[nb] = hi[nb] = offs[i];
            nb++;
        } else {
            hi[nb - 1] = offs[i];
        }
    }
    g.n_bands = nb;
    g.halo = (int)c->halo;
    int base = 0;
    for (int b = 0; b < nb; ++b) {
        const int delta = ((lo[b] + g.halo) % 4 + 4) % 4;
        g.lo[b] = lo[b];
        g.len[b] = (delta + threads + (hi[b] - lo[b]) + 3) / 4 * 4;
        g.base[b] = base;
        base += g.len[b];
    }
    g.cap = base;
    g.alloc_len = ((long long)c->n + 2 * c->halo) / 4 * 4;
    for (int o = 0; o < st.n_offsets; ++o) {
        int b = 0;
        while (b + 1 < nb && st.offsets[o] > hi[b]) ++b;
        const int delta = ((lo[b] + g.halo) % 4 + 4) % 4;
        g.rel[o] = g.base[b] + delta + (st.offsets[o] - lo[b]);
    }
    return true;
}

int build_line_factors(cg_ctx* c, const std::vector<uint8_t>& cls, int segment);

int alloc_vectors(cg_ctx* c) {
    const size_t n = (size_t)c->n;
    CG_TRY(dalloc_haloed(c, &c->d_V, n));
    CG_TRY(dalloc_haloed(c, &c->d_zp, n));
    CG_TRY(dalloc(c, &c->d_r, n * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_p, n * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_q, n * sizeof(double)));
    if (c->mixed()) {
        CG_TRY(dalloc_haloed(c, &c->d_z32, n));
        CG_TRY(dalloc(c, &c->d_r32, n * sizeof(float)));
        CG_TRY(dalloc(c, &c->d_p32, n * sizeof(float)));
        CG_TRY(dalloc(c, &c->d_q32, n * sizeof(float)));
        CG_TRY(dalloc_haloed(c, &c->d_e32, n));
        CG_TRY(dalloc(c, &c->d_Vprev, n * sizeof(double)));
        CG_TRY(dalloc_haloed(c, &c->d_m32a, n));
        CG_TRY(dalloc_haloed(c, &c->d_m32b, n));
    }
    CG_TRY(dalloc(c, &c->d_act, n * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_gs, sizeof(GridSync)));
    CG_TRY(dalloc(c, &c->d_ctl, sizeof(HostControl)));
    c->d_status = &c->d_ctl->status;
    c->d_step = &c->d_ctl->step;
    c->d_ring = c->d_ctl->ring;
    CG_TRY(dalloc(c, &c->d_refine, sizeof(int)));
    cudaStream_t s = c->stream;
    CG_CUDA(cudaMemsetAsync(c->d_gs, 0, sizeof(GridSync), s));
    CG_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
    CG_CUDA(cudaMemsetAsync(c->d_step, 0, sizeof(long long), s));
    CG_CUDA(cudaMemsetAsync(c->d_ring, 0, kRing * sizeof(int), s));
    CG_CUDA(cudaMemsetAsync(c->d_refine, 0, sizeof(int), s));
    CG_CUDA(cudaMemsetAsync(c->d_r, 0, n * sizeof(double), s));
    CG_CUDA(cudaMemsetAsync(c->d_p, 0, n * sizeof(double), s));
    CG_CUDA(cudaMemsetAsync(c->d_q, 0, n * sizeof(double), s));
    // launch shapes: the CG kernel is cooperative, so its grid must be co-resident
    int sms = 0;
    CG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    c->sms = sms;
    int per_sm = 0;
    CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_cg_kernel(c), 512, 0));
    if (per_sm < 1) return CG_ERR_UNSUPPORTED;
    const long long want = ((long long)n + 511) / 512;
    c->cg_blocks = (int)std::max(1LL, std::min({want, (long long)per_sm * sms, (long long)kMaxGridBlocks}));
    c->cg_threads = 512;
    const int blocks_512 = c->cg_blocks;
    c->pipe_nodes = 0;
    const bool want_line = c->want_line;
    c->line_pc = want_line;
    if (c->mixed() && c->slab && pick_pipe(c, 1)) {
        // one block of kPipeThreads per SM when the slab fills every SM with them (fewer
        // arrivals per grid reduction), else blocks of 512 so small slabs still spread
        // over many SMs; nodes per thread as that grid gives
        const int pt = (long long)n >= (long long)sms * kPipeThreads ? kPipeThreads : 512;
        const long long per_sm_guess = kPipeThreads / pt;
        const long long k0 = ((long long)n + sms * per_sm_guess * pt - 1) / (sms * per_sm_guess * pt);
        if (k0 <= 4 && plan_stage(c, pt)) {
            CgKernel kern0 = pick_pipe(c, (int)k0);
            // the x-line factors live after the staged windows; without room for both
            // the inner solve keeps Jacobi
            auto smem_of = [&](long long k) {
                return (size_t)k * ((size_t)c->stage.cap + (c->line_pc ? (size_t)kLineCoef * pt : 0)) * sizeof(float);
            };
            // the dynamic shared-memory limit is a property of the kernel for the whole
            // process, so it is raised once to the device's maximum (contexts with other
            // slab sizes launch the same kernels) and each launch passes its own size
            CG_TRY(allow_max_dynamic_smem(kern0, c->device));
            int per_sm_pipe = 0;
            for (int attempt = 0; attempt < 2; ++attempt) {
                const size_t smem0 = smem_of(k0);
                per_sm_pipe = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_pipe, kern0, pt, smem0) != cudaSuccess) {
                    cudaGetLastError();
                    per_sm_pipe = 0;
                }
                if (per_sm_pipe >= 1 || !c->line_pc) break;
                c->line_pc = false;
            }
            if (per_sm_pipe >= 1) {
                const long long blocks = std::max(1LL, std::min({((long long)n + pt - 1) / pt,
                                                                  (long long)per_sm_pipe * sms,
                                                                  (long long)kMaxGridBlocks}));
                const long long k = ((long long)n + blocks * pt - 1) / (blocks * pt);
                if (k <= k0) {
                    c->pipe_nodes = (int)k;
                    c->pipe_smem = smem_of(k);
                    CG_TRY(allow_max_dynamic_smem(pick_pipe(c, (int)k), c->device));
                    c->cg_blocks = (int)blocks;
                    c->cg_threads = pt;
                }
            }
        }
    }
    // the HBM-resident mixed solve takes the x-line preconditioner whenever it is asked for;
    // both solves cut the x-lines into the 32-node segments of a warp
    if (c->pipe_nodes == 0) c->line_pc = want_line;
    if (c->line_pc) {
        CG_TRY(build_line_factors(c, c->cls_host, 32));
        std::vector<uint8_t>().swap(c->cls_host);
    }
    if (c->ilu) {
        // one block while the level sweeps are short (block barriers between levels),
        // else the co-resident grid with grid barriers
        int per_sm_ilu = 0;
        CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ilu, cg_ilu_kernel, 1024, 0));
        if (per_sm_ilu < 1) return CG_ERR_UNSUPPORTED;
        const long long want_ilu = (long long)n <= kIluOneBlockNodes ? 1 : ((long long)n + 1023) / 1024;
        c->cg_blocks = (int)std::max(1LL, std::min({want_ilu, (long long)per_sm_ilu * sms, (long long)kMaxGridBlocks}));
        c->cg_threads = 1024;
        if (c->ilu_smem > 0) {
            c->cg_blocks = 1;
            c->cg_threads = kIluSmemThreads;
        }
    }
    CG_TRY(dalloc(c, &c->d_partials,
                  (size_t)2 * std::max(blocks_512, c->cg_blocks) * kPartialStride * sizeof(double)));
    c->ode_blocks = (int)std::max(1LL, std::min(((long long)n + 255) / 256, (long long)sms * 16));
    CG_CUDA(cudaStreamSynchronize(s));
    return CG_OK;
}

// Factors of the mixed solve's x-line inner preconditioner (kernels/cg_mixed.cuh):
// T = L D L^T on each segment of `segment` nodes aligned on a multiple of it (32: the
// nodes a warp holds in one register slot or grid-stride step), T the tridiagonal x
// part of A (sub-diagonal = the coefficient of offset -1, cut at the segment start),
// in FP64; stored per node as (a_i = -T_{i,i-1} / d_{i-1}, 1 / d_i).
int build_line_factors(cg_ctx* c, const std::vector<uint8_t>& cls, int segment) {
    const SlabStencil& st = c->stencil;
    c->line_segment = segment;
    const int no = st.n_offsets;
    std::vector<float2> ad((size_t)c->n);
    double dprev = 1.0;
    for (int i = 0; i < c->n; ++i) {
        const double* row = &st.a[(size_t)cls[i] * no];
        const double di = row[c->diag_slot];
        const double lo = (i % segment == 0) ? 0.0 : row[c->xm_slot];
        const double l = lo / dprev;
        const double d = di - l * lo;
        if (!(d > 0.0)) return CG_ERR_ARG;   // A is SPD, so every pivot is positive
        ad[i] = make_float2((float)(-l), (float)(1.0 / d));
        dprev = d;
    }
    CG_TRY(dalloc(c, &c->d_line_ad, ad.size() * sizeof(float2)));
    CG_CUDA(cudaMemcpyAsync(c->d_line_ad, ad.data(), ad.size() * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

// ILU(0) of A in natural order with no pivoting, on A's own pattern -- PETSc's
// bjacobi on one process factors the single diagonal block, the whole matrix,
// with ILU(0) -- and the level schedules of its two triangular solves (a row's
// level is one more than the highest level among the rows it reads).
int setup_ilu(cg_ctx* c) {
    const HostCsr& A = c->csr;
    const int n = A.n;
    std::vector<double> lu(A.a);
    std::vector<int> diag(n);
    for (int i = 0; i < n; ++i) {
        diag[i] = A.find(i, i);
        if (diag[i] < 0) return CG_ERR_ARG;
    }
    for (int i = 1; i < n; ++i) {
        const int end = A.rowptr[i + 1];
        for (int kk = A.rowptr[i]; kk < end && A.cols[kk] < i; ++kk) {
            const int k = A.cols[kk];
            lu[kk] /= lu[diag[k]];
            const double lik = lu[kk];
            // row i -= lik * (row k right of its diagonal), on row i's pattern only
            int jj = kk + 1;
            for (int kj = diag[k] + 1; kj < A.rowptr[k + 1]; ++kj) {
                const int j = A.cols[kj];
                while (jj < end && A.cols[jj] < j) ++jj;
                if (jj < end && A.cols[jj] == j) lu[jj] -= lik * lu[kj];
            }
        }
    }
    for (int i = 0; i < n; ++i)
        if (!(lu[diag[i]] != 0.0) || !std::isfinite(lu[diag[i]])) return CG_ERR_ARG;
    auto schedule = [&](bool forward, std::vector<int>& rows, std::vector<int>& ptr) {
        std::vector<int> level(n, 0);
        int top = 0;
        for (int s = 0; s < n; ++s) {
            const int i = forward ? s : n - 1 - s;
            int l = 0;
            const int b = forward ? A.rowptr[i] : diag[i] + 1;
            const int e = forward ? diag[i] : A.rowptr[i + 1];
            for (int k = b; k < e; ++k) l = std::max(l, level[A.cols[k]] + 1);
            level[i] = l;
            top = std::max(top, l);
        }
        ptr.assign(top + 2, 0);
        for (int i = 0; i < n; ++i) ptr[level[i] + 1]++;
        for (int l = 0; l <= top; ++l) ptr[l + 1] += ptr[l];
        rows.assign(n, 0);
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < n; ++i) rows[fill[level[i]]++] = i;   // ascending rows within a level
        return top + 1;
    };
    std::vector<int> frows, fptr, brows, bptr;
    const int fl = schedule(true, frows, fptr), bl = schedule(false, brows, bptr);
    cudaStream_t s = c->stream;
    double* d_lu = nullptr;
    int *d_diag = nullptr, *d_fr = nullptr, *d_fp = nullptr, *d_br = nullptr, *d_bp = nullptr;
    CG_TRY(dalloc(c, &d_lu, lu.size() * sizeof(double)));
    CG_TRY(dalloc(c, &d_diag, n * sizeof(int)));
    CG_TRY(dalloc(c, &d_fr, n * sizeof(int)));
    CG_TRY(dalloc(c, &d_fp, fptr.size() * sizeof(int)));
    CG_TRY(dalloc(c, &d_br, n * sizeof(int)));
    CG_TRY(dalloc(c, &d_bp, bptr.size() * sizeof(int)));
    CG_TRY(dalloc(c, &c->ilu_args.bvec, n * sizeof(double)));
    CG_TRY(dalloc(c, &c->ilu_args.wvec, n * sizeof(double)));
    CG_CUDA(cudaMemcpyAsync(d_lu, lu.data(), lu.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(d_diag, diag.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(d_fr, frows.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(d_fp, fptr.data(), fptr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(d_br, brows.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(d_bp, bptr.data(), bptr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaStreamSynchronize(s));
    c->ilu_args.lu = d_lu;
    c->ilu_args.diag = d_diag;
    c->ilu_args.f_rows = d_fr;
    c->ilu_args.f_ptr = d_fp;
    c->ilu_args.f_levels = fl;
    c->ilu_args.b_rows = d_br;
    c->ilu_args.b_ptr = d_bp;
    c->ilu_args.b_levels = bl;
    c->ilu = true;
    // small meshes: the one-block solve with its vectors in shared memory, when the packed
    // rows fit (at most kIluPackE entries either side of the diagonal, levels of at most
    // kIluSmemThreads rows, at most kIluSmemLevels levels a sweep)
    c->ilu_smem = 0;
    auto widest = [](const std::vector<int>& ptr) {
        int w = 0;
        for (size_t l = 0; l + 1 < ptr.size(); ++l) w = std::max(w, ptr[l + 1] - ptr[l]);
        return w;
    };
    int most_l = 0, most_u = 0;
    for (int i = 0; i < n; ++i) {
        most_l = std::max(most_l, diag[i] - A.rowptr[i]);
        most_u = std::max(most_u, A.rowptr[i + 1] - diag[i] - 1);
    }
    if (n <= kIluSmemNodes && fl <= kIluSmemLevels && bl <= kIluSmemLevels && most_l <= kIluPackE &&
        most_u <= kIluPackE && widest(fptr) <= kIluSmemThreads && widest(bptr) <= kIluSmemThreads) {
        const int pe = std::max(most_l, most_u) <= 4 ? 4 : kIluPackE;
        const size_t slots = (size_t)n * pe;
        std::vector<int> fcnt(n), fcol(slots, 0), bcnt(n), bcol(slots, 0);
        std::vector<double> fval(slots, 0.0), bval(slots, 0.0), bdg(n);
        for (int k = 0; k < n; ++k) {
            const int i = frows[k];
            fcnt[k] = diag[i] - A.rowptr[i];
            for (int e = 0; e < fcnt[k]; ++e) {
                fcol[(size_t)k * pe + e] = A.cols[A.rowptr[i] + e];
                fval[(size_t)k * pe + e] = lu[A.rowptr[i] + e];
            }
            const int j = brows[k];
            bcnt[k] = A.rowptr[j + 1] - diag[j] - 1;
            for (int e = 0; e < bcnt[k]; ++e) {
                bcol[(size_t)k * pe + e] = A.cols[diag[j] + 1 + e];
                bval[(size_t)k * pe + e] = lu[diag[j] + 1 + e];
            }
            bdg[k] = lu[diag[j]];
        }
        int *d_fcnt = nullptr, *d_fcol = nullptr, *d_bcnt = nullptr, *d_bcol = nullptr;
        double *d_fval = nullptr, *d_bval = nullptr, *d_bdg = nullptr;
        CG_TRY(dalloc(c, &d_fcnt, n * sizeof(int)));
        CG_TRY(dalloc(c, &d_fcol, slots * sizeof(int)));
        CG_TRY(dalloc(c, &d_fval, slots * sizeof(double)));
        CG_TRY(dalloc(c, &d_bcnt, n * sizeof(int)));
        CG_TRY(dalloc(c, &d_bcol, slots * sizeof(int)));
        CG_TRY(dalloc(c, &d_bval, slots * sizeof(double)));
        CG_TRY(dalloc(c, &d_bdg, n * sizeof(double)));
        CG_CUDA(cudaMemcpyAsync(d_fcnt, fcnt.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_fcol, fcol.data(), slots * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_fval, fval.data(), slots * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_bcnt, bcnt.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_bcol, bcol.data(), slots * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_bval, bval.data(), slots * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(d_bdg, bdg.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaStreamSynchronize(s));
        c->ilu_args.fk_cnt = d_fcnt;
        c->ilu_args.fk_col = d_fcol;
        c->ilu_args.fk_val = d_fval;
        c->ilu_args.bk_cnt = d_bcnt;
        c->ilu_args.bk_col = d_bcol;
        c->ilu_args.bk_val = d_bval;
        c->ilu_args.bk_dg = d_bdg;
        c->ilu_args.pack_e = pe;
        c->ilu_args.f_warps = (widest(fptr) + 31) / 32;
        c->ilu_args.b_warps = (widest(bptr) + 31) / 32;
        auto kern = pe == 4 ? cg_ilu_smem_kernel<4> : cg_ilu_smem_kernel<kIluPackE>;
        const size_t bytes = 2 * (size_t)n * sizeof(double) + (size_t)(fl + 1 + bl + 1) * sizeof(int);
        int optin = 0;
        CG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
        cudaFuncAttributes fa;
        CG_CUDA(cudaFuncGetAttributes(&fa, kern));
        if (bytes + fa.sharedSizeBytes <= (size_t)optin) {
            CG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         optin - (int)fa.sharedSizeBytes));
            c->ilu_smem = bytes;
        }
    }
    return CG_OK;
}

int upload_operator(cg_ctx* c) {
    cudaStream_t s = c->stream;
    if (c->slab) {
        const SlabStencil& st = c->stencil;
        const size_t tab = (size_t)st.n_classes * st.n_offsets;
        CG_TRY(dalloc(c, &c->d_atab, tab * sizeof(double)));
        CG_TRY(dalloc(c, &c->d_mtab, tab * sizeof(double)));
        CG_TRY(dalloc(c, &c->d_atab32, tab * sizeof(float)));
        CG_TRY(dalloc(c, &c->d_mtab32, tab * sizeof(float)));
        std::vector<float> a32(st.a.begin(), st.a.end()), m32(st.m.begin(), st.m.end());
        CG_CUDA(cudaMemcpyAsync(c->d_atab, st.a.data(), tab * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_mtab, st.m.data(), tab * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_atab32, a32.data(), tab * sizeof(float), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_mtab32, m32.data(), tab * sizeof(float), cudaMemcpyHostToDevice, s));
        std::vector<uint8_t> cls((size_t)c->n);
        std::vector<long long> count(st.n_classes, 0);
        const int NX = c->grid.NX(), NY = c->grid.NY(), NZ = c->grid.NZ();
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j)
                for (int i = 0; i < NX; ++i) {
                    const int cl = slab_class(c->grid, i, j, k);
                    cls[((size_t)k * NY + j) * NX + i] = (uint8_t)cl;
                    count[cl]++;
                }
        c->interior_cls = (int)(std::max_element(count.begin(), count.end()) - count.begin());
        // zero halo of the stencil-read vectors: the largest offset, plus slack for
        // the float4-aligned window copies of the pipelined solve, a multiple of 4
        long long far = 0;
        for (int o = 0; o < st.n_offsets; ++o) far = std::max<long long>(far, std::abs(st.offsets[o]));
        c->halo = (far + 8 + 3) / 4 * 4;
        CG_TRY(dalloc(c, &c->d_cls8, cls.size()));
        CG_CUDA(cudaMemcpyAsync(c->d_cls8, cls.data(), cls.size(), cudaMemcpyHostToDevice, s));
        c->diag_slot = c->xm_slot = c->xp_slot = -1;
        for (int o = 0; o < st.n_offsets; ++o) {
            if (st.offsets[o] == 0) c->diag_slot = o;
            if (st.offsets[o] == -1) c->xm_slot = o;
            if (st.offsets[o] == 1) c->xp_slot = o;
        }
        if (c->diag_slot < 0) return CG_ERR_ARG;
        c->want_line = c->mixed() && c->cfg.mixed_inner_preconditioner == CG_INNER_PC_LINE && c->xm_slot >= 0;
        if (c->want_line) c->cls_host = cls;
        CG_CUDA(cudaStreamSynchronize(s));
    } else {
        const HostCsr& m = c->csr;
        const size_t nnz = m.cols.size();
        CG_TRY(dalloc(c, &c->d_rowptr, (m.n + 1) * sizeof(int)));
        CG_TRY(dalloc(c, &c->d_cols, nnz * sizeof(int)));
        CG_TRY(dalloc(c, &c->d_aval, nnz * sizeof(double)));
        CG_TRY(dalloc(c, &c->d_mval, nnz * sizeof(double)));
        CG_TRY(dalloc(c, &c->d_dinv, m.n * sizeof(double)));
        std::vector<double> dinv(m.n);
        for (int i = 0; i < m.n; ++i) {
            const int k = m.find(i, i);
            if (k < 0 || m.a[k] == 0.0) return CG_ERR_ARG;
            dinv[i] = 1.0 / m.a[k];
        }
        CG_CUDA(cudaMemcpyAsync(c->d_rowptr, m.rowptr.data(), (m.n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_cols, m.cols.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_aval, m.a.data(), nnz * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_mval, m.m.data(), nnz * sizeof(double), cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_dinv, dinv.data(), m.n * sizeof(double), cudaMemcpyHostToDevice, s));
        if (c->cfg.ksp_preconditioner == CG_PC_BJACOBI) CG_TRY(setup_ilu(c));
        std::vector<float> a32, d32;
        if (c->mixed()) {
            a32.assign(m.a.begin(), m.a.end());
            d32.assign(dinv.begin(), dinv.end());
            CG_TRY(dalloc(c, &c->d_aval32, nnz * sizeof(float)));
            CG_TRY(dalloc(c, &c->d_dinv32, m.n * sizeof(float)));
            CG_CUDA(cudaMemcpyAsync(c->d_aval32, a32.data(), nnz * sizeof(float), cudaMemcpyHostToDevice, s));
            CG_CUDA(cudaMemcpyAsync(c->d_dinv32, d32.data(), m.n * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        CG_CUDA(cudaStreamSynchronize(s));
    }
    return alloc_vectors(c);
}

// Element data for state-variable interpolation: node lists, |det J| times the
// order-2 rule's reference weight, and each node's (element, local node) entries in
// ascending element order, stored column-major and padded with -1 (ELL).
int setup_svi(cg_ctx* c, int dim, int n, const double* xyz, int n_elems, const int* conn) {
    const int nb = dim + 1;
    const double wref = dim == 1 ? 0.5 : (dim == 2 ? 1.0 / 6.0 : 1.0 / 24.0);
    std::vector<double> wj(n_elems);
    for (int e = 0; e < n_elems; ++e) {
        const double* x0 = &xyz[(size_t)conn[e * nb] * 3];
        double d[3][3] = {{0}};
        for (int a = 1; a < nb; ++a)
            for (int k = 0; k < 3; ++k) d[a - 1][k] = xyz[(size_t)conn[e * nb + a] * 3 + k] - x0[k];
        double det;
        if (dim == 1) det = d[0][0];
        else if (dim == 2) det = d[0][0] * d[1][1] - d[0][1] * d[1][0];
        else
            det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) - d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                  d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
        wj[e] = std::fabs(det) * wref;
    }
    if (n_elems > (1 << 28)) return CG_ERR_UNSUPPORTED;   // entries 4e + j stay in int
    std::vector<int> deg(n, 0);
    for (int e = 0; e < n_elems; ++e)
        for (int a = 0; a < nb; ++a) deg[conn[e * nb + a]]++;
    int width = 0;
    for (int i = 0; i < n; ++i) width = std::max(width, deg[i]);
    std::vector<int> ell((size_t)width * n, -1);
    std::fill(deg.begin(), deg.end(), 0);
    for (int e = 0; e < n_elems; ++e)
        for (int a = 0; a < nb; ++a) {
            const int i = conn[e * nb + a];
            ell[(size_t)deg[i]++ * n + i] = 4 * e + a;
        }
    cudaStream_t s = c->stream;
    CG_TRY(dalloc(c, &c->d_econn, (size_t)n_elems * nb * sizeof(int)));
    CG_TRY(dalloc(c, &c->d_ewj, (size_t)n_elems * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_eflag, (size_t)n_elems));
    CG_TRY(dalloc(c, &c->d_ebuf, (size_t)n_elems * 4 * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_ell, std::max<size_t>(1, ell.size()) * sizeof(int)));
    CG_TRY(dalloc(c, &c->d_corr, (size_t)n * sizeof(double)));
    CG_CUDA(cudaMemcpyAsync(c->d_econn, conn, (size_t)n_elems * nb * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(c->d_ewj, wj.data(), wj.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(c->d_ell, ell.data(), ell.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemsetAsync(c->d_corr, 0, (size_t)n * sizeof(double), s));
    CG_CUDA(cudaStreamSynchronize(s));
    c->n_elems = n_elems;
    c->ell_width = width;
    c->svi = true;
    return CG_OK;
}

// B's values and Jacobi inverse on the device (after assembly and after fixing nodes).
int upload_bidomain_values(cg_ctx* c) {
    const size_t n2 = 2 * (size_t)c->n;
    std::vector<double> dinv(n2);
    for (size_t r = 0; r < n2; ++r) {
        double d = 0.0;
        for (int k = c->b_rp[r]; k < c->b_rp[r + 1]; ++k)
            if (c->b_ci[k] == (int)r) d = c->b_val[k];
        if (d == 0.0) return CG_ERR_ARG;
        dinv[r] = 1.0 / d;
    }
    CG_CUDA(cudaMemcpyAsync(c->d_bval, c->b_val.data(), c->b_val.size() * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    CG_CUDA(cudaMemcpyAsync(c->d_bdinv, dinv.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    c->graph_dirty = true;
    return CG_OK;
}

// The bidomain operator B on the interleaved unknowns (BidomainAssembler.cpp:41-89):
// rows 2i and 2i+1 carry node i's pattern twice (columns 2j, 2j+1), and element e adds
// Am Cm/dt M_e + K_i,e to the V-V block, K_i,e to both off-diagonal blocks and
// K_i,e + K_e,e to the phi_e-phi_e block, in ascending element order.
int setup_bidomain(cg_ctx* c, const double* xyz, int n_elems, const int* conn, const double* sigma_i,
                   const double* sigma_e) {
    const int n = c->n, dim = c->dim, nb = dim + 1;
    const HostCsr& A = c->csr;
    c->b_rp.assign(2 * (size_t)n + 1, 0);
    for (int i = 0; i < n; ++i) {
        const int len = 2 * (A.rowptr[i + 1] - A.rowptr[i]);
        c->b_rp[2 * i + 1] = c->b_rp[2 * i] + len;
        c->b_rp[2 * i + 2] = c->b_rp[2 * i + 1] + len;
    }
    const size_t nnz = (size_t)c->b_rp[2 * n];
    c->b_ci.resize(nnz);
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < 2; ++r) {
            int q = c->b_rp[2 * i + r];
            for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
                c->b_ci[q++] = 2 * A.cols[k];
                c->b_ci[q++] = 2 * A.cols[k] + 1;
            }
        }
    c->b_val.assign(nnz, 0.0);
    // position of (node i, node j) in A's row i: B's entries follow as 2 (k - rowptr[i])
    auto at = [&](int i, int j) { return A.find(i, j) - A.rowptr[i]; };
    const double ms = c->cfg.surface_area_to_volume_ratio * c->cfg.capacitance / c->cfg.pde_time_step;
    for (int e = 0; e < n_elems; ++e) {
        double X[12], Me[16], Ki[16], Me2[16], Ke[16];
        for (int a = 0; a < nb; ++a)
            for (int s2 = 0; s2 < 3; ++s2) X[a * 3 + s2] = xyz[(size_t)conn[(size_t)e * nb + a] * 3 + s2];
        if (!element_matrices(dim, X, sigma_i + (size_t)e * dim, false, Me, Ki) ||
            !element_matrices(dim, X, sigma_e + (size_t)e * dim, false, Me2, Ke))
            return CG_ERR_ARG;
        for (int a = 0; a < nb; ++a)
            for (int b2 = 0; b2 < nb; ++b2) {
                const int i = conn[(size_t)e * nb + a], j = conn[(size_t)e * nb + b2];
                const int off = 2 * at(i, j);
                const double ki = Ki[a * nb + b2];
                c->b_val[c->b_rp[2 * i] + off] += ms * Me[a * nb + b2] + ki;
                c->b_val[c->b_rp[2 * i] + off + 1] += ki;
                c->b_val[c->b_rp[2 * i + 1] + off] += ki;
                c->b_val[c->b_rp[2 * i + 1] + off + 1] += ki + Ke[a * nb + b2];
            }
    }
    const size_t n2 = 2 * (size_t)n;
    CG_TRY(dalloc(c, &c->d_brp, (n2 + 1) * sizeof(int)));
    CG_TRY(dalloc(c, &c->d_bci, nnz * sizeof(int)));
    CG_TRY(dalloc(c, &c->d_bval, nnz * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_bdinv, n2 * sizeof(double)));
    CG_TRY(dalloc(c, &c->d_u, n2 * sizeof(double)));
    for (double*& v : c->d_bvec) CG_TRY(dalloc(c, &v, n2 * sizeof(double)));
    CG_CUDA(cudaMemsetAsync(c->d_u, 0, n2 * sizeof(double), c->stream));
    CG_CUDA(cudaMemcpyAsync(c->d_brp, c->b_rp.data(), (n2 + 1) * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CG_CUDA(cudaMemcpyAsync(c->d_bci, c->b_ci.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    // one co-resident grid of 512-thread blocks over the 2n rows
    int sms = 1, per_sm = 0;
    CG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    CG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_bidomain_kernel, 512, 0));
    if (per_sm < 1) return CG_ERR_UNSUPPORTED;
    c->bido_blocks = (int)std::max(1LL, std::min({((long long)n2 + 511) / 512, (long long)per_sm * sms,
                                                 (long long)kMaxGridBlocks}));
    CG_TRY(dalloc(c, &c->d_partials, (size_t)2 * kMaxGridBlocks * kPartialStride * sizeof(double)));
    c->bido = true;
    c->bido_nullspace = true;
    return upload_bidomain_values(c);
}

}  // namespace

extern "C" {

int cg_set_bidomain_mesh(cg_ctx* c, int n_nodes, int dim, const double* xyz, int n_elems, const int* conn,
                         const double* sigma_i, const double* sigma_e) {
    if (!c || !sigma_e) return CG_ERR_ARG;
    if (c->have_mesh) return CG_ERR_ORDER;
    if (c->mixed() || c->cfg.solver != CG_SOLVER_MONODOMAIN || c->cfg.use_state_variable_interpolation ||
        c->cfg.use_mass_lumping || c->cfg.ksp_preconditioner == CG_PC_BJACOBI)
        return CG_ERR_UNSUPPORTED;
    CG_TRY(cg_set_mesh(c, n_nodes, dim, xyz, n_elems, conn, sigma_i));
    const int rc = setup_bidomain(c, xyz, n_elems, conn, sigma_i, sigma_e);
    if (rc != CG_OK) c->have_mesh = false;
    return rc;
}

int cg_set_fixed_extracellular_nodes(cg_ctx* c, const int* nodes, int n_fixed) {
    if (!c || n_fixed < 0 || (n_fixed > 0 && !nodes)) return CG_ERR_ARG;
    if (!c->bido) return CG_ERR_ORDER;
    if (c->steps != 0 || !c->bido_nullspace) return CG_ERR_ORDER;
    for (int k = 0; k < n_fixed; ++k)
        if (nodes[k] < 0 || nodes[k] >= c->n) return CG_ERR_ARG;
    if (n_fixed == 0) return CG_OK;
    CG_CUDA(cudaSetDevice(c->device));
    // Dirichlet phi_e = 0 on a symmetric matrix: zero the row and the column, 1 on the
    // diagonal (the column's moved contribution is value x column = 0)
    std::vector<char> fixed(2 * (size_t)c->n, 0);
    for (int k = 0; k < n_fixed; ++k) fixed[2 * (size_t)nodes[k] + 1] = 1;
    for (size_t r = 0; r < fixed.size(); ++r)
        for (int k = c->b_rp[r]; k < c->b_rp[r + 1]; ++k)
            if (fixed[r] || fixed[c->b_ci[k]]) c->b_val[k] = c->b_ci[k] == (int)r ? 1.0 : 0.0;
    c->bido_nullspace = false;
    return upload_bidomain_values(c);
}

int cg_get_extracellular_potential(cg_ctx* c, double* phi_e) {
    if (!c || !phi_e) return CG_ERR_ARG;
    if (!c->bido || !c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaMemcpy2D(phi_e, sizeof(double), c->d_u + 1, 2 * sizeof(double), sizeof(double), (size_t)c->n,
                         cudaMemcpyDeviceToHost));
    return CG_OK;
}

int cg_set_mesh(cg_ctx* c, int n_nodes, int dim, const double* xyz, int n_elems, const int* conn,
                const double* sigma) {
    if (!c || !xyz || !conn || !sigma || n_nodes <= 0 || n_elems <= 0 || dim < 1 || dim > 3) return CG_ERR_ARG;
    if (c->have_mesh) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    c->n = n_nodes;
    c->dim = dim;
    c->slab = false;
    const double mass_scale = c->cfg.surface_area_to_volume_ratio * c->cfg.capacitance / c->cfg.pde_time_step;
    if (!assemble(dim, n_nodes, xyz, n_elems, conn, sigma, mass_scale, c->cfg.use_mass_lumping != 0, c->csr))
        return CG_ERR_ARG;
    CG_TRY(upload_operator(c));
    if (c->cfg.use_state_variable_interpolation) CG_TRY(setup_svi(c, dim, n_nodes, xyz, n_elems, conn));
    c->have_mesh = true;
    return CG_OK;
}

int cg_set_slab_mesh(cg_ctx* c, int dim, double h, double width, double height, double depth,
                     const double* sigma, int* n_nodes_out) {
    if (!c || !sigma) return CG_ERR_ARG;
    if (c->have_mesh) return CG_ERR_ORDER;
    SlabGrid g;
    if (!slab_grid(dim, h, width, height, depth, g)) return CG_ERR_ARG;
    if (g.nodes() > (1LL << 31) - 1) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    std::vector<double> xyz;
    std::vector<int> conn;
    slab_mesh(g, xyz, conn);
    const int n_elems = (int)(conn.size() / (dim + 1));
    std::vector<double> sig((size_t)n_elems * dim);
    for (int e = 0; e < n_elems; ++e)
        for (int s = 0; s < dim; ++s) sig[(size_t)e * dim + s] = sigma[s];
    c->n = (int)g.nodes();
    c->dim = dim;
    c->grid = g;
    const double mass_scale = c->cfg.surface_area_to_volume_ratio * c->cfg.capacitance / c->cfg.pde_time_step;
    if (!assemble(dim, c->n, xyz.data(), n_elems, conn.data(), sig.data(), mass_scale,
                  c->cfg.use_mass_lumping != 0, c->csr))
        return CG_ERR_ARG;
    // the ILU(0) factors are per row, so bjacobi keeps the assembled CSR
    c->slab = c->cfg.ksp_preconditioner != CG_PC_BJACOBI && build_slab_stencil(g, c->csr, c->stencil);
    if (c->slab) {
        HostCsr empty;
        std::swap(c->csr, empty);
    }
    CG_TRY(upload_operator(c));
    if (c->cfg.use_state_variable_interpolation)
        CG_TRY(setup_svi(c, dim, c->n, xyz.data(), n_elems, conn.data()));
    c->have_mesh = true;
    if (n_nodes_out) *n_nodes_out = c->n;
    return CG_OK;
}

int cg_num_nodes(cg_ctx* c, int* n) {
    if (!c || !n) return CG_ERR_ARG;
    if (!c->have_mesh) return CG_ERR_ORDER;
    *n = c->n;
    return CG_OK;
}

}  // extern "C"

// --------------------------------------------------------------- cells --
namespace {

int ensure_stimulus_buffers(cg_ctx* c) {
    if (c->d_stim_id) return CG_OK;
    CG_TRY(dalloc(c, &c->d_stim_id, (size_t)c->n));
    CG_TRY(dalloc(c, &c->d_stims, 256 * sizeof(DevStimulus)));
    CG_CUDA(cudaMemsetAsync(c->d_stim_id, 0xFF, (size_t)c->n, c->stream));
    CG_CUDA(cudaMemsetAsync(c->d_stims, 0, 256 * sizeof(DevStimulus), c->stream));
    c->stim_id_host.assign(c->n, -1);
    return CG_OK;
}

template <typename T>
int upload_cells_t(cg_ctx* c, const double* init, const int* pset, const double* ptab, int nsets) {
    const size_t n = (size_t)c->n;
    const int S = c->n_states, P = c->n_params;
    if (!c->d_states) {
        T* p = nullptr;
        CG_TRY(dalloc(c, &p, (size_t)(S - 1) * n * sizeof(T)));
        c->d_states = p;
        CG_TRY(dalloc(c, &p, n * sizeof(T)));
        c->d_iion = p;
        CG_TRY(dalloc_haloed(c, &p, n));
        c->d_z = p;
    }
    CG_TRY(ensure_stimulus_buffers(c));
    std::vector<T> soa((size_t)(S - 1) * n);
    std::vector<double> v(n);
    const double* y0 = init_of(c->cfg.model);
    for (size_t i = 0; i < n; ++i) {
        const double* y = init ? init + i * S : y0;
        v[i] = y[0];
        for (int k = 1; k < S; ++k) soa[(size_t)(k - 1) * n + i] = (T)y[k];
    }
    cudaStream_t s = c->stream;
    CG_CUDA(cudaMemcpyAsync(c->d_states, soa.data(), soa.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemcpyAsync(c->d_V, v.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (c->d_Vprev) CG_CUDA(cudaMemcpyAsync(c->d_Vprev, c->d_V, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CG_CUDA(cudaMemsetAsync(c->d_iion, 0, n * sizeof(T), s));
    CG_CUDA(cudaMemsetAsync(c->d_z, 0, n * sizeof(T), s));
    std::vector<uint8_t> ps;
    std::vector<T> tab;
    if (pset && ptab && nsets > 0) {
        if (nsets > 255) return CG_ERR_ARG;
        ps.resize(n);
        for (size_t i = 0; i < n; ++i) {
            if (pset[i] < 0 || pset[i] >= nsets) return CG_ERR_ARG;
            ps[i] = (uint8_t)pset[i];
        }
        tab.resize((size_t)nsets * P);
        for (size_t k = 0; k < tab.size(); ++k) tab[k] = (T)ptab[k];
        if (!c->d_pset) CG_TRY(dalloc(c, &c->d_pset, n));
        T* dp = nullptr;
        CG_TRY(dalloc(c, &dp, tab.size() * sizeof(T)));
        c->d_params = dp;
        CG_CUDA(cudaMemcpyAsync(c->d_pset, ps.data(), n, cudaMemcpyHostToDevice, s));
        CG_CUDA(cudaMemcpyAsync(c->d_params, tab.data(), tab.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    } else {
        c->d_pset = nullptr;
        c->d_params = nullptr;
    }
    std::vector<double> neg(n, -1.0);
    CG_CUDA(cudaMemcpyAsync(c->d_act, neg.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    CG_CUDA(cudaMemsetAsync(c->d_step, 0, sizeof(long long), s));
    CG_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
    CG_CUDA(cudaStreamSynchronize(s));
    c->steps = 0;
    c->total_iters = 0;
    c->max_iters = 0;
    return CG_OK;
}

// The ODE methods whose kernel can read V^n from mapped host memory (cg_step_host);
// the others copy V in first.
constexpr bool host_input_method(int method) {
    return method == CG_ODE_FORWARD_EULER || method == CG_ODE_RUSH_LARSEN;
}

// One ode_kernel launch over the nodes [a.lo, a.hi) in the kernel's block shape
// (c->ode_blocks counts 256-thread blocks, so the grid keeps the same thread budget), or
// one operator-splitting half step over every node.
template <class M, typename T, int METHOD>
void launch_ode_kernel(cg_ctx* c, const OdeArgs<T>& a) {
    if (a.half) {
        ode_half_kernel<M, T, METHOD><<<c->ode_blocks, 256, 0, c->stream>>>(a);
        return;
    }
    // small meshes: smaller blocks, so that the cells spread over every SM (each thread's
    // step is a long chain of dependent FP64 or SFU operations: SMs, not warps, set the pace)
    const long long nodes = (long long)a.hi - a.lo;
    int tpb = OdeShape<M, T, METHOD>::kThreads;
    while (tpb > 32 && (nodes + tpb - 1) / tpb < c->sms) tpb /= 2;
    const long long cap = (long long)c->ode_blocks * 256 / tpb;
    const int blocks = (int)std::max(1LL, std::min(cap, (nodes + tpb - 1) / tpb));
    if constexpr (host_input_method(METHOD)) {
        if (a.v_in) {
            ode_kernel<M, T, METHOD, true><<<blocks, tpb, 0, c->stream>>>(a);
            return;
        }
    }
    ode_kernel<M, T, METHOD><<<blocks, tpb, 0, c->stream>>>(a);
}

template <class M, typename T>
void launch_ode(cg_ctx* c, int half = 0, int lo = 0, int hi = -1, bool reset_history = false,
                const double* v_in = nullptr) {
    OdeArgs<T> a;
    a.n = c->n;
    a.lo = lo;
    a.hi = hi < 0 ? c->n : hi;
    a.reset_history = reset_history ? 1 : 0;
    a.v_in = v_in;
    a.V = c->d_V;
    // the extrapolated guess replaces V^n in place, which splitting and SVI still need
    a.vprev = (c->cfg.solver == CG_SOLVER_OPERATOR_SPLITTING || c->svi) ? nullptr : c->d_Vprev;
    a.half = half;
    a.states = (T*)c->d_states;
    a.iion = (T*)c->d_iion;
    a.zrhs = (T*)c->d_z;
    a.stim_id = c->d_stim_id;
    a.stims = c->d_stims;
    a.pset = c->d_pset;
    a.params = (const T*)c->d_params;
    a.step = c->d_step;
    a.status = c->d_status;
    a.dt_ode = c->cfg.ode_time_step;
    a.dt_pde = c->cfg.pde_time_step;
    a.am = c->cfg.surface_area_to_volume_ratio;
    a.cm = c->cfg.capacitance;
    a.check_range = c->cfg.check_state_ranges;
    a.act = c->d_act;
    a.act_threshold = c->cfg.activation_threshold;
    if (c->cfg.ode_method == CG_ODE_RUSH_LARSEN)
        launch_ode_kernel<M, T, 1>(c, a);
    else if (c->cfg.ode_method == CG_ODE_BACKWARD_EULER)
        launch_ode_kernel<M, T, 2>(c, a);
    else if (c->cfg.ode_method == CG_ODE_GRL1)
        launch_ode_kernel<M, T, 3>(c, a);
    else if (c->cfg.ode_method == CG_ODE_GRL2)
        launch_ode_kernel<M, T, 4>(c, a);
    else
        launch_ode_kernel<M, T, 0>(c, a);
}

CgArgs make_cg_args(cg_ctx* c) {
    CgArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = c->n;
    if (c->slab) {
        const SlabStencil& st = c->stencil;
        a.slab.n_off = st.n_offsets;
        a.slab.n_cls = st.n_classes;
        a.slab.interior = c->interior_cls;
        for (int o = 0; o < st.n_offsets; ++o) {
            a.slab.ia[o] = st.a[(size_t)c->interior_cls * st.n_offsets + o];
            a.slab.im[o] = st.m[(size_t)c->interior_cls * st.n_offsets + o];
            a.slab.ia32[o] = (float)a.slab.ia[o];
        }
        for (int o = 0; o < st.n_offsets; ++o) a.slab.off[o] = st.offsets[o];
        a.slab.a_tab = c->d_atab;
        a.slab.m_tab = c->d_mtab;
        a.slab.a_tab32 = c->d_atab32;
        a.slab.m_tab32 = c->d_mtab32;
    } else {
        a.csr.rowptr = c->d_rowptr;
        a.csr.cols = c->d_cols;
        a.csr.a = c->d_aval;
        a.csr.m = c->d_mval;
        a.csr.dinv = c->d_dinv;
        a.csr.a32 = c->d_aval32;
        a.csr.dinv32 = c->d_dinv32;
    }
    a.x = c->d_V;
    a.zrhs = c->mixed() ? nullptr : (const double*)c->d_z;
    a.zrhs32 = c->mixed() ? (const float*)c->d_z : nullptr;
    a.cls8 = c->d_cls8;
    a.corr = c->svi ? c->d_corr : nullptr;
    a.r = c->d_r;
    a.zp = c->d_zp;
    a.p0 = c->d_p;
    a.q = c->d_q;
    a.r32 = c->d_r32;
    a.z32 = c->d_z32;
    a.p32 = c->d_p32;
    a.q32 = c->d_q32;
    a.e32 = c->d_e32;
    a.m32a = c->d_m32a;
    a.m32b = c->d_m32b;
    a.stage = c->stage;
    a.partials = c->d_partials;
    a.gs = c->d_gs;
    a.status = c->d_status;
    a.step = c->d_step;
    a.iters_ring = c->d_ring;
    a.ring = kRing;
    a.refine_out = c->d_refine;
    // KSPSetTolerances as LinearSystem sets them (LinearSystem.cpp:584-602, 755-762)
    a.rtol = c->cfg.use_absolute_tolerance ? DBL_EPSILON : c->cfg.ksp_tolerance;
    a.abstol = c->cfg.use_absolute_tolerance ? c->cfg.ksp_tolerance : 1e-50;
    a.dtol = 1e5;
    a.maxit = c->cfg.max_iterations;
    a.pc = c->cfg.ksp_preconditioner == CG_PC_JACOBI ? 1 : 0;
    a.diag_slot = c->diag_slot;
    a.xm_slot = c->xm_slot;
    a.xp_slot = c->xp_slot;
    a.line_pc = c->line_pc ? 1 : 0;
    a.line_ad = c->d_line_ad;
    a.max_refine = 20;
    return a;
}

cudaError_t launch_cg(cg_ctx* c) {
    CgArgs a = make_cg_args(c);
    if (c->ilu) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(c->cg_blocks);
        lc.blockDim = dim3(c->cg_threads);
        lc.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        if (c->ilu_smem > 0) {
            lc.dynamicSmemBytes = c->ilu_smem;
            return cudaLaunchKernelEx(&lc, c->ilu_args.pack_e == 4 ? cg_ilu_smem_kernel<4> : cg_ilu_smem_kernel<kIluPackE>,
                                      a, c->ilu_args);
        }
        return cudaLaunchKernelEx(&lc, cg_ilu_kernel, a, c->ilu_args);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->cg_blocks);
    cfg.blockDim = dim3(c->cg_threads);
    cfg.dynamicSmemBytes = c->pipe_nodes > 0 ? c->pipe_smem : 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pick_cg_kernel(c), a);
}

// The bidomain solve: u's V entries from the voltage, then the persistent CG on B.
cudaError_t launch_bidomain(cg_ctx* c) {
    bido_copy_voltage_kernel<<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, c->d_u);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    CgArgs a = make_cg_args(c);
    BidoArgs b;
    b.n2 = 2 * c->n;
    b.rp = c->d_brp;
    b.ci = c->d_bci;
    b.val = c->d_bval;
    b.dinv = c->cfg.ksp_preconditioner == CG_PC_JACOBI ? c->d_bdinv : nullptr;
    b.u = c->d_u;
    b.r = c->d_bvec[0];
    b.z = c->d_bvec[1];
    b.p = c->d_bvec[2];
    b.q = c->d_bvec[3];
    b.nullspace = c->bido_nullspace ? 1 : 0;
    b.inv_sqrt_n = 1.0 / std::sqrt((double)c->n);
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(c->bido_blocks);
    lc.blockDim = dim3(512);
    lc.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, cg_bidomain_kernel, a, b);
}

// The diffusion solve of a step (after the ODE launch).
cudaError_t launch_solve(cg_ctx* c) { return c->bido ? launch_bidomain(c) : launch_cg(c); }

// The ODE launch of a step: the whole step with V clamped (half 0), or one half of
// the operator-splitting step including V (half 1, 2); half 0 may cover the nodes
// [lo, hi) only.
void launch_odes(cg_ctx* c, int half, int lo = 0, int hi = -1, bool reset_history = false,
                 const double* v_in = nullptr) {
    const bool tt = c->cfg.model == CG_MODEL_TT06;
    if (c->mixed()) {
        if (tt) launch_ode<TenTusscher2006Epi, float>(c, half, lo, hi, reset_history, v_in);
        else launch_ode<LuoRudy1991, float>(c, half, lo, hi, reset_history, v_in);
    } else {
        if (tt) launch_ode<TenTusscher2006Epi, double>(c, half, lo, hi, reset_history, v_in);
        else launch_ode<LuoRudy1991, double>(c, half, lo, hi, reset_history, v_in);
    }
}

bool split(const cg_ctx* c) { return c->cfg.solver == CG_SOLVER_OPERATOR_SPLITTING; }

template <class M, typename T>
void launch_svi_t(cg_ctx* c) {
    SviArgs<T> a;
    a.n = c->n;
    a.dim = c->dim;
    a.V = c->d_V;
    a.states = (const T*)c->d_states;
    a.iion = (const T*)c->d_iion;
    a.pset = c->d_pset;
    a.params = (const T*)c->d_params;
    a.n_elems = c->n_elems;
    a.econn = c->d_econn;
    a.ewj = c->d_ewj;
    a.flag = c->d_eflag;
    a.ebuf = c->d_ebuf;
    a.ell = c->d_ell;
    a.ell_width = c->ell_width;
    a.corr = c->d_corr;
    a.am = c->cfg.surface_area_to_volume_ratio;
    a.cm = c->cfg.capacitance;
    // order-2 Gaussian rules: quadrature point q has basis value qa at node big[q]
    if (c->dim == 1) {
        const double r = std::sqrt(1.0 / 3.0);
        a.qa = (r + 1.0) / 2.0, a.qb = (-r + 1.0) / 2.0;
        a.big[0] = 0, a.big[1] = 1, a.big[2] = a.big[3] = 0;
    } else if (c->dim == 2) {
        a.qa = 2.0 / 3.0, a.qb = 1.0 / 6.0;
        a.big[0] = 1, a.big[1] = 0, a.big[2] = 2, a.big[3] = 0;
    } else {
        const double sf = 1.0 / std::sqrt(5.0);
        a.qa = (1.0 + 3.0 * sf) / 4.0, a.qb = (1.0 - sf) / 4.0;
        a.big[0] = 1, a.big[1] = 2, a.big[2] = 3, a.big[3] = 0;
    }
    const int eb = (int)std::max(1LL, std::min(((long long)a.n_elems + 255) / 256, (long long)c->ode_blocks * 8));
    svi_element_kernel<M, T><<<eb, 256, 0, c->stream>>>(a);
    svi_gather_kernel<<<c->ode_blocks, 256, 0, c->stream>>>(a.n, a.ell_width, a.ell, a.flag, a.ebuf, a.corr);
}

void launch_svi(cg_ctx* c) {
    const bool tt = c->cfg.model == CG_MODEL_TT06;
    if (c->mixed()) {
        if (tt) launch_svi_t<TenTusscher2006Epi, float>(c);
        else launch_svi_t<LuoRudy1991, float>(c);
    } else {
        if (tt) launch_svi_t<TenTusscher2006Epi, double>(c);
        else launch_svi_t<LuoRudy1991, double>(c);
    }
}

// Frames the next n_steps PDE steps add, and the frame written after step s.
long long out_frames_added(const cg_ctx* c, long long n_steps) {
    if (!c->out_every) return 0;
    const long long a = c->steps - c->out_origin, b = a + n_steps;
    return b / c->out_every - a / c->out_every;
}

void launch_frame(cg_ctx* c, double t) {
    if (c->d_act4)
        activation_modifier_kernel<<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, c->act4_threshold, t,
                                                                          c->d_act4);
    c->out_times.push_back(t);
    if (c->out_max == 0) return;   // modifiers only
    double* out = c->d_frames + (size_t)c->out_count * c->out_nv * c->n;
    if (c->mixed())
        frame_kernel<float><<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, (const float*)c->d_states,
                                                                   c->d_out_vars, c->out_nv, out);
    else
        frame_kernel<double><<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, (const double*)c->d_states,
                                                                    c->d_out_vars, c->out_nv, out);
    c->out_count++;
}

void out_after_step(cg_ctx* c, long long s) {
    if (c->out_every && (s - c->out_origin) % c->out_every == 0) launch_frame(c, (double)s * c->cfg.pde_time_step);
}

cudaError_t launch_step(cg_ctx* c) {
    launch_odes(c, split(c) ? 1 : 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (c->svi) {
        launch_svi(c);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    e = launch_solve(c);
    if (e != cudaSuccess || !split(c)) return e;
    launch_odes(c, 2);
    return cudaGetLastError();
}

// Everything one cg_step_host call puts on the stream after ev0: V in (in pieces the
// first step's ODE starts on as they arrive), the steps, ev1, V out and the control
// words.  In a capture (`capture`) the copy stream forks from the captured stream and
// the steps are plain launches.
// The address through which the device reads page-locked host memory p (unified
// addressing maps it), or null for memory the device cannot read.
const double* device_view(const double* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? static_cast<const double*>(at.devicePointer) : nullptr;
}

int enqueue_host_call(cg_ctx* c, const double* v_in, int n_steps, double* v_out, int keep_history, bool capture) {
    const size_t n = (size_t)c->n;
    int k0 = 0;
    const double* v_view = v_in ? device_view(v_in) : nullptr;
    if (v_in && v_view && n_steps > 0 && !split(c) && !c->svi && host_input_method(c->cfg.ode_method)) {
        // the first step's ODE reads V^n straight from the caller's page-locked buffer
        // (over the host link, while it computes) and stores it on the device
        launch_odes(c, 0, 0, -1, keep_history == 0, v_view);
        if (cudaGetLastError() != cudaSuccess || launch_solve(c) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        out_after_step(c, c->steps + 1);
        k0 = 1;
    } else if (v_in) {
        if (n_steps > 0 && !split(c) && !c->svi) {
            CG_CUDA(cudaEventRecord(c->fork_ev, c->stream));
            CG_CUDA(cudaStreamWaitEvent(c->copy_stream, c->fork_ev, 0));
            const int per = (int)((n + kHostChunks - 1) / kHostChunks);
            for (int k = 0; k < kHostChunks; ++k) {
                const int lo = k * per, hi = (int)std::min(n, (size_t)lo + per);
                if (lo >= hi) break;
                CG_CUDA(cudaMemcpyAsync(c->d_V + lo, v_in + lo, (size_t)(hi - lo) * sizeof(double),
                                        cudaMemcpyHostToDevice, c->copy_stream));
                CG_CUDA(cudaEventRecord(c->chunk_ev[k], c->copy_stream));
                CG_CUDA(cudaStreamWaitEvent(c->stream, c->chunk_ev[k], 0));
                launch_odes(c, 0, lo, hi, keep_history == 0);
            }
            if (cudaGetLastError() != cudaSuccess || launch_solve(c) != cudaSuccess) {
                cudaGetLastError();
                return CG_ERR_CUDA;
            }
            out_after_step(c, c->steps + 1);
            k0 = 1;
        } else {
            CG_CUDA(cudaMemcpyAsync(c->d_V, v_in, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            if (!keep_history && c->d_Vprev)
                CG_CUDA(cudaMemcpyAsync(c->d_Vprev, c->d_V, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        }
    }
    for (int k = k0; k < n_steps; ++k) {
        const cudaError_t e = (c->graph && !capture) ? cudaGraphLaunch(c->graph, c->stream) : launch_step(c);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        out_after_step(c, c->steps + k + 1);
    }
    // in a capture the record must be an external one, so that each replay records it
    CG_CUDA(capture ? cudaEventRecordWithFlags(c->ev1, c->stream, cudaEventRecordExternal)
                    : cudaEventRecord(c->ev1, c->stream));
    if (v_out) CG_CUDA(cudaMemcpyAsync(v_out, c->d_V, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CG_CUDA(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(HostControl), cudaMemcpyDeviceToHost, c->stream));
    return CG_OK;
}

// NULL, or page-locked (or mapped) host memory: a copy from it can be captured.
bool pinned(const void* p) {
    if (!p) return true;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

HostGraph* add_host_graph(cg_ctx* c, const double* in, double* out, int n_steps, int keep, cudaGraphExec_t exec);

// The call captured as a graph, or null when the capture failed (the error is kept in
// capture_error and the call runs as plain launches).
HostGraph* capture_host_call(cg_ctx* c, const double* v_in, int n_steps, double* v_out, int keep_history) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    int rc = CG_OK;
    if (e == cudaSuccess) {
        rc = enqueue_host_call(c, v_in, n_steps, v_out, keep_history, true);
        const cudaError_t le = cudaGetLastError();
        e = cudaStreamEndCapture(c->stream, &graph);
        if (e == cudaSuccess && le != cudaSuccess) e = le;
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess && rc == CG_OK) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess || rc != CG_OK) {
        c->capture_error = e != cudaSuccess ? (int)e : (int)last_cuda_error();
        cudaGetLastError();
        return nullptr;
    }
    return add_host_graph(c, v_in, v_out, n_steps, keep_history, exec);
}

HostGraph* find_host_graph(cg_ctx* c, const double* in, double* out, int n_steps, int keep) {
    for (HostGraph& g : c->host_graphs)
        if (g.exec && g.in == in && g.out == out && g.n_steps == n_steps && g.keep == (keep != 0)) return &g;
    return nullptr;
}

HostGraph* add_host_graph(cg_ctx* c, const double* in, double* out, int n_steps, int keep, cudaGraphExec_t exec) {
    HostGraph& g = c->host_graphs[c->host_graph_next];
    c->host_graph_next = (c->host_graph_next + 1) % kHostGraphs;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = HostGraph{in, out, n_steps, keep != 0, exec};
    return &g;
}

void drop_host_graphs(cg_ctx* c) {
    for (HostGraph& g : c->host_graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = HostGraph{};
    }
}

// The copy stream, chunk events and page-locked control words, made on first use.
int ensure_host_path(cg_ctx* c) {
    if (c->h_ctl) return CG_OK;
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    for (cudaEvent_t& e : c->chunk_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
    if (cudaMallocHost(&c->h_ctl, sizeof(HostControl)) != cudaSuccess) {
        cudaGetLastError();
        c->h_ctl = nullptr;
        return CG_ERR_NOMEM;
    }
    return CG_OK;
}

int build_graph(cg_ctx* c) {
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    cudaError_t le = launch_step(c);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess || !g) {
        c->capture_error = (int)(le != cudaSuccess ? le : ce);
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        return CG_ERR_CUDA;
    }
    cudaError_t ie = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        c->capture_error = (int)ie;
        cudaGetLastError();
        c->graph = nullptr;
        return CG_ERR_CUDA;
    }
    return CG_OK;
}

}  // namespace

extern "C" {

int cg_set_cells(cg_ctx* c, const double* init_states, const int* param_set, const double* param_table,
                 int n_param_sets) {
    if (!c) return CG_ERR_ARG;
    if (!c->have_mesh) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    const int rc = c->mixed() ? upload_cells_t<float>(c, init_states, param_set, param_table, n_param_sets)
                              : upload_cells_t<double>(c, init_states, param_set, param_table, n_param_sets);
    if (rc != CG_OK) return rc;
    c->have_cells = true;
    c->graph_dirty = true;
    return CG_OK;
}

int cg_set_stimulus(cg_ctx* c, const int* stim_id, const cg_stimulus* stims, int n_stims) {
    if (!c || n_stims < 0 || n_stims > 255 || (n_stims > 0 && (!stims || !stim_id))) return CG_ERR_ARG;
    if (!c->have_mesh) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)c->n;
    std::vector<uint8_t> ids(n, 0xFF);
    std::vector<int> host_ids(n, -1);
    if (stim_id)
        for (size_t i = 0; i < n; ++i) {
            if (stim_id[i] >= n_stims) return CG_ERR_ARG;
            if (stim_id[i] >= 0) {
                ids[i] = (uint8_t)stim_id[i];
                host_ids[i] = stim_id[i];
            }
        }
    std::vector<DevStimulus> d(std::max(1, n_stims));
    for (int k = 0; k < n_stims; ++k) {
        if (stims[k].kind == CG_STIM_REGULAR && !(stims[k].period > 0)) return CG_ERR_ARG;
        if (stims[k].kind < CG_STIM_NONE || stims[k].kind > CG_STIM_REGULAR) return CG_ERR_ARG;
        d[k] = to_dev(stims[k]);
    }
    CG_TRY(ensure_stimulus_buffers(c));
    c->stim_id_host = host_ids;
    c->stims_host.assign(stims, stims + n_stims);
    CG_CUDA(cudaMemcpyAsync(c->d_stim_id, ids.data(), n, cudaMemcpyHostToDevice, c->stream));
    CG_CUDA(cudaMemcpyAsync(c->d_stims, d.data(), d.size() * sizeof(DevStimulus), cudaMemcpyHostToDevice, c->stream));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    c->graph_dirty = true;
    return CG_OK;
}

int cg_step(cg_ctx* c, int n_steps) { return cg_step_host(c, nullptr, n_steps, nullptr, 1); }

int cg_step_host(cg_ctx* c, const double* v_in, int n_steps, double* v_out, int keep_history) {
    if (!c || n_steps < 0) return CG_ERR_ARG;
    if (!c->have_mesh || !c->have_cells) return CG_ERR_ORDER;
    if (n_steps == 0 && !v_in && !v_out) return CG_OK;
    CG_CUDA(cudaSetDevice(c->device));
    if (c->graph_dirty) {
        if (build_graph(c) != CG_OK) c->graph = nullptr;   // plain launches instead
        c->graph_dirty = false;
        drop_host_graphs(c);   // their kernel arguments may be out of date too
    }
    if (c->out_max && c->out_count + out_frames_added(c, n_steps) > c->out_max) return CG_ERR_NOMEM;
    CG_TRY(ensure_host_path(c));
    // a call with page-locked buffers and no printing-step output is replayed from a
    // graph of the whole call (launches, copies, read-back), built on its first use
    const bool replay = (v_in || v_out) && c->out_every == 0 && pinned(v_in) && pinned(v_out);
    HostGraph* g = replay ? find_host_graph(c, v_in, v_out, n_steps, keep_history) : nullptr;
    if (replay && !g) g = capture_host_call(c, v_in, n_steps, v_out, keep_history);
    c->host_call_graph = g != nullptr;
    // the timing starts here, after the host-side lookups and any capture
    CG_CUDA(cudaEventRecord(c->ev0, c->stream));
    if (g) {
        CG_CUDA(cudaGraphLaunch(g->exec, c->stream));
    } else {
        CG_TRY(enqueue_host_call(c, v_in, n_steps, v_out, keep_history, false));
    }
    CG_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) != cudaSuccess) {
        cudaGetLastError();   // leave no error behind for the next call's launch checks
        ms = 0.0f;
    }
    c->ms_last = ms;
    HostControl* h = c->h_ctl;
    const long long dstep = h->step;
    const long long from = std::max(c->steps, dstep - kRing);
    for (long long s = from; s < dstep; ++s) {
        const int it = h->ring[s % kRing];
        c->total_iters += it;
        c->max_iters = std::max(c->max_iters, it);
    }
    c->steps = dstep;
    return status_from_bits(h->status);
}

}  // extern "C"

// ------------------------------------------------------------- getters --
namespace {

template <typename T>
int read_states_t(cg_ctx* c, double* out, int node) {
    const size_t n = (size_t)c->n;
    const int S = c->n_states;
    if (node >= 0) {
        CG_CUDA(cudaMemcpy(out, c->d_V + node, sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 1; k < S; ++k) {
            T x;
            CG_CUDA(cudaMemcpy(&x, (T*)c->d_states + (size_t)(k - 1) * n + node, sizeof(T), cudaMemcpyDeviceToHost));
            out[k] = (double)x;
        }
        return CG_OK;
    }
    std::vector<double> v(n);
    CG_CUDA(cudaMemcpy(v.data(), c->d_V, n * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<T> soa((size_t)(S - 1) * n);
    CG_CUDA(cudaMemcpy(soa.data(), c->d_states, soa.size() * sizeof(T), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
        out[i * S] = v[i];
        for (int k = 1; k < S; ++k) out[i * S + k] = (double)soa[(size_t)(k - 1) * n + i];
    }
    return CG_OK;
}

template <typename T>
int read_vec_t(const void* d, size_t n, double* out) {
    std::vector<T> h(n);
    CG_CUDA(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) out[i] = (double)h[i];
    return CG_OK;
}

struct SnapshotHeader {
    char magic[8];
    int n, n_states, model, precision;
    long long step;
    long long bytes;
};

}  // namespace

extern "C" {

int cg_get_voltage(cg_ctx* c, double* v) {
    if (!c || !v) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaMemcpy(v, c->d_V, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost));
    return CG_OK;
}

int cg_set_voltage(cg_ctx* c, const double* v) {
    if (!c || !v) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaMemcpy(c->d_V, v, (size_t)c->n * sizeof(double), cudaMemcpyHostToDevice));
    // a voltage set from outside has no history: the next guess is V itself
    if (c->d_Vprev) CG_CUDA(cudaMemcpy(c->d_Vprev, c->d_V, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToDevice));
    return CG_OK;
}

int cg_get_states(cg_ctx* c, double* states) {
    if (!c || !states) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    return c->mixed() ? read_states_t<float>(c, states, -1) : read_states_t<double>(c, states, -1);
}

int cg_get_cell_state(cg_ctx* c, int node, double* state) {
    if (!c || !state) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    if (node < 0 || node >= c->n) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    return c->mixed() ? read_states_t<float>(c, state, node) : read_states_t<double>(c, state, node);
}

int cg_get_caches(cg_ctx* c, double* iion, double* istim) {
    if (!c) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    if (iion) CG_TRY(c->mixed() ? read_vec_t<float>(c->d_iion, c->n, iion) : read_vec_t<double>(c->d_iion, c->n, iion));
    if (istim) {
        // the cache holds GetIntracellularStimulus(t_{n+1}) of the last step
        const double t = (double)c->steps * c->cfg.pde_time_step;
        for (int i = 0; i < c->n; ++i) {
            const int s = c->stim_id_host.empty() ? -1 : c->stim_id_host[i];
            istim[i] = (s >= 0 && c->steps > 0) ? host_stim(c->stims_host[s], t) : 0.0;
        }
    }
    return CG_OK;
}

int cg_get_activation_times(cg_ctx* c, double* t) {
    if (!c || !t) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    const double now = (double)c->steps * c->cfg.pde_time_step;
    activation_kernel<<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, c->d_act, c->cfg.activation_threshold, now);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaStreamSynchronize(c->stream));
    CG_CUDA(cudaMemcpy(t, c->d_act, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost));
    return CG_OK;
}

int cg_get_stats(cg_ctx* c, cg_stats* s) {
    if (!c || !s) return CG_ERR_ARG;
    std::memset(s, 0, sizeof(*s));
    s->steps = c->steps;
    s->time = (double)c->steps * c->cfg.pde_time_step;
    s->total_cg_iterations = c->total_iters;
    s->max_cg_iterations = c->max_iters;
    s->operator_kind = c->slab ? 1 : 0;
    s->ms_last_call = c->ms_last;
    s->pipelined_nodes_per_thread = c->pipe_nodes;
    s->cg_blocks = c->cg_blocks;
    s->inner_preconditioner = !c->mixed() ? -1 : (c->line_pc ? CG_INNER_PC_LINE : CG_INNER_PC_JACOBI);
    s->inner_line_segment = c->line_pc ? c->line_segment : 0;
    s->step_graph = c->graph ? 1 : 0;
    s->host_call_graph = c->host_call_graph ? 1 : 0;
    s->capture_error = c->capture_error;
    if (c->have_cells && c->steps > 0) {
        CG_CUDA(cudaSetDevice(c->device));
        CG_CUDA(cudaMemcpy(&s->last_cg_iterations, c->d_ring + ((c->steps - 1) % kRing), sizeof(int),
                           cudaMemcpyDeviceToHost));
        CG_CUDA(cudaMemcpy(&s->refinement_sweeps, c->d_refine, sizeof(int), cudaMemcpyDeviceToHost));
        CG_CUDA(cudaMemcpy(&s->status_bits, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    }
    return CG_OK;
}

int cg_apply_inner_preconditioner(cg_ctx* c, const double* x, double* y) {
    if (!c || !x || !y) return CG_ERR_ARG;
    if (!c->have_mesh) return CG_ERR_ORDER;
    if (!c->line_pc || !c->d_line_ad) return CG_ERR_UNSUPPORTED;
    CG_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)c->n;
    std::vector<float> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = (float)x[i];
    float* d = nullptr;
    if (cudaMalloc(&d, 2 * n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_NOMEM;
    }
    int rc = CG_OK;
    if (cudaMemcpyAsync(d, h.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
        rc = CG_ERR_CUDA;
    } else {
        const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)c->ode_blocks);
        line_pc_apply_kernel<<<std::max(1, blocks), 256, 0, c->stream>>>(c->n, c->d_line_ad, d, d + n);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(h.data(), d + n, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = CG_ERR_CUDA;
    }
    cudaFree(d);
    cudaGetLastError();
    if (rc == CG_OK)
        for (size_t i = 0; i < n; ++i) y[i] = (double)h[i];
    return rc;
}

int cg_get_iteration_history(cg_ctx* c, int n, int* it) {
    if (!c || !it || n < 0) return CG_ERR_ARG;
    const long long avail = std::min<long long>(c->steps, kRing);
    const long long m = std::min<long long>(n, avail);
    if (m > 0) {
        CG_CUDA(cudaSetDevice(c->device));
        std::vector<int> ring(kRing);
        CG_CUDA(cudaMemcpy(ring.data(), c->d_ring, kRing * sizeof(int), cudaMemcpyDeviceToHost));
        for (long long k = 0; k < m; ++k) it[k] = ring[(c->steps - m + k) % kRing];
    }
    for (long long k = m; k < n; ++k) it[k] = 0;
    return CG_OK;
}

int cg_snapshot_size(cg_ctx* c, size_t* bytes) {
    if (c && c->bido) return CG_ERR_UNSUPPORTED;   // the snapshot holds V and the cells, not phi_e
    if (!c || !bytes) return CG_ERR_ARG;
    if (!c->have_cells) return CG_ERR_ORDER;
    const size_t n = (size_t)c->n, w = c->real_size();
    *bytes = sizeof(SnapshotHeader) + n * sizeof(double) * 2 + (size_t)(c->n_states - 1) * n * w + 2 * n * w;
    return CG_OK;
}

int cg_snapshot(cg_ctx* c, void* buf, size_t bytes) {
    if (c && c->bido) return CG_ERR_UNSUPPORTED;   // the snapshot holds V and the cells, not phi_e
    size_t need = 0;
    CG_TRY(cg_snapshot_size(c, &need));
    if (!buf || bytes < need) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)c->n, w = c->real_size();
    SnapshotHeader h{};
    std::memcpy(h.magic, "CHBSNAP1", 8);
    h.n = c->n;
    h.n_states = c->n_states;
    h.model = c->cfg.model;
    h.precision = c->cfg.precision;
    h.step = c->steps;
    h.bytes = (long long)need;
    char* p = (char*)buf;
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    CG_CUDA(cudaMemcpy(p, c->d_V, n * sizeof(double), cudaMemcpyDeviceToHost));
    p += n * sizeof(double);
    CG_CUDA(cudaMemcpy(p, c->d_act, n * sizeof(double), cudaMemcpyDeviceToHost));
    p += n * sizeof(double);
    CG_CUDA(cudaMemcpy(p, c->d_states, (size_t)(c->n_states - 1) * n * w, cudaMemcpyDeviceToHost));
    p += (size_t)(c->n_states - 1) * n * w;
    CG_CUDA(cudaMemcpy(p, c->d_iion, n * w, cudaMemcpyDeviceToHost));
    p += n * w;
    CG_CUDA(cudaMemcpy(p, c->d_z, n * w, cudaMemcpyDeviceToHost));
    return CG_OK;
}

int cg_restore(cg_ctx* c, const void* buf, size_t bytes) {
    if (c && c->bido) return CG_ERR_UNSUPPORTED;   // the snapshot holds V and the cells, not phi_e
    size_t need = 0;
    CG_TRY(cg_snapshot_size(c, &need));
    if (!buf || bytes < need) return CG_ERR_ARG;
    SnapshotHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (std::memcmp(h.magic, "CHBSNAP1", 8) != 0 || h.n != c->n || h.n_states != c->n_states ||
        h.model != c->cfg.model || h.precision != c->cfg.precision || h.bytes != (long long)need)
        return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)c->n, w = c->real_size();
    const char* p = (const char*)buf + sizeof(h);
    CG_CUDA(cudaMemcpy(c->d_V, p, n * sizeof(double), cudaMemcpyHostToDevice));
    if (c->d_Vprev) CG_CUDA(cudaMemcpy(c->d_Vprev, c->d_V, n * sizeof(double), cudaMemcpyDeviceToDevice));
    p += n * sizeof(double);
    CG_CUDA(cudaMemcpy(c->d_act, p, n * sizeof(double), cudaMemcpyHostToDevice));
    p += n * sizeof(double);
    CG_CUDA(cudaMemcpy(c->d_states, p, (size_t)(c->n_states - 1) * n * w, cudaMemcpyHostToDevice));
    p += (size_t)(c->n_states - 1) * n * w;
    CG_CUDA(cudaMemcpy(c->d_iion, p, n * w, cudaMemcpyHostToDevice));
    p += n * w;
    CG_CUDA(cudaMemcpy(c->d_z, p, n * w, cudaMemcpyHostToDevice));
    CG_CUDA(cudaMemcpy(c->d_step, &h.step, sizeof(long long), cudaMemcpyHostToDevice));
    CG_CUDA(cudaMemset(c->d_status, 0, sizeof(int)));
    c->steps = h.step;
    return CG_OK;
}

}  // extern "C"

extern "C" int cg_step_profiled(cg_ctx* c, int n_steps, double* ms_odes, double* ms_linear) {
    if (!c || n_steps < 0) return CG_ERR_ARG;
    if (!c->have_mesh || !c->have_cells) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    cudaEvent_t e[4];
    for (auto& x : e)
        if (cudaEventCreate(&x) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
    double t_ode = 0.0, t_cg = 0.0;
    int rc = CG_OK;
    if (c->out_max && c->out_count + out_frames_added(c, n_steps) > c->out_max) rc = CG_ERR_NOMEM;
    for (int k = 0; k < n_steps && rc == CG_OK; ++k) {
        cudaEventRecord(e[0], c->stream);
        launch_odes(c, split(c) ? 1 : 0);
        cudaEventRecord(e[1], c->stream);
        if (c->svi) launch_svi(c);   // part of assembling the RHS (ASSEMBLE_RHS)
        if (cudaGetLastError() != cudaSuccess || launch_solve(c) != cudaSuccess) rc = CG_ERR_CUDA;
        cudaEventRecord(e[2], c->stream);
        if (split(c)) launch_odes(c, 2);
        cudaEventRecord(e[3], c->stream);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e[3]) != cudaSuccess) rc = CG_ERR_CUDA;
        float a = 0.f, b = 0.f, d = 0.f;
        cudaEventElapsedTime(&a, e[0], e[1]);
        cudaEventElapsedTime(&b, e[1], e[2]);
        cudaEventElapsedTime(&d, e[2], e[3]);
        t_ode += a + d;
        t_cg += b;
        out_after_step(c, c->steps + k + 1);
    }
    for (auto& x : e) cudaEventDestroy(x);
    cudaGetLastError();
    if (ms_odes) *ms_odes = t_ode;
    if (ms_linear) *ms_linear = t_cg;
    if (rc != CG_OK) return rc;
    std::vector<HostControl> hc(1);
    CG_CUDA(cudaMemcpy(hc.data(), c->d_ctl, sizeof(HostControl), cudaMemcpyDeviceToHost));
    const long long dstep = hc[0].step;
    for (long long s = std::max(c->steps, dstep - kRing); s < dstep; ++s) {
        c->total_iters += hc[0].ring[s % kRing];
        c->max_iters = std::max(c->max_iters, hc[0].ring[s % kRing]);
    }
    c->steps = dstep;
    c->ms_last = t_ode + t_cg;
    return status_from_bits(hc[0].status);
}

// -------------------------------------------------------------- output --
extern "C" {

int cg_output_configure(cg_ctx* c, int printing_steps, int max_frames, const int* state_vars, int n_state_vars) {
    if (!c || printing_steps < 0 || n_state_vars < 0 || (n_state_vars > 0 && !state_vars)) return CG_ERR_ARG;
    if (!c->have_mesh || !c->have_cells) return CG_ERR_ORDER;
    for (int k = 0; k < n_state_vars; ++k)
        if (state_vars[k] < 1 || state_vars[k] >= c->n_states) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    if (c->d_frames) cudaFree(c->d_frames);
    if (c->d_out_vars) cudaFree(c->d_out_vars);
    if (c->d_act4) cudaFree(c->d_act4);
    c->d_frames = nullptr;
    c->d_out_vars = nullptr;
    c->d_act4 = nullptr;
    c->out_every = c->out_max = c->out_count = c->out_nv = 0;
    c->out_times.clear();
    if (printing_steps == 0) return CG_OK;
    if (max_frames < 0) return CG_ERR_ARG;
    const int nv = 1 + n_state_vars;
    const size_t bytes = (size_t)std::max(max_frames, 1) * nv * c->n * sizeof(double);
    if (cudaMalloc(&c->d_frames, bytes) != cudaSuccess || cudaMalloc(&c->d_out_vars, nv * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        if (c->d_frames) cudaFree(c->d_frames);
        c->d_frames = nullptr;
        return CG_ERR_NOMEM;
    }
    std::vector<int> vars(nv, 0);
    for (int k = 0; k < n_state_vars; ++k) vars[k + 1] = state_vars[k];
    CG_CUDA(cudaMemcpyAsync(c->d_out_vars, vars.data(), nv * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    c->out_every = printing_steps;
    c->out_max = max_frames;
    c->out_nv = nv;
    c->out_origin = c->steps;
    launch_frame(c, (double)c->steps * c->cfg.pde_time_step);   // the initial condition
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

int cg_output_frames(const cg_ctx* c, int* n_frames, double* times) {
    if (!c || !n_frames) return CG_ERR_ARG;
    *n_frames = c->out_count;
    if (times) std::copy(c->out_times.begin(), c->out_times.begin() + c->out_count, times);
    return CG_OK;
}

int cg_output_activation(cg_ctx* c, double threshold) {
    if (!c) return CG_ERR_ARG;
    if (!c->out_every) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    if (!c->d_act4) {
        if (cudaMalloc(&c->d_act4, 4 * (size_t)c->n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            c->d_act4 = nullptr;
            return CG_ERR_NOMEM;
        }
    }
    std::vector<double> init(4 * (size_t)c->n, -1.0);
    CG_CUDA(cudaMemcpyAsync(c->d_act4, init.data(), init.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->act4_threshold = threshold;
    // InitialiseAtStart then the initial condition (AbstractCardiacProblem.cpp:460-464)
    activation_modifier_kernel<<<c->ode_blocks, 256, 0, c->stream>>>(c->n, c->d_V, threshold,
                                                                      (double)c->steps * c->cfg.pde_time_step, c->d_act4);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaStreamSynchronize(c->stream));
    return CG_OK;
}

int cg_output_get_activation(cg_ctx* c, double* times) {
    if (!c || !times) return CG_ERR_ARG;
    if (!c->d_act4) return CG_ERR_ORDER;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)c->n;
    std::vector<double> buf(4 * n);
    CG_CUDA(cudaMemcpy(buf.data(), c->d_act4, buf.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 4; ++k) times[i * 4 + k] = buf[k * n + i];
    return CG_OK;
}

int cg_output_fetch(cg_ctx* c, int first, int count, double* data) {
    if (!c || !data || first < 0 || count < 0 || first + count > c->out_count) return CG_ERR_ARG;
    if (count == 0) return CG_OK;
    CG_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)c->n, nv = (size_t)c->out_nv, fb = nv * n;
    CG_CUDA(cudaStreamSynchronize(c->stream));
    if (nv == 1) {
        CG_CUDA(cudaMemcpy(data, c->d_frames + (size_t)first * fb, (size_t)count * fb * sizeof(double),
                           cudaMemcpyDeviceToHost));
        return CG_OK;
    }
    // device frames are variable-major; Hdf5DataWriter's Data dataset is [time][node][variable]
    std::vector<double> buf(fb);
    for (int f = 0; f < count; ++f) {
        CG_CUDA(cudaMemcpy(buf.data(), c->d_frames + (size_t)(first + f) * fb, fb * sizeof(double),
                           cudaMemcpyDeviceToHost));
        double* out = data + (size_t)f * fb;
        for (size_t v = 0; v < nv; ++v)
            for (size_t i = 0; i < n; ++i) out[i * nv + v] = buf[v * n + i];
    }
    return CG_OK;
}

}  // extern "C"

namespace {

struct DevBuf {
    std::vector<void*> p;
    template <typename P>
    int get(P** q, size_t count) {
        void* x = nullptr;
        if (cudaMalloc(&x, std::max<size_t>(count, 1) * sizeof(P)) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_NOMEM;
        }
        p.push_back(x);
        *q = (P*)x;
        return CG_OK;
    }
    ~DevBuf() {
        for (void* x : p) cudaFree(x);
    }
};

// CellProperties over every node's stored voltage frames; device results in a.
int run_cellprops(cg_ctx* c, DevBuf& db, CellPropsArgs& a, double percentage, double threshold, int cap) {
    if (c->out_count < 1) return CG_ERR_ORDER;
    const size_t n = (size_t)c->n;
    a.n = c->n;
    a.n_frames = c->out_count;
    a.nv = c->out_nv;
    a.cap = cap;
    a.frames = c->d_frames;
    a.threshold = threshold;
    a.percentage = percentage;
    double* times = nullptr;
    CG_TRY(db.get(&times, c->out_times.size()));
    CG_CUDA(cudaMemcpyAsync(times, c->out_times.data(), c->out_times.size() * sizeof(double),
                            cudaMemcpyHostToDevice, c->stream));
    a.times = times;
    CG_TRY(db.get(&a.onset, (size_t)cap * n));
    CG_TRY(db.get(&a.rest, (size_t)cap * n));
    CG_TRY(db.get(&a.peak, (size_t)cap * n));
    CG_TRY(db.get(&a.apd, (size_t)cap * n));
    CG_TRY(db.get(&a.up_time, (size_t)cap * n));
    CG_TRY(db.get(&a.up_vel, (size_t)cap * n));
    CG_TRY(db.get(&a.n_apd, n));
    CG_TRY(db.get(&a.n_up, n));
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((n + 127) / 128, (size_t)c->ode_blocks * 2));
    cellprops_kernel<<<blocks, 128, 0, c->stream>>>(a);
    CG_CUDA(cudaGetLastError());
    return CG_OK;
}

}  // namespace

extern "C" {

int cg_output_cell_properties(cg_ctx* c, double percentage, double threshold, int max_aps, double* apd, int* n_apd,
                              double* upstroke_time, double* max_upstroke_velocity, int* n_upstroke) {
    if (!c || max_aps < 1 || !(percentage > 0.0 && percentage < 100.0)) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    DevBuf db;
    CellPropsArgs a;
    CG_TRY(run_cellprops(c, db, a, percentage, threshold, max_aps));
    const size_t n = (size_t)c->n, cells = n * max_aps;
    CG_CUDA(cudaStreamSynchronize(c->stream));
    if (apd) CG_CUDA(cudaMemcpy(apd, a.apd, cells * sizeof(double), cudaMemcpyDeviceToHost));
    if (n_apd) CG_CUDA(cudaMemcpy(n_apd, a.n_apd, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (upstroke_time) CG_CUDA(cudaMemcpy(upstroke_time, a.up_time, cells * sizeof(double), cudaMemcpyDeviceToHost));
    if (max_upstroke_velocity)
        CG_CUDA(cudaMemcpy(max_upstroke_velocity, a.up_vel, cells * sizeof(double), cudaMemcpyDeviceToHost));
    if (n_upstroke) {
        CG_CUDA(cudaMemcpy(n_upstroke, a.n_up, n * sizeof(int), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) n_upstroke[i] = std::max(1, n_upstroke[i]);   // [0] when none
    }
    return CG_OK;
}

int cg_output_conduction_velocity(cg_ctx* c, int origin, const double* distances, double threshold, int max_aps,
                                  double* cv, int* n_cv) {
    if (!c || !distances || !cv || max_aps < 1 || origin < 0 || origin >= c->n) return CG_ERR_ARG;
    CG_CUDA(cudaSetDevice(c->device));
    CG_CUDA(cudaStreamSynchronize(c->stream));
    DevBuf db;
    CellPropsArgs a;
    CG_TRY(run_cellprops(c, db, a, 90.0, threshold, max_aps));
    const size_t n = (size_t)c->n;
    double *d_dist = nullptr, *d_cv = nullptr;
    int* d_ncv = nullptr;
    CG_TRY(db.get(&d_dist, n));
    CG_TRY(db.get(&d_cv, n * max_aps));
    CG_TRY(db.get(&d_ncv, n));
    CG_CUDA(cudaMemcpyAsync(d_dist, distances, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)c->ode_blocks));
    cv_kernel<<<blocks, 256, 0, c->stream>>>(c->n, max_aps, origin, d_dist, a.up_time, a.n_up, d_cv, d_ncv);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaStreamSynchronize(c->stream));
    CG_CUDA(cudaMemcpy(cv, d_cv, n * max_aps * sizeof(double), cudaMemcpyDeviceToHost));
    if (n_cv) CG_CUDA(cudaMemcpy(n_cv, d_ncv, n * sizeof(int), cudaMemcpyDeviceToHost));
    return CG_OK;
}

}  // extern "C"
