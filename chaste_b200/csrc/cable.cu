// Cables for parameter fitting (include/chaste_gpu.h, cg_cable_*): batched
// forward runs, one CTA per parameter set, and the checkpointed adjoint.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <set>
#include <vector>

#include "../../include/chaste_gpu.h"
#include "kernels/cable.cuh"

using namespace chb;

struct cg_cable {
    cg_cable_config cfg{};
    int S = 0, P = 0, device = 0, n_probes = 0;
    int* d_probes = nullptr;
    int* d_status = nullptr;
    double* d_ckpt = nullptr;
    double* d_seg = nullptr;
    size_t ckpt_sets = 0;       // sets the checkpoint buffers hold
    int ckpt_valid_sets = 0;    // sets written by the last keep_checkpoints forward
    ~cg_cable() {
        cudaFree(d_probes);
        cudaFree(d_status);
        cudaFree(d_ckpt);
        cudaFree(d_seg);
    }
};

namespace {

size_t smem_bytes() { return sizeof(CableShared); }

template <class M>
int configure_kernels() {
    static bool done = false;
    if (done) return CG_OK;
    if (cudaFuncSetAttribute(cable_forward_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes()) != cudaSuccess ||
        cudaFuncSetAttribute(cable_adjoint_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes()) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    done = true;
    return CG_OK;
}

CableArgs make_args(const cg_cable* c) {
    CableArgs a;
    std::memset(&a, 0, sizeof(a));
    const cg_cable_config& g = c->cfg;
    a.n = g.n_nodes;
    a.n_steps = g.n_steps;
    a.R = g.n_regions;
    a.n_probes = c->n_probes;
    a.n_stim = g.n_stimulated_nodes;
    a.ckpt_every = g.checkpoint_every;
    a.maxit = g.max_iterations;
    a.h = g.h;
    a.sigma0 = g.conductivity;
    a.am = g.surface_area_to_volume_ratio;
    a.cm = g.capacitance;
    a.dt = g.time_step;
    a.rtol = g.ksp_tolerance;
    a.stim_mag = g.stimulus_magnitude;
    a.stim_dur = g.stimulus_duration;
    a.probes = c->d_probes;
    a.status = c->d_status;
    return a;
}

int threads_for(int n) { return std::max(32, (n + 31) / 32 * 32); }

int finish(cg_cable* c, cudaStream_t st) {
    int status = 0;
    if (cudaMemcpyAsync(&status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (status & kStatusNaN) return CG_ERR_NAN;
    if (status & kStatusCgMaxIt) return CG_ERR_CG_MAXIT;
    return CG_OK;
}

size_t n_ckpt(const cg_cable* c) {
    return (size_t)((c->cfg.n_steps + c->cfg.checkpoint_every - 1) / c->cfg.checkpoint_every);
}

int ensure_checkpoints(cg_cable* c, int n_sets) {
    if ((size_t)n_sets <= c->ckpt_sets) return CG_OK;
    cudaFree(c->d_ckpt);
    cudaFree(c->d_seg);
    c->d_ckpt = c->d_seg = nullptr;
    c->ckpt_sets = 0;
    const size_t per = (size_t)c->S * c->cfg.n_nodes * sizeof(double);
    if (cudaMalloc(&c->d_ckpt, n_ckpt(c) * per * n_sets) != cudaSuccess ||
        cudaMalloc(&c->d_seg, (size_t)c->cfg.checkpoint_every * per * n_sets) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(c->d_ckpt);
        c->d_ckpt = nullptr;
        return CG_ERR_NOMEM;
    }
    c->ckpt_sets = n_sets;
    return CG_OK;
}

template <class M>
int launch(cg_cable* c, bool adjoint, int n_sets, CableArgs a, cudaStream_t st) {
    static_assert(M::kNumStates <= 32, "initial-state array too small");
    for (int k = 0; k < M::kNumStates; ++k) a.y0[k] = M::kInitialStates[k];
    int rc = configure_kernels<M>();
    if (rc != CG_OK) return rc;
    if (adjoint)
        cable_adjoint_kernel<M><<<n_sets, threads_for(c->cfg.n_nodes), smem_bytes(), st>>>(a);
    else
        cable_forward_kernel<M><<<n_sets, threads_for(c->cfg.n_nodes), smem_bytes(), st>>>(a);
    if (cudaGetLastError() != cudaSuccess) return CG_ERR_CUDA;
    return CG_OK;
}

int dispatch(cg_cable* c, bool adjoint, int n_sets, const CableArgs& a, cudaStream_t st) {
    if (c->cfg.model == CG_MODEL_LR91) return launch<LuoRudy1991>(c, adjoint, n_sets, a, st);
    return launch<TenTusscher2006Epi>(c, adjoint, n_sets, a, st);
}

}  // namespace

extern "C" {

void cg_cable_default_config(cg_cable_config* g) {
    if (!g) return;
    std::memset(g, 0, sizeof(*g));
    g->model = CG_MODEL_LR91;
    g->n_nodes = 1000;
    g->h = 0.01;
    g->conductivity = 1.75;
    g->surface_area_to_volume_ratio = 1400.0;
    g->capacitance = 1.0;
    g->time_step = 0.01;
    g->n_steps = 40000;
    g->n_regions = 4;
    g->n_stimulated_nodes = 2;
    g->stimulus_magnitude = -5e5;
    g->stimulus_duration = 0.5;
    g->ksp_tolerance = 1e-8;
    g->max_iterations = 10000;
    g->checkpoint_every = 200;
}

int cg_cable_create(const cg_cable_config* cfg, const int* probes, int n_probes, int device, cg_cable** out) {
    if (!cfg || !out || !probes || n_probes < 1) return CG_ERR_ARG;
    *out = nullptr;
    const cg_cable_config& g = *cfg;
    if (g.model != CG_MODEL_LR91 && g.model != CG_MODEL_TT06) return CG_ERR_ARG;
    if (g.n_nodes < 2 || g.n_nodes > kCableMaxNodes || g.n_regions < 1 || g.n_regions > kCableMaxRegions ||
        g.n_regions > g.n_nodes - 1 || g.n_steps < 1 || g.checkpoint_every < 1 || !(g.h > 0) ||
        !(g.time_step > 0) || !(g.ksp_tolerance > 0) || g.max_iterations < 1 || g.n_stimulated_nodes < 0 ||
        g.n_stimulated_nodes > g.n_nodes)
        return CG_ERR_ARG;
    std::set<int> seen;
    for (int k = 0; k < n_probes; ++k) {
        if (probes[k] < 0 || probes[k] >= g.n_nodes || !seen.insert(probes[k]).second) return CG_ERR_ARG;
    }
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return CG_ERR_CUDA;
    cg_cable* c = new (std::nothrow) cg_cable;
    if (!c) return CG_ERR_NOMEM;
    c->cfg = g;
    c->device = device;
    c->n_probes = n_probes;
    c->S = g.model == CG_MODEL_LR91 ? LuoRudy1991::kNumStates : TenTusscher2006Epi::kNumStates;
    c->P = g.model == CG_MODEL_LR91 ? LuoRudy1991::kNumParams : TenTusscher2006Epi::kNumParams;
    if (cudaMalloc(&c->d_probes, sizeof(int) * n_probes) != cudaSuccess ||
        cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return CG_ERR_NOMEM;
    }
    if (cudaMemcpy(c->d_probes, probes, sizeof(int) * n_probes, cudaMemcpyHostToDevice) != cudaSuccess) {
        delete c;
        return CG_ERR_CUDA;
    }
    *out = c;
    return CG_OK;
}

int cg_cable_forward(cg_cable* c, int n_sets, const double* d_params, const double* d_targets, double* d_loss,
                     double* d_traces, int* d_iterations, int keep_checkpoints, void* stream) {
    if (!c || n_sets < 1 || n_sets > 65535 || !d_params || (d_loss && !d_targets)) return CG_ERR_ARG;
    if (keep_checkpoints && !d_targets) return CG_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return CG_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    c->ckpt_valid_sets = 0;
    if (keep_checkpoints) {
        const int rc = ensure_checkpoints(c, n_sets);
        if (rc != CG_OK) return rc;
    }
    CableArgs a = make_args(c);
    a.params = d_params;
    a.targets = d_targets;
    a.loss = d_loss;
    a.traces = d_traces;
    a.iters = d_iterations;
    a.ckpt = keep_checkpoints ? c->d_ckpt : nullptr;
    if (cudaMemsetAsync(c->d_status, 0, sizeof(int), st) != cudaSuccess) return CG_ERR_CUDA;
    int rc = dispatch(c, false, n_sets, a, st);
    if (rc != CG_OK) return rc;
    rc = finish(c, st);
    if (rc == CG_OK && keep_checkpoints) c->ckpt_valid_sets = n_sets;
    return rc;
}

int cg_cable_backward(cg_cable* c, int n_sets, const double* d_params, const double* d_targets, double* d_grad,
                      void* stream) {
    if (!c || n_sets < 1 || !d_params || !d_targets || !d_grad) return CG_ERR_ARG;
    if (n_sets != c->ckpt_valid_sets) return CG_ERR_ORDER;
    if (cudaSetDevice(c->device) != cudaSuccess) return CG_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CableArgs a = make_args(c);
    a.params = d_params;
    a.targets = d_targets;
    a.ckpt = c->d_ckpt;
    a.seg = c->d_seg;
    a.grad = d_grad;
    if (cudaMemsetAsync(c->d_status, 0, sizeof(int), st) != cudaSuccess) return CG_ERR_CUDA;
    const int rc = dispatch(c, true, n_sets, a, st);
    if (rc != CG_OK) return rc;
    return finish(c, st);
}

int cg_cable_destroy(cg_cable* c) {
    if (!c) return CG_ERR_ARG;
    cudaSetDevice(c->device);
    delete c;
    return CG_OK;
}

}  // extern "C"
