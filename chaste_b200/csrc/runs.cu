// Mixed run populations (include/chaste_gpu.h, cg_runs_*): single-cell and cable
// runs of one cell model in one persistent launch of runs_kernel, replayed from a
// CUDA graph (kernels/runs.cuh).  The host packs the jobs -- cells sorted by
// length into groups of one block's worth, one job per cable -- and orders them by
// decreasing estimated cost; cg_runs_autotune picks threads per block and cells per
// thread by timing each shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/chaste_gpu.h"
#include "kernels/runs.cuh"

using namespace chb;

namespace {

struct HostRun {
    int kind;    // 0 cell, 1 cable
    int index;   // into cells / cables
};

}  // namespace

struct cg_runs {
    int model = 0, S = 0, P = 0, device = 0;
    int tpb = 128, cpt = 1;
    bool dirty = true;          // device buffers out of date with the runs added
    std::vector<HostRun> runs;
    std::vector<RunCell> cells;
    std::vector<double> cell_params;   // n_cells x P
    std::vector<RunCable> cables;
    std::vector<double> cable_params;
    std::vector<int> probes;
    long long trace_len = 0, cable_state_len = 0;
    int max_cable_nodes = 0;
    // device
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<void*> owned;
    RunsArgs args{};
    int blocks = 1;
    size_t smem = 0;
    std::vector<double> y0_cells, y0_cables;
    ~cg_runs() {
        release();
        if (stream) cudaStreamDestroy(stream);
    }
    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (void* p : owned) cudaFree(p);
        owned.clear();
    }
};

namespace {

template <typename T>
bool ralloc(cg_runs* r, T** p, size_t bytes) {
    void* q = nullptr;
    if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    r->owned.push_back(q);
    *p = static_cast<T*>(q);
    return true;
}

template <typename T>
bool upload(cg_runs* r, T** p, const std::vector<T>& v) {
    if (!ralloc(r, p, v.size() * sizeof(T))) return false;
    if (v.empty()) return true;
    if (cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

const void* kernel_for(int model, int cpt) {
    if (model == CG_MODEL_TT06)
        return cpt == 2 ? (const void*)runs_kernel<TenTusscher2006Epi, 2> : (const void*)runs_kernel<TenTusscher2006Epi, 1>;
    return cpt == 2 ? (const void*)runs_kernel<LuoRudy1991, 2> : (const void*)runs_kernel<LuoRudy1991, 1>;
}

// Estimated cost of a job in single-cell steps: a cable step is its nodes' ODE steps
// spread over the block plus the CG's block reductions (a few tens of dependent
// barriers), about as long as a dozen single-cell steps.
double cable_cost(const RunCable& c, int tpb) {
    const int npt = (c.n + tpb - 1) / tpb;
    return (double)c.n_steps * (12.0 + npt);
}

// Jobs (cells grouped by length, cables one each), longest first.  A run's steps
// are one dependent chain, so the population ends no sooner than its longest run:
// groups are cut small enough (down to one warp) that the cells spread over every
// block the GPU holds instead of crowding the threads of a few SMs.
void make_jobs(const cg_runs* r, int blocks_available, std::vector<RunJob>& jobs, std::vector<int>& order) {
    const int n_cells = (int)r->cells.size();
    order.resize(n_cells);
    for (int i = 0; i < n_cells; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return r->cells[x].n_steps > r->cells[y].n_steps; });
    std::vector<std::pair<double, RunJob>> cost;
    const int n_cables = (int)r->cables.size();
    const int for_cells = std::max(blocks_available - n_cables, std::max(1, blocks_available / 2));
    const int spread = (n_cells + for_cells - 1) / for_cells;
    const int group = std::min(r->tpb * r->cpt, std::max(32, (spread + 31) / 32 * 32));
    for (int f = 0; f < n_cells; f += group) {
        RunJob j{0, f, std::min(group, n_cells - f), 0};
        cost.push_back({(double)r->cells[order[f]].n_steps * r->cpt, j});
    }
    for (int c = 0; c < (int)r->cables.size(); ++c) cost.push_back({cable_cost(r->cables[c], r->tpb), RunJob{1, c, 1, 0}});
    std::stable_sort(cost.begin(), cost.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    jobs.clear();
    for (auto& c : cost) jobs.push_back(c.second);
}

// Shared memory of the launch shape and the blocks that fit on the GPU at once.
int configure(cg_runs* r, int smem_nodes, int* resident) {
    const void* k = kernel_for(r->model, r->cpt);
    r->smem = r->max_cable_nodes > 0 ? ((size_t)kRunsCableArrays * smem_nodes + 3 * 32) * sizeof(double) : 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r->smem) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    int sms = 1, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, r->tpb, r->smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return CG_ERR_UNSUPPORTED;
    }
    *resident = per_sm * sms;
    return CG_OK;
}

// Device buffers for the runs added so far, for the current launch shape.
int prepare(cg_runs* r) {
    if (!r->dirty) return CG_OK;
    r->release();
    const size_t n_cells = r->cells.size();
    const double* init = r->model == CG_MODEL_TT06 ? TenTusscher2006Epi::kInitialStates : LuoRudy1991::kInitialStates;
    r->y0_cells.resize((size_t)r->S * n_cells);
    for (int k = 0; k < r->S; ++k)
        for (size_t i = 0; i < n_cells; ++i) r->y0_cells[k * n_cells + i] = init[k];
    const int smem_nodes = (r->max_cable_nodes + 31) / 32 * 32;
    int resident = 1;
    int rc = configure(r, smem_nodes, &resident);
    if (rc != CG_OK) return rc;
    std::vector<RunJob> jobs;
    std::vector<int> order;
    make_jobs(r, resident, jobs, order);
    r->blocks = (int)std::max(1LL, std::min((long long)jobs.size(), (long long)resident));
    RunsArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n_jobs = (int)jobs.size();
    a.smem_nodes = smem_nodes;
    a.n_cells = (int)r->cells.size();
    RunJob* d_jobs = nullptr;
    RunCell* d_cells = nullptr;
    RunCable* d_cables = nullptr;
    int *d_order = nullptr, *d_probes = nullptr;
    double *d_cp = nullptr, *d_kp = nullptr;
    if (!upload(r, &d_jobs, jobs) || !upload(r, &d_cells, r->cells) || !upload(r, &d_order, order) ||
        !upload(r, &d_cp, r->cell_params) || !upload(r, &d_cables, r->cables) || !upload(r, &d_kp, r->cable_params) ||
        !upload(r, &d_probes, r->probes) || !ralloc(r, &a.next_job, sizeof(int)) ||
        !ralloc(r, &a.cell_y, r->y0_cells.size() * sizeof(double)) ||
        !ralloc(r, &a.cable_y, r->y0_cables.size() * sizeof(double)) ||
        !ralloc(r, &a.cable_iters, r->cables.size() * sizeof(long long)) ||
        !ralloc(r, &a.trace, (size_t)r->trace_len * sizeof(double)) || !ralloc(r, &a.status, sizeof(int))) {
        r->release();
        return CG_ERR_NOMEM;
    }
    a.jobs = d_jobs;
    a.cells = d_cells;
    a.cell_order = d_order;
    a.cell_params = d_cp;
    a.cables = d_cables;
    a.cable_params = d_kp;
    a.probes = d_probes;
    r->args = a;
    r->dirty = false;
    return CG_OK;
}

int reset(cg_runs* r) {
    const RunsArgs& a = r->args;
    if ((!r->y0_cells.empty() &&
         cudaMemcpyAsync(a.cell_y, r->y0_cells.data(), r->y0_cells.size() * sizeof(double), cudaMemcpyHostToDevice,
                         r->stream) != cudaSuccess) ||
        (!r->y0_cables.empty() &&
         cudaMemcpyAsync(a.cable_y, r->y0_cables.data(), r->y0_cables.size() * sizeof(double), cudaMemcpyHostToDevice,
                         r->stream) != cudaSuccess) ||
        cudaMemsetAsync(a.status, 0, sizeof(int), r->stream) != cudaSuccess ||
        cudaStreamSynchronize(r->stream) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    return CG_OK;
}

cudaError_t launch(cg_runs* r, long long steps_override) {
    cudaError_t e = cudaMemsetAsync(r->args.next_job, 0, sizeof(int), r->stream);
    if (e != cudaSuccess) return e;
    RunsArgs a = r->args;
    a.steps_override = steps_override;
    void* params[] = {&a};
    return cudaLaunchKernel(kernel_for(r->model, r->cpt), dim3(r->blocks), dim3(r->tpb), params, r->smem, r->stream);
}

int read_status(cg_runs* r) {
    int bits = 0;
    if (cudaMemcpy(&bits, r->args.status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (bits & kStatusNaN) return CG_ERR_NAN;
    if (bits & kStatusCgMaxIt) return CG_ERR_CG_MAXIT;
    return CG_OK;
}

int set_shape(cg_runs* r, int tpb, int cpt) {
    if (r->tpb != tpb || r->cpt != cpt) {
        r->tpb = tpb;
        r->cpt = cpt;
        r->dirty = true;
    }
    return CG_OK;
}

}  // namespace

extern "C" {

int cg_runs_create(int model, int device, cg_runs** out) {
    if (!out || (model != CG_MODEL_LR91 && model != CG_MODEL_TT06)) return CG_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) return CG_ERR_ARG;
    cg_runs* r = new (std::nothrow) cg_runs();
    if (!r) return CG_ERR_NOMEM;
    r->model = model;
    r->device = device;
    r->S = model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumStates : LuoRudy1991::kNumStates;
    r->P = model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumParams : LuoRudy1991::kNumParams;
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete r;
        return CG_ERR_CUDA;
    }
    *out = r;
    return CG_OK;
}

int cg_runs_add_cell(cg_runs* r, int method, const double* params, const cg_stimulus* stim, double dt, int n_steps,
                     int sample_every, int* id) {
    if (!r || !id || (method != CG_ODE_FORWARD_EULER && method != CG_ODE_RUSH_LARSEN) || !(dt > 0) || n_steps < 0 ||
        sample_every < 1 || n_steps % sample_every != 0)
        return CG_ERR_ARG;
    if (stim && stim->kind != CG_STIM_NONE && stim->kind != CG_STIM_SIMPLE && stim->kind != CG_STIM_REGULAR)
        return CG_ERR_ARG;
    RunCell c;
    std::memset(&c, 0, sizeof(c));
    c.method = method == CG_ODE_RUSH_LARSEN ? 1 : 0;
    c.n_steps = n_steps;
    c.sample_every = sample_every;
    c.dt = dt;
    c.tsamp = sample_every * dt;
    c.t_end = (double)(n_steps / sample_every) * c.tsamp;
    c.trace_off = r->trace_len;
    if (stim && stim->kind != CG_STIM_NONE) {
        c.stim.kind = stim->kind;
        c.stim.magnitude = stim->magnitude;
        c.stim.start = stim->start;
        c.stim.period = stim->period;
        c.stim.stop = stim->stop;
        c.stim.duration = stim->kind == CG_STIM_SIMPLE ? stim->duration + (stim->duration + stim->start) * DBL_EPSILON
                                                        : stim->duration + stim->period * DBL_EPSILON;
    }
    const int index = (int)r->cells.size();
    r->trace_len += n_steps / sample_every + 1;
    r->cells.push_back(c);
    for (int k = 0; k < r->P; ++k) r->cell_params.push_back(params ? params[k] : 1.0);
    r->runs.push_back({0, index});
    r->dirty = true;
    *id = (int)r->runs.size() - 1;
    return CG_OK;
}

int cg_runs_add_cable(cg_runs* r, const cg_cable_config* cfg, const double* params, const int* probes, int n_probes,
                      int sample_every, int* id) {
    if (!r || !cfg || !id || cfg->model != r->model || cfg->n_nodes < 2 || cfg->n_nodes > kCableMaxNodes ||
        cfg->n_steps < 0 || cfg->n_regions < 1 || cfg->n_regions > kCableMaxRegions || !(cfg->time_step > 0) ||
        !(cfg->h > 0) || cfg->max_iterations < 1 || n_probes < 0 || (n_probes > 0 && !probes) || sample_every < 1 ||
        cfg->n_steps % sample_every != 0)
        return CG_ERR_ARG;
    for (int k = 0; k < n_probes; ++k)
        if (probes[k] < 0 || probes[k] >= cfg->n_nodes) return CG_ERR_ARG;
    RunCable c;
    std::memset(&c, 0, sizeof(c));
    c.n = cfg->n_nodes;
    c.n_steps = cfg->n_steps;
    c.R = cfg->n_regions;
    c.n_stim = cfg->n_stimulated_nodes;
    c.n_probes = n_probes;
    c.maxit = cfg->max_iterations;
    c.sample_every = sample_every;
    c.h = cfg->h;
    c.sigma0 = cfg->conductivity;
    c.am = cfg->surface_area_to_volume_ratio;
    c.cm = cfg->capacitance;
    c.dt = cfg->time_step;
    c.rtol = cfg->ksp_tolerance;
    c.stim_mag = cfg->stimulus_magnitude;
    c.stim_dur = cfg->stimulus_duration + cfg->stimulus_duration * DBL_EPSILON;   // SimpleStimulus.cpp:50, start 0
    c.param_off = (long long)r->cable_params.size();
    c.probe_off = (long long)r->probes.size();
    c.trace_off = r->trace_len;
    c.state_off = r->cable_state_len;
    const int stride = r->P + 1;
    for (int k = 0; k < c.R * stride; ++k) r->cable_params.push_back(params ? params[k] : 1.0);
    for (int k = 0; k < n_probes; ++k) r->probes.push_back(probes[k]);
    r->trace_len += (long long)(c.n_steps / sample_every) * n_probes;
    r->cable_state_len += (long long)r->S * c.n;
    const double* init = r->model == CG_MODEL_TT06 ? TenTusscher2006Epi::kInitialStates : LuoRudy1991::kInitialStates;
    for (int k = 0; k < r->S; ++k)
        for (int i = 0; i < c.n; ++i) r->y0_cables.push_back(init[k]);
    r->max_cable_nodes = std::max(r->max_cable_nodes, c.n);
    const int index = (int)r->cables.size();
    r->cables.push_back(c);
    r->runs.push_back({1, index});
    r->dirty = true;
    *id = (int)r->runs.size() - 1;
    return CG_OK;
}

int cg_runs_set_shape(cg_runs* r, int threads_per_block, int cells_per_thread) {
    if (!r || threads_per_block < 32 || threads_per_block > kRunsMaxThreads || threads_per_block % 32 != 0 ||
        (cells_per_thread != 1 && cells_per_thread != 2))
        return CG_ERR_ARG;
    return set_shape(r, threads_per_block, cells_per_thread);
}

int cg_runs_shape(const cg_runs* r, int* threads_per_block, int* cells_per_thread) {
    if (!r) return CG_ERR_ARG;
    if (threads_per_block) *threads_per_block = r->tpb;
    if (cells_per_thread) *cells_per_thread = r->cpt;
    return CG_OK;
}

int cg_runs_autotune(cg_runs* r, int steps, int* threads_per_block, int* cells_per_thread) {
    if (!r || steps <= 0 || r->runs.empty()) return CG_ERR_ARG;
    cudaSetDevice(r->device);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int best_tpb = r->tpb, best_cpt = r->cpt;
    const int tpbs[3] = {64, 128, 256};
    int rc = CG_OK;
    for (int cand = 0; cand < 6 && rc == CG_OK; ++cand) {
        set_shape(r, tpbs[cand % 3], cand < 3 ? 1 : 2);
        rc = prepare(r);
        if (rc == CG_ERR_UNSUPPORTED) {   // this shape does not fit on an SM
            rc = CG_OK;
            continue;
        }
        if (rc == CG_OK) rc = reset(r);
        if (rc != CG_OK) break;
        cudaEventRecord(e0, r->stream);
        if (launch(r, steps) != cudaSuccess) {
            cudaGetLastError();
            rc = CG_ERR_CUDA;
            break;
        }
        cudaEventRecord(e1, r->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaGetLastError();
            rc = CG_ERR_CUDA;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            best_tpb = r->tpb;
            best_cpt = r->cpt;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != CG_OK) return rc;
    set_shape(r, best_tpb, best_cpt);
    if ((rc = prepare(r)) != CG_OK || (rc = reset(r)) != CG_OK) return rc;
    if (threads_per_block) *threads_per_block = best_tpb;
    if (cells_per_thread) *cells_per_thread = best_cpt;
    return CG_OK;
}

int cg_runs_run(cg_runs* r, double* ms) {
    if (!r || r->runs.empty()) return CG_ERR_ARG;
    cudaSetDevice(r->device);
    int rc = prepare(r);
    if (rc == CG_OK) rc = reset(r);
    if (rc != CG_OK) return rc;
    if (!r->graph) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        const cudaError_t le = launch(r, 0);
        const cudaError_t ce = cudaStreamEndCapture(r->stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess || cudaGraphInstantiate(&r->graph, g, 0) != cudaSuccess) {
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            r->graph = nullptr;
            return CG_ERR_CUDA;
        }
        cudaGraphDestroy(g);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, r->stream);
    bool ok = cudaGraphLaunch(r->graph, r->stream) == cudaSuccess;
    cudaEventRecord(e1, r->stream);
    ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (ms) *ms = t;
    return read_status(r);
}

int cg_runs_result(cg_runs* r, int id, double* states, double* trace, int* n_samples, long long* cg_iterations) {
    if (!r || id < 0 || id >= (int)r->runs.size() || r->dirty) return CG_ERR_ARG;
    cudaSetDevice(r->device);
    const HostRun& h = r->runs[id];
    const RunsArgs& a = r->args;
    if (h.kind == 0) {
        const RunCell& c = r->cells[h.index];
        const int ns = c.n_steps / c.sample_every + 1;
        if (n_samples) *n_samples = ns;
        if (cg_iterations) *cg_iterations = 0;
        if (trace && cudaMemcpy(trace, a.trace + c.trace_off, ns * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return CG_ERR_CUDA;
        if (states) {
            const size_t n = r->cells.size();
            // state k of cell i lies at k * n + i: one strided copy
            if (cudaMemcpy2D(states, sizeof(double), a.cell_y + h.index, n * sizeof(double), sizeof(double), r->S,
                             cudaMemcpyDeviceToHost) != cudaSuccess)
                return CG_ERR_CUDA;
        }
        return CG_OK;
    }
    const RunCable& c = r->cables[h.index];
    const int ns = c.n_steps / c.sample_every;
    if (n_samples) *n_samples = ns;
    if (trace && cudaMemcpy(trace, a.trace + c.trace_off, (size_t)ns * c.n_probes * sizeof(double),
                            cudaMemcpyDeviceToHost) != cudaSuccess)
        return CG_ERR_CUDA;
    if (cg_iterations &&
        cudaMemcpy(cg_iterations, a.cable_iters + h.index, sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CG_ERR_CUDA;
    if (states) {
        std::vector<double> s((size_t)r->S * c.n);
        if (cudaMemcpy(s.data(), a.cable_y + c.state_off, s.size() * sizeof(double), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return CG_ERR_CUDA;
        for (int i = 0; i < c.n; ++i)
            for (int k = 0; k < r->S; ++k) states[(size_t)i * r->S + k] = s[(size_t)k * c.n + i];
    }
    return CG_OK;
}

int cg_runs_destroy(cg_runs* r) {
    if (!r) return CG_ERR_ARG;
    cudaSetDevice(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    delete r;
    return CG_OK;
}

}  // extern "C"
