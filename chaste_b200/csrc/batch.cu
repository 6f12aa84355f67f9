// Batched single-cell populations (include/chaste_gpu.h, cg_batch_*).  Two engines:
//   persistent (default): one CUDA graph holding ONE launch of population_kernel that
//     runs every beat of every cell from a work queue (kernels/population.cuh);
//   per beat: one CUDA graph holding batch_kernel, the per-beat error kernel and the
//     beat counter, replayed once per beat (kernels/batch.cuh).
// cg_batch_autotune times both (and the per-beat kernel's launch shapes) and keeps
// the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/chaste_gpu.h"
#include "kernels/population.cuh"

using namespace chb;

struct cg_batch {
    int model = 0, n = 0, S = 0, P = 0, max_beats = 0, max_aps = 0, sample_every = 10, device = 0;
    int tpb = 64;
    int cpt = 1;            // cells per thread
    int engine = CG_BATCH_PERSISTENT;
    int pop_blocks = 1;     // persistent engine: co-resident blocks of kPopThreads
    long long steps_per_beat = 0;
    double dt = 0.01;
    DevStimulus stim{};
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<void*> owned;
    int* d_beats = nullptr;
    double* d_params = nullptr;
    double* d_y64 = nullptr;
    float* d_y32 = nullptr;
    ApdTracker* d_trk = nullptr;
    double* d_apd = nullptr;
    float* d_vsamp = nullptr;
    float* d_maxdv = nullptr;
    long long* d_launch = nullptr;
    int* d_status = nullptr;
    int* d_order = nullptr;   // cells by decreasing beat count (the persistent engine's queue)
    int* d_next = nullptr;    // its work-queue counter
    std::vector<double> y0;   // initial states, SoA
    ~cg_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : owned) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

template <typename P>
bool balloc(cg_batch* b, P** p, size_t bytes) {
    void* q = nullptr;
    if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    b->owned.push_back(q);
    *p = static_cast<P*>(q);
    return true;
}

BatchArgs batch_args(const cg_batch* b, long long steps_override) {
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n_cells = b->n;
    a.max_aps = b->max_aps;
    a.max_beats = b->max_beats;
    a.sample_every = b->sample_every;
    a.blocks_per_precision = (b->n + b->tpb * b->cpt - 1) / (b->tpb * b->cpt);
    a.steps_per_beat = b->steps_per_beat;
    a.dt = b->dt;
    a.cm = 1.0;
    a.stim = b->stim;
    a.beats = b->d_beats;
    a.params = b->d_params;
    a.y64 = b->d_y64;
    a.y32 = b->d_y32;
    a.trk = b->d_trk;
    a.apd = b->d_apd;
    a.vsamp = b->d_vsamp;
    a.launch = b->d_launch;
    a.steps_override = steps_override;
    a.status = b->d_status;
    return a;
}

cudaError_t launch_beat(cg_batch* b, long long steps_override, bool with_error) {
    BatchArgs a = batch_args(b, steps_override);
    const int grid = 2 * a.blocks_per_precision;
    const bool tt = b->model == CG_MODEL_TT06;
    if (b->cpt == 2) {
        if (tt) batch_kernel<TenTusscher2006Epi, 2><<<grid, b->tpb, 0, b->stream>>>(a);
        else batch_kernel<LuoRudy1991, 2><<<grid, b->tpb, 0, b->stream>>>(a);
    } else {
        if (tt) batch_kernel<TenTusscher2006Epi, 1><<<grid, b->tpb, 0, b->stream>>>(a);
        else batch_kernel<LuoRudy1991, 1><<<grid, b->tpb, 0, b->stream>>>(a);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !with_error) return e;
    batch_beat_error_kernel<<<(b->n + 255) / 256, 256, 0, b->stream>>>(a, b->d_maxdv);
    batch_advance_kernel<<<1, 1, 0, b->stream>>>(b->d_launch);
    return cudaGetLastError();
}

PopArgs pop_args(const cg_batch* b, long long steps_override) {
    PopArgs pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.b = batch_args(b, steps_override);
    pa.order = b->d_order;
    pa.n_groups = (b->n + 31) / 32;
    pa.next_group = b->d_next;
    pa.max_dv = b->d_maxdv;
    return pa;
}

cudaError_t launch_population(cg_batch* b, long long steps_override) {
    cudaError_t e = cudaMemsetAsync(b->d_next, 0, sizeof(int), b->stream);
    if (e != cudaSuccess) return e;
    const PopArgs pa = pop_args(b, steps_override);
    if (b->model == CG_MODEL_TT06) population_kernel<TenTusscher2006Epi><<<b->pop_blocks, kPopThreads, 0, b->stream>>>(pa);
    else population_kernel<LuoRudy1991><<<b->pop_blocks, kPopThreads, 0, b->stream>>>(pa);
    return cudaGetLastError();
}

// A run (or, with steps_override, the first steps of one) of the current engine.
cudaError_t launch_engine(cg_batch* b, long long steps_override) {
    return b->engine == CG_BATCH_PERSISTENT ? launch_population(b, steps_override)
                                            : launch_beat(b, steps_override, false);
}

int reset_states(cg_batch* b) {
    const size_t n = b->n;
    std::vector<float> y32(b->y0.begin(), b->y0.end());
    if (cudaMemcpyAsync(b->d_y64, b->y0.data(), b->y0.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
        cudaMemcpyAsync(b->d_y32, y32.data(), y32.size() * sizeof(float), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_trk, 0, 2 * n * sizeof(ApdTracker), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_launch, 0, sizeof(long long), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_status, 0, sizeof(int), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_maxdv, 0, n * b->max_beats * sizeof(float), b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    std::vector<double> nan((size_t)2 * n * b->max_aps, -1.0);
    if (cudaMemcpy(b->d_apd, nan.data(), nan.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    return CG_OK;
}

}  // namespace

extern "C" {

int cg_batch_create(int model, int n_cells, const int* beats, const double* params, const cg_stimulus* stim,
                    double dt, double beat_length, int max_aps, int device, cg_batch** out) {
    if (!out || !beats || !stim || n_cells <= 0 || !(dt > 0) || !(beat_length > 0) || max_aps <= 0) return CG_ERR_ARG;
    if (model != CG_MODEL_LR91 && model != CG_MODEL_TT06) return CG_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) return CG_ERR_ARG;
    cg_batch* b = new (std::nothrow) cg_batch();
    if (!b) return CG_ERR_NOMEM;
    b->model = model;
    b->n = n_cells;
    b->device = device;
    b->S = model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumStates : LuoRudy1991::kNumStates;
    b->P = model == CG_MODEL_TT06 ? TenTusscher2006Epi::kNumParams : LuoRudy1991::kNumParams;
    b->dt = dt;
    b->steps_per_beat = (long long)(beat_length / dt + 0.5);
    b->max_aps = max_aps;
    int mb = 0;
    for (int i = 0; i < n_cells; ++i) {
        if (beats[i] < 0) {
            delete b;
            return CG_ERR_ARG;
        }
        mb = std::max(mb, beats[i]);
    }
    b->max_beats = std::max(1, mb);
    b->stim.kind = stim->kind;
    b->stim.magnitude = stim->magnitude;
    b->stim.start = stim->start;
    b->stim.period = stim->period;
    b->stim.stop = stim->stop;
    b->stim.duration = stim->kind == CG_STIM_SIMPLE ? stim->duration + (stim->duration + stim->start) * DBL_EPSILON
                                                    : stim->duration + stim->period * DBL_EPSILON;
    const size_t n = n_cells;
    const long long nsamp = (b->steps_per_beat + b->sample_every - 1) / b->sample_every;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        !balloc(b, &b->d_beats, n * sizeof(int)) || !balloc(b, &b->d_params, n * b->P * sizeof(double)) ||
        !balloc(b, &b->d_y64, n * b->S * sizeof(double)) || !balloc(b, &b->d_y32, n * b->S * sizeof(float)) ||
        !balloc(b, &b->d_trk, 2 * n * sizeof(ApdTracker)) || !balloc(b, &b->d_apd, 2 * n * max_aps * sizeof(double)) ||
        !balloc(b, &b->d_vsamp, 2 * (size_t)nsamp * n * sizeof(float)) ||
        !balloc(b, &b->d_maxdv, n * b->max_beats * sizeof(float)) || !balloc(b, &b->d_launch, sizeof(long long)) ||
        !balloc(b, &b->d_status, sizeof(int)) || !balloc(b, &b->d_order, n * sizeof(int)) ||
        !balloc(b, &b->d_next, sizeof(int))) {
        cudaGetLastError();
        delete b;
        return CG_ERR_NOMEM;
    }
    std::vector<double> p(n * b->P, 1.0);
    if (params) std::memcpy(p.data(), params, p.size() * sizeof(double));
    const double* init = model == CG_MODEL_TT06 ? TenTusscher2006Epi::kInitialStates : LuoRudy1991::kInitialStates;
    b->y0.resize(n * b->S);
    for (int k = 0; k < b->S; ++k)
        for (size_t i = 0; i < n; ++i) b->y0[k * n + i] = init[k];
    // the persistent engine's queue: longest runs first (ties by cell index), so each
    // group of 32 cells has about one length and the long runs start at once
    std::vector<int> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return beats[x] > beats[y]; });
    int sms = 1, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (model == CG_MODEL_TT06)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, population_kernel<TenTusscher2006Epi>, kPopThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, population_kernel<LuoRudy1991>, kPopThreads, 0);
    b->pop_blocks = (int)std::max(1LL, std::min((long long)(n + 31) / 32, (long long)std::max(per_sm, 1) * sms));
    if (cudaMemcpy(b->d_order, order.data(), n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_beats, beats, n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_params, p.data(), p.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return CG_ERR_CUDA;
    }
    const int rc = reset_states(b);
    if (rc != CG_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return CG_OK;
}

int cg_batch_autotune(cg_batch* b, int steps, int* threads_per_block) {
    if (!b || steps <= 0) return CG_ERR_ARG;
    cudaSetDevice(b->device);
    const int cands[4] = {32, 64, 128, 256};
    float best = 1e30f;
    int best_tpb = b->tpb, best_cpt = b->cpt;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best_engine = b->engine;
    for (int cand = 0; cand < 9; ++cand) {
        // candidates 0-7: the per-beat kernel's shapes; 8: the persistent engine
        const int c = cands[cand % 4];
        b->engine = cand < 8 ? CG_BATCH_PER_BEAT : CG_BATCH_PERSISTENT;
        b->tpb = cand < 8 ? c : best_tpb;
        b->cpt = cand < 8 ? (cand < 4 ? 1 : 2) : best_cpt;
        int rc = reset_states(b);
        if (rc != CG_OK) return rc;
        cudaEventRecord(e0, b->stream);
        if (launch_engine(b, steps) != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return CG_ERR_CUDA;
        }
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            best_engine = b->engine;
            if (cand < 8) {
                best_tpb = c;
                best_cpt = b->cpt;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->engine = best_engine;
    b->tpb = best_tpb;
    b->cpt = best_cpt;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (threads_per_block) *threads_per_block = best_tpb;
    return reset_states(b);
}

int cg_batch_set_launch_shape(cg_batch* b, int threads_per_block, int cells_per_thread) {
    if (!b || threads_per_block < 32 || threads_per_block > 1024 || threads_per_block % 32 != 0 ||
        (cells_per_thread != 1 && cells_per_thread != 2))
        return CG_ERR_ARG;
    b->tpb = threads_per_block;
    b->cpt = cells_per_thread;
    b->engine = CG_BATCH_PER_BEAT;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return CG_OK;
}

int cg_batch_launch_shape(const cg_batch* b, int* threads_per_block, int* cells_per_thread) {
    if (!b) return CG_ERR_ARG;
    if (threads_per_block) *threads_per_block = b->tpb;
    if (cells_per_thread) *cells_per_thread = b->cpt;
    return CG_OK;
}

int cg_batch_set_engine(cg_batch* b, int engine) {
    if (!b || (engine != CG_BATCH_PER_BEAT && engine != CG_BATCH_PERSISTENT)) return CG_ERR_ARG;
    b->engine = engine;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return CG_OK;
}

int cg_batch_engine(const cg_batch* b, int* engine) {
    if (!b || !engine) return CG_ERR_ARG;
    *engine = b->engine;
    return CG_OK;
}

int cg_batch_run(cg_batch* b, double* ms) {
    if (!b) return CG_ERR_ARG;
    cudaSetDevice(b->device);
    if (!b->graph) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        const cudaError_t le = b->engine == CG_BATCH_PERSISTENT ? launch_population(b, 0) : launch_beat(b, 0, true);
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess || cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) {
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            b->graph = nullptr;
            return CG_ERR_CUDA;
        }
        cudaGraphDestroy(g);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, b->stream);
    bool ok = true;
    const int replays = b->engine == CG_BATCH_PERSISTENT ? 1 : b->max_beats;
    for (int k = 0; k < replays && ok; ++k) ok = cudaGraphLaunch(b->graph, b->stream) == cudaSuccess;
    cudaEventRecord(e1, b->stream);
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
    int bits = 0;
    if (cudaMemcpy(&bits, b->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return CG_ERR_CUDA;
    return bits ? CG_ERR_NAN : CG_OK;
}

int cg_batch_results(cg_batch* b, double* apd64, double* apd32, int* n_ap64, int* n_ap32, float* max_dv,
                     double* states64, double* states32) {
    if (!b) return CG_ERR_ARG;
    cudaSetDevice(b->device);
    const size_t n = b->n;
    std::vector<double> apd(2 * n * b->max_aps);
    std::vector<ApdTracker> trk(2 * n);
    if (cudaMemcpy(apd.data(), b->d_apd, apd.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(trk.data(), b->d_trk, trk.size() * sizeof(ApdTracker), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CG_ERR_CUDA;
    if (apd64) std::memcpy(apd64, apd.data(), n * b->max_aps * sizeof(double));
    if (apd32) std::memcpy(apd32, apd.data() + n * b->max_aps, n * b->max_aps * sizeof(double));
    for (size_t i = 0; i < n; ++i) {
        if (n_ap64) n_ap64[i] = trk[i].n_ap;
        if (n_ap32) n_ap32[i] = trk[n + i].n_ap;
    }
    if (max_dv && cudaMemcpy(max_dv, b->d_maxdv, n * b->max_beats * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CG_ERR_CUDA;
    std::vector<double> y64(n * b->S);
    std::vector<float> y32(n * b->S);
    if (cudaMemcpy(y64.data(), b->d_y64, y64.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(y32.data(), b->d_y32, y32.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CG_ERR_CUDA;
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < b->S; ++k) {
            if (states64) states64[i * b->S + k] = y64[k * n + i];
            if (states32) states32[i * b->S + k] = y32[k * n + i];
        }
    return CG_OK;
}

int cg_batch_destroy(cg_batch* b) {
    if (!b) return CG_ERR_ARG;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    return CG_OK;
}

}  // extern "C"
