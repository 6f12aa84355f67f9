// Device-side helpers shared by the tissue kernels.
#pragma once

#include <cfloat>
#include <cstdint>

#include <cuda/atomic>

namespace chb {

// Status bits written by kernels (never a trap: the host reads them).
enum : int {
    kStatusCgMaxIt = 1,
    kStatusCgDiverged = 2,
    kStatusNaN = 4,
    kStatusStateRange = 8,
    kStatusBarrierTimeout = 16,
};

// Stimulus as evaluated on the device; durations already padded on the host
// exactly as SimpleStimulus.cpp:50 / RegularStimulus.cpp:55 do.
struct DevStimulus {
    int kind;          // 0 none, 1 simple, 2 regular
    double magnitude;
    double duration;   // padded
    double start;
    double period;
    double stop;
};

__device__ __forceinline__ double stimulus_value(const DevStimulus& s, double t) {
    if (s.kind == 1) return (s.start <= t && t <= s.duration + s.start) ? s.magnitude : 0.0;
    if (s.kind == 2) {
        if (t < s.start) return 0.0;
        const double beat = fmod(t - s.start, s.period);
        return (beat >= 0 && beat <= s.duration && t <= s.stop) ? s.magnitude : 0.0;
    }
    return 0.0;
}

// TimeStepper time arithmetic (global/src/TimeStepper.cpp:43-135).
struct DevTimeStepper {
    double start, end, dt, eps, time, next;
    unsigned steps;
    __device__ DevTimeStepper(double s, double e, double d)
        : start(s), end(e), dt(d), eps(e > 1.0 ? DBL_EPSILON * e : DBL_EPSILON), time(s), steps(0) {
        next = calc();
    }
    __device__ double calc() const {
        double n = start + (steps + 1) * dt;
        if (end - n <= eps) n = end;
        return n;
    }
    __device__ bool at_end() const { return time >= end; }
    __device__ void advance() {
        steps++;
        time = next;
        next = calc();
    }
};

// ------------------------------------------------------------------------
// Grid-wide reduction + barrier for persistent kernels launched cooperatively
// (all blocks co-resident).  Every wait is bounded: on timeout the block sets
// kStatusBarrierTimeout and returns false, and later waits see the flag and
// return at once, so the kernel always terminates.
struct GridSync {
    unsigned int count;
    unsigned int gen;
    double result[8];
};

constexpr long long kBarrierSpinLimit = 20000000;   // x ~100 ns sleep ~ 2 s
constexpr int kMaxGridBlocks = 512;                  // largest grid a persistent kernel is launched with

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Reduce NV per-thread values over the block into smem_out[NV].
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* smem /* 32*NV */, double* smem_out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[warp * NV + k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? smem[lane * NV + k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) smem_out[k] = s;
        }
    }
    __syncthreads();
}

// All blocks contribute NV partial sums; out[] receives the grid totals,
// identical in every block because the last block to arrive sums the partials
// in a fixed order (lane l takes blocks l, l+32, ..., then a fixed shuffle tree).
template <int NV>
__device__ bool grid_reduce(GridSync* gs, double* partials, const double* block_vals,
                            double* out, int* status) {
    const int lane = threadIdx.x & 31;
    __shared__ int s_ok;
    __shared__ double s_res[8];
    if (threadIdx.x < 32) {
        unsigned my_gen = 0, ticket = 0;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = block_vals[k];
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(gs->gen);
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
            my_gen = gen.load(cuda::memory_order_acquire);
            ticket = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        }
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
        my_gen = __shfl_sync(0xffffffffu, my_gen, 0);
        int ok = 1;
        if (ticket == gridDim.x - 1) {
            __threadfence();
            __syncwarp();
            // all loads of a lane are issued before any is used (grids of at most
            // kMaxGridBlocks blocks), so the reduction costs one L2 round trip
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                double vals[kMaxGridBlocks / 32];
#pragma unroll
                for (int m = 0; m < kMaxGridBlocks / 32; ++m) {
                    const unsigned b = lane + 32u * m;
                    vals[m] = b < gridDim.x ? __ldcg(&partials[b * NV + k]) : 0.0;
                }
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < kMaxGridBlocks / 32; ++m) s += vals[m];
                s = warp_sum(s);
                if (lane == 0) gs->result[k] = s;
            }
            __syncwarp();
            if (lane == 0) {
                cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(gs->gen);
                cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
                cnt.store(0u, cuda::memory_order_relaxed);
                gen.fetch_add(1u, cuda::memory_order_release);
            }
        } else if (lane == 0) {
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(gs->gen);
            long long spins = 0;
            while (gen.load(cuda::memory_order_acquire) == my_gen) {
                if (++spins > kBarrierSpinLimit || (*(volatile int*)status & kStatusBarrierTimeout)) {
                    atomicOr(status, kStatusBarrierTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (lane == 0) {
            __threadfence();
            s_ok = ok;
            if (ok)
                for (int k = 0; k < NV; ++k) s_res[k] = __ldcg(&gs->result[k]);
        }
    }
    __syncthreads();
    if (!s_ok) return false;
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = s_res[k];
    return true;
}

}  // namespace chb
