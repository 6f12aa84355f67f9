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
// (all blocks co-resident).
//
// Arrival is a monotonic counter: at its k-th reduction (k = 0, 1, ...) a block
// writes its partial sums into buffer k % 2, adds 1 to `count` (release) and
// waits until `count` reaches (k + 1) * gridDim (acquire).  Every block then
// sums all partials itself, lane l taking blocks l, l+32, ... and a fixed
// shuffle tree finishing, so all blocks obtain bitwise the same totals with
// no broadcast round trip.  Two buffers suffice: a block can write round k+1
// only after every block has arrived at round k, i.e. has finished reading
// round k-1.  The counter is returned to zero by the last block to leave the
// kernel (grid_exit), so each launch starts from zero.
//
// Every wait is bounded (about 2 s of %globaltimer): on timeout the block sets
// kStatusBarrierTimeout and returns false, and later waits see the flag and
// return at once, so the kernel always terminates.
struct GridSync {
    unsigned int count;
    unsigned int gen;     // unused (layout kept)
    unsigned int exit;
    unsigned int pad;
    double result[8];
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;
constexpr int kMaxGridBlocks = 512;                  // largest grid a persistent kernel is launched with
constexpr int kPartialStride = 4;                    // doubles per block and buffer (NV <= 4)

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One thread waits until *counter >= target (acquire), for at most limit_ns of
// %globaltimer.  On timeout, or when another waiter has already timed out, it sets
// kStatusBarrierTimeout and returns false: every wait of a kernel ends.
__device__ __forceinline__ bool wait_count(unsigned* counter, unsigned target, int* status,
                                           unsigned long long limit_ns = kBarrierTimeoutNs) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(*counter);
    if (cnt.load(cuda::memory_order_acquire) >= target) return true;
    const unsigned long long t0 = global_ns();
    while (cnt.load(cuda::memory_order_acquire) < target) {
        if ((*(volatile int*)status & kStatusBarrierTimeout) || global_ns() - t0 > limit_ns) {
            atomicOr(status, kStatusBarrierTimeout);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

// Block and grid reduction in one: every thread contributes v[NV]; out[] receives
// the grid totals, identical in every block.  The block's sum is formed by each
// warp's shuffle tree and then warp 0's over the warps (so thread 0 holds it and
// arrives without a further block barrier); partials: 2 x gridDim x
// kPartialStride doubles; `round` counts this block's reductions in the launch
// (start at 0; same sequence in every block).  The partials are read back by the
// first kReduceWarps warps, thread t taking blocks t, t + 32 kReduceWarps, ... (at
// most 4 loads, issued together), then each warp's shuffle tree and the warps in
// order: the order is fixed, so every block gets bitwise the same sums.
// Needs blockDim >= 32 * kReduceWarps; red holds 32 * NV doubles.
constexpr int kReduceWarps = 4;

// The same reduction for a kernel that always runs as one block (the shared-memory
// bjacobi solve): the block's sums are the totals, with no global partials, atomics or
// polling.  (Taken inside grid_reduce whenever gridDim is 1, the branch pushed the
// HBM-resident mixed solve from 16 to 156 bytes of spills a thread and 0.49 to 0.61 ms
// per solve on the 2.1M-node slab.)
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* red, double* out, unsigned& round) {
    __shared__ double s_tot[2][kPartialStride];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp * NV + k] = v[k];
    __syncthreads();
    // two buffers by round parity: round r + 1 writes the other one, so a thread still
    // reading round r's totals is never overwritten
    const unsigned par = round & 1u;
    round++;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double b = warp_sum(lane < nw ? red[lane * NV + k] : 0.0);
            if (lane == 0) s_tot[par][k] = b;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = s_tot[par][k];
}

template <int NV>
__device__ bool grid_reduce(double (&v)[NV], double* red, GridSync* gs, double* partials, double* out, int* status,
                            unsigned& round) {
    static_assert(NV >= 1 && NV <= kPartialStride, "at most four sums per reduction");

    constexpr int kLoads = kMaxGridBlocks / (32 * kReduceWarps);
    __shared__ int s_ok;
    __shared__ double s_part[kReduceWarps][kPartialStride];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp * NV + k] = v[k];
    __syncthreads();
    double* buf = partials + (size_t)(round & 1u) * gridDim.x * kPartialStride;
    const unsigned target = (round + 1u) * gridDim.x;
    round++;
    if (warp == 0) {
        double b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) b[k] = warp_sum(lane < nw ? red[lane * NV + k] : 0.0);
        if (lane == 0) {
            int ok = 1;
#pragma unroll
            for (int k = 0; k < NV; ++k) buf[blockIdx.x * kPartialStride + k] = b[k];
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
            cnt.fetch_add(1u, cuda::memory_order_release);
            ok = wait_count(&gs->count, target, status) ? 1 : 0;
            s_ok = ok;
        }
    }
    __syncthreads();
    if (!s_ok) return false;
    // thread 0's acquire load and the block barrier order these loads after every
    // block's release (the pattern of a cooperative-groups grid sync), so the
    // reading warps need no fence of their own
    if (warp < kReduceWarps) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double vals[kLoads];
#pragma unroll
            for (int m = 0; m < kLoads; ++m) {
                const unsigned bb = threadIdx.x + 32u * kReduceWarps * m;
                vals[m] = bb < gridDim.x ? __ldcg(&buf[bb * kPartialStride + k]) : 0.0;
            }
            double sum = 0.0;
#pragma unroll
            for (int m = 0; m < kLoads; ++m) sum += vals[m];
            sum = warp_sum(sum);
            if (lane == 0) s_part[warp][k] = sum;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double sum = s_part[0][k];
#pragma unroll
        for (int w = 1; w < kReduceWarps; ++w) sum += s_part[w][k];
        out[k] = sum;
    }
    // no trailing barrier: the next reduction writes s_part / s_ok / red only after
    // its own block barrier, which every thread reaches after reading these
    return true;
}

// Called once by every block as it leaves a kernel that used grid_reduce: the
// last block out returns the arrival counter to zero for the next launch.
__device__ __forceinline__ void grid_exit(GridSync* gs) {
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> ex(gs->exit);
        if (ex.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
            cnt.store(0u, cuda::memory_order_relaxed);
            ex.store(0u, cuda::memory_order_release);
        }
    }
}

}  // namespace chb
