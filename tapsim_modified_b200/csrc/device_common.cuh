// Shared device definitions for the TAPSim hot-path kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace tgd {

// Makes device dev current for a scope (dev < 0: leaves the current device
// alone) and gives the caller's current device back at the scope's end.  A
// handle's buffers, streams and events live on the device that was current
// when it was created; the entry points run under one of these, so a caller
// whose current device is another one still reaches the handle's memory.
struct ScopedDevice {
    int prev = -1;
    explicit ScopedDevice(int dev) {
        if (dev < 0 || cudaGetDevice(&prev) != cudaSuccess || prev == dev) {
            prev = -1;
            return;
        }
        if (cudaSetDevice(dev) != cudaSuccess) prev = -1;
    }
    ~ScopedDevice() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    ScopedDevice(const ScopedDevice&) = delete;
    ScopedDevice& operator=(const ScopedDevice&) = delete;
};

// per-node flag bits
enum : uint8_t {
    F_HULL = 1,        // Geometry_3d::NodeData::boundary
    F_DIRICHLET = 2,   // Grid_3d::Node DIRICHLET
    F_NEUMANN = 4,     // Grid_3d::Node NEUMANN
    F_SURFACE = 8,     // member of the Surface_3d::Table node set
    F_FREE = 16        // listed in a free-row list
};

// device-side status bits (accumulated, read by the host after a call)
enum : int {
    S_NAN = 1,
    S_SINGULAR = 2,
    S_NOT_SURFACE = 4,
    S_WALK_LIMIT = 8,
    S_UNKNOWN_TYPE = 16,
    S_ZERO_WEIGHT = 32,
    S_CAPACITY = 64,
    S_TIMEOUT = 128    // a bounded wait inside a kernel ran out
};

struct DType {
    float epsilon;
    float evap_field;
    float evap_energy;  // [eV], EVAPORATION_ACTIVATION_ENERGY
    float charge_density;
    float phi;
    uint8_t removable, neumann, dirichlet, present;
};

constexpr double kEpsilon0 = 8.85418781762e-12;  // As/(Vm), grid_3d.h:283

__device__ __forceinline__ void atomic_max_double_nonneg(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// monotone map float -> uint32 (total order, -0 < +0 ignored)
__device__ __forceinline__ uint32_t float_order_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sums of two doubles into *outA, *outB (one atomicAdd each per
// block, one shared-memory pass).
template <int BLOCK>
__device__ __forceinline__ void block_sum2_atomic(double a, double b, double* outA, double* outB) {
    __shared__ double red[2][BLOCK / 32];
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = a;
        red[1][wid] = b;
    }
    __syncthreads();
    if (wid == 0) {
        double sa = lane < BLOCK / 32 ? red[0][lane] : 0.0;
        double sb = lane < BLOCK / 32 ? red[1][lane] : 0.0;
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            if (sa != 0.0) atomicAdd(outA, sa);
            if (sb != 0.0) atomicAdd(outB, sb);
        }
    }
    __syncthreads();
}

// Block-wide sum of a double into *out (one atomicAdd per block).
template <int BLOCK>
__device__ __forceinline__ void block_sum_atomic(double v, double* out) {
    __shared__ double red[BLOCK / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double s = lane < BLOCK / 32 ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0 && s != 0.0) atomicAdd(out, s);
    }
    __syncthreads();
}

template <int BLOCK>
__device__ __forceinline__ void block_max_atomic_u64(unsigned long long v, unsigned long long* out) {
    __shared__ unsigned long long red[BLOCK / 32];
    v = warp_max_u64(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        unsigned long long s = lane < BLOCK / 32 ? red[lane] : 0ull;
        s = warp_max_u64(s);
        if (lane == 0 && s != 0ull) atomicMax(out, s);
    }
    __syncthreads();
}

// Runs f() (a cudaError_t-returning setup such as cudaFuncSetAttribute,
// which holds per device) the first time it is reached with each current
// device 0..63; `done` is the caller's bit set of devices already set up.
// Concurrent first calls may both run f, which must be idempotent.
template <class F>
inline cudaError_t once_per_device(std::atomic<uint64_t>& done, F f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev >= 0 && dev < 64 ? (1ull << dev) : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = f();
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
    return e;
}


}  // namespace tgd
