// Device layout and shared helpers of the VVM step kernels (sm_100a).
//
// Every 2D field of a case is one x-contiguous array [nz][pitch] with the
// reference's ghost cells kept in place (i = 0 and nx-1, k = 0 and nz-1), so
// cell (i, k) of the reference's model.var[i][k] lives at k*pitch + i. Rows
// are padded to a multiple of 32 cells: a warp reading one row segment touches
// whole 128-byte lines. Profiles are [nz] doubles.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vvm {

constexpr int kPad = 32;

struct Dims {
    int nx, nz, pitch;  // pitch >= nx, multiple of kPad
    __host__ __device__ __forceinline__ size_t at(int i, int k) const {
        return (size_t)k * pitch + i;
    }
    __host__ __device__ __forceinline__ size_t cells() const { return (size_t)nz * pitch; }
};

// Physical constants and grid metrics of one case (src/Declare.hpp:78-96,
// src/main.cpp:68-72). Reciprocals are formed exactly as the reference
// forms them.
struct Consts {
    double dx, dz, dt, rdx, r2dx, rdz, r2dz, rdx2, rdz2;
    double gravity, cp, cv, rd, lv, p0;
};

template <typename T>
__device__ __forceinline__ T plus_part(T v) { return T(0.5) * (v + fabs(v)); }   // Advection.cpp:17-19
template <typename T>
__device__ __forceinline__ T minus_part(T v) { return T(0.5) * (v - fabs(v)); }  // Advection.cpp:21-23

// std::max / std::min semantics (the first argument wins ties and NaN), as
// used throughout the reference's microphysics and turbulence.
template <typename T>
__device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }

// Writes the value of interior cell (i, k) and every ghost cell that
// BoundaryProcess2D_center (src/Boundary.cpp:9-19) fills from it: the
// periodic x ghosts of rows 1..nz-2, then the zero-gradient z ghosts of every
// column including the corner cells. Each ghost cell has exactly one source
// cell, so a grid over the interior fills the halo without a second pass.
template <typename T>
__device__ __forceinline__ void store_center(T* a, const Dims& d, int i, int k, T v) {
    const bool gl = (i == d.nx - 2), gr = (i == 1);
    a[d.at(i, k)] = v;
    if (gl) a[d.at(0, k)] = v;
    if (gr) a[d.at(d.nx - 1, k)] = v;
    if (k == 1) {
        a[d.at(i, 0)] = v;
        if (gl) a[d.at(0, 0)] = v;
        if (gr) a[d.at(d.nx - 1, 0)] = v;
    }
    if (k == d.nz - 2) {
        a[d.at(i, d.nz - 1)] = v;
        if (gl) a[d.at(0, d.nz - 1)] = v;
        if (gr) a[d.at(d.nx - 1, d.nz - 1)] = v;
    }
}

// Same for BoundaryProcess2D_westdown (src/Boundary.cpp:21-30) on a field
// whose interior values exist for k = 2..nz-2: periodic x ghosts, rows 0, 1
// and nz-1 zero everywhere (written by the k = 2 and k = nz-2 cells).
template <typename T>
__device__ __forceinline__ void store_westdown(T* a, const Dims& d, int i, int k, T v) {
    const bool gl = (i == d.nx - 2), gr = (i == 1);
    a[d.at(i, k)] = v;
    if (gl) a[d.at(0, k)] = v;
    if (gr) a[d.at(d.nx - 1, k)] = v;
    if (k == 2) {
        a[d.at(i, 0)] = T(0);
        a[d.at(i, 1)] = T(0);
        if (gl) { a[d.at(0, 0)] = T(0); a[d.at(0, 1)] = T(0); }
        if (gr) { a[d.at(d.nx - 1, 0)] = T(0); a[d.at(d.nx - 1, 1)] = T(0); }
    }
    if (k == d.nz - 2) {
        a[d.at(i, d.nz - 1)] = T(0);
        if (gl) a[d.at(0, d.nz - 1)] = T(0);
        if (gr) a[d.at(d.nx - 1, d.nz - 1)] = T(0);
    }
}

// Warp and block sums in a fixed order (deterministic for a fixed launch
// shape). All reductions of the step accumulate in FP64.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums N values per thread over the (1D or 2D) block; every thread gets the
// totals. `sh` needs 32*N doubles of shared memory.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* sh) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = tid & 31, wid = tid >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int j = 0; j < N; j++) v[j] = warp_sum(v[j]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < N; j++) sh[j * 32 + wid] = v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < N; j++) {
        double t = (lane < nw) ? sh[j * 32 + lane] : 0.0;
        v[j] = warp_sum(t);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Shared-memory barriers and TMA loads (sm_100a PTX).

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// One-arrival barrier for a block's TMA loads (call from one thread, then
// __syncthreads before any thread waits on it).
__device__ __forceinline__ void mbar_init1(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Waits for phase `parity` of the barrier, polling at most kStageSpinLimit
// times; false if it gave up.
constexpr int kStageSpinLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < kStageSpinLimit; it++)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// 2D tiled TMA load of a box at (x, y) into shared memory (no multicast);
// completion counted on `bar`. x times the element size must be a multiple
// of 16 bytes; y and x may be negative or out of range (zero fill).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Grid-wide finish of per-block partial sums without a second launch. Every
// block calls it once, after its thread 0 has written the block's partial;
// it returns true in the one block that arrives last (thread 0 fences its
// partial, then counts in: no block waits for another), which may then read
// all partials (__ldcg) and finish the sum in a fixed order. That block also
// puts the counter back to 0 for the next launch; `count` starts at 0.
__device__ __forceinline__ bool arrive_last(unsigned* count, unsigned nblocks) {
    __shared__ int last;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(count, 1u);
        last = (prev == nblocks - 1);
        if (last) atomicExch(count, 0u);
    }
    __syncthreads();
    if (last) __threadfence();
    return last != 0;
}

}  // namespace vvm
