// Grouped launches: many independent cases of one grid shape in one launch.
//
// A batch of cases steps as one CUDA graph. Launched case by case, a step of
// a small case is ~25 short kernels, and a few hundred cases make thousands
// of graph nodes: the GPU's launch rate, not its bandwidth, then sets the
// step time. A grouped launch runs one kernel for every case of a group at
// once: blockIdx.z is the case, and each case's arguments come from an array
// of argument packs in device memory (one pack a case, the kernel's own
// parameter list laid out as a struct). The kernel bodies are the single-case
// kernels' bodies (`k_*_body`), so a case computes exactly what it computes
// alone.
//
// Inside a graph loop (a WHILE node the group runs while any of its cases
// needs another iteration) a grouped kernel is gated: a case whose own loop
// has ended (its flag is 0) skips the iteration, as it would have left its
// own loop.
#pragma once

#include <cuda.h>

#include <utility>

#include "step_kernels.cuh"

namespace vvm {

template <typename... A>
struct KPack {};
template <typename H, typename... R>
struct KPack<H, R...> {
    H h;
    KPack<R...> r;
};

inline KPack<> kpack() { return {}; }
template <typename H, typename... R>
KPack<H, R...> kpack(const H& h, const R&... r) {
    KPack<H, R...> p;
    p.h = h;
    p.r = kpack(r...);
    return p;
}

template <size_t I, typename H, typename... R>
__device__ __forceinline__ const auto& kget(const KPack<H, R...>& p) {
    if constexpr (I == 0) return p.h;
    else return kget<I - 1>(p.r);
}

template <auto Body, typename... A, size_t... I>
__device__ __forceinline__ void kcall(const KPack<A...>& p, std::index_sequence<I...>) {
    Body(kget<I>(p)...);
}

// The body `Body` for case blockIdx.z with the arguments packs[blockIdx.z];
// gate (null outside loops): the cases' loop flags.
template <auto Body, int MAXT, int MINB, typename... A>
__global__ void __launch_bounds__(MAXT, MINB)
    k_grouped(const KPack<A...>* __restrict__ packs, const int* const* __restrict__ gate) {
    if (gate && !*(const volatile int*)gate[blockIdx.z]) return;
    kcall<Body>(packs[blockIdx.z], std::index_sequence_for<A...>{});
}

// The scalar advection's pack: its four tensor maps stay in global memory,
// where TMA reads them.
template <typename T>
struct PAdvPack {
    CUtensorMap m[4];
    PAdvArgs<T> a;
};

// A tensor map that a host copy wrote to global memory, made visible to the
// TMA unit's proxy before its first use.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(m))
                 : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kPAdvBX * kPAdvBZ, 4)
    k_padv_grouped(const PAdvPack<T>* __restrict__ packs, const int* const* __restrict__ gate) {
    if (gate && !*(const volatile int*)gate[blockIdx.z]) return;
    const PAdvPack<T>& p = packs[blockIdx.z];
    if (threadIdx.x == 0 && threadIdx.y == 0)
        for (int f = 0; f < 4; f++) tensormap_acquire(&p.m[f]);
    k_padv_body<T>(&p.m[0], &p.m[1], &p.m[2], &p.m[3], p.a);
}

// The group's loop condition: another iteration while any case's flag is set.
__global__ void k_group_cond(const int* const* __restrict__ flags, int n, cudaGraphConditionalHandle h) {
    int any = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) any |= (*(const volatile int*)flags[i] != 0);
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// Clears `bytes` bytes at ptrs[blockIdx.z] (a device memset a case).
__global__ void k_group_zero(unsigned char* const* __restrict__ ptrs, size_t bytes) {
    unsigned char* p = ptrs[blockIdx.z];
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < bytes; j += (size_t)gridDim.x * blockDim.x)
        p[j] = 0;
}

}  // namespace vvm
