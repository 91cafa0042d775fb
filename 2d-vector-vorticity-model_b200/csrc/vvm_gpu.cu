// libvvmgpu.so: the B200 VVM time step behind the C ABI of include/vvm_gpu.h.
//
// Host code: device memory of one context, coefficient profiles formed with
// the reference's expressions, the multigrid-preconditioned CG of cal_w, and
// the launch sequence of one step (src/Iteration.cpp:262-434).
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <tuple>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/vvm_gpu.h"
#include "poisson_kernels.cuh"
#include "spectral_kernels.cuh"
#include "learned_kernels.cuh"
#include "step_kernels.cuh"
#include "grouped.cuh"

using namespace vvm;

// ===========================================================================
// Non-template kernels

namespace vvm {

__device__ __forceinline__ void k_nvp_final_body(const double* partial, int nblocks, double* nvp) {
    __shared__ double sh[32 * 6];
    nvp_finish(partial, nblocks, nvp, sh);
}
__global__ void k_nvp_final(const double* partial, int nblocks, double* nvp) { k_nvp_final_body(partial, nblocks, nvp); }

__device__ __forceinline__ void k_cg_scalar_body(const double* partial, int n, CGScalars* sc, int mode) {
    __shared__ double sh[32];
    double s[1] = {0};
    for (int b = threadIdx.x; b < n; b += blockDim.x) s[0] += partial[b];
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        double v = s[0];
        switch (mode) {
            case CG_SET_BB: sc->bb = v; break;
            case CG_SET_RR: sc->rr = v; break;
            case CG_SET_RZ: sc->rz = v; break;
            case CG_PQ_ALPHA: sc->pq = v; sc->alpha = (v != 0.0) ? sc->rz / v : 0.0; break;
            case CG_RZ_BETA:
                sc->rz_new = v;
                sc->beta = (sc->rz != 0.0) ? v / sc->rz : 0.0;
                sc->rz = v;
                break;
            case CG_SET_NRM: sc->nrm = v; break;
            case CG_FCG_BETA: sc->beta = (sc->pq != 0.0) ? -v / sc->pq : 0.0; break;   // -(z, q) / (p, q)
            case CG_NET_DSD: sc->dsd = v; break;
            case CG_NET_GAMMA: sc->gam = (sc->dsd > 0.0) ? v / sc->dsd : 0.0; break;     // (d, r1) / (d, S d)
        }
    }
}
__global__ void k_cg_scalar(const double* partial, int n, CGScalars* sc, int mode) { k_cg_scalar_body(partial, n, sc, mode); }

__device__ __forceinline__ void k_cg_scalar_it_body(const double* partial, int n, CGScalars* sc, const CGCtl* ctl) {
    __shared__ double sh[32];
    double s[1] = {0};
    for (int b = threadIdx.x; b < n; b += blockDim.x) s[0] += partial[b];
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        double v = s[0];
        sc->rz_new = v;
        sc->beta = (ctl->it == 0 || sc->rz == 0.0) ? 0.0 : v / sc->rz;
        sc->rz = v;
    }
}
__global__ void k_cg_scalar_it(const double* partial, int n, CGScalars* sc, const CGCtl* ctl) { k_cg_scalar_it_body(partial, n, sc, ctl); }

__global__ void k_zero_if_b0(int NX, int NK, int pitch, const CGScalars* sc, double* W) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK && sc->bb == 0.0) W[(size_t)kk * pitch + ii] = 0.0;
}

__device__ __forceinline__ void k_loop_plain_body(const CGScalars* sc, CGCtl* ctl, cudaGraphConditionalHandle h, double tol2,
                             int maxit, int init, long long* exec, int body_kernels) {
    if (init) ctl->it = 0;
    else { ctl->it++; *exec += body_kernels; }
    const double rr = sc->rr, bb = sc->bb;
    bool more = (bb > 0.0) && (rr > tol2 * bb) && (ctl->it < maxit) && isfinite(rr);
    ctl->total = ctl->it;
    ctl->relres = (bb > 0.0) ? sqrt(rr / bb) : 0.0;
    ctl->more = more ? 1 : 0;
    if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
}
__global__ void k_loop_plain(const CGScalars* sc, CGCtl* ctl, cudaGraphConditionalHandle h, double tol2,
                             int maxit, int init, long long* exec, int body_kernels) { k_loop_plain_body(sc, ctl, h, tol2, maxit, init, exec, body_kernels); }

__global__ void k_loop_inner(const CGScalars* sc, CGCtl* ctl, cudaGraphConditionalHandle h, double rtol2,
                             int maxit, int init, long long* exec, int body_kernels) {
    if (init) {
        ctl->it = 0;
        ctl->rr0 = sc->rr;
    } else {
        ctl->it++;
        *exec += body_kernels;
    }
    const double rr = sc->rr;
    bool more = (ctl->rr0 > 0.0) && (rr > rtol2 * ctl->rr0) && (ctl->it < maxit) && isfinite(rr);
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void k_loop_outer(const CGScalars* sc64, CGCtl* ctl, const CGCtl* inner,
                             cudaGraphConditionalHandle h, double tol2, int maxit, int init, long long* exec,
                             int body_kernels) {
    if (init) {
        ctl->outer = 0;
        ctl->total = 0;
    } else {
        ctl->outer++;
        ctl->total += (inner->it > 0 ? inner->it : 1);
        *exec += body_kernels;
    }
    const double rr = sc64->rr, bb = sc64->bb;
    ctl->relres = (bb > 0.0) ? sqrt(rr / bb) : 0.0;
    bool more = (bb > 0.0) && (rr > tol2 * bb) && isfinite(rr) && (ctl->total < maxit) && (ctl->outer < 20);
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

// b = rhow_k^2 (zetap[i+1][k] - zetap[i][k]) dx for k = 2..nz-2, i = 1..nx-2
// (PoissonSolver.cpp:444-450); stores f = -b / rw_k and the block partials of
// ||b||^2, which the block that arrives last sums in a fixed order into
// sc->bb (arrive: a counter at 0, left at 0). rw_k is the row's residual
// weight: rhow_k on uniform levels, rhow_k / a_k on stretched ones (a_k the
// centre spacing around face k over dx).
template <typename T>
__device__ __forceinline__ void k_poisson_rhs_body(const Dims& d, double dx, const double* rhow, const double* rw, const T* zetap, double* f,
                              int pitch_f, double* partial, unsigned* arrive, CGScalars* sc) {
    __shared__ double sh[32];
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (ii < d.nx - 2 && kk < d.nz - 3) {
        const int i = ii + 1, k = kk + 2;
        double b = rhow[k] * rhow[k] * ((double)zetap[d.at(i + 1, k)] - (double)zetap[d.at(i, k)]) * dx;
        f[(size_t)kk * pitch_f + ii] = -b / rw[k];
        s[0] = b * b;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
    const unsigned nb = gridDim.x * gridDim.y;
    if (!arrive_last(arrive, nb)) return;
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.x + blockDim.x * threadIdx.y;
    double t[1] = {0};
    for (int q = tid; q < (int)nb; q += nt) t[0] += __ldcg(partial + q);
    block_sum(t, sh);
    if (tid == 0) sc->bb = t[0];
}
template <typename T>
__global__ void k_poisson_rhs(Dims d, double dx, const double* rhow, const double* rw, const T* zetap, double* f,
                              int pitch_f, double* partial, unsigned* arrive, CGScalars* sc) {
    k_poisson_rhs_body<T>(d, dx, rhow, rw, zetap, f, pitch_f, partial, arrive, sc);
}

// Reference-ordered b vector ((k-2)*NX + (i-1)) to f = -b/rw_k, partial ||b||^2.
__global__ void k_rhs_from_b(int NX, int NK, const double* rw, const double* b, double* f,
                             int pitch_f, double* partial) {
    __shared__ double sh[32];
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (ii < NX && kk < NK) {
        double bv = b[(size_t)kk * NX + ii];
        f[(size_t)kk * pitch_f + ii] = -bv / rw[kk + 2];
        s[0] = bv * bv;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

__global__ void k_pack_solution(int NX, int NK, const double* x, int pitch, double* out) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK) out[(size_t)kk * NX + ii] = x[(size_t)kk * pitch + ii];
}

__global__ void k_unpack_solution(int NX, int NK, const double* in, double* x, int pitch) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK) x[(size_t)kk * pitch + ii] = in[(size_t)kk * NX + ii];
}

// w = W / rhow_k for k = 2..nz-2 (PoissonSolver.cpp:469-475), westdown halo.
template <typename T>
__device__ __forceinline__ void k_w_from_W_body(const Dims& d, const double* rhow, const double* W, int pitch_f, T* w) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 2 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx - 2 || k > d.nz - 2) return;
    double v = W[(size_t)(k - 2) * pitch_f + (i - 1)] / rhow[k];
    store_westdown(w, d, i, k, T(v));
}
template <typename T>
__global__ void k_w_from_W(Dims d, const double* rhow, const double* W, int pitch_f, T* w) { k_w_from_W_body<T>(d, rhow, W, pitch_f, w); }

// The streamfunction formulation (PoissonSolver::calpsiuw, STREAMFUNCTION,
// src/PoissonSolver.cpp:124-177). Its matrix (src/PoissonSolver.cpp:726-756,
// POISSONPARAM = 0) is -S with S the symmetric w-equation operator of
// uniform levels; the right-hand side is b = zetap dx^2 over k = 2..nz-2,
// i = 1..nx-2. So S psi = f with f = -b, and ||f - S psi|| / ||f|| is the
// reference's ||b - A psi|| / ||b|| (an unweighted residual).
template <typename T>
__global__ void k_psi_rhs(Dims d, double dx, const T* zetap, double* f, int pitch_f, double* partial) {
    __shared__ double sh[32];
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (ii < d.nx - 2 && kk < d.nz - 3) {
        const double b = (double)zetap[d.at(ii + 1, kk + 2)] * dx * dx;
        f[(size_t)kk * pitch_f + ii] = -b;
        s[0] = b * b;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// psi with its ghosts (periodic columns, zero at k = 0, 1, nz-1), then
//   u = -(rhow_{k+1} psi_{i,k+1} - rhow_k psi_{i,k}) rdz / rhou_k,
//   w = (psi_{i+1,k} - psi_{i,k}) rdx,   i = 1..nx-2, k = 1..nz-2,
// with u's centre halo and w's westdown halo (w = 0 at k = 0, 1, nz-1: the
// routine's zeroing loop over i < nz, line 172, is overwritten by that halo).
// One thread a cell of the padded [nz][pitch] arrays, ghosts included: a
// ghost takes the value of the interior cell the halo copies into it.
template <typename T>
__global__ void k_psi_uw(Dims d, const double* rhou, const double* rhow, double rdx, double rdz, const double* X,
                         int pitch_x, double* psi, T* u, T* w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= d.nx || k >= d.nz) return;
    const int NX = d.nx - 2, nz = d.nz;
    auto P = [&](int ii, int kk) -> double {   // psi at interior column ii (1..NX, wrapped), level kk
        if (kk <= 1 || kk >= nz - 1) return 0.0;
        const int c = (ii - 1 + NX) % NX;
        return X[(size_t)(kk - 2) * pitch_x + c];
    };
    const int iw = (i == 0) ? NX : (i == d.nx - 1 ? 1 : i);   // periodic ghost columns
    psi[d.at(i, k)] = P(iw, k);
    const int ku = k < 1 ? 1 : (k > nz - 2 ? nz - 2 : k);        // u: zero-gradient rows
    const double uv = -(rhow[ku + 1] * P(iw, ku + 1) - rhow[ku] * P(iw, ku)) * rdz / rhou[ku];
    u[d.at(i, k)] = T(uv);
    double wv = 0.0;
    if (k >= 2 && k <= nz - 2) wv = (P(iw + 1, k) - P(iw, k)) * rdx;
    w[d.at(i, k)] = T(wv);
}

// Initial guess of the next cal_w from the last two solutions:
// W <- 2 W - Wprev, Wprev <- W (old).
__global__ void k_extrapolate(int NX, int NK, int pitch, double* W, double* Wprev) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK) {
        size_t id = (size_t)kk * pitch + ii;
        double w = W[id];
        W[id] = 2.0 * w - Wprev[id];
        Wprev[id] = w;
    }
}

// x64 += (double) d32 (iterative refinement).
__global__ void k_refine_add(int NX, int NK, int pitch, double* x, const float* dlt) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK) {
        size_t id = (size_t)kk * pitch + ii;
        x[id] += (double)dlt[id];
    }
}

__global__ void k_to_float(int NX, int NK, int pitch, const double* a, float* b) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii < NX && kk < NK) {
        size_t id = (size_t)kk * pitch + ii;
        b[id] = (float)a[id];
    }
}

// Host [nx][nz] (k fast, stride sk per element) <-> device [nz][pitch].
// `ref` (optional, [nz]) is subtracted on the way in and added on the way
// out: the mixed step stores th and qv as perturbations from a profile.
template <typename T>
__global__ void k_from_host_layout(Dims d, const double* src, int sk, int off, const double* ref, T* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < d.nx && k < d.nz) {
        double v = src[((size_t)i * d.nz + k) * sk + off];
        if (ref) v -= ref[k];
        dst[d.at(i, k)] = T(v);
    }
}

template <typename T>
__global__ void k_to_host_layout(Dims d, const T* src, int sk, int off, const double* ref, double* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < d.nx && k < d.nz) {
        double v = (double)src[d.at(i, k)];
        if (ref) v += ref[k];
        dst[((size_t)i * d.nz + k) * sk + off] = v;
    }
}

}  // namespace vvm

// ===========================================================================
// Host helpers

namespace {

struct CudaError {
    std::string msg;
};

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw CudaError{std::string(#call) + ": " + cudaGetErrorString(e_)};             \
    } while (0)

#define CKL()                                                                                \
    do {                                                                                     \
        cudaError_t e_ = cudaGetLastError();                                                 \
        if (e_ != cudaSuccess) throw CudaError{std::string("launch: ") + cudaGetErrorString(e_)}; \
    } while (0)

inline int round_up(int a, int b) { return (a + b - 1) / b * b; }
inline int cdiv(int a, int b) { return (a + b - 1) / b; }

// Owns device allocations of one context.
// Host -> device copy of set-up data, complete on return (a plain cudaMemcpy
// from pageable memory may return before its DMA ends, and work on a
// non-blocking stream is not ordered after the legacy stream).
inline void upload_now(void* dst, const void* src, size_t nb) {
    CK(cudaMemcpy(dst, src, nb, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(nullptr));
}

struct Arena {
    std::vector<void*> ptrs;
    std::vector<size_t> bytes;
    template <typename X>
    X* alloc(size_t n) {
        void* p = nullptr;
        const size_t nb = std::max<size_t>(n, 1) * sizeof(X);
        CK(cudaMalloc(&p, nb));
        CK(cudaMemset(p, 0, nb));
        // complete before returning: a context's stream may be non-blocking,
        // and work on it is not ordered after the legacy stream
        CK(cudaStreamSynchronize(nullptr));
        ptrs.push_back(p);
        bytes.push_back(nb);
        return static_cast<X*>(p);
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

// Multigrid hierarchy for the symmetric w-equation operator, precision P.
//
// Levels halve the column count while it is even (x-semicoarsening); a
// power-of-two NX ends at one column, whose operator has no x part and is
// solved exactly by one line solve. Otherwise the coarsest level has an odd
// column count (at most kMaxOddCoarse) and gets 2*nc + 8 damped line sweeps.
// Levels of at most 32 columns run inside one block (k_mg_coarse_cycle).
constexpr int kMaxOddCoarse = 256;
// Dynamic shared memory of the Fourier-mode coarse solve at most (f / solution
// and the reduced-system bands, next to 32 KB of static tiles within 227 KB).
constexpr int kModeSmemMax = 192 * 1024;

struct Recorder;

// Launch counter and, when enabled, per-kernel-class device time from CUDA
// events recorded around each launch on the launching stream.
struct Stats {
    bool on = false;
    Recorder* rec = nullptr;   // set while a step is recorded for a grouped launch (no work issued)
    long long launches = 0;
    double ms[VVM_K_COUNT] = {};
    long long cnt[VVM_K_COUNT] = {};
    struct Rec {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t ev() {
        if (pool.empty()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    void resolve() {
        for (auto& r : pending) {
            CK(cudaEventSynchronize(r.b));
            float t = 0;
            CK(cudaEventElapsedTime(&t, r.a, r.b));
            ms[r.id] += t;
            cnt[r.id]++;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    void reset() {
        resolve();
        for (int i = 0; i < VVM_K_COUNT; i++) { ms[i] = 0; cnt[i] = 0; }
        launches = 0;
    }
    ~Stats() {
        for (auto& r : pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct Timed {
    Stats* s;
    int id;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    Timed(Stats* s_, int id_, cudaStream_t st_) : s(s_), id(id_), st(st_) {
        if (!s) return;
        // a recording issues no work: a launch here has no grouped form
        if (s->rec) throw CudaError{"grouped launch: a kernel of the step has no grouped form"};
        s->launches++;
        if (s->on) {
            a = s->ev();
            CK(cudaEventRecord(a, st));
        }
    }
    ~Timed() {
        if (!a) return;
        cudaEvent_t b = s->ev();
        cudaEventRecord(b, st);
        s->pending.push_back({id, a, b});
        if (s->pending.size() > 8192) s->resolve();
    }
};

#define LAUNCH(S, ID, ST, ...)      \
    do {                            \
        Timed t_((S), (ID), (ST));  \
        __VA_ARGS__;                \
    } while (0)

// ---------------------------------------------------------------- recording
//
// A batch steps the cases of one shape as grouped launches (grouped.cuh).
// To build them, each case's step is first recorded instead of issued: the
// kernels with their launch shapes and argument packs, the clears of small
// control blocks, and the graph loops with the points where a case decides
// whether its loop goes on (its flag, an int in device memory). The batch
// then checks that the recordings of a group agree op for op and replays
// them side by side.
struct RecOp {
    enum Kind { KERNEL, ZERO, COND_NEXT, COND_LOOP, LOOP_BEGIN, LOOP_END } kind = KERNEL;
    const void* fn = nullptr;           // KERNEL: the grouped kernel
    dim3 grid, block;
    size_t smem = 0;
    std::vector<unsigned char> pack;    // KERNEL: this case's arguments
    size_t align = 16;
    void* ptr = nullptr;                // ZERO: what to clear; COND_*: the case's loop flag (int)
    size_t bytes = 0;                   // ZERO
};
struct Recorder {
    std::vector<RecOp> ops;
};

template <typename X>
struct same_t {
    using type = X;
};

inline void record_kernel(Stats* s, const void* fn, dim3 g, dim3 b, size_t smem, const void* pack, size_t size,
                          size_t align) {
    RecOp op;
    op.kind = RecOp::KERNEL;
    op.fn = fn;
    op.grid = g;
    op.block = b;
    op.smem = smem;
    op.pack.assign(static_cast<const unsigned char*>(pack), static_cast<const unsigned char*>(pack) + size);
    op.align = align;
    s->rec->ops.push_back(std::move(op));
}

// Launches kernel k (body Body) on st, or records it when a step is being
// recorded. MAXT and MINB: the launch bounds of its grouped form, the
// largest block it is launched with and the blocks a SM its own
// __launch_bounds__ asks for.
template <auto Body, int MAXT, int MINB = 1, typename... A>
void klaunch(Stats* s, int id, cudaStream_t st, void (*k)(A...), dim3 g, dim3 b, size_t smem,
             typename same_t<A>::type... args) {
    if (s && s->rec) {
        if ((int)(b.x * b.y * b.z) > MAXT) throw CudaError{"grouped launch: block larger than its launch bounds"};
        const KPack<A...> p = kpack<A...>(args...);
        record_kernel(s, reinterpret_cast<const void*>(&k_grouped<Body, MAXT, MINB, A...>), g, b, smem, &p,
                      sizeof(p), alignof(KPack<A...>));
        return;
    }
    LAUNCH(s, id, st, k<<<g, b, smem, st>>>(args...));
    CKL();
}

// cudaMemsetAsync(p, 0, bytes, st), or its record.
inline void zero_async(Stats* s, void* p, size_t bytes, cudaStream_t st) {
    if (s && s->rec) {
        RecOp op;
        op.kind = RecOp::ZERO;
        op.ptr = p;
        op.bytes = bytes;
        s->rec->ops.push_back(std::move(op));
        return;
    }
    CK(cudaMemsetAsync(p, 0, bytes, st));
}

// Marks where a case has decided whether a graph loop runs (another) pass:
// its flag `more` (next: the loop that opens next; else the innermost open
// loop). Only recordings keep it: a case's own graph sets its conditions in
// the deciding kernels.
inline void record_cond(Stats* s, int* more, bool next) {
    if (!(s && s->rec)) return;
    RecOp op;
    op.kind = next ? RecOp::COND_NEXT : RecOp::COND_LOOP;
    op.ptr = more;
    s->rec->ops.push_back(std::move(op));
}

struct HostLine {   // host copy of one level's line factors
    std::vector<double> lo, inv, cp, gL, gR;
    // banded LU of the 2S x 2S reduced system (lower and upper bandwidth 2):
    // [5][2S] = l1, l2, u1, u2, 1/diag
    std::vector<double> band;
};


// Segment factors, spikes and reduced inverse of tridiag(-rd, xdiag + ru + rd, -ru)
// (first row without the -rd coupling, last without -ru: W = 0 beyond).
static HostLine factor_partitioned(const std::vector<double>& xdiag, const std::vector<double>& ru,
                                   const std::vector<double>& rd, int S) {
    const int NK = (int)xdiag.size();
    HostLine h;
    h.lo.assign(NK, 0.0);
    h.inv.assign(NK, 0.0);
    h.cp.assign(NK, 0.0);
    h.gL.assign(NK, 0.0);
    h.gR.assign(NK, 0.0);
    std::vector<double> first(S), last(S);
    for (int s = 0; s < S; s++) {
        int a = (s * NK) / S, b = ((s + 1) * NK) / S;
        double cprev = 0.0;
        for (int j = a; j < b; j++) {
            double l = (j > a) ? -rd[j] : 0.0;
            double u = (j < b - 1) ? -ru[j] : 0.0;
            double den = (xdiag[j] + ru[j] + rd[j]) - l * cprev;
            h.lo[j] = l;
            h.inv[j] = 1.0 / den;
            h.cp[j] = u * h.inv[j];
            cprev = h.cp[j];
        }
        auto solve = [&](std::vector<double>& v) {   // v on [a, b) in place
            double prev = 0.0;
            for (int j = a; j < b; j++) { prev = (v[j] - h.lo[j] * prev) * h.inv[j]; v[j] = prev; }
            double next = 0.0;
            for (int j = b - 1; j >= a; j--) { next = v[j] - h.cp[j] * next; v[j] = next; }
        };
        std::vector<double> e(NK, 0.0);
        if (a > 0) { e[a] = -rd[a]; solve(e); for (int j = a; j < b; j++) h.gL[j] = e[j]; }
        std::fill(e.begin(), e.end(), 0.0);
        if (b < NK) { e[b - 1] = -ru[b - 1]; solve(e); for (int j = a; j < b; j++) h.gR[j] = e[j]; }
    }
    // Reduced system of the segment ends, unknowns (first_s, last_s):
    //   x_j + gL_s[j] last_{s-1} + gR_s[j] first_{s+1} = y_j,  j = a_s, b_s - 1.
    // In the order (first_0, last_0, first_1, ...) it is pentadiagonal; its LU
    // without pivoting (I + small spikes) stays in the band.
    const int n = 2 * S;
    std::vector<double> M((size_t)n * n, 0.0);
    for (int s = 0; s < S; s++) {
        int a = (s * NK) / S, b = ((s + 1) * NK) / S;
        for (int r = 0; r < 2; r++) {
            int row = 2 * s + r, j = r ? b - 1 : a;
            M[(size_t)row * n + row] += 1.0;
            if (s > 0) M[(size_t)row * n + 2 * (s - 1) + 1] += h.gL[j];
            if (s + 1 < S) M[(size_t)row * n + 2 * (s + 1)] += h.gR[j];
        }
    }
    for (int c = 0; c < n; c++)        // Doolittle in place: M = L U
        for (int r = c + 1; r < n && r <= c + 2; r++) {
            double f = M[(size_t)r * n + c] / M[(size_t)c * n + c];
            M[(size_t)r * n + c] = f;
            for (int j = c + 1; j < n && j <= c + 2; j++) M[(size_t)r * n + j] -= f * M[(size_t)c * n + j];
        }
    h.band.assign((size_t)5 * n, 0.0);
    for (int i = 0; i < n; i++) {
        h.band[0 * n + i] = (i >= 1) ? M[(size_t)i * n + i - 1] : 0.0;
        h.band[1 * n + i] = (i >= 2) ? M[(size_t)i * n + i - 2] : 0.0;
        h.band[2 * n + i] = (i + 1 < n) ? M[(size_t)i * n + i + 1] : 0.0;
        h.band[3 * n + i] = (i + 2 < n) ? M[(size_t)i * n + i + 2] : 0.0;
        h.band[4 * n + i] = 1.0 / M[(size_t)i * n + i];
    }
    return h;
}

template <typename P>
struct Multigrid {
    int NK = 0, nlev = 0, S = 0, LS = 8, lc = 0;   // lc: first level run in the coarse block
    bool modes = false;        // level lc is solved exactly by Fourier modes
    ModeSolve ms{};
    size_t mode_smem = 0;
    bool exact_coarsest = true;
    int coarse_sweeps = 1;
    std::vector<int> nx, pitch;
    std::vector<P*> f, x, y;
    std::vector<LineLevel> lines;
    double *ru = nullptr, *rd = nullptr;
    P omega = P(2.0 / 3.0);
    Stats* stats = nullptr;

    double* upload(Arena& ar, const std::vector<double>& v) {
        double* d = ar.alloc<double>(v.size());
        upload_now(d, v.data(), v.size() * sizeof(double));
        return d;
    }

    void build(Arena& ar, int NX, int NKr, const std::vector<double>& cx0, const std::vector<double>& ru_h,
               const std::vector<double>& rd_h) {
        NK = NKr;
        LS = NK <= 256 ? 8 : (NK <= 512 ? 16 : 32);
        S = (NK + LS - 1) / LS;
        int n = NX;
        nx.push_back(n);
        while (n % 2 == 0 && n > 1) {
            n /= 2;
            nx.push_back(n);
        }
        nlev = (int)nx.size();
        exact_coarsest = (nx.back() == 1);
        coarse_sweeps = exact_coarsest ? 1 : 2 * nx.back() + 8;
        lc = nlev - 1;
        while (lc > 0 && nx[lc - 1] <= 32) lc--;
        if (nlev - lc > kMaxCoarseLevels) lc = nlev - kMaxCoarseLevels;
        // exact Fourier-mode solve on the first level of at most 32 columns
        // when its shared-memory tiles (f / solution and the reduced-system
        // bands, next to 32 KB of static tiles) fit in 227 KB
        for (int l = 0; l < nlev; l++) {
            if (nx[l] <= 32 && ((size_t)NK + 10 * (size_t)S) * nx[l] * sizeof(P) <= (size_t)kModeSmemMax) {
                modes = true;
                lc = l;
                nlev = l + 1;   // coarser levels are not needed
                nx.resize(nlev);
                break;
            }
        }
        ru = upload(ar, ru_h);
        rd = upload(ar, rd_h);
        for (int l = 0; l < nlev; l++) {
            int pl = round_up(nx[l], kPad);
            pitch.push_back(pl);
            f.push_back(l == 0 ? nullptr : ar.alloc<P>((size_t)NK * pl));
            x.push_back(ar.alloc<P>((size_t)NK * pl));
            y.push_back(ar.alloc<P>((size_t)NK * pl));
            std::vector<double> c(NK), xd(NK);
            double sc = std::pow(0.25, l);
            bool exact = (l == nlev - 1) && exact_coarsest;
            for (int k = 0; k < NK; k++) {
                c[k] = cx0[k] * sc;
                xd[k] = exact ? 0.0 : 2.0 * c[k];
            }
            HostLine h = factor_partitioned(xd, ru_h, rd_h, S);
            LineLevel L{nx[l], pl, NK, S, upload(ar, c), upload(ar, h.lo), upload(ar, h.inv), upload(ar, h.cp),
                        upload(ar, h.gL), upload(ar, h.gR), upload(ar, h.band)};
            lines.push_back(L);
            if (modes && l == lc) build_modes(ar, c, ru_h, rd_h, pl);
        }
    }

    // Orthonormal real Fourier basis of nc periodic columns and the per-mode
    // partitioned factors of (cx mu_m + ru + rd, -ru, -rd).
    void build_modes(Arena& ar, const std::vector<double>& c, const std::vector<double>& ru_h,
                     const std::vector<double>& rd_h, int pl) {
        const int nc = nx[lc];
        const double pi = 3.14159265358979323846;
        std::vector<double> Q((size_t)nc * nc, 0.0), mu(nc, 0.0);
        int m = 0;
        for (int j = 0; j < nc; j++) Q[(size_t)j * nc + m] = 1.0 / std::sqrt((double)nc);
        mu[m++] = 0.0;
        for (int fr = 1; 2 * fr < nc; fr++) {
            for (int j = 0; j < nc; j++) {
                Q[(size_t)j * nc + m] = std::sqrt(2.0 / nc) * std::cos(2 * pi * fr * j / nc);
                Q[(size_t)j * nc + m + 1] = std::sqrt(2.0 / nc) * std::sin(2 * pi * fr * j / nc);
            }
            mu[m] = mu[m + 1] = 2.0 - 2.0 * std::cos(2 * pi * fr / nc);
            m += 2;
        }
        if (nc % 2 == 0) {
            for (int j = 0; j < nc; j++) Q[(size_t)j * nc + m] = ((j & 1) ? -1.0 : 1.0) / std::sqrt((double)nc);
            mu[m++] = 4.0;
        }
        std::vector<double> lo((size_t)NK * nc), inv((size_t)NK * nc), cp((size_t)NK * nc), gL((size_t)NK * nc),
            gR((size_t)NK * nc), Mi((size_t)5 * 2 * S * nc);
        const size_t S2 = 2 * (size_t)S;
        for (int q = 0; q < nc; q++) {   // mode fastest: lanes (modes) read consecutive words
            std::vector<double> xd(NK);
            for (int k = 0; k < NK; k++) xd[k] = c[k] * mu[q];
            HostLine h = factor_partitioned(xd, ru_h, rd_h, S);
            for (int k = 0; k < NK; k++) {
                lo[(size_t)k * nc + q] = h.lo[k];
                inv[(size_t)k * nc + q] = h.inv[k];
                cp[(size_t)k * nc + q] = h.cp[k];
                gL[(size_t)k * nc + q] = h.gL[k];
                gR[(size_t)k * nc + q] = h.gR[k];
            }
            for (size_t e = 0; e < 5 * S2; e++) Mi[e * nc + q] = h.band[e];
        }
        ms = ModeSolve{nc, pl, NK, S, upload(ar, Q), upload(ar, lo), upload(ar, inv), upload(ar, cp),
                       upload(ar, gL), upload(ar, gR), upload(ar, Mi)};
        mode_smem = ((size_t)NK * nc + (size_t)10 * S * nc) * sizeof(P);
        auto setattr = [&](auto kern) {
            // the attribute is per kernel, not per context: set the largest any
            // context may use (the fit test above), so contexts of other sizes
            // in the same process never lower it under each other
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kModeSmemMax));
        };
        if (LS == 8) setattr(k_coarse_modes<P, 8>);
        else if (LS == 16) setattr(k_coarse_modes<P, 16>);
        else setattr(k_coarse_modes<P, 32>);
    }

    ZOps zops() const { return ZOps{ru, rd, NK}; }

    void sweep(int l, const P* fl, const P* xin, const P* xc, int pc, int nc, P* out, P om, cudaStream_t st) {
        SweepArgs<P> a{lines[l], zops(), fl, xin, xc, pc, nc, out, om};
        dim3 g(cdiv(nx[l], 32)), b(32 * S);
        if (LS == 8) LAUNCH(stats, VVM_K_MG_SWEEP, st, k_line_sweep<P, 8><<<g, b, 0, st>>>(a));
        else if (LS == 16) LAUNCH(stats, VVM_K_MG_SWEEP, st, k_line_sweep<P, 16><<<g, b, 0, st>>>(a));
        else LAUNCH(stats, VVM_K_MG_SWEEP, st, k_line_sweep<P, 32><<<g, b, 0, st>>>(a));
        CKL();
    }

    // z = M r (one V(1,1) cycle); returns the buffer holding z.
    P* apply(const P* r, cudaStream_t st) {
        const P* fl = r;
        for (int l = 0; l < lc; l++) {
            // pre-smoothing from zero fused with the restriction of its residual
            dim3 g(cdiv(nx[l], kOwned)), b(32 * S);
            if (LS == 8) LAUNCH(stats, VVM_K_MG_SWEEP, st, k_presmooth_restrict<P, 8><<<g, b, 0, st>>>(lines[l], zops(), fl, x[l], f[l + 1], pitch[l + 1], omega));
            else if (LS == 16) LAUNCH(stats, VVM_K_MG_SWEEP, st, k_presmooth_restrict<P, 16><<<g, b, 0, st>>>(lines[l], zops(), fl, x[l], f[l + 1], pitch[l + 1], omega));
            else LAUNCH(stats, VVM_K_MG_SWEEP, st, k_presmooth_restrict<P, 32><<<g, b, 0, st>>>(lines[l], zops(), fl, x[l], f[l + 1], pitch[l + 1], omega));
            CKL();
            fl = f[l + 1];
        }
        P* res;
        if (modes) {
            P* out = (lc == 0) ? y[0] : x[lc];
            if (LS == 8) LAUNCH(stats, VVM_K_MG_COARSE, st, k_coarse_modes<P, 8><<<1, 32 * S, mode_smem, st>>>(ms, fl, out));
            else if (LS == 16) LAUNCH(stats, VVM_K_MG_COARSE, st, k_coarse_modes<P, 16><<<1, 32 * S, mode_smem, st>>>(ms, fl, out));
            else LAUNCH(stats, VVM_K_MG_COARSE, st, k_coarse_modes<P, 32><<<1, 32 * S, mode_smem, st>>>(ms, fl, out));
            CKL();
            res = out;
        } else {
            // levels lc..nlev-1 in one block
            CoarseCycleArgs<P> ca{};
            ca.nlev = nlev - lc;
            for (int j = 0; j < ca.nlev; j++) {
                ca.L[j] = lines[lc + j];
                ca.f[j] = f[lc + j];
                ca.x[j] = x[lc + j];
                ca.y[j] = y[lc + j];
            }
            ca.z = zops();
            ca.f0 = fl;
            ca.omega = omega;
            ca.coarse_sweeps = coarse_sweeps;
            if (LS == 8) LAUNCH(stats, VVM_K_MG_COARSE, st, k_mg_coarse_cycle<P, 8><<<1, 32 * S, 0, st>>>(ca));
            else if (LS == 16) LAUNCH(stats, VVM_K_MG_COARSE, st, k_mg_coarse_cycle<P, 16><<<1, 32 * S, 0, st>>>(ca));
            else LAUNCH(stats, VVM_K_MG_COARSE, st, k_mg_coarse_cycle<P, 32><<<1, 32 * S, 0, st>>>(ca));
            CKL();
            res = y[lc];
        }
        for (int l = lc - 1; l >= 0; l--) {
            const P* fl2 = (l == 0) ? r : f[l];
            sweep(l, fl2, x[l], res, pitch[l + 1], nx[l + 1], y[l], omega, st);
            res = y[l];
        }
        return res;
    }
};

// Exact Fourier-mode preconditioner (spectral_kernels.cuh); NX a power of two.
template <typename P>
struct Spectral {
    SpecArgs<P> a{};
    P* out = nullptr;
    size_t smem = 0;
    int threads = 0;
    Stats* stats = nullptr;

    static bool supports(int NX) { return NX >= 4 && NX <= 8192 && (NX & (NX - 1)) == 0; }

    static P* upload(Arena& ar, const std::vector<double>& v) {
        std::vector<P> h(v.begin(), v.end());
        P* d = ar.alloc<P>(h.size());
        upload_now(d, h.data(), h.size() * sizeof(P));
        return d;
    }

    void build(Arena& ar, int NX, int NK, int pitch, const std::vector<double>& cx0, const std::vector<double>& ru,
               const std::vector<double>& rd) {
        int logN = 0;
        while ((1 << logN) < NX) logN++;
        const int M = NX / 2 + 1, mp = round_up(M, 32);
        const double pi = 3.14159265358979323846;
        std::vector<double> twr(NX / 2), twi(NX / 2);
        for (int j = 0; j < NX / 2; j++) {
            twr[j] = std::cos(2.0 * pi * j / NX);
            twi[j] = -std::sin(2.0 * pi * j / NX);
        }
        // twisted factorisation of each mode's z operator (spectral_kernels.cuh):
        // rows 0..mid eliminated downwards, mid+1..NK-1 upwards
        const int mid = (NK - 1) / 2;
        std::vector<double> inv((size_t)NK * mp, 0.0), cp((size_t)NK * mp, 0.0), den(mp, 0.0);
        for (int m = 0; m < M; m++) {
            const double mu = 2.0 - 2.0 * std::cos(2.0 * pi * m / NX);
            double up_over_piv = 0.0;   // ru_{k-1} / piv_{k-1}
            for (int k = 0; k <= mid; k++) {
                const double piv = cx0[k] * mu + ru[k] + rd[k] - (k > 0 ? rd[k] * up_over_piv : 0.0);
                inv[(size_t)k * mp + m] = 1.0 / piv;
                cp[(size_t)k * mp + m] = -ru[k] / piv;
                up_over_piv = ru[k] / piv;
            }
            double dn_over_piv = 0.0;   // rd_{k+1} / piv_{k+1}
            for (int k = NK - 1; k > mid; k--) {
                const double piv = cx0[k] * mu + ru[k] + rd[k] - (k + 1 < NK ? ru[k] * dn_over_piv : 0.0);
                inv[(size_t)k * mp + m] = 1.0 / piv;
                cp[(size_t)k * mp + m] = -rd[k] / piv;
                dn_over_piv = rd[k] / piv;
            }
            den[m] = 1.0 / (1.0 - cp[(size_t)mid * mp + m] * cp[(size_t)(mid + 1) * mp + m]);
        }
        a.NX = NX;
        a.logN = logN;
        a.NK = NK;
        a.pitch = pitch;
        a.mpitch = mp;
        a.mid = mid;
        a.twr = upload(ar, twr);
        a.twi = upload(ar, twi);
        a.inv = upload(ar, inv);
        a.cp = upload(ar, cp);
        a.den = upload(ar, den);
        a.rd = upload(ar, rd);
        a.ru = upload(ar, ru);
        a.sre = ar.alloc<P>((size_t)NK * mp);
        a.sim = ar.alloc<P>((size_t)NK * mp);
        out = ar.alloc<P>((size_t)NK * pitch);
        smem = 3 * (size_t)NX * sizeof(P);   // the row pair (re, im) and the twiddles
        threads = std::max(32, std::min(NX / 2, 512));
        // per-kernel attribute: the largest row any context may have (NX = 8192)
        const int smax = 3 * 8192 * (int)sizeof(P);
        CK(cudaFuncSetAttribute(k_spec_forward<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
        CK(cudaFuncSetAttribute(k_spec_inverse<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
    }

    // dst = S^{-1} r (to round-off).
    void apply_to(const P* r, P* dst, cudaStream_t st) {
        const int rows2 = cdiv(a.NK, 2);
        klaunch<k_spec_forward_body<P>, 1024>(stats, VVM_K_MG_SWEEP, st, k_spec_forward<P>, dim3(rows2), dim3(threads),
                                              smem, a, r);
        klaunch<k_spec_modes_seg_body<P>, 64 * kModeSegs>(stats, VVM_K_MG_COARSE, st, k_spec_modes_seg<P>,
                                                          dim3(cdiv(a.NX / 2 + 1, 32)), dim3(64 * kModeSegs), 0, a);
        klaunch<k_spec_inverse_body<P>, 1024>(stats, VVM_K_MG_SWEEP, st, k_spec_inverse<P>, dim3(rows2), dim3(threads),
                                              smem, a, dst);
    }
    // z = S^{-1} r; returns the buffer holding z.
    P* apply(const P* r, cudaStream_t st) {
        apply_to(r, out, st);
        return out;
    }
};

// ---------------------------------------------------------------- learned net

// Solver layout (FP64 [NK][pitch]) -> network layout (FP32 [H0][W0], rows
// >= NK zero): x = scale_k (a - sub) / sqrt(*nrm2) (sub, scale may be null);
// and back: a = scale_k z sqrt(*nrm2). The per-row scales map between the
// solver's variables and the network's (LearnedNet::set_operator).
__global__ void k_net_in(const double* a, const double* sub, int NX, int NK, int pitch, float* x, int H0,
                         const double* nrm2, const double* scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NX || k >= H0) return;
    const double s = (*nrm2 > 0) ? 1.0 / sqrt(*nrm2) : 0.0;
    const size_t e = (size_t)k * pitch + i;
    x[(size_t)k * NX + i] = (k < NK) ? (float)((a[e] - (sub ? sub[e] : 0.0)) * s * (scale ? scale[k] : 1.0)) : 0.f;
}

// partial sums of (scale_k a)^2: the norm of the network's input.
__global__ void k_net_sdot(VecArgs<double> v, const double* a, const double* scale, double* partial) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        const double x = a[(size_t)kk * v.pitch + i] * scale[kk];
        s[0] = x * x;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// White noise in the solver layout: a[k][i] = N(0, 1) from a counter hash
// (Box-Muller on two 32-bit uniforms), seeded.
__global__ void k_white_noise(double* a, int NX, int NK, int pitch, unsigned seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NX || k >= NK) return;
    auto mix = [](unsigned x) {
        x ^= x >> 16;
        x *= 0x7feb352du;
        x ^= x >> 15;
        x *= 0x846ca68bu;
        x ^= x >> 16;
        return x;
    };
    const unsigned id = (unsigned)(k * NX + i);
    const unsigned h1 = mix(id * 2u + 1u + seed * 0x9E3779B9u), h2 = mix(id * 2u + 2u + seed * 0x85EBCA6Bu);
    const double u1 = (h1 + 1.0) / 4294967297.0, u2 = h2 / 4294967296.0;
    a[(size_t)k * pitch + i] = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

__global__ void k_net_out(const float* z, int NX, int NK, int pitch, double* a, const double* nrm2,
                          const double* scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NX || k >= NK) return;
    a[(size_t)k * pitch + i] = (double)z[(size_t)k * NX + i] * sqrt(*nrm2 > 0 ? *nrm2 : 0.0) * (scale ? scale[k] : 1.0);
}

// Truncated flexible CG of the learned preconditioner (fcg_learned): up to
// kFcgM-1 earlier directions (or their S images), in ring slots `slot`.
constexpr int kFcgM = 8;
// Device state of the flexible-CG loop. Iteration k (from 0) writes ring
// slot k % kFcgM and orthogonalises against the fcg_cnt(k) slots before it,
// newest first, so the kernels of one recorded iteration serve every pass of
// a graph loop.
struct FcgCtl {
    int k;           // iterations done
    int converged;   // the loop stopped on the tolerance (or ||b|| = 0)
};
__device__ __forceinline__ int fcg_cnt(int k) { return k < kFcgM - 1 ? k : kFcgM - 1; }
__device__ __forceinline__ int fcg_prev(int k, int j) { return (k - 1 - j) % kFcgM; }

// The direction ring in device memory: ring[s] = p_s, ring[kFcgM + s] = q_s = S p_s.
using FcgRing = double* const*;

// Partials of (z, q_j), j < fcg_cnt(k): row j of `partial` holds one value a block.
__global__ void k_fcg_multidot(VecArgs<double> v, const double* z, FcgRing ring, const FcgCtl* ctl, double* partial) {
    __shared__ double sh[kFcgM * 32];
    const int k = ctl->k, cnt = fcg_cnt(k);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[kFcgM] = {};
    if (i < v.nx && kk < v.NK) {
        const size_t id = (size_t)kk * v.pitch + i;
        const double zv = z[id];
#pragma unroll
        for (int j = 0; j < kFcgM; j++)
            if (j < cnt) s[j] = zv * ring[kFcgM + fcg_prev(k, j)][id];
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const int b = blockIdx.x + gridDim.x * blockIdx.y, nb = gridDim.x * gridDim.y;
        for (int j = 0; j < cnt; j++) partial[(size_t)j * nb + b] = s[j];
    }
}

// beta_j = (z, q_j) / (p_j, q_j), the sums finished in a fixed order (one block).
__global__ void k_fcg_beta(const double* partial, int npart, const FcgCtl* ctl, const double* pq, double* beta) {
    __shared__ double sh[32];
    const int k = ctl->k, cnt = fcg_cnt(k);
    for (int j = 0; j < cnt; j++) {
        double s[1] = {0};
        for (int b = threadIdx.x; b < npart; b += blockDim.x) s[0] += partial[(size_t)j * npart + b];
        block_sum(s, sh);
        if (threadIdx.x == 0) {
            const double d = pq[fcg_prev(k, j)];
            beta[j] = (d != 0.0) ? s[0] / d : 0.0;
        }
    }
}

// p_k = z - sum_j beta_j p_j.
__global__ void k_fcg_dir(VecArgs<double> v, const double* z, FcgRing ring, const FcgCtl* ctl, const double* beta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= v.nx || kk >= v.NK) return;
    const int k = ctl->k, cnt = fcg_cnt(k);
    const size_t id = (size_t)kk * v.pitch + i;
    double y = z[id];
    for (int j = 0; j < cnt; j++) y -= beta[j] * ring[fcg_prev(k, j)][id];
    ring[k % kFcgM][id] = y;
}

// q_k = S p_k and the partials of (p_k, q_k) and (p_k, r).
__global__ void k_fcg_spmv(VecArgs<double> v, FcgRing ring, const FcgCtl* ctl, const double* r, double* ppq,
                           double* ppr) {
    __shared__ double sh[2 * 32];
    const int slot = ctl->k % kFcgM;
    const double* p = ring[slot];
    double* q = ring[kFcgM + slot];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[2] = {0, 0};
    if (i < v.nx && kk < v.NK) {
        const double y = s_apply(p, v.pitch, v.nx, v.NK, v.z, v.cx, kk, i);
        const size_t id = (size_t)kk * v.pitch + i;
        q[id] = y;
        s[0] = p[id] * y;
        s[1] = p[id] * r[id];
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const int b = blockIdx.x + gridDim.x * blockIdx.y;
        ppq[b] = s[0];
        ppr[b] = s[1];
    }
}

// alpha = (p, r) / (p, q) from the partials of both; keeps (p, q) for the ring slot.
__global__ void k_fcg_alpha(const double* ppq, const double* ppr, int npart, CGScalars* sc, double* pq,
                            const FcgCtl* ctl) {
    __shared__ double sh[64];
    double s[2] = {0, 0};
    for (int b = threadIdx.x; b < npart; b += blockDim.x) {
        s[0] += ppq[b];
        s[1] += ppr[b];
    }
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        sc->pq = s[0];
        sc->alpha = (s[0] != 0.0) ? s[1] / s[0] : 0.0;
        pq[ctl->k % kFcgM] = s[0];
    }
}

// x += alpha p_k; r -= alpha q_k; partial ||rhow r||^2.
__global__ void k_fcg_update(VecArgs<double> v, const CGScalars* sc, FcgRing ring, const FcgCtl* ctl, double* x,
                             double* r, double* partial) {
    __shared__ double sh[32];
    const int slot = ctl->k % kFcgM;
    const double* p = ring[slot];
    const double* q = ring[kFcgM + slot];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        const double al = sc->alpha;
        const size_t id = (size_t)kk * v.pitch + i;
        x[id] = x[id] + al * p[id];
        const double rn = r[id] - al * q[id];
        r[id] = rn;
        const double wr = v.rhow_k[kk] * rn;
        s[0] = wr * wr;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// Loop condition of the flexible-CG loop (one block): ||rhow r||^2 from the
// partials, in a fixed order, into sc->rr; `init` starts the loop (k = 0),
// otherwise iteration k has finished (k + 1, and its body's kernels counted
// in *exec). Continues while ||rhow r||^2 > tol^2 ||b||^2 and k < cap.
__global__ void k_fcg_loop(const double* partial, int npart, CGScalars* sc, FcgCtl* ctl,
                           cudaGraphConditionalHandle h, double tol2, int cap, int init, long long* exec,
                           int body_kernels) {
    __shared__ double sh[32];
    double s[1] = {0};
    for (int b = threadIdx.x; b < npart; b += blockDim.x) s[0] += partial[b];
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        const double rr = s[0], bb = sc->bb;
        sc->rr = rr;
        if (init) {
            ctl->k = 0;
        } else {
            ctl->k++;
            *exec += body_kernels;
        }
        const bool above = (bb > 0.0) && !(rr <= tol2 * bb);   // a NaN residual counts as above
        ctl->converged = !above;
        cudaGraphSetConditional(h, (above && isfinite(rr) && ctl->k < cap) ? 1u : 0u);
    }
}

// z += gam d (the Galerkin-scaled network correction).
__global__ void k_net_galerkin(int NX, int NK, int pitch, const CGScalars* sc, const double* d, double* z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= NX || k >= NK) return;
    const size_t e = (size_t)k * pitch + i;
    z[e] += sc->gam * d[e];
}

// The learned preconditioner (learned_kernels.cuh): a linear 4-level network,
// lift 1 -> 32, three levels of (2x2 average pool, 3x3 conv 32 -> 32 on the
// tensor cores), three levels of (nearest upsampling + the skip from the same
// level, 3x3 conv), projection 32 -> 1. Level 0 is the cal_w grid padded to
// H0 = round_up(NK, 8) rows (W0 = NX, a multiple of 8). FP32 master weights
// with Adam; BF16 operands and activations, FP32 accumulation.
// The 3x3 32 -> 32 convolution of the learned preconditioner: rows of at
// least kCBox pixels (W a multiple of 8) go to the streamed TMA kernel, the
// rest to the one-row-tile kernel. Tensor maps (3D {64, W / 8, 4 H} over the
// chunk-major BF16 activations, boxes {64, 18, 1} and {64, 1, 1}) are encoded
// through the driver's cuTensorMapEncodeTiled and cached per (tensor, H, W,
// box width): the map is a function of those alone.
// The driver's tensor-map encoder (looked up once).
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) throw CudaError{"cuTensorMapEncodeTiled: not found in the driver"};
        enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    return enc;
}

// Tensor map of one field buffer for the stencils' TMA staging: nz rows of
// nx columns (the pitch padding outside it, so loads past column nx-1 or row
// nz-1 fill zeros), element size 8 (FP64) or 4 (FP32), box {bx, by}. Cached
// per (buffer, shape, box): the map is a function of those alone.
CUtensorMap field_map(const void* p, int nx, int nz, int pitch, int elem, int bx, int by) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, int, int, int, int>, CUtensorMap> cache;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(p, nx, nz, pitch, elem, bx, by);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)nz};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * (cuuint64_t)elem};
    cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by}, es[2] = {1, 1};
    CUresult r = enc(&m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                     const_cast<void*>(p), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError{"cuTensorMapEncodeTiled (field) failed"};
    cache.emplace(key, m);
    return m;
}

CUtensorMap conv_map(const void* p, int H, int W, int boxw) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, int>, CUtensorMap> cache;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(p, H, W, boxw);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    // chunk-major activations as {64 elements (8 pixels x 8 channels), W / 8
    // pixel blocks, 4 H chunk rows}; boxw counts pixels (a multiple of 8)
    CUtensorMap m;
    cuuint64_t dims[3] = {64, (cuuint64_t)(W / 8), (cuuint64_t)(4 * H)};
    cuuint64_t strides[2] = {128, (cuuint64_t)W * 16};
    cuuint32_t box[3] = {64, (cuuint32_t)(boxw / 8), 1}, es[3] = {1, 1, 1};
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(p), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError{"cuTensorMapEncodeTiled failed"};
    cache.emplace(key, m);
    return m;
}

// Output rows per CTA of the streamed kernel: the fewest that fit the grid
// into one wave of two CTAs a SM (its shared memory allows two); a grid just
// over a wave would run its last CTAs alone, doubling the time.
int conv_rows_per_cta(int H, int W) {
    static int sms[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) {
        CK(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(k_conv32_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvStreamSmem));
    }
    const long strips = cdiv(W, kConvTile), slots = 2L * sms[dev];
    const long groups = std::max(1L, std::min((long)H, slots / strips));
    return (int)((H + groups - 1) / groups);
}

void conv32(const __nv_bfloat16* in, __nv_bfloat16* out, const uint4* w, int H, int W, int* err, cudaStream_t st,
            Stats* stats) {
    if (W >= kCBox && W % 8 == 0) {
        const int R = conv_rows_per_cta(H, W);
        const CUtensorMap trow = conv_map(in, H, W, kCBox), twrap = conv_map(in, H, W, 8);
        ConvStreamArgs a{in, out, w, H, W, R, err};
        const int grid = cdiv(W, kConvTile) * cdiv(H, R);
        LAUNCH(stats, VVM_K_CONV, st, k_conv32_stream<<<grid, kCThreads, kConvStreamSmem, st>>>(trow, twrap, a));
    } else {
        ConvArgs a{in, out, w, H, W, err};
        LAUNCH(stats, VVM_K_CONV, st, k_conv32_tc<<<H * cdiv(W, kConvTile), kConvTile, 0, st>>>(a));
    }
    CKL();
}

struct LearnedNet {
    static constexpr int kLift = 0, kConvs = 9 * kNetC, kConvSize = 9 * kNetC * kNetC;
    static constexpr int kProj = kConvs + 6 * kConvSize, kParams = kProj + 9 * kNetC;
    // conv order in the parameter array: D1 D2 D3 (down, levels 1-3), U2 U1 U0 (up)
    int NX = 0, NK = 0, H[4] = {}, W[4] = {};
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    uint4 *pk = nullptr, *pkT = nullptr;       // packed forward / adjoint operands, 6 x 1152
    float *x0 = nullptr, *z0 = nullptr, *dz = nullptr;
    __nv_bfloat16 *h[4] = {}, *pl[4] = {}, *u[3] = {}, *gg[3] = {};
    __nv_bfloat16 *dgb[4] = {}, *dub[3] = {}, *dpb[4] = {}, *dh3 = nullptr;
    double *part = nullptr, *lt = nullptr;
    float *op = nullptr, *sz = nullptr, *st = nullptr;   // rows' cx, ru, rd, diagonal ([4][H0]) for the loss; S z, S t
    double *dsc = nullptr, *dsc_inv = nullptr;             // per row D_k^{-1/2}, D_k^{1/2} ([NK])
    int* err = nullptr;
    int adam_t = 0;
    Stats* stats = nullptr;

    static bool supports(int NX, int NK) { return NX >= 8 && NX % 8 == 0 && NK >= 1; }

    // the cal_w operator's row coefficients (cx = 1/rhow_k, ru = 1/rhou_k,
    // rd = 1/rhou_{k-1}, k = kk + 2) in the network's rows
    // The network works in the variables of S~ = D^{-1/2} S D^{-1/2}, D the
    // diagonal of S (2 cx_k + ru_k + rd_k): every row of S~ has diagonal 1, so
    // its coefficients vary little from level to level even where the
    // densities span orders of magnitude (deep or stretched levels), which a
    // translation-invariant network needs. Input D^{-1/2} r, output mapped
    // back by D^{-1/2}, target D^{1/2} e; (e, S e) = (D^{1/2} e, S~ D^{1/2} e).
    void set_operator(const std::vector<double>& rhou, const std::vector<double>& rhow,
                      const std::vector<double>& ma, const std::vector<double>& mh) {
        std::vector<double> cx(NK), ru(NK), rd(NK), s(NK), si(NK);
        for (int kk = 0; kk < NK; kk++) {
            const int k = kk + 2;
            cx[kk] = ma[k] / rhow[k];
            ru[kk] = mh[k] / rhou[k];
            rd[kk] = mh[k - 1] / rhou[k - 1];
            const double dg = 2.0 * cx[kk] + ru[kk] + rd[kk];
            s[kk] = 1.0 / std::sqrt(dg);
            si[kk] = std::sqrt(dg);
        }
        std::vector<float> h(4 * (size_t)H[0], 0.f);
        for (int kk = 0; kk < NK; kk++) {
            h[kk] = (float)(cx[kk] * s[kk] * s[kk]);
            h[H[0] + kk] = (float)(ru[kk] * s[kk] * (kk + 1 < NK ? s[kk + 1] : s[kk]));
            h[2 * H[0] + kk] = (float)(rd[kk] * s[kk] * (kk > 0 ? s[kk - 1] : s[kk]));
            h[3 * H[0] + kk] = 1.f;
        }
        upload_now(dsc, s.data(), NK * sizeof(double));
        upload_now(dsc_inv, si.data(), NK * sizeof(double));
        upload_now(op, h.data(), h.size() * sizeof(float));
    }

    void build(Arena& ar, int NXr, int NKr, int seed) {
        NX = NXr;
        NK = NKr;
        H[0] = round_up(NK, 8);
        W[0] = NX;
        for (int l = 1; l < 4; l++) {
            H[l] = H[l - 1] / 2;
            W[l] = W[l - 1] / 2;
        }
        w = ar.alloc<float>(kParams);
        g = ar.alloc<float>(kParams);
        m = ar.alloc<float>(kParams);
        v = ar.alloc<float>(kParams);
        pk = ar.alloc<uint4>(6 * 9 * 4 * kNetC);
        pkT = ar.alloc<uint4>(6 * 9 * 4 * kNetC);
        const size_t n0 = (size_t)H[0] * W[0];
        x0 = ar.alloc<float>(n0);
        z0 = ar.alloc<float>(n0);
        dz = ar.alloc<float>(n0);
        for (int l = 0; l < 4; l++) {
            const size_t nl = (size_t)H[l] * W[l] * kNetC;
            h[l] = ar.alloc<__nv_bfloat16>(nl);
            dgb[l] = ar.alloc<__nv_bfloat16>(nl);
            dpb[l] = ar.alloc<__nv_bfloat16>(nl);
            if (l > 0) pl[l] = ar.alloc<__nv_bfloat16>(nl);
            if (l < 3) {
                u[l] = ar.alloc<__nv_bfloat16>(nl);
                gg[l] = ar.alloc<__nv_bfloat16>(nl);
                dub[l] = ar.alloc<__nv_bfloat16>(nl);
            }
        }
        dh3 = ar.alloc<__nv_bfloat16>((size_t)H[3] * W[3] * kNetC);
        part = ar.alloc<double>(3 * 1024);
        lt = ar.alloc<double>(4);
        op = ar.alloc<float>(4 * (size_t)H[0]);
        dsc = ar.alloc<double>(NK);
        dsc_inv = ar.alloc<double>(NK);
        sz = ar.alloc<float>(n0);
        st = ar.alloc<float>(n0);
        err = ar.alloc<int>(1);
        init_weights(seed);
    }

    // Seeded initial weights: N(0, 1/fan_in) per layer (fan_in = 9 inputs for
    // the lift, 9 * 32 otherwise), so each layer keeps the signal's scale.
    void init_weights(int seed) {
        std::vector<float> hw(kParams);
        uint64_t st = 0x9E3779B97F4A7C15ull ^ (uint64_t)seed;
        auto next = [&]() {   // xorshift64*
            st ^= st >> 12;
            st ^= st << 25;
            st ^= st >> 27;
            return (double)((st * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0);
        };
        auto normal = [&]() {
            double u1 = next(), u2 = next();
            if (u1 < 1e-300) u1 = 1e-300;
            return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
        };
        for (int j = 0; j < kParams; j++) {
            const double fan = (j < kConvs || j >= kProj) ? 9.0 : 9.0 * kNetC;
            hw[j] = (float)(normal() / std::sqrt(fan));
        }
        set_weights(hw.data());
    }

    void set_weights(const float* hw) {
        CK(cudaMemcpy(w, hw, kParams * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemset(m, 0, kParams * sizeof(float)));
        CK(cudaMemset(v, 0, kParams * sizeof(float)));
        adam_t = 0;
        pack(nullptr);
        CK(cudaStreamSynchronize(nullptr));
    }

    void pack(cudaStream_t st) {
        for (int c = 0; c < 6; c++) {
            const float* wc = w + kConvs + (size_t)c * kConvSize;
            LAUNCH(stats, VVM_K_LEARNED, st, k_pack_conv32<<<cdiv(9 * 4 * kNetC, 128), 128, 0, st>>>(wc, pk + (size_t)c * 1152, 0));
            CKL();
            LAUNCH(stats, VVM_K_LEARNED, st, k_pack_conv32<<<cdiv(9 * 4 * kNetC, 128), 128, 0, st>>>(wc, pkT + (size_t)c * 1152, 1));
            CKL();
        }
    }

    void conv(int c, bool adj, const __nv_bfloat16* in, __nv_bfloat16* out, int l, cudaStream_t st) {
        conv32(in, out, (adj ? pkT : pk) + (size_t)c * 1152, H[l], W[l], err, st, stats);
    }
    void sum4(const __nv_bfloat16* in, __nv_bfloat16* out, int lo, float mult, cudaStream_t st) {
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_sum4<<<cdiv(H[lo] * W[lo] * 4, 256), 256, 0, st>>>(in, out, H[lo], W[lo], mult));
        CKL();
    }
    void up_add(const __nv_bfloat16* lo, const __nv_bfloat16* skip, __nv_bfloat16* out, int l, float mult,
                cudaStream_t st) {
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_up_add<<<cdiv(H[l] * W[l] * 4, 256), 256, 0, st>>>(lo, skip, out, H[l], W[l], mult));
        CKL();
    }
    void wgrad(const __nv_bfloat16* X, const __nv_bfloat16* dY, int c, int l, cudaStream_t st) {
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_wgrad32<<<H[l] * cdiv(W[l], kConvTile), 256, 0, st>>>(X, dY, g + kConvs + (size_t)c * kConvSize, H[l], W[l]));
        CKL();
    }

    // z0 = net(x0), z0 rows >= NK set to zero.
    void forward(cudaStream_t st) {
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_lift<<<cdiv(4 * H[0] * W[0], 256), 256, 0, st>>>(x0, w + kLift, h[0], H[0], W[0]));
        CKL();
        for (int l = 1; l < 4; l++) {   // down: pool, conv D_l
            sum4(h[l - 1], pl[l], l, 0.25f, st);
            conv(l - 1, false, pl[l], h[l], l, st);
        }
        const __nv_bfloat16* lower = h[3];
        for (int l = 2; l >= 0; l--) {   // up: upsample + skip, conv U_l (index 3 + (2 - l))
            up_add(lower, h[l], u[l], l, 1.f, st);
            conv(3 + (2 - l), false, u[l], gg[l], l, st);
            lower = gg[l];
        }
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_proj<<<cdiv(4 * H[0] * W[0], 256), 256, 0, st>>>(gg[0], w + kProj, z0, H[0], W[0], NK, 1.f));
        CKL();
    }

    // The six 32 -> 32 convolutions of forward() alone, on the activations a
    // forward() left (for timing them).
    void convs_only(cudaStream_t st) {
        for (int l = 1; l < 4; l++) conv(l - 1, false, pl[l], h[l], l, st);
        for (int l = 2; l >= 0; l--) conv(3 + (2 - l), false, u[l], gg[l], l, st);
    }

    // g += d loss / d w for the gradient dz of the output (after forward()).
    void backward(cudaStream_t st) {
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_wgrad_edge<<<H[0], 9 * kNetC, 0, st>>>(dz, gg[0], g + kProj, H[0], W[0], 1));
        CKL();
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_proj_adj<<<cdiv(H[0] * W[0], 128), 128, 0, st>>>(dz, w + kProj, dgb[0], H[0], W[0]));
        CKL();
        // up path, level 0 first: du_l = U_l^T dg_l; dg_{l+1} = up^T du_l; dh_l = du_l
        for (int l = 0; l <= 2; l++) {
            const int c = 3 + (2 - l);
            conv(c, true, dgb[l], dub[l], l, st);
            wgrad(u[l], dgb[l], c, l, st);
            sum4(dub[l], l < 2 ? dgb[l + 1] : dh3, l + 1, 1.f, st);
        }
        // down path, level 3 first: dp_l = D_l^T dh_l; dh_{l-1} += pool^T dp_l
        const __nv_bfloat16* dh = dh3;
        for (int l = 3; l >= 1; l--) {
            conv(l - 1, true, dh, dpb[l], l, st);
            wgrad(pl[l], dh, l - 1, l, st);
            up_add(dpb[l], dub[l - 1], dub[l - 1], l - 1, 0.25f, st);   // dh_{l-1} lives in du_{l-1}
            dh = dub[l - 1];
        }
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_wgrad_edge<<<H[0], 9 * kNetC, 0, st>>>(x0, dub[0], g + kLift, H[0], W[0], 0));
        CKL();
    }

    // loss of z0 against target t (FP32 [H0][W0]): the S-norm error left by
    // the best multiple of z0, into lt[0]; dz = mult * dL/dz.
    void loss(const float* t, float mult, cudaStream_t s) {
        const size_t n = (size_t)H[0] * W[0];
        LAUNCH(stats, VVM_K_LEARNED, s, k_net_loss_partial<<<1024, 256, 0, s>>>(z0, t, op, H[0], W[0], NK, sz, st, part));
        CKL();
        LAUNCH(stats, VVM_K_LEARNED, s, k_net_loss_final<<<1, 1024, 0, s>>>(part, 1024, lt));
        CKL();
        LAUNCH(stats, VVM_K_LEARNED, s, k_net_loss_grad<<<1024, 256, 0, s>>>(sz, st, n, lt, dz, mult));
        CKL();
    }

    void adam(float lr, cudaStream_t st) {
        adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = 1.f - std::pow(b1, (float)adam_t), bc2 = 1.f - std::pow(b2, (float)adam_t);
        LAUNCH(stats, VVM_K_LEARNED, st, k_net_adam<<<cdiv(kParams, 256), 256, 0, st>>>(w, g, m, v, kParams, lr, b1, b2, 1e-8f, bc1, bc2));
        CKL();
        pack(st);
    }
};

// Preconditioned CG on S d = g in precision P with the level-0 vectors below.
template <typename P>
struct PCG {
    Multigrid<P> mg;
    Spectral<P> sp;
    bool spectral = false;   // Fourier-mode preconditioner instead of the V-cycle
    int NX = 0, NK = 0, pitch = 0;
    P *r = nullptr, *p = nullptr, *q = nullptr;
    double* partial = nullptr;
    int npart = 0;
    double* rhow_k = nullptr;
    CGScalars* sc = nullptr;
    CGScalars* sc_host = nullptr;
    CGCtl* ctl = nullptr;   // loop state of graph-captured solves
    unsigned* arrive = nullptr;   // arrival counter of k_cg_check's last block
    Stats* stats = nullptr;

    // S = -diag(1/rw) A in symmetric form: cx_k = a_k / rhow_k, ru_k = h_k /
    // rhou_k, rd_k = h_{k-1} / rhou_{k-1}, rw_k = rhow_k / a_k (a = h = 1 on
    // uniform levels: the reference's matrix, PoissonSolver.cpp:760-796).
    // `unweighted`: residual weight 1 on every row (the streamfunction
    // system, whose reference residual carries no rhow).
    void build(Arena& ar, int NXr, int NKr, const std::vector<double>& rhou, const std::vector<double>& rhow,
               const std::vector<double>& a, const std::vector<double>& h, bool unweighted = false) {
        NX = NXr;
        NK = NKr;
        std::vector<double> cx0(NK), ru(NK), rd(NK), rw(NK);
        for (int kk = 0; kk < NK; kk++) {
            int k = kk + 2;
            cx0[kk] = a[k] / rhow[k];
            ru[kk] = h[k] / rhou[k];
            rd[kk] = h[k - 1] / rhou[k - 1];
            rw[kk] = unweighted ? 1.0 : rhow[k] / a[k];
        }
        mg.stats = stats;
        mg.build(ar, NX, NK, cx0, ru, rd);
        pitch = mg.pitch[0];
        if (spectral) {
            sp.stats = stats;
            sp.build(ar, NX, NK, pitch, cx0, ru, rd);
        }
        r = ar.alloc<P>((size_t)NK * pitch);
        p = ar.alloc<P>((size_t)NK * pitch);
        q = ar.alloc<P>((size_t)NK * pitch);
        dim3 g = grid();
        npart = g.x * g.y;
        partial = ar.alloc<double>(npart);
        rhow_k = ar.alloc<double>(NK);
        upload_now(rhow_k, rw.data(), NK * sizeof(double));
        sc = ar.alloc<CGScalars>(1);
        ctl = ar.alloc<CGCtl>(1);
        arrive = ar.alloc<unsigned>(1);
        CK(cudaMallocHost(&sc_host, sizeof(CGScalars)));
    }
    void release() {
        if (sc_host) cudaFreeHost(sc_host);
        sc_host = nullptr;
    }
    dim3 block() const { return dim3(64, 4); }
    dim3 grid() const { return dim3(cdiv(NX, 64), cdiv(NK, 4)); }
    VecArgs<P> vargs() const { return VecArgs<P>{NX, pitch, NK, mg.zops(), mg.lines[0].cx, rhow_k}; }
    P* precond(const P* r, cudaStream_t st) { return spectral ? sp.apply(r, st) : mg.apply(r, st); }

    double read_rr(cudaStream_t st) {
        CK(cudaMemcpyAsync(sc_host, sc, sizeof(CGScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return sc_host->rr;
    }

    // One PCG iteration for a graph-captured loop (x, r resident, r holding
    // the current residual): z = M r, beta (0 on the loop's first pass),
    // p, q = S p, alpha, x += alpha p, r -= alpha q, ||rhow r||^2. Returns the
    // number of kernels recorded.
    int record_iteration(P* x, cudaStream_t st) {
        const long long n0 = stats->launches;
        VecArgs<P> v = vargs();
        dim3 B = block(), G = grid();
        P* z = precond(r, st);
        klaunch<k_cg_dot_body<P>, 256>(stats, VVM_K_CG, st, k_cg_dot<P>, G, B, 0, v, (const P*)r, (const P*)z, partial);
        klaunch<k_cg_scalar_it_body, 1024>(stats, VVM_K_CG, st, k_cg_scalar_it, dim3(1), dim3(1024), 0,
                                           (const double*)partial, npart, sc, (const CGCtl*)ctl);
        klaunch<k_cg_dir_it_body<P>, 256>(stats, VVM_K_CG, st, k_cg_dir_it<P>, G, B, 0, v, (const CGScalars*)sc,
                                          (const CGCtl*)ctl, (const P*)z, p);
        klaunch<k_cg_spmv_body<P>, 256>(stats, VVM_K_CG, st, k_cg_spmv<P>, G, B, 0, v, (const P*)p, q, partial);
        klaunch<k_cg_scalar_body, 1024>(stats, VVM_K_CG, st, k_cg_scalar, dim3(1), dim3(1024), 0,
                                        (const double*)partial, npart, sc, (int)CG_PQ_ALPHA);
        klaunch<k_cg_update_body<P>, 256>(stats, VVM_K_CG, st, k_cg_update<P>, G, B, 0, v, (const CGScalars*)sc, x, r,
                                          (const P*)p, (const P*)q, partial);
        klaunch<k_cg_scalar_body, 1024>(stats, VVM_K_CG, st, k_cg_scalar, dim3(1), dim3(1024), 0,
                                        (const double*)partial, npart, sc, (int)CG_SET_RR);
        return (int)(stats->launches - n0);
    }

    // Solves S x = g. x holds the initial guess when `warm`, else it is zeroed.
    // Stops when ||rhow (g - S x)||^2 <= rtol^2 * ref2; ref2 < 0 takes the
    // initial residual as the reference. Returns iterations; relres out
    // (relative to ref2). The stopping tests are the ones the graph-captured
    // loops evaluate on the device (k_loop_plain / k_loop_inner).
    int solve(const P* g, P* x, bool warm, double ref2, double rtol, int maxit, cudaStream_t st,
              double* relres) {
        VecArgs<P> v = vargs();
        dim3 B = block(), G = grid();
        if (!warm) CK(cudaMemsetAsync(x, 0, (size_t)NK * pitch * sizeof(P), st));
        LAUNCH(stats, VVM_K_CG, st, k_cg_residual<P><<<G, B, 0, st>>>(v, g, x, r, partial));
        CKL();
        LAUNCH(stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(partial, npart, sc, CG_SET_RR));
        CKL();
        double rr = read_rr(st);
        if (ref2 < 0.0) ref2 = rr;
        const double stop2 = (rtol * rtol) * ref2;
        if (!(ref2 > 0.0) || !(rr > stop2)) {
            *relres = (ref2 > 0) ? std::sqrt(rr / ref2) : 0.0;
            return 0;
        }
        P* z = precond(r, st);
        LAUNCH(stats, VVM_K_CG, st, k_cg_dot<P><<<G, B, 0, st>>>(v, r, z, partial));
        CKL();
        LAUNCH(stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(partial, npart, sc, CG_SET_RZ));
        CKL();
        LAUNCH(stats, VVM_K_CG, st, k_cg_dir<P><<<G, B, 0, st>>>(v, sc, z, p, 1));
        CKL();
        int it = 0;
        for (it = 1; it <= maxit; it++) {
            LAUNCH(stats, VVM_K_CG, st, k_cg_spmv<P><<<G, B, 0, st>>>(v, p, q, partial));
            CKL();
            LAUNCH(stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(partial, npart, sc, CG_PQ_ALPHA));
            CKL();
            LAUNCH(stats, VVM_K_CG, st, k_cg_update<P><<<G, B, 0, st>>>(v, sc, x, r, p, q, partial));
            CKL();
            LAUNCH(stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(partial, npart, sc, CG_SET_RR));
            CKL();
            rr = read_rr(st);
            if (!(rr > stop2) || !std::isfinite(rr) || it >= maxit) break;
            z = precond(r, st);
            LAUNCH(stats, VVM_K_CG, st, k_cg_dot<P><<<G, B, 0, st>>>(v, r, z, partial));
            CKL();
            LAUNCH(stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(partial, npart, sc, CG_RZ_BETA));
            CKL();
            LAUNCH(stats, VVM_K_CG, st, k_cg_dir<P><<<G, B, 0, st>>>(v, sc, z, p, 0));
            CKL();
        }
        *relres = std::sqrt(rr / ref2);
        return it > maxit ? maxit : it;
    }
};

enum { H_ZETA = 0, H_BUOY, H_TH, H_QV, H_QC, H_QR, H_VT, NHIST };

template <typename T>
struct Fields {
    T *zeta[2] = {}, *th[2] = {}, *qv[2] = {}, *qc[2] = {}, *qr[2] = {};
    T *u = nullptr, *w = nullptr, *RKM = nullptr, *RKH = nullptr;
    T* hist[NHIST][2] = {};
    T *d_auto = nullptr, *d_accr = nullptr, *d_evap = nullptr, *d_cond = nullptr;
    T *precip = nullptr, *th_forcing = nullptr;
    T* gsA = nullptr;                                   // Gauss-Seidel constant terms, [5][cells]
    T *gsC = nullptr, *gsB = nullptr;                   // and coefficients (cluster schedule; on first use)
    T *gsRight = nullptr, *gsTop = nullptr;             // Gauss-Seidel tile outflows (k_gs_tiles)
};

}  // namespace

// ===========================================================================
// Context

struct vvm_gpu_ctx {
    vvm_gpu_desc desc{};
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    Dims d{};
    Consts c{};
    bool mixed = false;
    bool spectral = false;   // VVM_SOLVER_SPECTRAL
    int tune_gs_tr = 0;      // rows of a Gauss-Seidel tile (0: automatic)
    GSTileCtl* gsctl = nullptr;   // pass state of the Gauss-Seidel tiles
    int* sc_host_i = nullptr;     // pinned: the tiles' "another pass" flag read by the host loop
    // learned preconditioner (VVM_SOLVER_LEARNED)
    std::unique_ptr<LearnedNet> net;
    double* z64 = nullptr;   // preconditioned residual, solver layout
    double *za64 = nullptr, *r164 = nullptr, *d64 = nullptr, *sd64 = nullptr;   // the learned cycle's work arrays
    double *fcg_p[kFcgM] = {}, *fcg_q[kFcgM] = {};   // flexible-CG direction ring and its S images
    double *fcg_part = nullptr, *fcg_pq = nullptr, *fcg_beta = nullptr;
    double** fcg_ring = nullptr;        // device copy of {fcg_p, fcg_q} (FcgRing)
    FcgCtl* fcg_ctl = nullptr;          // flexible-CG loop state
    FcgCtl* fcg_host = nullptr;         // pinned copy of it
    cudaGraphExec_t fcg_exec = nullptr; // the flexible-CG loop alone (fcg_graph)
    double fcg_tol = 0;
    int fcg_cap = 0, fcg_mode = -1;
    long long fcg_static = 0;           // kernels of fcg_exec outside its loop
    int learned_mode = 0;    // 0: the cycle with the network; 1: without it; 2: identity
    int learned_cap = 200;   // flexible-CG iterations before the multigrid-PCG fallback
    int learned_iters = 0, learned_fallback = 0;
    bool learned_collect = false;   // training-pair collection: solve with the plain solver
    int tune_fft = 0;        // threads of a row-FFT block (0: automatic)
    int tune_group = 0;      // in a batch: cases a grouped launch takes at most (0: the batch's limit)
    Arena ar;
    Fields<double> f64;
    Fields<float> f32;
    int cur = 0;       // buffer index of the "now" time level
    int step = 0;
    // The reference's nextTimeStep copies each future array into the present
    // one (src/Iteration.cpp:153-204), so after a whole step the model's *p
    // arrays equal the present ones. Here the rotation is a pointer swap and
    // the future buffers keep the previous level until the next step
    // overwrites them; true while that holds, so a state download returns the
    // present level for the *p arrays, as the reference's model holds them.
    bool fut_is_now = false;
    bool has_state = false, has_forcing_th = false, has_q = false;
    // profiles
    double *rhou = nullptr, *rhow = nullptr, *thvb = nullptr, *thb = nullptr, *qvb = nullptr,
           *thb_init = nullptr, *qvb0 = nullptr, *pib = nullptr, *pb = nullptr, *lambda2 = nullptr,
           *z = nullptr, *z_zeta = nullptr, *vt_c1 = nullptr, *vt_fac = nullptr, *pc = nullptr,
           *dtcgr_th = nullptr, *dtcgr_zeta = nullptr, *q1ls = nullptr, *q2ls = nullptr;
    double pf1 = 0, pf2 = 0;
    // perturbation profiles of th (0) and qv (1); used by the mixed step
    double *pref[2] = {}, *pd0[2] = {}, *ps0[2] = {}, *pg0[2] = {}, *pdn[2] = {};
    std::vector<double> h_rhou, h_rhow;
    // vertical metric of the cal_w operator: a_k = (z_k - z_{k-1}) / dx, h_k =
    // dx / (2 (z_k - z_zeta_k)); exactly 1 on uniform levels. `stretched`:
    // non-uniform levels, which only the Poisson entries support.
    std::vector<double> h_a, h_h;
    std::vector<double> h_forcing;   // [nx][nz] host copy of the last regenerated th forcing
    bool stretched = false;
    double* rwres = nullptr;   // [nz] residual weight rw_k = rhow_k / a_k
    // vertical level metric of the step's stencils (Profiles::r2dzc ...)
    double *lv_r2dzc = nullptr, *lv_r2dzw = nullptr, *lv_rdzc = nullptr, *lv_r2dzcc = nullptr, *lv_kmax = nullptr,
           *gsM_cz = nullptr, *gsM_rhod = nullptr, *gsS_cz = nullptr, *gsS_rhod = nullptr, *lv_dzw = nullptr;
    double lv_rdz_up = 0, lv_rdz_dn = 0, lv_rdz_c = 0, lv_hfac = 1;
    double* ubar = nullptr;   // [0] ubarTop, [1] ubarTopp
    double* dubar = nullptr;  // [2]
    double *partial = nullptr, *nvp = nullptr;
    int npart = 0;
    double* staging = nullptr;   // nx*nz*2 doubles
    // Poisson
    bool poisson_ready = false;
    std::unique_ptr<PCG<double>> pcg64;
    std::unique_ptr<PCG<float>> pcg32;
    double *Wf = nullptr, *W = nullptr, *r64 = nullptr;   // level-0 layout, FP64
    // streamfunction formulation (VVM_FLAG_STREAMFUNCTION / vvm_gpu_calpsiuw)
    std::unique_ptr<PCG<double>> pcg_psi;
    double *psi_f = nullptr, *psi_x = nullptr;   // right-hand side and solution, solver layout
    double* psi = nullptr;                       // [nz][pitch] field with its ghosts
    double* Wprev = nullptr;   // previous cal_w solution (initial-guess extrapolation)
    int nsolves = 0;
    // CUDA graphs of one whole step, by (time-level buffer, step parity)
    cudaGraphExec_t gexec[2][2] = {};
    long long gstatic[2][2] = {};      // kernels outside the solver loops
    cudaStream_t cap[2] = {};          // streams for capturing loop bodies
    cudaStream_t side = nullptr;       // the step's second chain (run_step)
    cudaEvent_t fork_ev[3] = {};       // its fork, meeting and join points
    cudaStream_t xfer = nullptr;       // host copies of the prognostic transfers
    cudaEvent_t xev[2][2] = {};        // per staging slot: [0] its copy done, [1] its layout kernel done
    bool branches = true;              // use them (off inside a batch: the cases are the branches)
    CGCtl* wctl = nullptr;             // outer loop state of the mixed solve
    long long* d_exec = nullptr;       // kernels executed inside graph loops
    int* d_err = nullptr;              // device error word (kGSErrWait), checked when the host syncs
    bool last_graph = false;           // the last cal_w ran inside a graph
    bool graphs_off = false;
    float *g32 = nullptr, *d32 = nullptr;
    double* wpartial = nullptr;
    int wnpart = 0;
    double* sc_host = nullptr;
    int last_iters = 0;
    double last_relres = 0;
    Stats stats;
    std::string err;

    void drop_graphs() {
        for (auto& row : gexec)
            for (auto& g : row)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
        if (fcg_exec) cudaGraphExecDestroy(fcg_exec);
        fcg_exec = nullptr;
    }

    ~vvm_gpu_ctx() {
        drop_graphs();
        if (fcg_host) cudaFreeHost(fcg_host);
        for (auto s : cap)
            if (s) cudaStreamDestroy(s);
        if (side) cudaStreamDestroy(side);
        for (auto e : fork_ev)
            if (e) cudaEventDestroy(e);
        if (xfer) cudaStreamDestroy(xfer);
        for (auto& row : xev)
            for (auto e : row)
                if (e) cudaEventDestroy(e);
        if (pcg64) pcg64->release();
        if (pcg32) pcg32->release();
        if (pcg_psi) pcg_psi->release();
        if (sc_host) cudaFreeHost(sc_host);
        if (sc_host_i) cudaFreeHost(sc_host_i);
        if (own) cudaStreamDestroy(own);
    }

    Profiles profiles() const {
        return Profiles{rhou, rhow, thvb, thb_init, qvb0, pib, pb, lambda2, vt_c1, vt_fac, pc,
                        dtcgr_th, dtcgr_zeta, q1ls, q2ls, pf1, pf2,
                        {pref[0], pref[1]}, {pd0[0], pd0[1]}, {ps0[0], ps0[1]}, {pg0[0], pg0[1]},
                        {pdn[0], pdn[1]},
                        lv_r2dzc, lv_r2dzw, lv_rdzc, lv_r2dzcc, lv_kmax, gsM_cz, gsM_rhod, gsS_cz, gsS_rhod, lv_dzw,
                        lv_rdz_up, lv_rdz_dn, lv_rdz_c, lv_hfac};
    }
    // profile subtracted from a stored field (mixed step: th and qv only)
    const double* offset_th() const { return mixed ? pref[0] : nullptr; }
    const double* offset_qv() const { return mixed ? pref[1] : nullptr; }
    dim3 blk() const { return dim3(64, 4); }
    dim3 grid_interior(int k0) const { return dim3(cdiv(d.nx - 2, 64), cdiv(d.nz - 1 - k0, 4)); }
    // k_padv's tiles of kPAdvBX x kPAdvBZ interior cells
    dim3 padv_blk() const { return dim3(kPAdvBX, kPAdvBZ); }
    dim3 padv_grid() const { return dim3(cdiv(d.nx - 2, kPAdvBX), cdiv(d.nz - 2, kPAdvBZ)); }
    dim3 grid_all() const { return dim3(cdiv(d.nx, 64), cdiv(d.nz, 4)); }
};

namespace {

std::string g_create_error;

int fail(vvm_gpu_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    else g_create_error = msg;
    return code;
}

template <typename T>
Fields<T>& fields(vvm_gpu_ctx* c);
template <>
Fields<double>& fields<double>(vvm_gpu_ctx* c) { return c->f64; }
template <>
Fields<float>& fields<float>(vvm_gpu_ctx* c) { return c->f32; }

template <typename T>
void alloc_fields(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    size_t n = c->d.cells();
    for (int b = 0; b < 2; b++) {
        F.zeta[b] = c->ar.alloc<T>(n);
        F.th[b] = c->ar.alloc<T>(n);
        F.qv[b] = c->ar.alloc<T>(n);
        F.qc[b] = c->ar.alloc<T>(n);
        F.qr[b] = c->ar.alloc<T>(n);
    }
    F.u = c->ar.alloc<T>(n);
    F.w = c->ar.alloc<T>(n);
    F.RKM = c->ar.alloc<T>(n);
    F.RKH = c->ar.alloc<T>(n);
    for (int h = 0; h < NHIST; h++)
        for (int s = 0; s < 2; s++) F.hist[h][s] = c->ar.alloc<T>(n);
    F.d_auto = c->ar.alloc<T>(n);
    F.d_accr = c->ar.alloc<T>(n);
    F.d_evap = c->ar.alloc<T>(n);
    F.d_cond = c->ar.alloc<T>(n);
    F.precip = c->ar.alloc<T>(c->d.nx);
    F.th_forcing = c->ar.alloc<T>(n);
    F.gsA = c->ar.alloc<T>(5 * n);
    // tile outflows for any tile height in kGSTileRows
    const size_t nc = cdiv(c->d.pitch, kGTCols), rows = c->d.nz - 2;
    F.gsRight = c->ar.alloc<T>(2 * 5 * nc * (rows + kGSTileRowsMax));
    F.gsTop = c->ar.alloc<T>(2 * 5 * nc * (size_t)cdiv((int)rows, kGSTileRowsMin) * kGTCols);
    if (!c->gsctl) c->gsctl = c->ar.alloc<GSTileCtl>(1);
    if (!c->sc_host_i) CK(cudaMallocHost(&c->sc_host_i, sizeof(int)));
}

// ---------------------------------------------------------------- routines

template <typename T>
void launch_pzeta(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    int now = c->cur, fut = 1 - c->cur;
    AB2 ab = AB2::of(c->step);
    PZetaArgs<T> a{c->d, c->c, c->profiles(), F.zeta[now], F.u, F.w, F.th[now], F.qv[now], F.qc[now], F.qr[now],
                   F.zeta[fut], F.hist[H_ZETA][ab.sn], F.hist[H_ZETA][ab.so], F.hist[H_BUOY][ab.sn],
                   F.hist[H_BUOY][ab.so], ab};
    dim3 g(cdiv(c->d.nx - 2, kPZBX), cdiv(c->d.nz - 3, kPZBZ));
    klaunch<k_pzeta_body<T>, kPZBX * kPZBZ>(&c->stats, VVM_K_PZETA, c->stream, k_pzeta<T>, g, dim3(kPZBX, kPZBZ), 0, a);
}

template <typename T>
void launch_padv(vvm_gpu_ctx* c, int mask, int nvp_mask, bool vt, bool precip) {
    Fields<T>& F = fields<T>(c);
    int now = c->cur, fut = 1 - c->cur;
    AB2 ab = AB2::of(c->step);
    PAdvArgs<T> a{};
    a.d = c->d;
    a.c = c->c;
    a.p = c->profiles();
    a.u = F.u;
    a.w = F.w;
    T* nows[4] = {F.th[now], F.qv[now], F.qc[now], F.qr[now]};
    T* futs[4] = {F.th[fut], F.qv[fut], F.qc[fut], F.qr[fut]};
    int hid[4] = {H_TH, H_QV, H_QC, H_QR};
    for (int f = 0; f < 4; f++) {
        a.now[f] = nows[f];
        a.fut[f] = futs[f];
        a.hn[f] = F.hist[hid[f]][ab.sn];
        a.ho[f] = F.hist[hid[f]][ab.so];
    }
    a.hvt_n = F.hist[H_VT][ab.sn];
    a.hvt_o = F.hist[H_VT][ab.so];
    a.precip = F.precip;
    a.partial = c->partial;
    a.mask = mask;
    a.nvp_mask = nvp_mask;
    a.do_vt = vt;
    a.do_precip = precip;
    a.ab = ab;
    a.err = c->d_err;
    dim3 g = c->padv_grid();
    CUtensorMap m[4];
    for (int f = 0; f < 4; f++)
        m[f] = field_map(a.now[f], c->d.nx, c->d.nz, c->d.pitch, (int)sizeof(T), kPAdvVX, kPAdvVZ);
    if (c->stats.rec) {
        PAdvPack<T> p;
        for (int f = 0; f < 4; f++) p.m[f] = m[f];
        p.a = a;
        record_kernel(&c->stats, reinterpret_cast<const void*>(&k_padv_grouped<T>), g, c->padv_blk(),
                      sizeof(PAdvShared<T>), &p, sizeof(p), alignof(PAdvPack<T>));
    } else {
        LAUNCH(&c->stats, VVM_K_PADV, c->stream,
               k_padv<T><<<g, c->padv_blk(), sizeof(PAdvShared<T>), c->stream>>>(m[0], m[1], m[2], m[3], a));
        CKL();
    }
    if (nvp_mask)
        klaunch<k_nvp_final_body, 1024>(&c->stats, VVM_K_APPLY, c->stream, k_nvp_final, dim3(1), dim3(1024), 0,
                                        (const double*)c->partial, (int)(g.x * g.y), c->nvp);
}

template <typename T>
void launch_apply(vvm_gpu_ctx* c, int mask, int nvp_mask, bool forcing, bool halo) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    ApplyArgs<T> a{};
    a.d = c->d;
    a.c = c->c;
    a.p = c->profiles();
    a.fut[0] = F.th[fut];
    a.fut[1] = F.qv[fut];
    a.fut[2] = F.qc[fut];
    a.fut[3] = F.qr[fut];
    a.nvp = c->nvp;
    a.th_forcing = F.th_forcing;
    a.mask = mask;
    a.nvp_mask = nvp_mask;
    a.forcing = forcing && c->has_q;
    // status_for_adding_forcing (Iteration.cpp:276-277)
    a.forcing_th = forcing && c->has_forcing_th && (c->step * c->desc.dt <= c->desc.addforcingtime);
    a.halo = halo;
    klaunch<k_apply_body<T>, 256>(&c->stats, VVM_K_APPLY, c->stream, k_apply<T>, c->grid_interior(1), c->blk(), 0, a);
}

template <typename T>
void launch_halo_all(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    HaloArgs<T> a{c->d, F.zeta[fut], F.w, {F.th[fut], F.u, F.qv[fut], F.qc[fut], F.qr[fut]}};
    LAUNCH(&c->stats, VVM_K_APPLY, c->stream, k_halo_all<T><<<c->grid_interior(1), c->blk(), 0, c->stream>>>(a));
    CKL();
}

template <typename T>
void launch_pubartop(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    PubarArgs<T> a{c->d, c->c, c->profiles(), F.u, F.w, F.RKM, c->ubar, c->dubar, AB2::of(c->step)};
    klaunch<k_pubartop_body<T>, 1024>(&c->stats, VVM_K_PUBAR, c->stream, k_pubartop<T>, dim3(1), dim3(1024), 0, a);
}

// finish_advection: the step's own sequence, where the finish of the
// advection (k_apply's NVP rescaling and AddForcing of th, qv, qc, qr, whose
// NVP sums k_padv left) is applied as Kessler reads each value.
template <typename T>
void launch_kessler(vvm_gpu_ctx* c, bool halo, bool finish_advection = false) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    KesslerArgs<T> a{c->d, c->c, c->profiles(), F.th[fut], F.qv[fut], F.qc[fut], F.qr[fut],
                     F.d_auto, F.d_accr, F.d_evap, F.d_cond, c->partial, 1};
    if (finish_advection) {
        a.do_pre = 1;
        a.pre.nvp = c->nvp;
        a.pre.th_forcing = F.th_forcing;
        a.pre.nvp_mask = F_QV | F_QC | F_QR;
        a.pre.forcing = c->has_q;
        // status_for_adding_forcing (Iteration.cpp:276-277), as launch_apply forms it
        a.pre.forcing_th = c->has_forcing_th && (c->step * c->desc.dt <= c->desc.addforcingtime);
    }
    dim3 g = c->grid_interior(1);
    klaunch<k_kessler_body<T>, 256>(&c->stats, VVM_K_KESSLER, c->stream, k_kessler<T>, g, c->blk(), 0, a);
    klaunch<k_nvp_final_body, 1024>(&c->stats, VVM_K_APPLY, c->stream, k_nvp_final, dim3(1), dim3(1024), 0,
                                    (const double*)c->partial, (int)(g.x * g.y), c->nvp);
    launch_apply<T>(c, halo ? (F_TH | F_QV | F_QC | F_QR) : (F_QV | F_QC | F_QR), F_QV | F_QC | F_QR, false, halo);
}

cudaGraphConditionalHandle new_handle(cudaStream_t st) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    return h;
}

// A handle for a WHILE node of the graph being captured on st whose value
// resets to 0 at each launch of the graph; 0 while a step is recorded (the
// recorded kernels then set no condition: the group's own kernel does).
cudaGraphConditionalHandle new_handle_reset(Stats* s, cudaStream_t st) {
    if (s && s->rec) return 0;
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    return h;
}
cudaGraphConditionalHandle new_handle(Stats* s, cudaStream_t st) {
    if (s && s->rec) return 0;
    return new_handle(st);
}

// Appends a WHILE node (condition h) to the graph being captured on st and
// returns its body graph; capture on st continues after the node.
cudaGraph_t add_while(cudaStream_t st, cudaGraphConditionalHandle h) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &p));
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return p.conditional.phGraph_out[0];
}

// add_while, or the start of a loop in a recording (no body graph).
cudaGraph_t add_while(Stats* s, cudaStream_t st, cudaGraphConditionalHandle h) {
    if (s && s->rec) {
        RecOp op;
        op.kind = RecOp::LOOP_BEGIN;
        s->rec->ops.push_back(std::move(op));
        return nullptr;
    }
    return add_while(st, h);
}

struct BodyCapture {   // stream capture into a conditional node's body graph
    cudaStream_t s;
    Stats* stats = nullptr;   // recording: the loop's end is marked instead
    bool active = false;      // capturing on s (not yet ended)
    BodyCapture(cudaStream_t s_, cudaGraph_t body, Stats* st = nullptr) : s(s_), stats(st) {
        if (stats && stats->rec) return;
        CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        active = true;
    }
    void end() {
        if (stats && stats->rec) {
            RecOp op;
            op.kind = RecOp::LOOP_END;
            stats->rec->ops.push_back(std::move(op));
            return;
        }
        active = false;
        cudaGraph_t g;
        CK(cudaStreamEndCapture(s, &g));
    }
    // An error between the start and end() leaves the stream out of capture
    // mode again, so the context's capture streams stay usable.
    ~BodyCapture() {
        if (!active) return;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        (void)cudaGetLastError();
    }
};

// The cluster schedule's launch shape for a padded row of `pitch` cells of
// `elem` bytes: chunks of 32*kGSPer cells (one warp each) over a cluster of cs
// CTAs of w warps, coefficient rows d ahead.
constexpr int kGSPer = 4;
struct GSPlan {
    int cs, w, d;
    size_t smem;
};
inline GSPlan gs_plan(int pitch, int nz, size_t elem) {
    GSPlan p{};
    const int gwn = cdiv(pitch, 32 * kGSPer);
    p.cs = gwn >= 8 ? 8 : (gwn >= 4 ? 4 : (gwn >= 2 ? 2 : 1));
    p.w = cdiv(gwn, p.cs);   // <= kGSClusterWarps for pitch <= 8224 (checked at create)
    const size_t row = 3 * (size_t)p.w * 32 * kGSPer * elem;
    const size_t tab = 2 * (size_t)nz * elem;   // nudging scalars
    p.d = (8 * row + tab <= kGSRingBytes) ? 8 : (4 * row + tab <= kGSRingBytes ? 4 : 2);
    p.smem = p.d * row + tab;
    return p;
}

template <typename T, int D, int CS>
void gs_launch(vvm_gpu_ctx* c, const GSArgs<T>& g, const GSPlan& p) {
    LAUNCH(&c->stats, VVM_K_GS, c->stream, k_gs_cluster<T, kGSPer, D, CS><<<5 * CS, 32 * p.w, p.smem, c->stream>>>(g));
}

template <typename T, int D>
void gs_launch_d(vvm_gpu_ctx* c, const GSArgs<T>& g, const GSPlan& p) {
    if (p.cs == 8) gs_launch<T, D, 8>(c, g, p);
    else if (p.cs == 4) gs_launch<T, D, 4>(c, g, p);
    else if (p.cs == 2) gs_launch<T, D, 2>(c, g, p);
    else gs_launch<T, D, 1>(c, g, p);
}

template <typename T, int D>
void gs_set_smem_d() {
    const int mx = (int)kGSRingBytes;
    CK(cudaFuncSetAttribute(k_gs_cluster<T, kGSPer, D, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(k_gs_cluster<T, kGSPer, D, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(k_gs_cluster<T, kGSPer, D, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(k_gs_cluster<T, kGSPer, D, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
}

template <typename T>
void gs_set_smem() {
    gs_set_smem_d<T, 8>();
    gs_set_smem_d<T, 4>();
    gs_set_smem_d<T, 2>();
}

// The cluster schedule's coefficient arrays and shared-memory limits, made
// when the schedule is chosen (never during a graph capture).
template <typename T>
void ensure_gs_cluster_t(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    if (F.gsC) return;
    CK(cudaStreamSynchronize(c->stream));
    F.gsC = c->ar.alloc<T>(5 * c->d.cells());
    F.gsB = c->ar.alloc<T>(5 * c->d.cells());
    gs_set_smem<T>();
}
inline void ensure_gs_cluster(vvm_gpu_ctx* c) {
    if (c->mixed) ensure_gs_cluster_t<float>(c);
    else ensure_gs_cluster_t<double>(c);
}

// The cluster schedule: coefficients, then one cluster a field (k_gs_cluster).
template <typename T>
void launch_gs_cluster(vvm_gpu_ctx* c, GSArgs<T> g) {
    Fields<T>& F = fields<T>(c);
    if (!F.gsC) throw CudaError{"Gauss-Seidel cluster schedule used before it was set up"};
    g.C = F.gsC;
    g.B = F.gsB;
    g.err = c->d_err;
    dim3 cb(64, 4), cgr(cdiv(c->d.pitch, 64), cdiv(c->d.nz - 2, 4), 5);
    LAUNCH(&c->stats, VVM_K_GS, c->stream, k_gs_coeffs<T><<<cgr, cb, 0, c->stream>>>(g));
    CKL();
    const GSPlan p = gs_plan(c->d.pitch, c->d.nz, sizeof(T));
    if (p.d == 8) gs_launch_d<T, 8>(c, g, p);
    else if (p.d == 4) gs_launch_d<T, 4>(c, g, p);
    else gs_launch_d<T, 2>(c, g, p);
    CKL();
}

// Later Gauss-Seidel passes a step graph runs before its WHILE node (the
// typical sweep is pass 1 and two more).
constexpr int kGSGraphPasses = 2;
// The Gauss-Seidel schedule: kGSSchedCluster (one cluster a field) or a tile
// height. Automatic: tiles of 16 rows in FP64, 8 in FP32 (the fastest at
// 2048 x 256 on a B200: FP64 0.365 / 0.376 ms a step with 16 / 8 rows, FP32
// 0.305 / 0.301 ms); a batch's autotuner also tries the cluster schedule.
constexpr int kGSSchedCluster = 1;
inline int gs_tile_rows(const vvm_gpu_ctx* c) {
    return c->tune_gs_tr ? c->tune_gs_tr : (c->mixed ? kGSTileRowsDefault : 2 * kGSTileRowsDefault);
}
inline bool gs_schedule_ok(int v) { return v == 0 || v == kGSSchedCluster || gs_tile_rows_ok(v); }

template <typename T>
void launch_turbulence(vvm_gpu_ctx* c, bool nudge, long long* recorded_in_loops = nullptr) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    RKArgs<T> r{c->d, c->c, c->profiles(), F.u, F.w, F.th[fut], F.RKM, F.RKH};
    klaunch<k_rkm_rkh_body<T>, 256>(&c->stats, VVM_K_RKM, c->stream, k_rkm_rkh<T>, c->grid_interior(1), c->blk(), 0, r);
    GSArgs<T> g{c->d, c->c, c->profiles(), {F.zeta[fut], F.th[fut], F.qv[fut], F.qc[fut], F.qr[fut]},
                F.RKM, F.RKH, 0x1f, nudge ? 1 : 0, F.gsA, nullptr, nullptr, nullptr};
    if (c->tune_gs_tr == kGSSchedCluster) {
        launch_gs_cluster<T>(c, g);
        return;
    }
    // the recurrence: tiles and passes (see k_gs_tiles)
    const int tr = gs_tile_rows(c);
    const int nb = cdiv(c->d.nz - 2, tr), nc = cdiv(c->d.pitch, kGTCols);
    GSTileArgs<T> t{nb, nc, tr, F.gsRight, F.gsTop, c->gsctl, recorded_in_loops ? c->d_exec : nullptr};
    const int tblocks = cdiv(5 * nb * nc, 4);
    const int maxp = std::max(2, nb + nc - 1);
    cudaStream_t st = c->stream;
    zero_async(&c->stats, c->gsctl, sizeof(GSTileCtl), st);   // a fresh sweep
    klaunch<k_gs_tiles_body<T, true>, 128, kGSTileMinBlocks<T>>(&c->stats, VVM_K_GS, st, k_gs_tiles<T, true>, dim3(tblocks), dim3(128), 0,
                                              g, t, (cudaGraphConditionalHandle)0);   // pass 1
    if (recorded_in_loops) {
        // graph capture: the typical passes 2..kGSGraphPasses+1 unconditionally
        // (each returns at once if the sweep already converged, and the last
        // block of each sets the condition below), then a WHILE node that runs
        // further passes only when they are needed
        const cudaGraphConditionalHandle h = new_handle_reset(&c->stats, st);
        GSTileArgs<T> tu = t;
        tu.exec = nullptr;   // counted with the graph's static kernels
        for (int p = 0; p < kGSGraphPasses; p++)
            klaunch<k_gs_tiles_body<T, false>, 128, kGSTileMinBlocks<T>>(&c->stats, VVM_K_GS, st, k_gs_tiles<T, false>, dim3(tblocks),
                                                       dim3(128), 0, g, tu, h);
        record_cond(&c->stats, &c->gsctl->more, true);
        cudaGraph_t body = add_while(&c->stats, st, h);
        BodyCapture bc(c->cap[0], body, &c->stats);
        const long long n0 = c->stats.launches;
        klaunch<k_gs_tiles_body<T, false>, 128, kGSTileMinBlocks<T>>(&c->stats, VVM_K_GS, bc.s, k_gs_tiles<T, false>, dim3(tblocks),
                                                   dim3(128), 0, g, t, h);
        record_cond(&c->stats, &c->gsctl->more, false);
        bc.end();
        *recorded_in_loops += c->stats.launches - n0;
        return;
    }
    for (int p = 2; p <= maxp; p++) {
        LAUNCH(&c->stats, VVM_K_GS, st, k_gs_tiles<T, false><<<tblocks, 128, 0, st>>>(g, t, 0));
        CKL();
        CK(cudaMemcpyAsync(c->sc_host_i, &c->gsctl->more, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (!*c->sc_host_i) break;
    }
}

template <typename T>
void launch_nudge(vvm_gpu_ctx* c, bool th_zeta, bool qv) {
    Fields<T>& F = fields<T>(c);
    int now = c->cur, fut = 1 - c->cur;
    NudgeArgs<T> a{c->d, c->c, c->profiles(), F.th[fut], F.zeta[fut], F.qv[fut], F.qv[now],
                   th_zeta ? 1 : 0, (th_zeta && c->desc.case_id != 2) ? 1 : 0,
                   qv ? c->desc.moisture_nudge_time : 0.0};
    klaunch<k_nudge_body<T>, 256>(&c->stats, VVM_K_MEAN, c->stream, k_nudge<T>, c->grid_all(), c->blk(), 0, a);
    CKL();
}

template <typename T>
void launch_update_mean(vvm_gpu_ctx* c, bool rotate) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    MeanArgs<T> a{c->d, c->offset_th(), c->offset_qv(), F.th[fut], F.qv[fut], c->thb, c->qvb, c->thvb,
                  c->ubar, rotate ? 1 : 0};
    klaunch<k_update_mean_body<T>, 256>(&c->stats, VVM_K_MEAN, c->stream, k_update_mean<T>, dim3(c->d.nz - 2),
                                        dim3(256), 0, a);
}

// ---------------------------------------------------------------- Poisson

// Applies the launch-shape knobs that live inside the solver objects.
void apply_tuning(vvm_gpu_ctx* c) {
    if (c->pcg64 && c->pcg64->spectral) {
        const int half = std::max(32, (c->d.nx - 2) / 2);
        const int def = std::min(half, 512);
        c->pcg64->sp.threads = c->tune_fft > 0 ? std::max(32, std::min(c->tune_fft, std::min(half, 1024))) : def;
    }
}

void ensure_poisson(vvm_gpu_ctx* c) {
    if (c->poisson_ready) return;
    c->drop_graphs();
    int NX = c->d.nx - 2, NK = c->d.nz - 3;
    c->pcg64.reset(new PCG<double>());
    c->pcg64->stats = &c->stats;
    c->pcg64->spectral = c->spectral;
    c->pcg64->build(c->ar, NX, NK, c->h_rhou, c->h_rhow, c->h_a, c->h_h);
    int pitch = c->pcg64->pitch;
    c->Wf = c->ar.alloc<double>((size_t)NK * pitch);
    c->W = c->ar.alloc<double>((size_t)NK * pitch);
    c->r64 = c->ar.alloc<double>((size_t)NK * pitch);
    c->Wprev = c->ar.alloc<double>((size_t)NK * pitch);
    c->nsolves = 0;
    if (c->mixed && !c->spectral) {
        c->pcg32.reset(new PCG<float>());
        c->pcg32->stats = &c->stats;
        c->pcg32->build(c->ar, NX, NK, c->h_rhou, c->h_rhow, c->h_a, c->h_h);
        c->g32 = c->ar.alloc<float>((size_t)NK * pitch);
        c->d32 = c->ar.alloc<float>((size_t)NK * pitch);
    }
    dim3 g(cdiv(NX, 64), cdiv(NK, 4));
    c->wnpart = g.x * g.y;
    c->wpartial = c->ar.alloc<double>(c->wnpart);
    if (!c->sc_host) CK(cudaMallocHost(&c->sc_host, sizeof(double)));
    c->poisson_ready = true;
    apply_tuning(c);
}

double read_scalar(vvm_gpu_ctx* c, const double* dptr) {
    CK(cudaMemcpyAsync(c->sc_host, dptr, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return *c->sc_host;
}

void ensure_learned(vvm_gpu_ctx* c) {
    ensure_poisson(c);
    if (c->net) return;
    const int NX = c->d.nx - 2, NK = c->d.nz - 3;
    if (!LearnedNet::supports(NX, NK)) throw CudaError{"learned preconditioner: NX must be a multiple of 8"};
    c->net.reset(new LearnedNet());
    c->net->stats = &c->stats;
    c->net->build(c->ar, NX, NK, 1);
    c->net->set_operator(c->h_rhou, c->h_rhow, c->h_a, c->h_h);
    const size_t n = (size_t)NK * c->pcg64->pitch;
    c->z64 = c->ar.alloc<double>(n);
    c->za64 = c->ar.alloc<double>(n);
    c->r164 = c->ar.alloc<double>(n);
    c->d64 = c->ar.alloc<double>(n);
    c->sd64 = c->ar.alloc<double>(n);
    for (int j = 0; j < kFcgM; j++) {
        c->fcg_p[j] = c->ar.alloc<double>(n);
        c->fcg_q[j] = c->ar.alloc<double>(n);
    }
    c->fcg_part = c->ar.alloc<double>((size_t)kFcgM * c->pcg64->npart);
    c->fcg_pq = c->ar.alloc<double>(kFcgM);
    c->fcg_beta = c->ar.alloc<double>(kFcgM);
    double* ring[2 * kFcgM];
    for (int j = 0; j < kFcgM; j++) {
        ring[j] = c->fcg_p[j];
        ring[kFcgM + j] = c->fcg_q[j];
    }
    c->fcg_ring = c->ar.alloc<double*>(2 * kFcgM);
    upload_now(c->fcg_ring, ring, sizeof(ring));
    c->fcg_ctl = c->ar.alloc<FcgCtl>(1);
    CK(cudaMallocHost(&c->fcg_host, sizeof(FcgCtl)));
    (void)conv_rows_per_cta(c->net->H[0], c->net->W[0]);   // the convolution's one-time setup, outside any capture
}

// z64 = M r: a two-level cycle whose coarse correction is the network.
//   za = L r                      (L: the exact z-line solve, the multigrid's
//                                  level-0 line operator)
//   r1 = r - S za
//   d  = ||r1|| net(r1 / ||r1||)  (BF16 operands; trained on e1 = S^{-1} r1)
//   za += gam d, gam = (d, r1) / (d, S d)
//   z  = za + L (r - S za)
// gam minimises the S-norm error of za along d, so an application is never
// worse than the same cycle without the network, whatever the network says.
// Mode 1 runs the cycle without the network (the method without it), mode 2
// is the identity.
void learned_precond(vvm_gpu_ctx* c, const double* r, cudaStream_t st) {
    PCG<double>& P = *c->pcg64;
    LearnedNet& N = *c->net;
    VecArgs<double> v = P.vargs();
    dim3 B = P.block(), G = P.grid();
    if (c->learned_mode == 2) {
        CK(cudaMemcpyAsync(c->z64, r, (size_t)P.NK * P.pitch * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return;
    }
    P.mg.sweep(0, r, nullptr, nullptr, 0, 0, c->za64, 1.0, st);
    if (c->learned_mode == 0) {
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_residual<double><<<G, B, 0, st>>>(v, r, c->za64, c->r164, P.partial));
        CKL();
        LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_sdot<<<G, B, 0, st>>>(v, c->r164, N.dsc, P.partial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, CG_SET_NRM));
        CKL();
        dim3 g0(cdiv(P.NX, 64), cdiv(N.H[0], 4));
        LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_in<<<g0, B, 0, st>>>(c->r164, nullptr, P.NX, P.NK, P.pitch, N.x0, N.H[0], &P.sc->nrm, N.dsc));
        CKL();
        N.forward(st);
        LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_out<<<G, B, 0, st>>>(N.z0, P.NX, P.NK, P.pitch, c->d64, &P.sc->nrm, N.dsc));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_spmv<double><<<G, B, 0, st>>>(v, c->d64, c->sd64, P.partial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, CG_NET_DSD));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_dot<double><<<G, B, 0, st>>>(v, c->d64, c->r164, P.partial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, CG_NET_GAMMA));
        CKL();
        LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_galerkin<<<G, B, 0, st>>>(P.NX, P.NK, P.pitch, P.sc, c->d64, c->za64));
        CKL();
    }
    P.mg.sweep(0, r, c->za64, nullptr, 0, 0, c->z64, 1.0, st);
}

// Flexible CG with truncated orthogonalisation: the new direction is made
// S-orthogonal to the last kFcgM-1 directions,
//   p_k = z_k - sum_j ((z_k, q_j) / (p_j, q_j)) p_j,  q_j = S p_j,
// alpha_k = (p_k, r_k) / (p_k, q_k). With a preconditioner that varies from
// one application to the next (the network's Galerkin step makes it
// nonlinear), keeping only the previous direction loses the Krylov speed-up;
// a few more restore it. Directions and their S images live in a ring of
// kFcgM slots. On S W = Wf from W = 0, preconditioned by learned_precond, to
// the FP64 residual ||rhow r||^2 <= tol^2 bb, at most `cap` iterations.
//
// Recorded into the stream's capture as a WHILE node whose body is one
// iteration: the kernels take the ring slots from the iteration count on the
// device (FcgCtl), and k_fcg_loop tests the residual after every iteration,
// so the host never waits inside the loop. Returns the kernels recorded
// inside the loop body.
long long record_fcg(vvm_gpu_ctx* c, double tol, int cap) {
    PCG<double>& P = *c->pcg64;
    VecArgs<double> v = P.vargs();
    dim3 B = P.block(), G = P.grid();
    cudaStream_t st = c->stream;
    CK(cudaMemsetAsync(c->W, 0, (size_t)P.NK * P.pitch * sizeof(double), st));
    LAUNCH(&c->stats, VVM_K_CG, st, k_cg_residual<double><<<G, B, 0, st>>>(v, c->Wf, c->W, P.r, P.partial));
    CKL();
    cudaGraphConditionalHandle h = new_handle(st);
    LAUNCH(&c->stats, VVM_K_CG, st,
           k_fcg_loop<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, c->fcg_ctl, h, tol * tol, cap, 1, c->d_exec, 0));
    CKL();
    cudaGraph_t body = add_while(st, h);
    BodyCapture bc(c->cap[0], body);
    cudaStream_t bs = bc.s;
    const long long n0 = c->stats.launches;
    learned_precond(c, P.r, bs);
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_multidot<<<G, B, 0, bs>>>(v, c->z64, c->fcg_ring, c->fcg_ctl, c->fcg_part));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_beta<<<1, 1024, 0, bs>>>(c->fcg_part, P.npart, c->fcg_ctl, c->fcg_pq, c->fcg_beta));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_dir<<<G, B, 0, bs>>>(v, c->z64, c->fcg_ring, c->fcg_ctl, c->fcg_beta));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_spmv<<<G, B, 0, bs>>>(v, c->fcg_ring, c->fcg_ctl, P.r, P.partial, c->fcg_part));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_alpha<<<1, 1024, 0, bs>>>(P.partial, c->fcg_part, P.npart, P.sc, c->fcg_pq, c->fcg_ctl));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, bs, k_fcg_update<<<G, B, 0, bs>>>(v, P.sc, c->fcg_ring, c->fcg_ctl, c->W, P.r, P.partial));
    CKL();
    const int nb = (int)(c->stats.launches - n0);
    LAUNCH(&c->stats, VVM_K_CG, bs,
           k_fcg_loop<<<1, 1024, 0, bs>>>(P.partial, P.npart, P.sc, c->fcg_ctl, h, tol * tol, cap, 0, c->d_exec, nb + 1));
    CKL();
    bc.end();
    return c->stats.launches - n0;
}

// The flexible-CG loop alone as an instantiated graph, kept per context for
// its (tol, cap, mode).
cudaGraphExec_t fcg_graph(vvm_gpu_ctx* c, double tol, int cap) {
    if (c->fcg_exec && c->fcg_tol == tol && c->fcg_cap == cap && c->fcg_mode == c->learned_mode) return c->fcg_exec;
    if (c->fcg_exec) cudaGraphExecDestroy(c->fcg_exec);
    c->fcg_exec = nullptr;
    const long long l0 = c->stats.launches;
    const bool timing = c->stats.on;   // no per-launch events inside a capture
    c->stats.on = false;
    cudaStream_t saved = c->stream;
    c->stream = c->own;
    cudaGraph_t g = nullptr;
    long long in_loop = 0;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    try {
        in_loop = record_fcg(c, tol, cap);
    } catch (...) {
        cudaStreamEndCapture(c->stream, &g);
        if (g) cudaGraphDestroy(g);
        c->stream = saved;
        c->stats.launches = l0;
        c->stats.on = timing;
        throw;
    }
    CK(cudaStreamEndCapture(c->stream, &g));
    c->stream = saved;
    c->stats.on = timing;
    c->fcg_static = c->stats.launches - l0 - in_loop;
    c->stats.launches = l0;
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw CudaError{std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
    c->fcg_exec = ex;
    c->fcg_tol = tol;
    c->fcg_cap = cap;
    c->fcg_mode = c->learned_mode;
    return ex;
}

// Runs the flexible-CG loop (one graph launch, one wait at the end). Returns
// the iterations run, or -cap if the tolerance was not reached.
int fcg_learned(vvm_gpu_ctx* c, double bb, double tol, int cap, double* relres) {
    cudaGraphExec_t ex = fcg_graph(c, tol, cap);
    cudaEvent_t e0 = nullptr;   // profiling: the whole loop counts as the learned class
    if (c->stats.on) {
        e0 = c->stats.ev();
        CK(cudaEventRecord(e0, c->stream));
    }
    CK(cudaGraphLaunch(ex, c->stream));
    if (e0) {
        cudaEvent_t e1 = c->stats.ev();
        CK(cudaEventRecord(e1, c->stream));
        c->stats.pending.push_back({VVM_K_LEARNED, e0, e1});
    }
    c->stats.launches += c->fcg_static;
    PCG<double>& P = *c->pcg64;
    CK(cudaMemcpyAsync(P.sc_host, P.sc, sizeof(CGScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->fcg_host, c->fcg_ctl, sizeof(FcgCtl), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const FcgCtl h = *c->fcg_host;
    const double rr = P.sc_host->rr;
    *relres = (bb > 0.0) ? std::sqrt(rr / bb) : 0.0;
    return h.converged ? h.k : -cap;
}

// Solves S W = Wf (FP64 rhs in c->Wf, ||b||^2 = bb) into c->W.
int solve_w(vvm_gpu_ctx* c, double bb, double tol, bool warm) {
    int maxit = c->desc.poisson_maxit > 0 ? c->desc.poisson_maxit : 200;
    if (bb == 0.0) {
        CK(cudaMemsetAsync(c->W, 0, (size_t)c->pcg64->NK * c->pcg64->pitch * sizeof(double), c->stream));
        c->last_iters = 0;
        c->last_relres = 0.0;
        return VVM_GPU_OK;
    }
    if (c->desc.solver == VVM_SOLVER_LEARNED && !c->learned_collect) {
        ensure_learned(c);
        double rel = 0;
        int it = fcg_learned(c, bb, tol, c->learned_cap, &rel);
        c->learned_fallback = (it < 0) ? 1 : 0;
        c->learned_iters = (it < 0) ? c->learned_cap : it;
        if (it < 0) {   // the plain multigrid-PCG takes over from the current iterate
            it = c->learned_cap + c->pcg64->solve(c->Wf, c->W, true, bb, tol, maxit, c->stream, &rel);
        }
        c->last_iters = it;
        c->last_relres = rel;
        return (rel <= tol) ? VVM_GPU_OK : VVM_GPU_ENOCONV;
    }
    if (c->spectral) {   // direct solve W = S^{-1} f, checked; CG from there if the check fails
        double rel = 0;
        c->pcg64->sp.apply_to(c->Wf, c->W, c->stream);
        int it = c->pcg64->solve(c->Wf, c->W, true, bb, tol, maxit, c->stream, &rel);
        c->last_iters = it;
        c->last_relres = rel;
        return (rel <= tol) ? VVM_GPU_OK : VVM_GPU_ENOCONV;
    }
    if (!c->mixed) {
        double rel = 0;
        int it = c->pcg64->solve(c->Wf, c->W, warm, bb, tol, maxit, c->stream, &rel);
        c->last_iters = it;
        c->last_relres = rel;
        return (rel <= tol) ? VVM_GPU_OK : VVM_GPU_ENOCONV;
    }
    // Mixed precision: FP64 residual and correction, FP32 inner PCG.
    PCG<double>& P64 = *c->pcg64;
    PCG<float>& P32 = *c->pcg32;
    VecArgs<double> v = P64.vargs();
    dim3 B = P64.block(), G = P64.grid();
    if (!warm) CK(cudaMemsetAsync(c->W, 0, (size_t)P64.NK * P64.pitch * sizeof(double), c->stream));
    int total = 0;
    double rel = 0;
    for (int outer = 0;; outer++) {
        LAUNCH(&c->stats, VVM_K_CG, c->stream, k_cg_residual<double><<<G, B, 0, c->stream>>>(v, c->Wf, c->W, c->r64, c->wpartial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, c->stream, k_cg_scalar<<<1, 1024, 0, c->stream>>>(c->wpartial, c->wnpart, P64.sc, CG_SET_RR));
        CKL();
        double rr = P64.read_rr(c->stream);
        rel = std::sqrt(rr / bb);
        if (!(rr > (tol * tol) * bb) || !std::isfinite(rr) || total >= maxit || outer >= 20) break;
        LAUNCH(&c->stats, VVM_K_CG, c->stream, k_to_float<<<G, B, 0, c->stream>>>(P64.NX, P64.NK, P64.pitch, c->r64, c->g32));
        CKL();
        double irel = 0;
        // inner: reduce its initial residual by 1e-4
        int it = P32.solve(c->g32, c->d32, false, -1.0, 1e-4, maxit, c->stream, &irel);
        total += std::max(it, 1);
        LAUNCH(&c->stats, VVM_K_CG, c->stream, k_refine_add<<<G, B, 0, c->stream>>>(P64.NX, P64.NK, P64.pitch, c->W, c->d32));
        CKL();
    }
    c->last_iters = total;
    c->last_relres = rel;
    return (rel <= tol) ? VVM_GPU_OK : VVM_GPU_ENOCONV;
}

// ---------------------------------------------------------------- graphs

// Records the cal_w solve with device-side loop control (graph capture on
// c->stream). The FP64 step: one PCG loop to tol. The mixed step: FP64
// residual refinement around an FP32 PCG loop. Returns the number of
// kernels recorded inside loop bodies (excluded from the per-launch count).
long long record_solve(vvm_gpu_ctx* c, double tol, int maxit, bool warm) {
    PCG<double>& P64 = *c->pcg64;
    cudaStream_t st = c->stream;
    dim3 B = P64.block(), G = P64.grid();
    VecArgs<double> v = P64.vargs();
    const long long n_start = c->stats.launches;
    long long in_bodies = 0;
    const bool learned = (c->desc.solver == VVM_SOLVER_LEARNED && !c->learned_collect);
    // learned: the flexible-CG loop, then the check below, whose plain PCG
    // loop runs only if the flexible CG stopped at its cap (the fallback)
    if (learned) in_bodies += record_fcg(c, tol, c->learned_cap);
    if (c->spectral) P64.sp.apply_to(c->Wf, c->W, st);   // direct solve; the loop below checks it
    else if (!warm && !learned) CK(cudaMemsetAsync(c->W, 0, (size_t)P64.NK * P64.pitch * sizeof(double), st));
    if (!c->mixed || c->spectral || learned) {
        cudaGraphConditionalHandle h = new_handle(&c->stats, st);
        klaunch<k_cg_check_body<double>, 256>(&c->stats, VVM_K_CG, st, k_cg_check<double>, G, B, 0, v,
                                              (const double*)c->Wf, c->W, P64.r, P64.partial, P64.sc, P64.ctl,
                                              P64.arrive, h, tol * tol, maxit);
        record_cond(&c->stats, &P64.ctl->more, true);
        cudaGraph_t body = add_while(&c->stats, st, h);
        BodyCapture bc(c->cap[0], body, &c->stats);
        const long long n0 = c->stats.launches;
        int nb = P64.record_iteration(c->W, bc.s);
        klaunch<k_loop_plain_body, 32>(&c->stats, VVM_K_CG, bc.s, k_loop_plain, dim3(1), dim3(1), 0,
                                       (const CGScalars*)P64.sc, P64.ctl, h, tol * tol, maxit, 0, c->d_exec, nb + 1);
        record_cond(&c->stats, &P64.ctl->more, false);
        bc.end();
        in_bodies += c->stats.launches - n0;
        return in_bodies;
    }
    PCG<float>& P32 = *c->pcg32;
    VecArgs<float> v32 = P32.vargs();
    LAUNCH(&c->stats, VVM_K_CG, st, k_zero_if_b0<<<G, B, 0, st>>>(P64.NX, P64.NK, P64.pitch, P64.sc, c->W));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, st, k_cg_residual<double><<<G, B, 0, st>>>(v, c->Wf, c->W, c->r64, c->wpartial));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(c->wpartial, c->wnpart, P64.sc, CG_SET_RR));
    CKL();
    cudaGraphConditionalHandle ho = new_handle(st);
    LAUNCH(&c->stats, VVM_K_CG, st, k_loop_outer<<<1, 1, 0, st>>>(P64.sc, c->wctl, P32.ctl, ho, tol * tol, maxit, 1, c->d_exec, 0));
    CKL();
    cudaGraph_t outer = add_while(st, ho);
    {
        BodyCapture oc(c->cap[0], outer);
        cudaStream_t os = oc.s;
        const long long n0 = c->stats.launches;
        LAUNCH(&c->stats, VVM_K_CG, os, k_to_float<<<G, B, 0, os>>>(P64.NX, P64.NK, P64.pitch, c->r64, c->g32));
        CKL();
        CK(cudaMemsetAsync(c->d32, 0, (size_t)P32.NK * P32.pitch * sizeof(float), os));
        LAUNCH(&c->stats, VVM_K_CG, os, k_cg_residual<float><<<G, B, 0, os>>>(v32, c->g32, c->d32, P32.r, P32.partial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, os, k_cg_scalar<<<1, 1024, 0, os>>>(P32.partial, P32.npart, P32.sc, CG_SET_RR));
        CKL();
        cudaGraphConditionalHandle hi = new_handle(os);
        LAUNCH(&c->stats, VVM_K_CG, os, k_loop_inner<<<1, 1, 0, os>>>(P32.sc, P32.ctl, hi, 1e-8, maxit, 1, c->d_exec, 0));
        CKL();
        cudaGraph_t inner = add_while(os, hi);
        long long n_inner;
        {
            BodyCapture ic(c->cap[1], inner);
            const long long m0 = c->stats.launches;
            int nb = P32.record_iteration(c->d32, ic.s);
            LAUNCH(&c->stats, VVM_K_CG, ic.s, k_loop_inner<<<1, 1, 0, ic.s>>>(P32.sc, P32.ctl, hi, 1e-8, maxit, 0, c->d_exec, nb + 1));
            CKL();
            ic.end();
            n_inner = c->stats.launches - m0;
        }
        LAUNCH(&c->stats, VVM_K_CG, os, k_refine_add<<<G, B, 0, os>>>(P64.NX, P64.NK, P64.pitch, c->W, c->d32));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, os, k_cg_residual<double><<<G, B, 0, os>>>(v, c->Wf, c->W, c->r64, c->wpartial));
        CKL();
        LAUNCH(&c->stats, VVM_K_CG, os, k_cg_scalar<<<1, 1024, 0, os>>>(c->wpartial, c->wnpart, P64.sc, CG_SET_RR));
        CKL();
        const int n_outer = (int)(c->stats.launches - n0 - n_inner) + 1;   // + its own check
        LAUNCH(&c->stats, VVM_K_CG, os, k_loop_outer<<<1, 1, 0, os>>>(P64.sc, c->wctl, P32.ctl, ho, tol * tol, maxit, 0, c->d_exec, n_outer));
        CKL();
        oc.end();
        in_bodies += c->stats.launches - n0;
    }
    (void)n_start;
    return in_bodies;
}

template <typename T>
// before_w: an event the velocity update (k_w_from_W, which writes w) waits
// for, when kernels that read w run beside the solve.
int launch_cal_w(vvm_gpu_ctx* c, long long* recorded_in_loops = nullptr, cudaEvent_t before_w = nullptr) {
    ensure_poisson(c);
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    int NX = c->d.nx - 2, NK = c->d.nz - 3;
    int pitch = c->pcg64->pitch;
    dim3 B(64, 4), G(cdiv(NX, 64), cdiv(NK, 4));
    klaunch<k_poisson_rhs_body<T>, 256>(&c->stats, VVM_K_POISSON_RHS, c->stream, k_poisson_rhs<T>, G, B, 0, c->d,
                                        c->c.dx, (const double*)c->rhow, (const double*)c->rwres,
                                        (const T*)F.zeta[fut], c->Wf, pitch, c->wpartial, c->pcg64->arrive,
                                        c->pcg64->sc);   // sets sc->bb
    const bool warm = c->desc.warm_start != 0;
    const int maxit = c->desc.poisson_maxit > 0 ? c->desc.poisson_maxit : 200;
    if (recorded_in_loops) {   // graph capture: the loops run on the device
        if (warm && !c->spectral) {
            LAUNCH(&c->stats, VVM_K_POISSON_RHS, c->stream, k_extrapolate<<<G, B, 0, c->stream>>>(NX, NK, pitch, c->W, c->Wprev));
            CKL();
        }
        *recorded_in_loops = record_solve(c, c->desc.poisson_tol, maxit, warm);
        c->nsolves++;
        if (before_w) CK(cudaStreamWaitEvent(c->stream, before_w, 0));
        klaunch<k_w_from_W_body<T>, 256>(&c->stats, VVM_K_POISSON_RHS, c->stream, k_w_from_W<T>, c->grid_interior(2),
                                         c->blk(), 0, c->d, (const double*)c->rhow, (const double*)c->W, pitch, F.w);
        return VVM_GPU_OK;
    }
    CK(cudaMemcpyAsync(c->sc_host, &c->pcg64->sc->bb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double bb = *c->sc_host;
    if (warm && !c->spectral) {
        // the previous solution(s) as the initial guess: linear extrapolation
        // once two exist (the reference starts every solve from zero)
        if (c->nsolves >= 2) {
            LAUNCH(&c->stats, VVM_K_POISSON_RHS, c->stream, k_extrapolate<<<G, B, 0, c->stream>>>(NX, NK, pitch, c->W, c->Wprev));
            CKL();
        } else {
            CK(cudaMemcpyAsync(c->Wprev, c->W, (size_t)NK * pitch * sizeof(double), cudaMemcpyDeviceToDevice,
                               c->stream));
        }
    }
    int rc = solve_w(c, bb, c->desc.poisson_tol, warm);
    c->nsolves++;
    if (before_w) CK(cudaStreamWaitEvent(c->stream, before_w, 0));
    LAUNCH(&c->stats, VVM_K_POISSON_RHS, c->stream, k_w_from_W<T><<<c->grid_interior(2), c->blk(), 0, c->stream>>>(c->d, c->rhow, c->W, pitch, F.w));
    CKL();
    return rc;
}

template <typename T>
void launch_cal_u(vvm_gpu_ctx* c) {
    Fields<T>& F = fields<T>(c);
    int fut = 1 - c->cur;
    CalUArgs<T> a{c->d, c->c, c->profiles(), F.u, F.w, F.zeta[fut], c->ubar};
    klaunch<k_cal_u_columns_body<T>, 32 * kColSeg>(&c->stats, VVM_K_CAL_U, c->stream, k_cal_u_columns<T>,
                                                   dim3(cdiv(c->d.nx - 2, 32)), dim3(32 * kColSeg), 0, a);
}

// The psi system's solver: the w-equation's operator on uniform levels with
// an unweighted residual; the exact Fourier-mode solve when NX is a power of
// two (checked, CG from there), multigrid-PCG otherwise.
void ensure_psi(vvm_gpu_ctx* c) {
    if (c->pcg_psi) return;
    const int NX = c->d.nx - 2, NK = c->d.nz - 3;
    std::vector<double> one(c->d.nz, 1.0);
    c->pcg_psi.reset(new PCG<double>());
    c->pcg_psi->stats = &c->stats;
    c->pcg_psi->spectral = Spectral<double>::supports(NX);
    c->pcg_psi->build(c->ar, NX, NK, c->h_rhou, c->h_rhow, one, one, true);
    const int pitch = c->pcg_psi->pitch;
    c->psi_f = c->ar.alloc<double>((size_t)NK * pitch);
    c->psi_x = c->ar.alloc<double>((size_t)NK * pitch);
    c->psi = c->ar.alloc<double>(c->d.cells());
    if (!c->sc_host) CK(cudaMallocHost(&c->sc_host, sizeof(double)));
    if (!c->wpartial) {
        dim3 g(cdiv(NX, 64), cdiv(NK, 4));
        c->wnpart = g.x * g.y;
        c->wpartial = c->ar.alloc<double>(c->wnpart);
    }
}

// PoissonSolver::calpsiuw (src/PoissonSolver.cpp:124-177): psi from zetap,
// then u and w from psi, each with the halos the routine applies. The solve
// starts from zero as the reference's does and stops at desc.poisson_tol.
template <typename T>
int launch_calpsiuw(vvm_gpu_ctx* c) {
    ensure_psi(c);
    PCG<double>& P = *c->pcg_psi;
    Fields<T>& F = fields<T>(c);
    const int fut = 1 - c->cur;
    const int NX = c->d.nx - 2, NK = c->d.nz - 3, pitch = P.pitch;
    dim3 B(64, 4), G(cdiv(NX, 64), cdiv(NK, 4));
    LAUNCH(&c->stats, VVM_K_POISSON_RHS, c->stream, k_psi_rhs<T><<<G, B, 0, c->stream>>>(c->d, c->c.dx, F.zeta[fut], c->psi_f, pitch, c->wpartial));
    CKL();
    LAUNCH(&c->stats, VVM_K_CG, c->stream, k_cg_scalar<<<1, 1024, 0, c->stream>>>(c->wpartial, c->wnpart, P.sc, CG_SET_BB));
    CKL();
    CK(cudaMemcpyAsync(c->sc_host, &P.sc->bb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double bb = *c->sc_host;
    const int maxit = c->desc.poisson_maxit > 0 ? c->desc.poisson_maxit : 200;
    double rel = 0.0;
    int it = 0;
    if (bb == 0.0) {
        CK(cudaMemsetAsync(c->psi_x, 0, (size_t)NK * pitch * sizeof(double), c->stream));
    } else if (P.spectral) {
        P.sp.apply_to(c->psi_f, c->psi_x, c->stream);
        it = P.solve(c->psi_f, c->psi_x, true, bb, c->desc.poisson_tol, maxit, c->stream, &rel);
    } else {
        it = P.solve(c->psi_f, c->psi_x, false, bb, c->desc.poisson_tol, maxit, c->stream, &rel);
    }
    c->last_iters = it;
    c->last_relres = rel;
    LAUNCH(&c->stats, VVM_K_POISSON_RHS, c->stream, k_psi_uw<T><<<c->grid_all(), c->blk(), 0, c->stream>>>(c->d, c->rhou, c->rhow, c->c.rdx, c->c.rdz, c->psi_x, pitch, c->psi, F.u, F.w));
    CKL();
    return (rel <= c->desc.poisson_tol) ? VVM_GPU_OK : VVM_GPU_ENOCONV;
}

// ---------------------------------------------------------------- one step

// Fork/join of a step's second chain: the side stream waits for everything
// issued on the context's stream so far (fork), and the context's stream
// waits for everything issued on the side stream (join). Inside a stream
// capture these become branches of the graph.
void fork_side(vvm_gpu_ctx* c, int e) {
    CK(cudaEventRecord(c->fork_ev[e], c->stream));
    CK(cudaStreamWaitEvent(c->side, c->fork_ev[e], 0));
}
void join_side(vvm_gpu_ctx* c, int e) {
    CK(cudaEventRecord(c->fork_ev[e], c->side));
    CK(cudaStreamWaitEvent(c->stream, c->fork_ev[e], 0));
}
struct OnStream {   // issues a scope's launches on another stream
    vvm_gpu_ctx* c;
    cudaStream_t saved;
    OnStream(vvm_gpu_ctx* c_, cudaStream_t s) : c(c_), saved(c_->stream) { c->stream = s; }
    ~OnStream() { c->stream = saved; }
};

template <typename T>
int run_step(vvm_gpu_ctx* c, long long* recorded_in_loops = nullptr) {
    c->step++;                                                 // Iteration.cpp:246
    const bool sf = (c->desc.flags & VVM_FLAG_STREAMFUNCTION) != 0;
    // The step's kernels form two chains (in a captured step, two branches of
    // the graph; the results are those of the reference's order, since
    // neither chain reads what the other writes before they meet):
    //  main: pzeta_pt (writes zetap and its tendencies), cal_w up to its
    //        solution W, then, once the side chain has read w and u and
    //        written ubarTopp, w from W and cal_u (which reads ubarTopp);
    //  side: pubarTop_pt (reads u, w, RKM; writes ubar, dubar), the scalar
    //        advection (writes the future th, qv, qc, qr and their
    //        tendencies), their NVP rescaling and AddForcing, Kessler, its
    //        NVP and the halos of th, qv, qc, qr.
    // They meet before the turbulence. A batch's cases are already parallel
    // branches of its graph: there every case runs as one chain, in the
    // reference's order; so does a profiled step, whose event timers should
    // each see one kernel at a time.
    const bool br = c->branches && !c->stats.on;
    int rc = VVM_GPU_OK;
    if (br) {
        fork_side(c, 0);
        {
            OnStream os(c, c->side);
            if (!sf) launch_pubartop<T>(c);                    // pubarTop_pt
            launch_padv<T>(c, F_TH | F_QV | F_QC | F_QR, F_QV | F_QC | F_QR, true, true);  // pth, pqv, pqc, pqr
            CK(cudaEventRecord(c->fork_ev[1], c->side));   // u and w read, ubarTopp written
            launch_kessler<T>(c, true, true);                  // NVP + AddForcing, Kessler + NVP x3 + halos
        }
        try {
            launch_pzeta<T>(c);                                // pzeta_pt
            if (sf) {
                CK(cudaStreamWaitEvent(c->stream, c->fork_ev[1], 0));
                rc = launch_calpsiuw<T>(c);                    // calpsiuw (Iteration.cpp:289-290)
            } else {
                rc = launch_cal_w<T>(c, recorded_in_loops, c->fork_ev[1]);   // cal_w
                launch_cal_u<T>(c);                            // cal_u
            }
        } catch (...) {
            join_side(c, 2);
            throw;
        }
        join_side(c, 2);
    } else {
        launch_pzeta<T>(c);                                    // pzeta_pt
        launch_padv<T>(c, F_TH | F_QV | F_QC | F_QR, F_QV | F_QC | F_QR, true, true);  // pth, pqv, pqc, pqr
        if (sf) {
            rc = launch_calpsiuw<T>(c);
        } else {
            launch_pubartop<T>(c);
            rc = launch_cal_w<T>(c, recorded_in_loops);
            launch_cal_u<T>(c);
        }
        // NVP and AddForcing of the advected fields run inside Kessler's
        // kernel (nothing before it reads th, qv, qc, qr; their halos come
        // after it)
        launch_kessler<T>(c, true, true);
    }
    // The first updateMean of the step (Iteration.cpp:408) only writes thb,
    // qvb, thvb, which nextTimeStep's updateMean overwrites before any read.
    launch_turbulence<T>(c, true, recorded_in_loops);          // RKM_RKH + diffusion + theta/zeta nudging
    if (c->desc.moisture_nudge_time != 0.0) launch_nudge<T>(c, false, true);
    launch_update_mean<T>(c, true);                            // nextTimeStep: means, ubarTop
    c->cur = 1 - c->cur;                                       // time levels by pointer swap
    return rc;
}

// The step as one CUDA graph: every kernel of run_step, with the cal_w
// iterations as device-controlled WHILE nodes (no host round trip). Graphs
// are keyed by the time-level buffer and the parity of the step they run
// (the AB2 slots alternate with it) and captured on first use.
template <typename T>
cudaGraphExec_t step_graph(vvm_gpu_ctx* c) {
    const int b = c->cur, par = (c->step + 1) & 1;
    if (c->gexec[b][par]) return c->gexec[b][par];
    ensure_poisson(c);
    if (c->desc.solver == VVM_SOLVER_LEARNED) ensure_learned(c);   // allocations stay outside the capture
    const int step0 = c->step, cur0 = c->cur, ns0 = c->nsolves;
    const long long l0 = c->stats.launches;
    cudaStream_t saved = c->stream;
    c->stream = c->own;
    cudaGraph_t g = nullptr;
    long long in_loops = 0;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    try {
        run_step<T>(c, &in_loops);
    } catch (...) {
        cudaStreamEndCapture(c->stream, &g);
        if (g) cudaGraphDestroy(g);
        c->stream = saved;
        c->step = step0;
        c->cur = cur0;
        c->nsolves = ns0;
        throw;
    }
    CK(cudaStreamEndCapture(c->stream, &g));
    c->stream = saved;
    c->step = step0;
    c->cur = cur0;
    c->nsolves = ns0;
    c->gstatic[b][par] = c->stats.launches - l0 - in_loops;
    c->stats.launches = l0;
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw CudaError{std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
    c->gexec[b][par] = ex;
    return ex;
}

int regen_forcing(vvm_gpu_ctx* c, int t, double lo, double hi, double sd);

// After a graph step the solve's loop state lives on the device: brings
// last_iters / last_relres (and the learned solver's counts) to the host.
void sync_graph_solve(vvm_gpu_ctx* c) {
    if (!c->last_graph || !c->poisson_ready) return;
    CGCtl h{};
    CK(cudaStreamSynchronize(c->stream));
    const bool learned = (c->desc.solver == VVM_SOLVER_LEARNED) && c->fcg_ctl;
    const bool refined = c->mixed && !c->spectral && !learned;   // FP32 inner loops in an FP64 outer loop
    CK(cudaMemcpy(&h, refined ? c->wctl : c->pcg64->ctl, sizeof(CGCtl), cudaMemcpyDeviceToHost));
    c->last_iters = h.total;
    c->last_relres = h.relres;
    if (learned) {
        FcgCtl f{};
        CK(cudaMemcpy(&f, c->fcg_ctl, sizeof(FcgCtl), cudaMemcpyDeviceToHost));
        c->learned_iters = f.k;
        c->learned_fallback = f.converged ? 0 : 1;
        c->last_iters += f.k;
    }
}

template <typename T>
int step_once(vvm_gpu_ctx* c) {
    const bool forcing_now = c->has_forcing_th && ((c->step + 1) * c->desc.dt <= c->desc.addforcingtime);
    const bool warm = c->desc.warm_start != 0;
    const bool use_graph = !c->graphs_off && !c->stats.on && c->step >= 0 && !forcing_now &&
                           c->poisson_ready && (!warm || c->nsolves >= 2) && !c->learned_collect &&
                           !(c->desc.flags & VVM_FLAG_STREAMFUNCTION);
    if (!use_graph) {
        c->last_graph = false;
        // TimeMarching makes the step's forcing field before AddForcing
        // (src/Iteration.cpp:276-283); nothing before AddForcing reads it
        if (forcing_now && !(c->desc.flags & VVM_FLAG_FIXED_FORCING))
            if (int rc = regen_forcing(c, c->step + 1, -0.001, 0.001, 1.)) return rc;
        const int rc = run_step<T>(c);
        c->fut_is_now = true;
        return rc;
    }
    cudaGraphExec_t ex = step_graph<T>(c);
    const int b = c->cur, par = (c->step + 1) & 1;
    CK(cudaGraphLaunch(ex, c->stream));
    c->stats.launches += c->gstatic[b][par];
    c->step++;
    c->cur = 1 - c->cur;
    c->nsolves++;
    c->last_graph = true;
    c->fut_is_now = true;
    return VVM_GPU_OK;
}

// ---------------------------------------------------------------- snapshots

// A device copy of every buffer of a context plus its host-side counters:
// the autotuner runs real steps and puts the cases back exactly afterwards.
struct Snapshot {
    std::vector<void*> copies;
    int step = 0, cur = 0, nsolves = 0, last_iters = 0;
    bool fut_is_now = false;
    double last_relres = 0;
    long long launches = 0;
    void take(vvm_gpu_ctx* c) {
        CK(cudaStreamSynchronize(c->stream));
        for (size_t j = 0; j < c->ar.ptrs.size(); j++) {
            void* q = nullptr;
            CK(cudaMalloc(&q, c->ar.bytes[j]));
            CK(cudaMemcpyAsync(q, c->ar.ptrs[j], c->ar.bytes[j], cudaMemcpyDeviceToDevice, c->stream));
            copies.push_back(q);
        }
        CK(cudaStreamSynchronize(c->stream));
        step = c->step;
        cur = c->cur;
        fut_is_now = c->fut_is_now;
        nsolves = c->nsolves;
        last_iters = c->last_iters;
        last_relres = c->last_relres;
        launches = c->stats.launches;
    }
    void restore(vvm_gpu_ctx* c) {
        CK(cudaStreamSynchronize(c->stream));
        for (size_t j = 0; j < copies.size(); j++)
            CK(cudaMemcpyAsync(c->ar.ptrs[j], copies[j], c->ar.bytes[j], cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->step = step;
        c->cur = cur;
        c->fut_is_now = fut_is_now;
        c->nsolves = nsolves;
        c->last_iters = last_iters;
        c->last_relres = last_relres;
        c->stats.launches = launches;
    }
    ~Snapshot() {
        for (void* q : copies) cudaFree(q);
    }
};

// True when the case's next step may run from a captured graph (the test of
// step_once).
bool graph_ready(vvm_gpu_ctx* c) {
    const bool forcing_now = c->has_forcing_th && ((c->step + 1) * c->desc.dt <= c->desc.addforcingtime);
    const bool warm = c->desc.warm_start != 0;
    return !c->graphs_off && !c->stats.on && c->step >= 0 && !forcing_now && c->poisson_ready &&
           (!warm || c->nsolves >= 2) && !c->learned_collect && !(c->desc.flags & VVM_FLAG_STREAMFUNCTION);
}

}  // namespace

// ---------------------------------------------------------------- batches

// Cases a grouped launch takes at most, unless the autotuner chose otherwise:
// larger groups of a shape are split into parallel sub-groups.
constexpr int kGroupMaxDefault = 32;
// Grids of more cells step case by case unless the autotuner chose grouped
// launches for them. Measured on a B200 (mixed step, spectral cal_w), ms a
// step grouped / case by case: 256 cases of 256 x 64 2.0 / 10.4, 64 of
// 512 x 96 1.40 / 1.83, 64 of 1024 x 96 2.6 / 2.38, 48 of 2048 x 128 4.8 / 3.9.
// A small case's step is launch-bound, so one launch for many cases wins; a
// large case fills the GPU itself, and independent chains of kernels (one a
// case) then overlap their phases, which a group's lock-step launches cannot.
constexpr long long kGroupCellsMax = 65536;

// Independent cases of any sizes that advance together: one CUDA graph per
// step holds every case's step as a parallel branch (captured by forking the
// batch stream to each case's stream and joining back), keyed like a case's
// own graphs by (time-level buffer, step parity).
struct vvm_gpu_batch {
    int device = 0;
    std::vector<vvm_gpu_ctx*> cases;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t gexec[2][2] = {};
    std::vector<long long> gstatic[2][2];   // kernels outside loops, per case
    std::vector<void*> gbufs[2][2];         // device arrays of the grouped launches of gexec
    int group_max = kGroupMaxDefault;       // cases a grouped launch takes at most (0: no grouping)
    int last_groups = 0;                    // grouped groups of the last capture
    std::string err;

    void drop_graphs() {
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                if (gexec[i][j]) {
                    cudaGraphExecDestroy(gexec[i][j]);
                    gexec[i][j] = nullptr;
                }
                for (void* q : gbufs[i][j]) cudaFree(q);
                gbufs[i][j].clear();
            }
    }
    ~vvm_gpu_batch() {
        drop_graphs();
        for (auto* c : cases) vvm_gpu_destroy(c);
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int batch_fail(vvm_gpu_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

// ------------------------------------------------------- grouped launches
//
// Cases of one grid shape, precision and tuning whose step runs the exact
// Fourier-mode cal_w and the tiled Gauss-Seidel passes step as grouped
// launches (grouped.cuh), up to group_limit cases a group (small grids by
// default, larger ones where the autotuner chose it): each case's step is
// recorded, the recordings are
// checked to agree op for op (kernel, launch shape, pack size, loop
// structure), and then replayed side by side, one launch a kernel for the
// whole group, blockIdx.z the case. Groups whose recordings differ step case
// by case.

bool groupable(const vvm_gpu_ctx* c) {
    return c->spectral && c->desc.solver != VVM_SOLVER_LEARNED && c->tune_gs_tr != kGSSchedCluster &&
           !(c->desc.flags & VVM_FLAG_STREAMFUNCTION) && !c->stats.on;
}

// Records case c's next step into r without issuing work; false when some
// launch of it has no grouped form. The case's host-side step state is put
// back.
bool record_step(vvm_gpu_ctx* c, Recorder& r) {
    const int step = c->step, cur = c->cur, ns = c->nsolves;
    const long long l0 = c->stats.launches;
    c->stats.rec = &r;
    c->branches = false;
    bool ok = true;
    long long in_loops = 0;
    try {
        if (c->mixed) run_step<float>(c, &in_loops);
        else run_step<double>(c, &in_loops);
    } catch (const CudaError&) {
        ok = false;
    }
    c->stats.rec = nullptr;
    c->branches = true;
    c->step = step;
    c->cur = cur;
    c->nsolves = ns;
    c->stats.launches = l0;
    return ok;
}

// The most cases a grouped launch of c's shape takes (< 2: none).
int group_limit(const vvm_gpu_batch* b, const vvm_gpu_ctx* c) {
    if (b->group_max < 2) return 0;
    if (c->tune_group > 0) return std::min(c->tune_group, b->group_max);
    return (long long)(c->d.nx - 2) * (c->d.nz - 2) <= kGroupCellsMax ? b->group_max : 1;
}

bool same_ops(const Recorder& a, const Recorder& b) {
    if (a.ops.size() != b.ops.size()) return false;
    for (size_t j = 0; j < a.ops.size(); j++) {
        const RecOp &x = a.ops[j], &y = b.ops[j];
        if (x.kind != y.kind) return false;
        if (x.kind == RecOp::KERNEL &&
            (x.fn != y.fn || x.grid.x != y.grid.x || x.grid.y != y.grid.y || x.grid.z != 1 || y.grid.z != 1 ||
             x.block.x != y.block.x || x.block.y != y.block.y || x.block.z != y.block.z || x.smem != y.smem ||
             x.pack.size() != y.pack.size()))
            return false;
        if (x.kind == RecOp::ZERO && x.bytes != y.bytes) return false;
    }
    return true;
}

// The device arrays of one group's replay: per kernel op the n argument
// packs, per clear the n targets, per condition point the n flags.
struct GroupArrays {
    std::vector<size_t> off;   // per op: offset of its array in the blob
    std::vector<unsigned char> host;
    void* dev = nullptr;
};

GroupArrays group_arrays(const std::vector<Recorder>& recs) {
    const size_t n = recs.size(), nops = recs[0].ops.size();
    GroupArrays A;
    A.off.assign(nops, 0);
    size_t at = 0;
    auto place = [&](size_t bytes) {
        at = (at + 255) / 256 * 256;
        const size_t o = at;
        at += bytes;
        return o;
    };
    std::vector<size_t> stride(nops, 0);
    for (size_t j = 0; j < nops; j++) {
        const RecOp& op = recs[0].ops[j];
        if (op.kind == RecOp::KERNEL) {
            stride[j] = op.pack.size();   // sizeof the pack: the kernel indexes packs[blockIdx.z]
            A.off[j] = place(stride[j] * n);
        } else if (op.kind == RecOp::ZERO || op.kind == RecOp::COND_NEXT || op.kind == RecOp::COND_LOOP) {
            A.off[j] = place(sizeof(void*) * n);
        }
    }
    A.host.assign(std::max<size_t>(at, 1), 0);
    for (size_t j = 0; j < nops; j++) {
        const RecOp::Kind k = recs[0].ops[j].kind;
        for (size_t i = 0; i < n; i++) {
            const RecOp& op = recs[i].ops[j];
            if (k == RecOp::KERNEL) memcpy(&A.host[A.off[j] + i * stride[j]], op.pack.data(), op.pack.size());
            else if (k == RecOp::ZERO || k == RecOp::COND_NEXT || k == RecOp::COND_LOOP)
                memcpy(&A.host[A.off[j] + i * sizeof(void*)], &op.ptr, sizeof(void*));
        }
    }
    CK(cudaMalloc(&A.dev, A.host.size()));
    upload_now(A.dev, A.host.data(), A.host.size());
    for (size_t j = 0; j < nops; j++) {   // kernels needing more than 48 KB of dynamic shared memory
        const RecOp& op = recs[0].ops[j];
        if (op.kind == RecOp::KERNEL && op.smem > 48 * 1024)
            CK(cudaFuncSetAttribute(op.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)op.smem));
    }
    return A;
}

// Issues the group's step on st (under capture): one launch a kernel op,
// blockIdx.z the case; loops as WHILE nodes whose condition a one-block
// kernel sets from the cases' flags. Loop bodies are captured on cap[depth].
// Returns the kernels issued outside loops.
long long group_replay(const std::vector<Recorder>& recs, const GroupArrays& A, cudaStream_t st,
                       const cudaStream_t* cap, int ncap) {
    const int n = (int)recs.size();
    const std::vector<RecOp>& ops = recs[0].ops;
    char* base = static_cast<char*>(A.dev);
    struct Loop {
        cudaGraphConditionalHandle h;
        void* flags;
        std::unique_ptr<BodyCapture> bc;
    };
    std::vector<Loop> open;
    cudaGraphConditionalHandle next_h = 0;
    void* next_flags = nullptr;
    long long outside = 0;
    auto cur = [&]() { return open.empty() ? st : open.back().bc->s; };
    for (size_t j = 0; j < ops.size(); j++) {
        const RecOp& op = ops[j];
        void* arr = base + A.off[j];
        switch (op.kind) {
        case RecOp::KERNEL: {
            void* gate = open.empty() ? nullptr : open.back().flags;
            void* args[2] = {&arr, &gate};
            CK(cudaLaunchKernel(op.fn, dim3(op.grid.x, op.grid.y, n), op.block, args, op.smem, cur()));
            if (open.empty()) outside++;
            break;
        }
        case RecOp::ZERO:
            k_group_zero<<<dim3(1, 1, n), 128, 0, cur()>>>(reinterpret_cast<unsigned char* const*>(arr), op.bytes);
            CKL();
            if (open.empty()) outside++;
            break;
        case RecOp::COND_NEXT:
            next_h = new_handle(cur());
            next_flags = arr;
            k_group_cond<<<1, 256, 0, cur()>>>(reinterpret_cast<const int* const*>(arr), n, next_h);
            CKL();
            if (open.empty()) outside++;
            break;
        case RecOp::COND_LOOP:
            if (open.empty()) throw CudaError{"grouped launch: a loop condition outside a loop"};
            k_group_cond<<<1, 256, 0, cur()>>>(reinterpret_cast<const int* const*>(arr), n, open.back().h);
            CKL();
            break;
        case RecOp::LOOP_BEGIN: {
            if (!next_flags || (int)open.size() >= ncap) throw CudaError{"grouped launch: unsupported loop"};
            cudaGraph_t body = add_while(cur(), next_h);
            Loop L{next_h, next_flags, nullptr};
            L.bc.reset(new BodyCapture(cap[open.size()], body));
            open.push_back(std::move(L));
            next_flags = nullptr;
            break;
        }
        case RecOp::LOOP_END:
            if (open.empty()) throw CudaError{"grouped launch: unbalanced loop"};
            open.back().bc->end();
            open.pop_back();
            break;
        }
    }
    if (!open.empty()) throw CudaError{"grouped launch: unbalanced loop"};
    return outside;
}

// Captures one step of the cases `idx` as a graph on the batch stream;
// gstatic receives each case's kernel count outside loops (a grouped
// launch counts once, for the group's first case); bufs the device arrays
// the graph's grouped launches read.
cudaGraphExec_t batch_capture(vvm_gpu_batch* b, const std::vector<int>& idx, std::vector<long long>& gstatic,
                              std::vector<void*>& bufs) {
    gstatic.assign(b->cases.size(), 0);
    struct Saved {
        cudaStream_t stream;
        int step, cur, nsolves;
        long long launches;
    };
    std::vector<Saved> sv;
    for (int i : idx) {
        vvm_gpu_ctx* c = b->cases[i];
        ensure_poisson(c);
        if (c->desc.solver == VVM_SOLVER_LEARNED) ensure_learned(c);
        sv.push_back({c->stream, c->step, c->cur, c->nsolves, c->stats.launches});
    }
    auto put_back = [&]() {
        for (size_t j = 0; j < idx.size(); j++) {
            vvm_gpu_ctx* c = b->cases[idx[j]];
            c->stream = sv[j].stream;
            c->step = sv[j].step;
            c->cur = sv[j].cur;
            c->nsolves = sv[j].nsolves;
            c->stats.launches = sv[j].launches;
        }
    };
    // groups of cases that can step as grouped launches, recorded and checked
    std::vector<std::vector<int>> groups;
    std::vector<std::vector<Recorder>> recs;
    std::vector<int> alone;
    {
        std::vector<std::vector<int>> cand;
        std::vector<std::array<int, 5>> keys;
        for (int i : idx) {
            vvm_gpu_ctx* c = b->cases[i];
            const int lim = group_limit(b, c);
            if (lim < 2 || !groupable(c)) {
                alone.push_back(i);
                continue;
            }
            const std::array<int, 5> k = {c->d.nx, c->d.nz, c->mixed ? 1 : 0, c->tune_gs_tr, c->tune_fft};
            size_t gi = 0;
            while (gi < keys.size() && keys[gi] != k) gi++;
            if (gi == keys.size()) {
                keys.push_back(k);
                cand.emplace_back();
            }
            cand[gi].push_back(i);
        }
        // split each shape's cases into sub-groups of at most `lim`, sizes as even as possible
        std::vector<std::vector<int>> parts;
        for (auto& gidx : cand) {
            const int lim = group_limit(b, b->cases[gidx[0]]);
            const int m = (int)gidx.size(), np = (m + lim - 1) / lim;
            for (int q = 0, at = 0; q < np; q++) {
                const int sz = m / np + (q < m % np ? 1 : 0);
                parts.emplace_back(gidx.begin() + at, gidx.begin() + at + sz);
                at += sz;
            }
        }
        for (auto& gidx : parts) {
            std::vector<Recorder> r(gidx.size());
            bool ok = gidx.size() >= 2;
            for (size_t j = 0; ok && j < gidx.size(); j++) ok = record_step(b->cases[gidx[j]], r[j]);
            for (size_t j = 1; ok && j < gidx.size(); j++) ok = same_ops(r[0], r[j]);
            if (ok) {
                groups.push_back(gidx);
                recs.push_back(std::move(r));
            } else {
                alone.insert(alone.end(), gidx.begin(), gidx.end());
            }
        }
    }
    std::vector<GroupArrays> arrays;
    try {
        for (auto& r : recs) arrays.push_back(group_arrays(r));
    } catch (...) {
        for (auto& A : arrays) cudaFree(A.dev);
        throw;
    }
    for (auto& A : arrays) bufs.push_back(A.dev);
    b->last_groups = (int)groups.size();
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    try {
        CK(cudaEventRecord(b->fork, b->stream));
        for (size_t gi = 0; gi < groups.size(); gi++) {
            vvm_gpu_ctx* c0 = b->cases[groups[gi][0]];
            CK(cudaStreamWaitEvent(c0->own, b->fork, 0));
            gstatic[groups[gi][0]] = group_replay(recs[gi], arrays[gi], c0->own, c0->cap, 2);
            CK(cudaEventRecord(b->joins[groups[gi][0]], c0->own));
            CK(cudaStreamWaitEvent(b->stream, b->joins[groups[gi][0]], 0));
        }
        for (int i : alone) {
            vvm_gpu_ctx* c = b->cases[i];
            c->stream = c->own;
            CK(cudaStreamWaitEvent(c->own, b->fork, 0));
            const long long l0 = c->stats.launches;
            long long in_loops = 0;
            c->branches = false;   // one chain a case: the cases are the graph's branches
            try {
                if (c->mixed) run_step<float>(c, &in_loops);
                else run_step<double>(c, &in_loops);
            } catch (...) {
                c->branches = true;
                throw;
            }
            c->branches = true;
            gstatic[i] = c->stats.launches - l0 - in_loops;
            CK(cudaEventRecord(b->joins[i], c->own));
            CK(cudaStreamWaitEvent(b->stream, b->joins[i], 0));
        }
    } catch (...) {
        cudaStreamEndCapture(b->stream, &g);
        if (g) cudaGraphDestroy(g);
        put_back();
        throw;
    }
    CK(cudaStreamEndCapture(b->stream, &g));
    put_back();
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw CudaError{std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
    return ex;
}

// Orders the batch stream after every case's stream (into = true) or every
// case's stream after the batch stream.
void batch_fence(vvm_gpu_batch* b, bool into) {
    for (size_t i = 0; i < b->cases.size(); i++) {
        vvm_gpu_ctx* c = b->cases[i];
        if (into) {
            CK(cudaEventRecord(b->joins[i], c->stream));
            CK(cudaStreamWaitEvent(b->stream, b->joins[i], 0));
        } else {
            CK(cudaEventRecord(b->joins[i], b->stream));
            CK(cudaStreamWaitEvent(c->stream, b->joins[i], 0));
        }
    }
}

int batch_step(vvm_gpu_batch* b, int nsteps) {
    int worst = VVM_GPU_OK;
    std::vector<int> all(b->cases.size());
    for (size_t i = 0; i < all.size(); i++) all[i] = (int)i;
    bool on_batch = false;   // work since the last fence sits on the batch stream
    for (int s = 0; s < nsteps; s++) {
        vvm_gpu_ctx* c0 = b->cases[0];
        bool ready = true;
        for (auto* c : b->cases) {
            if (c->step != c0->step || c->cur != c0->cur)
                return batch_fail(b, VVM_GPU_ESTATE, "batch_step: the cases are not at the same step");
            ready = ready && graph_ready(c);
        }
        if (!ready) {   // the first steps, or timers on: each case on its own stream
            if (on_batch) {
                batch_fence(b, false);
                on_batch = false;
            }
            for (auto* c : b->cases) {
                int rc = c->mixed ? step_once<float>(c) : step_once<double>(c);
                if (rc != VVM_GPU_OK) worst = rc;
            }
            continue;
        }
        const int bi = c0->cur, par = (c0->step + 1) & 1;
        if (!b->gexec[bi][par]) b->gexec[bi][par] = batch_capture(b, all, b->gstatic[bi][par], b->gbufs[bi][par]);
        if (!on_batch) {
            batch_fence(b, true);
            on_batch = true;
        }
        CK(cudaGraphLaunch(b->gexec[bi][par], b->stream));
        for (size_t i = 0; i < b->cases.size(); i++) {
            vvm_gpu_ctx* c = b->cases[i];
            c->stats.launches += b->gstatic[bi][par][i];
            c->step++;
            c->cur = 1 - c->cur;
            c->nsolves++;
            c->last_graph = true;
            c->fut_is_now = true;
        }
    }
    if (on_batch) batch_fence(b, false);
    return worst;
}

// Milliseconds a step of the cases `idx` takes as one graph (one launch to
// warm up, then `reps` timed launches of the same graph on the batch stream).
double batch_time(vvm_gpu_batch* b, const std::vector<int>& idx, int reps) {
    std::vector<long long> gs;
    std::vector<void*> bufs;
    struct Free {
        std::vector<void*>& v;
        ~Free() {
            for (void* q : v) cudaFree(q);
        }
    } free_bufs{bufs};
    cudaGraphExec_t ex = batch_capture(b, idx, gs, bufs);
    float ms = 0;
    try {
        CK(cudaGraphLaunch(ex, b->stream));
        CK(cudaEventRecord(b->t0, b->stream));
        for (int r = 0; r < reps; r++) CK(cudaGraphLaunch(ex, b->stream));
        CK(cudaEventRecord(b->t1, b->stream));
        CK(cudaEventSynchronize(b->t1));
        CK(cudaEventElapsedTime(&ms, b->t0, b->t1));
    } catch (...) {
        cudaStreamSynchronize(b->stream);
        cudaGraphExecDestroy(ex);
        throw;
    }
    cudaGraphExecDestroy(ex);
    return ms / std::max(reps, 1);
}

// Autotuner: for each group of cases with the same grid, precision and
// solver, coordinate descent over the launch-shape knobs that leave the
// arithmetic unchanged (the Gauss-Seidel schedule: tile height or one cluster
// a field; the row-FFT block; the cases a grouped launch takes), timing one
// step of the group's cases as a graph per candidate. Every case is put back
// exactly afterwards.
int batch_autotune(vvm_gpu_batch* b, int reps, int* ngroups) {
    const size_t n = b->cases.size();
    CK(cudaStreamSynchronize(b->stream));
    std::vector<std::unique_ptr<Snapshot>> snaps(n);
    for (size_t i = 0; i < n; i++) {
        snaps[i].reset(new Snapshot());
        snaps[i]->take(b->cases[i]);
    }
    int rc = VVM_GPU_OK;
    // bring every case to a step that runs from a graph (restored below)
    for (int guard = 0; guard < 4 && rc == VVM_GPU_OK; guard++) {
        bool ready = true;
        for (auto* c : b->cases) ready = ready && graph_ready(c);
        if (ready) break;
        rc = batch_step(b, 1);
    }
    std::vector<std::vector<int>> groups;
    std::vector<std::array<int, 4>> keys;
    for (size_t i = 0; i < n; i++) {
        vvm_gpu_ctx* c = b->cases[i];
        std::array<int, 4> k = {c->d.nx, c->d.nz, c->mixed ? 1 : 0, c->spectral ? 1 : 0};
        size_t gi = 0;
        while (gi < keys.size() && keys[gi] != k) gi++;
        if (gi == keys.size()) {
            keys.push_back(k);
            groups.emplace_back();
        }
        groups[gi].push_back((int)i);
    }
    auto set_all = [&](const std::vector<int>& idx, int tr, int fft) {
        for (int i : idx) {
            vvm_gpu_ctx* c = b->cases[i];
            if (tr == kGSSchedCluster) ensure_gs_cluster(c);
            c->tune_gs_tr = tr;
            c->tune_fft = fft;
            apply_tuning(c);
        }
    };
    for (size_t gi = 0; gi < groups.size() && rc == VVM_GPU_OK; gi++) {
        const std::vector<int>& idx = groups[gi];
        vvm_gpu_ctx* c = b->cases[idx[0]];
        int best_cs = c->tune_gs_tr, best_fft = c->tune_fft;
        double best = batch_time(b, idx, reps);
        for (int tr : {kGSSchedCluster, 4, 8, 16, 32}) {   // Gauss-Seidel schedule: cluster, tile rows
            set_all(idx, tr, best_fft);
            const double t = batch_time(b, idx, reps);
            if (t < best) {
                best = t;
                best_cs = tr;
            }
        }
        set_all(idx, best_cs, best_fft);
        if (c->spectral) {
            for (int th : {128, 256, 512}) {
                set_all(idx, best_cs, th);
                const double t = batch_time(b, idx, reps);
                if (t < best) {
                    best = t;
                    best_fft = th;
                }
            }
        }
        set_all(idx, best_cs, best_fft);
        // cases a grouped launch takes: one launch for all of them, sub-groups
        // as parallel branches, or (1) every case its own branch
        if (idx.size() >= 2 && groupable(c)) {
            const int m = (int)idx.size();
            int best_grp = 0;
            for (int gsz : {1, m, (m + 1) / 2, (m + 3) / 4, (m + 7) / 8}) {
                if (gsz < 2 && gsz != 1) continue;
                for (int i : idx) b->cases[i]->tune_group = gsz;
                const double t = batch_time(b, idx, reps);
                if (t < best) {
                    best = t;
                    best_grp = gsz;
                }
            }
            for (int i : idx) b->cases[i]->tune_group = best_grp;
        }
    }
    CK(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < n; i++) {
        snaps[i]->restore(b->cases[i]);
        b->cases[i]->drop_graphs();
    }
    b->drop_graphs();
    if (ngroups) *ngroups = (int)groups.size();
    return rc;
}

template <typename Fn>
int batch_guarded(vvm_gpu_batch* b, Fn fn) {
    if (!b) return VVM_GPU_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    int rc;
    try {
        rc = fn();
    } catch (const CudaError& e) {
        rc = batch_fail(b, VVM_GPU_ECUDA, e.msg);
    }
    if (prev != b->device) cudaSetDevice(prev);
    return rc;
}

// ---------------------------------------------------------------- transfer

template <typename T>
void upload_field(vvm_gpu_ctx* c, const double* host, int sk, int off, T* dst, const double* ref = nullptr) {
    size_t n = (size_t)c->d.nx * c->d.nz * sk;
    CK(cudaMemcpyAsync(c->staging, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    dim3 b(32, 8), g(cdiv(c->d.nx, 32), cdiv(c->d.nz, 8));
    LAUNCH(&c->stats, VVM_K_MEAN, c->stream, k_from_host_layout<T><<<g, b, 0, c->stream>>>(c->d, c->staging, sk, off, ref, dst));
    CKL();
}

// Init::RandomPerturbation (src/Init.cpp:488-515) on the host, with the
// reference's own generator so the numbers are the same: std::mt19937 seeded
// with t, std::normal_distribution<> of mean 0 and deviation 1 scaled by sd
// and drawn again until inside [lo, hi], for the interior cells with
// z = (k - 0.5) dz < 200 m (k outer, i inner; the others 0), then the ghost
// images of BoundaryProcess2D_center (src/Boundary.cpp:9-19). out is
// [nx][nz]. A cell that takes more than kMaxDraws draws fails (EINVAL).
constexpr long long kMaxDraws = 1ll << 28;   // ~5 s of draws; [-0.001, 0.001] needs ~1250 a cell
int random_perturbation(int NX, int NZ, double dz, int t, double lo, double hi, double sd, double* out) {
    if (NX < 1 || NZ < 1 || !out || !(dz > 0) || !(lo <= hi) || !(sd > 0)) return VVM_GPU_EINVAL;
    const int nx = NX + 2, nz = NZ + 2;
    std::mt19937 gen(t);
    std::normal_distribution<> dist(0.0, 1.0);
    for (int k = 1; k < nz - 1; k++) {
        const double z = (k - 0.5) * dz;
        for (int i = 1; i < nx - 1; i++) {
            double v = 0.;
            if (z < 200) {
                long long n = 0;
                do {
                    v = 0. + sd * dist(gen);
                    if (++n > kMaxDraws) return VVM_GPU_EINVAL;
                } while (v < lo || v > hi);
            }
            out[(size_t)i * nz + k] = v;
        }
    }
    for (int k = 1; k <= nz - 2; k++) {
        out[k] = out[(size_t)(nx - 2) * nz + k];
        out[(size_t)(nx - 1) * nz + k] = out[(size_t)nz + k];
    }
    for (int i = 0; i < nx; i++) {
        out[(size_t)i * nz] = out[(size_t)i * nz + 1];
        out[(size_t)i * nz + nz - 1] = out[(size_t)i * nz + nz - 2];
    }
    return VVM_GPU_OK;
}

template <typename T>
void upload_forcing(vvm_gpu_ctx* c) {
    upload_field<T>(c, c->h_forcing.data(), 1, 0, fields<T>(c).th_forcing);
}

// The field of step t into the device's init_th_forcing (stream-ordered).
int regen_forcing(vvm_gpu_ctx* c, int t, double lo, double hi, double sd) {
    c->h_forcing.assign((size_t)c->d.nx * c->d.nz, 0.);
    if (int rc = random_perturbation(c->d.nx - 2, c->d.nz - 2, c->desc.dz, t, lo, hi, sd, c->h_forcing.data()))
        return fail(c, rc, "random_perturbation: needs min_range <= max_range and standard_deviation > 0");
    (c->mixed ? upload_forcing<float> : upload_forcing<double>)(c);
    c->has_forcing_th = true;
    return VVM_GPU_OK;
}

template <typename T>
void download_field(vvm_gpu_ctx* c, const T* src, int sk, int off, double* host, bool first_of_pair,
                    const double* ref = nullptr) {
    size_t n = (size_t)c->d.nx * c->d.nz * sk;
    dim3 b(32, 8), g(cdiv(c->d.nx, 32), cdiv(c->d.nz, 8));
    LAUNCH(&c->stats, VVM_K_MEAN, c->stream, k_to_host_layout<T><<<g, b, 0, c->stream>>>(c->d, src, sk, off, ref, c->staging));
    CKL();
    if (!first_of_pair) {
        CK(cudaMemcpyAsync(host, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
}

void upload_profile(vvm_gpu_ctx* c, const double* h, double* dptr) {
    CK(cudaMemcpyAsync(dptr, h, c->d.nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
}

template <typename T>
int upload_prognostic_t(vvm_gpu_ctx* c, const vvm_gpu_host_state* s) {
    Fields<T>& F = fields<T>(c);
    int now = c->cur, fut = 1 - c->cur;
    const double* req[] = {s->zeta, s->th, s->qv, s->qc, s->qr, s->u, s->w};
    for (const double* p : req)
        if (!p) return fail(c, VVM_GPU_EINVAL, "upload: prognostic field pointer is NULL");
    // the fields' copies back to back on the copy stream, two staging slots
    // alternating, each slot's layout kernel on the context's stream: the
    // link stays busy while the previous field is rearranged
    struct { const double* h; T* dptr; const double* ref; } m[] = {
        {s->zeta, F.zeta[now], nullptr}, {s->th, F.th[now], c->offset_th()}, {s->qv, F.qv[now], c->offset_qv()},
        {s->qc, F.qc[now], nullptr}, {s->qr, F.qr[now], nullptr}, {s->u, F.u, nullptr}, {s->w, F.w, nullptr}};
    const size_t n = (size_t)c->d.nx * c->d.nz;
    const dim3 b(32, 8), g(cdiv(c->d.nx, 32), cdiv(c->d.nz, 8));
    // no copy into staging before the work already on the context's stream
    // (which may read it) is done
    CK(cudaEventRecord(c->xev[0][1], c->stream));
    CK(cudaEventRecord(c->xev[1][1], c->stream));
    for (int f = 0; f < 7; f++) {
        const int slot = f & 1;
        double* st = c->staging + slot * n;
        CK(cudaStreamWaitEvent(c->xfer, c->xev[slot][1], 0));   // the slot's last reader is done
        CK(cudaMemcpyAsync(st, m[f].h, n * sizeof(double), cudaMemcpyHostToDevice, c->xfer));
        CK(cudaEventRecord(c->xev[slot][0], c->xfer));
        CK(cudaStreamWaitEvent(c->stream, c->xev[slot][0], 0));
        LAUNCH(&c->stats, VVM_K_MEAN, c->stream,
               k_from_host_layout<T><<<g, b, 0, c->stream>>>(c->d, st, 1, 0, m[f].ref, m[f].dptr));
        CKL();
        CK(cudaEventRecord(c->xev[slot][1], c->stream));
    }
    (void)fut;
    return VVM_GPU_OK;
}

template <typename T>
int upload_state_t(vvm_gpu_ctx* c, const vvm_gpu_host_state* s) {
    Fields<T>& F = fields<T>(c);
    int rc = upload_prognostic_t<T>(c, s);
    if (rc) return rc;
    int fut = 1 - c->cur;
    size_t n = c->d.cells();
    auto up_or_zero = [&](const double* h, int sk, int off, T* dst, const double* ref = nullptr) {
        if (h) upload_field<T>(c, h, sk, off, dst, ref);
        else CK(cudaMemsetAsync(dst, 0, n * sizeof(T), c->stream));
    };
    up_or_zero(s->zetap, 1, 0, F.zeta[fut]);
    up_or_zero(s->thp, 1, 0, F.th[fut], c->offset_th());
    up_or_zero(s->qvp, 1, 0, F.qv[fut], c->offset_qv());
    up_or_zero(s->qcp, 1, 0, F.qc[fut]);
    up_or_zero(s->qrp, 1, 0, F.qr[fut]);
    up_or_zero(s->RKM, 1, 0, F.RKM);
    up_or_zero(s->RKH, 1, 0, F.RKH);
    double* hs[NHIST] = {s->dzeta_advect, s->dth_buoyancy, s->dth_advect, s->dqv_advect,
                         s->dqc_advect, s->dqr_advect, s->dqr_VT};
    for (int h = 0; h < NHIST; h++)
        for (int sl = 0; sl < 2; sl++) up_or_zero(hs[h], 2, sl, F.hist[h][sl]);
    // regenerated each forced step unless the uploaded field is to be kept
    c->has_forcing_th = (s->init_th_forcing != nullptr) || !(c->desc.flags & VVM_FLAG_FIXED_FORCING);
    up_or_zero(s->init_th_forcing, 1, 0, F.th_forcing);
    if (s->precip) {
        std::vector<T> pr(c->d.nx);
        for (int i = 0; i < c->d.nx; i++) pr[i] = T(s->precip[i]);
        CK(cudaMemcpyAsync(F.precip, pr.data(), c->d.nx * sizeof(T), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return VVM_GPU_OK;
}

// Coefficient profiles (double) with the reference's expressions.
int upload_profiles(vvm_gpu_ctx* c, const vvm_gpu_host_state* s) {
    const int nz = c->d.nz;
    const double* req[] = {s->rhou, s->rhow, s->thb, s->thvb, s->qvb, s->pib, s->pb,
                           s->thb_init, s->qvb0, s->z, s->z_zeta, s->lambda2};
    for (const double* p : req)
        if (!p) return fail(c, VVM_GPU_EINVAL, "upload: profile pointer is NULL");
    upload_profile(c, s->rhou, c->rhou);
    upload_profile(c, s->rhow, c->rhow);
    upload_profile(c, s->thb, c->thb);
    upload_profile(c, s->thvb, c->thvb);
    upload_profile(c, s->qvb, c->qvb);
    upload_profile(c, s->pib, c->pib);
    upload_profile(c, s->pb, c->pb);
    upload_profile(c, s->thb_init, c->thb_init);
    upload_profile(c, s->qvb0, c->qvb0);
    upload_profile(c, s->z, c->z);
    upload_profile(c, s->z_zeta, c->z_zeta);
    upload_profile(c, s->lambda2, c->lambda2);
    const vvm_gpu_desc& D = c->desc;
    std::vector<double> vt1(nz), vtf(nz), pc(nz), cth(nz, 0.0), cze(nz, 0.0), q1(nz, 0.0), q2(nz, 0.0);
    for (int k = 0; k < nz; k++) {
        vt1[k] = 1E-3 * s->rhow[k] * 0.5;                            // Advection.cpp:165
        vtf[k] = std::pow(s->rhow[k] / s->rhow[1], -0.5);
        pc[k] = 380. / (std::pow(s->pib[k], D.cp / D.rd) * D.p0);    // MicroPhysics.cpp:10
    }
    // Vertical level metric of the stencils (the C restatement's levels(),
    // oracle/vvm_oracle.c, formula for formula): with dc[k] = 2 (z[k] -
    // z_zeta[k]) the thickness of centre cell k and dw[k] = z[k] - z[k-1] the
    // distance between the centres around face k (mirror centres beyond the
    // surface and the top: dw[1] = dc[1], dw[nz-1] = dc[nz-2]), a flux
    // divergence at a centre is over dc, at a face over dw, a gradient across
    // two centres over z[k+1] - z[k-1]. Uniform levels (every spacing within
    // 1e-9 dz of dz) take the reference's constants exactly.
    bool lv_uniform = true;
    for (int k = 1; k <= nz - 2; k++)
        if (std::fabs(2.0 * (s->z[k] - s->z_zeta[k]) - D.dz) > 1e-9 * D.dz) lv_uniform = false;
    for (int k = 2; k <= nz - 2; k++)
        if (std::fabs((s->z[k] - s->z[k - 1]) - D.dz) > 1e-9 * D.dz) lv_uniform = false;
    {
        std::vector<double> r2c(nz), r2w(nz), rc(nz), r2cc(nz), km(nz), mcz(nz), mrd(nz), scz(nz), srd(nz), dzw(nz);
        const double rdz = 1.0 / D.dz, r2dz = rdz / 2.0, rdz2 = rdz * rdz;
        if (lv_uniform) {
            for (int k = 0; k < nz; k++) {
                r2c[k] = r2dz; r2w[k] = r2dz; rc[k] = rdz; r2cc[k] = r2dz;
                km[k] = 0.8 * D.dx * D.dz / D.dt;
                mcz[k] = rdz2 * D.dt / s->rhow[k];       // Turbulent.cpp:84
                mrd[k] = k > 0 ? 1.0 * s->rhou[k - 1] : 0.0;
                scz[k] = rdz2 * D.dt / s->rhou[k];       // Turbulent.cpp:108
                srd[k] = 1.0 * s->rhow[k];
                dzw[k] = D.dz;
            }
            c->lv_rdz_up = c->lv_rdz_dn = c->lv_rdz_c = rdz;
            c->lv_hfac = 1.0;
        } else {
            std::vector<double> dc(nz), dw(nz);
            for (int k = 1; k <= nz - 2; k++) dc[k] = 2.0 * (s->z[k] - s->z_zeta[k]);
            dc[0] = dc[1];
            dc[nz - 1] = dc[nz - 2];
            for (int k = 2; k <= nz - 2; k++) dw[k] = s->z[k] - s->z[k - 1];
            dw[1] = dc[1];
            dw[0] = dc[1];
            dw[nz - 1] = dc[nz - 2];
            for (int k = 0; k < nz; k++) {
                r2c[k] = (1.0 / dc[k]) / 2.0;
                r2w[k] = (1.0 / dw[k]) / 2.0;
                rc[k] = 1.0 / dc[k];
                km[k] = 0.8 * D.dx * dc[k] / D.dt;
                dzw[k] = dw[k];
                r2cc[k] = r2dz;
                mcz[k] = scz[k] = 0.0;
                mrd[k] = srd[k] = 0.0;
            }
            for (int k = 1; k <= nz - 2; k++) {
                const double zm = (k == 1) ? s->z[1] - dc[1] : s->z[k - 1];
                const double zp = (k == nz - 2) ? s->z[nz - 2] + dc[nz - 2] : s->z[k + 1];
                r2cc[k] = 1.0 / (zp - zm);
                mcz[k] = ((1.0 / dw[k]) * (1.0 / dc[k])) * D.dt / s->rhow[k];
                mrd[k] = (dc[k] / dc[k - 1]) * s->rhou[k - 1];
                scz[k] = ((1.0 / dc[k]) * (1.0 / dw[k + 1])) * D.dt / s->rhou[k];
                srd[k] = (dw[k + 1] / dw[k]) * s->rhow[k];
            }
            c->lv_rdz_up = 1.0 / dw[nz - 1];
            c->lv_rdz_dn = 1.0 / dw[nz - 2];
            c->lv_rdz_c = 1.0 / dc[nz - 2];
            c->lv_hfac = D.dx / dc[nz - 2];
        }
        upload_profile(c, r2c.data(), c->lv_r2dzc);
        upload_profile(c, r2w.data(), c->lv_r2dzw);
        upload_profile(c, rc.data(), c->lv_rdzc);
        upload_profile(c, r2cc.data(), c->lv_r2dzcc);
        upload_profile(c, km.data(), c->lv_kmax);
        upload_profile(c, mcz.data(), c->gsM_cz);
        upload_profile(c, mrd.data(), c->gsM_rhod);
        upload_profile(c, scz.data(), c->gsS_cz);
        upload_profile(c, srd.data(), c->gsS_rhod);
        upload_profile(c, dzw.data(), c->lv_dzw);
    }
    // the first nudged level (NumericalProcess.cpp:62: 12000 / dz + 1); on
    // stretched levels the last face at or below 12 km
    int ks = (int)(12000. / D.dz + 1);
    if (!lv_uniform) {
        ks = 1;
        for (int k = 1; k <= nz - 1; k++)
            if (s->z_zeta[k] <= 12000.) ks = k;
    }
    if (ks < nz - 1 && (nz - 1) - ks >= 0) {
        const double* z = s->z;
        const double* zz = s->z_zeta;
        int kb = (nz - 1) - ks;
        for (int k = ks; k < nz - 1; k++) {
            double CGR = (1. / 3600.) * (z[k] - z[kb]) / (z[nz - 1] - z[kb]);
            cth[k] = D.dt * CGR;
            if (D.case_id != 2) {
                double CGRz = (1. / 360.) * (zz[k] - zz[kb]) / (zz[nz - 1] - zz[kb]);
                cze[k] = D.dt * CGRz;
            }
        }
    }
    c->has_q = false;
    if (s->Q1LS) { q1.assign(s->Q1LS, s->Q1LS + nz); c->has_q = true; }
    if (s->Q2LS) { q2.assign(s->Q2LS, s->Q2LS + nz); c->has_q = true; }
    upload_profile(c, vt1.data(), c->vt_c1);
    upload_profile(c, vtf.data(), c->vt_fac);
    upload_profile(c, pc.data(), c->pc);
    upload_profile(c, cth.data(), c->dtcgr_th);
    upload_profile(c, cze.data(), c->dtcgr_zeta);
    upload_profile(c, q1.data(), c->q1ls);
    upload_profile(c, q2.data(), c->q2ls);
    // perturbation profiles (reference profile with its 1D center halo)
    const double* tgt[2] = {s->thb_init, s->qvb0};
    for (int j = 0; j < 2; j++) {
        std::vector<double> r(tgt[j], tgt[j] + nz), d0(nz, 0.0), s0(nz, 0.0), g0(nz, 0.0), dn(nz, 0.0);
        r[0] = r[1];
        r[nz - 1] = r[nz - 2];
        for (int k = 1; k < nz; k++) {
            d0[k] = r[k] - r[k - 1];
            s0[k] = r[k] + r[k - 1];
        }
        for (int k = 1; k < nz - 1; k++) g0[k] = r[k + 1] - r[k - 1];
        for (int k = 0; k < nz; k++) dn[k] = r[k] - tgt[j][k];
        upload_profile(c, r.data(), c->pref[j]);
        upload_profile(c, d0.data(), c->pd0[j]);
        upload_profile(c, s0.data(), c->ps0[j]);
        upload_profile(c, g0.data(), c->pg0[j]);
        upload_profile(c, dn.data(), c->pdn[j]);
    }
    c->pf1 = 1E-3 * s->rhou[1];                                      // Iteration.cpp:115
    c->pf2 = std::pow(s->rhou[1] / s->rhow[1], -0.5);
    // vertical metric from the level heights: uniform levels (every spacing
    // equal to dz) keep the reference's operator exactly (a = h = 1, whatever
    // dx is, as the reference's matrix assumes); otherwise the stretched one
    std::vector<double> ma(nz, 1.0), mh(nz, 1.0);
    bool uniform = true;
    for (int k = 1; k < nz - 1; k++) {
        const double dzu = 2.0 * (s->z[k] - s->z_zeta[k]);
        if (!(dzu > 0)) return fail(c, VVM_GPU_EINVAL, "upload: level heights z must lie above z_zeta");
        if (std::fabs(dzu - c->desc.dz) > 1e-9 * c->desc.dz) uniform = false;
        mh[k] = c->desc.dx / dzu;
    }
    for (int k = 2; k < nz - 1; k++) {
        const double dzw = s->z[k] - s->z[k - 1];
        if (!(dzw > 0)) return fail(c, VVM_GPU_EINVAL, "upload: level heights z must increase");
        if (std::fabs(dzw - c->desc.dz) > 1e-9 * c->desc.dz) uniform = false;
        ma[k] = dzw / c->desc.dx;
    }
    if (uniform) {
        std::fill(ma.begin(), ma.end(), 1.0);
        std::fill(mh.begin(), mh.end(), 1.0);
    }
    c->stretched = !uniform;
    std::vector<double> rw(nz);
    for (int k = 0; k < nz; k++) rw[k] = s->rhow[k] / ma[k];
    upload_profile(c, rw.data(), c->rwres);
    bool changed = c->h_rhou.empty() ||
                   !std::equal(c->h_rhou.begin(), c->h_rhou.end(), s->rhou) ||
                   !std::equal(c->h_rhow.begin(), c->h_rhow.end(), s->rhow) || c->h_a != ma || c->h_h != mh;
    c->h_rhou.assign(s->rhou, s->rhou + nz);
    c->h_rhow.assign(s->rhow, s->rhow + nz);
    c->h_a = ma;
    c->h_h = mh;
    if (changed && c->poisson_ready) {
        // the elliptic operator depends on rhou/rhow: rebuild on next use
        c->poisson_ready = false;
        c->pcg64.reset();
        c->pcg32.reset();
    }
    double ub[2] = {s->ubarTop, s->ubarTopp};
    CK(cudaMemcpyAsync(c->ubar, ub, sizeof(ub), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->dubar, s->dubarTop_advect, 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->step = s->step;
    return VVM_GPU_OK;
}

template <typename T>
int download_prognostic_t(vvm_gpu_ctx* c, vvm_gpu_host_state* s) {
    Fields<T>& F = fields<T>(c);
    int now = c->cur;
    struct { double* h; T* dptr; const double* ref; } m[] = {
        {s->zeta, F.zeta[now], nullptr}, {s->th, F.th[now], c->offset_th()}, {s->qv, F.qv[now], c->offset_qv()},
        {s->qc, F.qc[now], nullptr}, {s->qr, F.qr[now], nullptr}, {s->u, F.u, nullptr}, {s->w, F.w, nullptr}};
    // each field's layout kernel into one of two staging slots on the
    // context's stream, its copy to the host on the copy stream: the link
    // stays busy while the next field is rearranged; one wait at the end
    const size_t n = (size_t)c->d.nx * c->d.nz;
    const dim3 b(32, 8), g(cdiv(c->d.nx, 32), cdiv(c->d.nz, 8));
    int f = 0;
    for (auto& e : m) {
        if (!e.h) continue;
        const int slot = f++ & 1;
        double* st = c->staging + slot * n;
        CK(cudaStreamWaitEvent(c->stream, c->xev[slot][0], 0));   // the slot's last copy is done
        LAUNCH(&c->stats, VVM_K_MEAN, c->stream,
               k_to_host_layout<T><<<g, b, 0, c->stream>>>(c->d, e.dptr, 1, 0, e.ref, st));
        CKL();
        CK(cudaEventRecord(c->xev[slot][1], c->stream));
        CK(cudaStreamWaitEvent(c->xfer, c->xev[slot][1], 0));
        CK(cudaMemcpyAsync(e.h, st, n * sizeof(double), cudaMemcpyDeviceToHost, c->xfer));
        CK(cudaEventRecord(c->xev[slot][0], c->xfer));
    }
    // later work on the context's stream may reuse the staging slots
    CK(cudaEventRecord(c->xev[0][0], c->xfer));
    CK(cudaStreamWaitEvent(c->stream, c->xev[0][0], 0));
    CK(cudaStreamSynchronize(c->xfer));
    return VVM_GPU_OK;
}

template <typename T>
int download_state_t(vvm_gpu_ctx* c, vvm_gpu_host_state* s) {
    Fields<T>& F = fields<T>(c);
    download_prognostic_t<T>(c, s);
    const int fut = c->fut_is_now ? c->cur : 1 - c->cur;
    struct { double* h; T* dptr; const double* ref; } m[] = {
        {s->zetap, F.zeta[fut], nullptr}, {s->thp, F.th[fut], c->offset_th()}, {s->qvp, F.qv[fut], c->offset_qv()},
        {s->qcp, F.qc[fut], nullptr}, {s->qrp, F.qr[fut], nullptr}, {s->RKM, F.RKM, nullptr},
        {s->RKH, F.RKH, nullptr}};
    for (auto& e : m)
        if (e.h) download_field<T>(c, e.dptr, 1, 0, e.h, false, e.ref);
    double* hs[NHIST] = {s->dzeta_advect, s->dth_buoyancy, s->dth_advect, s->dqv_advect,
                         s->dqc_advect, s->dqr_advect, s->dqr_VT};
    for (int h = 0; h < NHIST; h++) {
        if (!hs[h]) continue;
        download_field<T>(c, F.hist[h][0], 2, 0, hs[h], true);
        download_field<T>(c, F.hist[h][1], 2, 1, hs[h], false);
    }
    auto down_prof = [&](double* h, const double* dptr) {
        if (h) CK(cudaMemcpy(h, dptr, c->d.nz * sizeof(double), cudaMemcpyDeviceToHost));
    };
    CK(cudaStreamSynchronize(c->stream));
    down_prof(s->thb, c->thb);
    down_prof(s->qvb, c->qvb);
    down_prof(s->thvb, c->thvb);
    down_prof(s->rhou, c->rhou);
    down_prof(s->rhow, c->rhow);
    if (s->precip) {
        std::vector<T> pr(c->d.nx);
        CK(cudaMemcpy(pr.data(), F.precip, c->d.nx * sizeof(T), cudaMemcpyDeviceToHost));
        for (int i = 0; i < c->d.nx; i++) s->precip[i] = (double)pr[i];
    }
    double ub[2];
    CK(cudaMemcpy(ub, c->ubar, sizeof(ub), cudaMemcpyDeviceToHost));
    s->ubarTop = ub[0];
    s->ubarTopp = ub[1];
    CK(cudaMemcpy(s->dubarTop_advect, c->dubar, 2 * sizeof(double), cudaMemcpyDeviceToHost));
    s->step = c->step;
    return VVM_GPU_OK;
}

// Runs `fn` with the context's device current, mapping exceptions to statuses.
template <typename Fn>
int guarded(vvm_gpu_ctx* c, Fn fn) {
    if (!c) return VVM_GPU_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    int rc;
    try {
        rc = fn();
    } catch (const CudaError& e) {
        rc = fail(c, VVM_GPU_ECUDA, e.msg);
    }
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

#define DISPATCH(c, fn) ((c)->mixed ? fn<float> : fn<double>)

int need_state(vvm_gpu_ctx* c) {
    return c->has_state ? VVM_GPU_OK : fail(c, VVM_GPU_ESTATE, "no state uploaded");
}

// The streamfunction formulation keeps the reference's psi matrix, which
// assumes uniform levels; every other entry takes stretched levels.
int need_uniform(vvm_gpu_ctx* c) {
    return c->stretched ? fail(c, VVM_GPU_EINVAL,
                               "stretched vertical levels: the streamfunction formulation needs uniform levels")
                        : VVM_GPU_OK;
}


// Reads and clears the device error word (after the stream's work is done).
int device_errors(vvm_gpu_ctx* c) {
    if (!c->d_err) return VVM_GPU_OK;
    int h = 0;
    CK(cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!h) return VVM_GPU_OK;
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return fail(c, VVM_GPU_ECUDA, "Gauss-Seidel diffusion (cluster schedule): a wait between warps gave up; "
                                  "the state is invalid");
}

}  // namespace

// Message of a failed context-free entry, returned by vvm_gpu_last_error(NULL, ...).
void vvm_set_context_free_error(const std::string& msg) { g_create_error = msg; }

// ===========================================================================
// C ABI

extern "C" {

void vvm_gpu_desc_default(vvm_gpu_desc* d, int NX, int NZ, double dx, double dz, double dt) {
    std::memset(d, 0, sizeof(*d));
    d->NX = NX;
    d->NZ = NZ;
    d->dx = dx;
    d->dz = dz;
    d->dt = dt;
    d->gravity = 9.80665;
    d->cp = 1003.5;
    d->cv = 716.5;
    d->rd = 287.;
    d->lv = 2.5E6;
    d->p0 = 1E5;
    d->psurf = 96500.;
    d->poisson_tol = 1e-10;
    d->poisson_maxit = 200;
    d->case_id = 1;
    d->precision = VVM_PREC_FP64;
    d->solver = VVM_SOLVER_MGPCG;
    d->warm_start = 1;
}

int vvm_gpu_create(const vvm_gpu_desc* desc, int device, vvm_gpu_ctx** out) {
    if (!desc || !out) return fail(nullptr, VVM_GPU_EINVAL, "create: NULL argument");
    *out = nullptr;
    const vvm_gpu_desc& D = *desc;
    if (D.NX < 4 || D.NZ < 4) return fail(nullptr, VVM_GPU_EINVAL, "create: NX and NZ must be >= 4");
    if (D.NX > kGSMaxNX || gs_plan(round_up(D.NX + 2, kPad), D.NZ + 2, 8).w > kGSClusterWarps)
        return fail(nullptr, VVM_GPU_EINVAL, "create: NX exceeds 8192");
    if (D.NZ - 1 > 32 * kMaxSeg)
        return fail(nullptr, VVM_GPU_EINVAL, "create: NZ exceeds 1025");
    {
        int odd = D.NX;
        while (odd % 2 == 0) odd /= 2;
        if (odd > kMaxOddCoarse)
            return fail(nullptr, VVM_GPU_EINVAL, "create: the odd factor of NX must be <= 256");
    }
    if (!(D.dx > 0) || !(D.dz > 0) || !(D.dt > 0)) return fail(nullptr, VVM_GPU_EINVAL, "create: dx, dz, dt must be > 0");
    if (D.precision != VVM_PREC_FP64 && D.precision != VVM_PREC_MIXED)
        return fail(nullptr, VVM_GPU_EINVAL, "create: unknown precision");
    if (D.flags & ~(VVM_FLAG_FIXED_FORCING | VVM_FLAG_STREAMFUNCTION))
        return fail(nullptr, VVM_GPU_EINVAL, "create: unknown flags");
    if (D.solver != VVM_SOLVER_MGPCG && D.solver != VVM_SOLVER_LEARNED && D.solver != VVM_SOLVER_SPECTRAL)
        return fail(nullptr, VVM_GPU_EINVAL, "create: unknown solver");
    if (D.solver == VVM_SOLVER_SPECTRAL && !Spectral<double>::supports(D.NX))
        return fail(nullptr, VVM_GPU_EINVAL, "create: the spectral solver needs NX a power of two (4..8192)");
    std::unique_ptr<vvm_gpu_ctx> c(new vvm_gpu_ctx());
    c->desc = D;
    c->device = device;
    c->mixed = (D.precision == VVM_PREC_MIXED);
    c->spectral = (D.solver == VVM_SOLVER_SPECTRAL);
    // the learned solver's iterations are checked on the host (no graph)
    c->graphs_off = false;
    int prev = 0;
    cudaGetDevice(&prev);
    try {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
        c->stream = c->own;
        c->d.nx = D.NX + 2;
        c->d.nz = D.NZ + 2;
        c->d.pitch = round_up(c->d.nx, kPad);
        Consts& k = c->c;
        k.dx = D.dx;
        k.dz = D.dz;
        k.dt = D.dt;
        k.rdx = 1.0 / D.dx;                      // Declare.hpp:80-83
        k.r2dx = k.rdx / 2.0;
        k.rdz = 1.0 / D.dz;
        k.r2dz = k.rdz / 2.0;
        k.rdx2 = k.rdx * k.rdx;
        k.rdz2 = k.rdz * k.rdz;
        k.gravity = D.gravity;
        k.cp = D.cp;
        k.cv = D.cv;
        k.rd = D.rd;
        k.lv = D.lv;
        k.p0 = D.p0;
        if (c->mixed) alloc_fields<float>(c.get());
        else alloc_fields<double>(c.get());
        int nz = c->d.nz;
        double** profs[] = {&c->rhou, &c->rhow, &c->thvb, &c->thb, &c->qvb, &c->thb_init, &c->qvb0,
                            &c->pib, &c->pb, &c->lambda2, &c->z, &c->z_zeta, &c->vt_c1, &c->vt_fac,
                            &c->pc, &c->dtcgr_th, &c->dtcgr_zeta, &c->q1ls, &c->q2ls, &c->rwres,
                            &c->lv_r2dzc, &c->lv_r2dzw, &c->lv_rdzc, &c->lv_r2dzcc, &c->lv_kmax, &c->gsM_cz,
                            &c->gsM_rhod, &c->gsS_cz, &c->gsS_rhod, &c->lv_dzw};
        for (double** p : profs) *p = c->ar.alloc<double>(nz);
        for (int j = 0; j < 2; j++) {
            c->pref[j] = c->ar.alloc<double>(nz);
            c->pd0[j] = c->ar.alloc<double>(nz);
            c->ps0[j] = c->ar.alloc<double>(nz);
            c->pg0[j] = c->ar.alloc<double>(nz);
            c->pdn[j] = c->ar.alloc<double>(nz);
        }
        c->ubar = c->ar.alloc<double>(2);
        c->dubar = c->ar.alloc<double>(2);
        // block partials of k_padv and k_kessler (NegativeValueProcess sums)
        dim3 g = c->grid_interior(1), ga = c->padv_grid();
        c->npart = std::max(g.x * g.y, ga.x * ga.y);
        c->partial = c->ar.alloc<double>((size_t)c->npart * 6);
        CK(cudaFuncSetAttribute(k_padv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(PAdvShared<double>)));
        CK(cudaFuncSetAttribute(k_padv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(PAdvShared<float>)));
        c->nvp = c->ar.alloc<double>(6);
        c->staging = c->ar.alloc<double>((size_t)c->d.nx * c->d.nz * 2);
        c->wctl = c->ar.alloc<CGCtl>(1);
        c->d_exec = c->ar.alloc<long long>(1);
        c->d_err = c->ar.alloc<int>(1);
        for (auto& cs : c->cap) CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        for (auto& e : c->fork_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaStreamCreateWithFlags(&c->xfer, cudaStreamNonBlocking));
        for (auto& row : c->xev)
            for (auto& e : row) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    } catch (const CudaError& e) {
        cudaSetDevice(prev);
        return fail(nullptr, VVM_GPU_ECUDA, e.msg);
    }
    cudaSetDevice(prev);
    *out = c.release();
    return VVM_GPU_OK;
}

int vvm_gpu_destroy(vvm_gpu_ctx* ctx) {
    if (!ctx) return VVM_GPU_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    delete ctx;
    cudaSetDevice(prev);
    return VVM_GPU_OK;
}

int vvm_gpu_set_stream(vvm_gpu_ctx* ctx, void* stream) {
    if (!ctx) return VVM_GPU_EINVAL;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
    return VVM_GPU_OK;
}

int vvm_gpu_synchronize(vvm_gpu_ctx* ctx) {
    return guarded(ctx, [&] {
        CK(cudaStreamSynchronize(ctx->stream));
        return device_errors(ctx);
    });
}

int vvm_gpu_last_error(vvm_gpu_ctx* ctx, char* buf, size_t len) {
    const std::string& m = ctx ? ctx->err : g_create_error;
    if (buf && len) {
        std::snprintf(buf, len, "%s", m.c_str());
    }
    return VVM_GPU_OK;
}

int vvm_gpu_upload_state(vvm_gpu_ctx* ctx, const vvm_gpu_host_state* st) {
    if (!st) return fail(ctx, VVM_GPU_EINVAL, "upload: NULL state");
    return guarded(ctx, [&] {
        ctx->drop_graphs();   // kernel arguments depend on the uploaded flags
        int rc = upload_profiles(ctx, st);
        if (rc) return rc;
        if (ctx->poisson_ready) {   // a new state: no solver history
            CK(cudaMemsetAsync(ctx->W, 0, (size_t)ctx->pcg64->NK * ctx->pcg64->pitch * sizeof(double), ctx->stream));
            ctx->nsolves = 0;
        }
        rc = DISPATCH(ctx, upload_state_t)(ctx, st);
        if (rc) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->has_state = true;
        ctx->fut_is_now = false;
        return VVM_GPU_OK;
    });
}

int vvm_gpu_download_state(vvm_gpu_ctx* ctx, vvm_gpu_host_state* st) {
    if (!st) return fail(ctx, VVM_GPU_EINVAL, "download: NULL state");
    return guarded(ctx, [&] {
        if (int rc = need_state(ctx)) return rc;
        if (int rc = DISPATCH(ctx, download_state_t)(ctx, st)) return rc;
        return device_errors(ctx);
    });
}

int vvm_gpu_upload_prognostic(vvm_gpu_ctx* ctx, const vvm_gpu_host_state* st) {
    if (!st) return fail(ctx, VVM_GPU_EINVAL, "upload: NULL state");
    return guarded(ctx, [&] { return need_state(ctx) ? need_state(ctx) : DISPATCH(ctx, upload_prognostic_t)(ctx, st); });
}

int vvm_gpu_download_prognostic(vvm_gpu_ctx* ctx, vvm_gpu_host_state* st) {
    if (!st) return fail(ctx, VVM_GPU_EINVAL, "download: NULL state");
    return guarded(ctx, [&] {
        if (int rc = need_state(ctx)) return rc;
        if (int rc = DISPATCH(ctx, download_prognostic_t)(ctx, st)) return rc;
        return device_errors(ctx);
    });
}

int vvm_gpu_set_step(vvm_gpu_ctx* ctx, int step) {
    if (!ctx) return VVM_GPU_EINVAL;
    ctx->step = step;
    return VVM_GPU_OK;
}

int vvm_gpu_get_step(vvm_gpu_ctx* ctx, int* step) {
    if (!ctx || !step) return VVM_GPU_EINVAL;
    *step = ctx->step;
    return VVM_GPU_OK;
}

#define ROUTINE(name, ...)                                                    \
    int name(vvm_gpu_ctx* ctx) {                                              \
        return guarded(ctx, [&]() -> int {                                    \
            if (int rc = need_state(ctx)) return rc;                          \
            ctx->fut_is_now = false;                                          \
            __VA_ARGS__;                                                      \
        });                                                                   \
    }

ROUTINE(vvm_gpu_pzeta, { DISPATCH(ctx, launch_pzeta)(ctx); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_pth, {
    DISPATCH(ctx, launch_padv)(ctx, F_TH, 0, false, false);
    DISPATCH(ctx, launch_apply)(ctx, F_TH, 0, false, true);
    return VVM_GPU_OK;
})
ROUTINE(vvm_gpu_pqv, {
    DISPATCH(ctx, launch_padv)(ctx, F_QV, F_QV, false, false);
    DISPATCH(ctx, launch_apply)(ctx, F_QV, F_QV, false, true);
    return VVM_GPU_OK;
})
ROUTINE(vvm_gpu_pqc, {
    DISPATCH(ctx, launch_padv)(ctx, F_QC, F_QC, false, false);
    DISPATCH(ctx, launch_apply)(ctx, F_QC, F_QC, false, true);
    return VVM_GPU_OK;
})
ROUTINE(vvm_gpu_pqr, {
    DISPATCH(ctx, launch_padv)(ctx, F_QR, F_QR, true, true);
    DISPATCH(ctx, launch_apply)(ctx, F_QR, F_QR, false, true);
    return VVM_GPU_OK;
})
ROUTINE(vvm_gpu_add_forcing, { DISPATCH(ctx, launch_apply)(ctx, F_TH | F_QV, 0, true, false); return VVM_GPU_OK; })

int vvm_gpu_random_perturbation(vvm_gpu_ctx* ctx, int t, double min_range, double max_range,
                                double standard_deviation) {
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        return regen_forcing(ctx, t, min_range, max_range, standard_deviation);
    });
}

int vvm_gpu_random_perturbation_host(int NX, int NZ, double dz, int t, double min_range, double max_range,
                                     double standard_deviation, double* out) {
    return random_perturbation(NX, NZ, dz, t, min_range, max_range, standard_deviation, out);
}
ROUTINE(vvm_gpu_halo_all, { DISPATCH(ctx, launch_halo_all)(ctx); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_pubartop, { DISPATCH(ctx, launch_pubartop)(ctx); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_cal_w, { ctx->last_graph = false; return DISPATCH(ctx, launch_cal_w)(ctx, nullptr, nullptr); })
ROUTINE(vvm_gpu_cal_u, { DISPATCH(ctx, launch_cal_u)(ctx); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_kessler, { DISPATCH(ctx, launch_kessler)(ctx, false, false); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_update_mean, { DISPATCH(ctx, launch_update_mean)(ctx, false); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_turbulence, { DISPATCH(ctx, launch_turbulence)(ctx, false, nullptr); return VVM_GPU_OK; })
ROUTINE(vvm_gpu_nudge, {
    DISPATCH(ctx, launch_nudge)(ctx, true, ctx->desc.moisture_nudge_time != 0.0);
    return VVM_GPU_OK;
})
ROUTINE(vvm_gpu_calpsiuw, {
    if (int rc = need_uniform(ctx)) return rc;   // the reference's psi matrix assumes uniform levels
    return DISPATCH(ctx, launch_calpsiuw)(ctx);
})

int vvm_gpu_download_psi(vvm_gpu_ctx* ctx, double* psi) {
    return guarded(ctx, [&]() -> int {
        if (!psi) return fail(ctx, VVM_GPU_EINVAL, "download_psi: NULL argument");
        if (!ctx->psi) return fail(ctx, VVM_GPU_ESTATE, "download_psi: calpsiuw has not run");
        download_field<double>(ctx, ctx->psi, 1, 0, psi, false);
        return VVM_GPU_OK;
    });
}

ROUTINE(vvm_gpu_next_step, {
    DISPATCH(ctx, launch_update_mean)(ctx, true);
    ctx->cur = 1 - ctx->cur;
    ctx->fut_is_now = true;
    return VVM_GPU_OK;
})

int vvm_gpu_step(vvm_gpu_ctx* ctx, int nsteps) {
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        if (nsteps < 0) return fail(ctx, VVM_GPU_EINVAL, "step: nsteps < 0");
        if (ctx->desc.flags & VVM_FLAG_STREAMFUNCTION)
            if (int rc = need_uniform(ctx)) return rc;
        int worst = VVM_GPU_OK;
        for (int s = 0; s < nsteps; s++) {
            int rc = DISPATCH(ctx, step_once)(ctx);
            if (rc != VVM_GPU_OK) worst = rc;
        }
        if (worst == VVM_GPU_ENOCONV) fail(ctx, worst, "cal_w: Poisson solve did not reach its tolerance");
        return worst;
    });
}

int vvm_gpu_poisson_solve_device(vvm_gpu_ctx* ctx, const double* d_b, double* d_W, double tol, int* iters,
                                 double* relres) {
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        ensure_poisson(ctx);
        int NX = ctx->d.nx - 2, NK = ctx->d.nz - 3, pitch = ctx->pcg64->pitch;
        dim3 B(64, 4), G(cdiv(NX, 64), cdiv(NK, 4));
        LAUNCH(&ctx->stats, VVM_K_POISSON_RHS, ctx->stream, k_rhs_from_b<<<G, B, 0, ctx->stream>>>(NX, NK, ctx->rwres, d_b, ctx->Wf, pitch, ctx->wpartial));
        CKL();
        LAUNCH(&ctx->stats, VVM_K_CG, ctx->stream, k_cg_scalar<<<1, 1024, 0, ctx->stream>>>(ctx->wpartial, ctx->wnpart, ctx->pcg64->sc, CG_SET_BB));
        CKL();
        double bb = read_scalar(ctx, &ctx->pcg64->sc->bb);
        bool warm = ctx->desc.warm_start != 0;
        if (warm) {
            LAUNCH(&ctx->stats, VVM_K_POISSON_RHS, ctx->stream, k_unpack_solution<<<G, B, 0, ctx->stream>>>(NX, NK, d_W, ctx->W, pitch));
            CKL();
        }
        int rc = solve_w(ctx, bb, tol, warm);
        ctx->last_graph = false;
        LAUNCH(&ctx->stats, VVM_K_POISSON_RHS, ctx->stream, k_pack_solution<<<G, B, 0, ctx->stream>>>(NX, NK, ctx->W, pitch, d_W));
        CKL();
        CK(cudaStreamSynchronize(ctx->stream));
        if (iters) *iters = ctx->last_iters;
        if (relres) *relres = ctx->last_relres;
        if (rc == VVM_GPU_ENOCONV) fail(ctx, rc, "poisson_solve: tolerance not reached");
        return rc;
    });
}

int vvm_gpu_poisson_solve(vvm_gpu_ctx* ctx, const double* b, double* W, double tol, int* iters,
                          double* relres) {
    if (!b || !W) return fail(ctx, VVM_GPU_EINVAL, "poisson_solve: NULL argument");
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        size_t n = (size_t)(ctx->d.nx - 2) * (ctx->d.nz - 3);
        double* db = ctx->staging;
        double* dw = ctx->staging + n;
        CK(cudaMemcpyAsync(db, b, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(dw, W, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        int rc = vvm_gpu_poisson_solve_device(ctx, db, dw, tol, iters, relres);
        CK(cudaMemcpyAsync(W, dw, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return rc;
    });
}

int vvm_gpu_profile(vvm_gpu_ctx* ctx, int enable) {
    return guarded(ctx, [&]() -> int {
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->stats.reset();
        CK(cudaMemsetAsync(ctx->d_exec, 0, sizeof(long long), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->stats.on = (enable != 0);
        return VVM_GPU_OK;
    });
}

int vvm_gpu_profile_read(vvm_gpu_ctx* ctx, int kernel_class, double* ms, long long* launches) {
    if (kernel_class < 0 || kernel_class >= VVM_K_COUNT) return fail(ctx, VVM_GPU_EINVAL, "profile_read: bad class");
    return guarded(ctx, [&]() -> int {
        ctx->stats.resolve();
        if (ms) *ms = ctx->stats.ms[kernel_class];
        if (launches) *launches = ctx->stats.cnt[kernel_class];
        return VVM_GPU_OK;
    });
}

int vvm_gpu_launch_count(vvm_gpu_ctx* ctx, long long* launches) {
    if (!ctx || !launches) return VVM_GPU_EINVAL;
    return guarded(ctx, [&]() -> int {
        long long in_loops = 0;
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(&in_loops, ctx->d_exec, sizeof(long long), cudaMemcpyDeviceToHost));
        *launches = ctx->stats.launches + in_loops;
        return VVM_GPU_OK;
    });
}

int vvm_gpu_conv3x3_c32(const float* x, const float* w, float* y, int H, int W, int adjoint, int device) {
    if (!x || !w || !y || H < 1 || W < 1) return fail(nullptr, VVM_GPU_EINVAL, "conv3x3_c32: bad arguments");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int rc = VVM_GPU_OK;
    try {
        Arena ar;
        const size_t n = (size_t)H * W * kNetC;
        float* fx = ar.alloc<float>(n);
        float* fw = ar.alloc<float>(9 * kNetC * kNetC);
        int* err = ar.alloc<int>(1);
        __nv_bfloat16* bx = ar.alloc<__nv_bfloat16>(n);
        __nv_bfloat16* by = ar.alloc<__nv_bfloat16>(n);
        uint4* pw = ar.alloc<uint4>(9 * 4 * kNetC);
        CK(cudaMemcpy(fx, x, n * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(fw, w, 9 * kNetC * kNetC * sizeof(float), cudaMemcpyHostToDevice));
        k_nhwc_to_act<<<256, 256>>>(fx, bx, H, W);
        CKL();
        k_pack_conv32<<<cdiv(9 * 4 * kNetC, 128), 128>>>(fw, pw, adjoint ? 1 : 0);
        CKL();
        conv32(bx, by, pw, H, W, err, nullptr, nullptr);
        k_act_to_nhwc<<<256, 256>>>(by, fx, H, W);
        CKL();
        CK(cudaMemcpy(y, fx, n * sizeof(float), cudaMemcpyDeviceToHost));
        int h = 0;
        CK(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) rc = fail(nullptr, VVM_GPU_ECUDA, "conv3x3_c32: an MMA completion wait gave up");
    } catch (const CudaError& e) {
        rc = fail(nullptr, VVM_GPU_ECUDA, e.msg);
    }
    cudaSetDevice(prev);
    return rc;
}

int vvm_gpu_learned_shape(vvm_gpu_ctx* ctx, int* H0, int* W0, int* nparams) {
    if (!ctx) return VVM_GPU_EINVAL;
    const int NX = ctx->d.nx - 2, NK = ctx->d.nz - 3;
    if (!LearnedNet::supports(NX, NK)) return fail(ctx, VVM_GPU_EINVAL, "learned: NX must be a multiple of 8");
    if (H0) *H0 = round_up(NK, 8);
    if (W0) *W0 = NX;
    if (nparams) *nparams = LearnedNet::kParams;
    return VVM_GPU_OK;
}

int vvm_gpu_learned_weights(vvm_gpu_ctx* ctx, float* get, const float* set, int n) {
    if (!ctx) return VVM_GPU_EINVAL;
    if (n != LearnedNet::kParams) return fail(ctx, VVM_GPU_EINVAL, "learned_weights: wrong parameter count");
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        ensure_learned(ctx);
        CK(cudaStreamSynchronize(ctx->stream));
        if (set) ctx->net->set_weights(set);
        if (get) CK(cudaMemcpy(get, ctx->net->w, n * sizeof(float), cudaMemcpyDeviceToHost));
        return VVM_GPU_OK;
    });
}

// Network input x and target t as host [H0][W0] FP32; out: z = net(x) (if
// z), the gradient of L = ||z - t||^2 / ||t||^2 with respect to the weights
// (if grad and t) and L.
int vvm_gpu_learned_eval(vvm_gpu_ctx* ctx, const float* x, const float* t, float* z, float* grad, double* loss) {
    if (!ctx || !x) return VVM_GPU_EINVAL;
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        ensure_learned(ctx);
        LearnedNet& N = *ctx->net;
        cudaStream_t st = ctx->stream;
        const size_t n0 = (size_t)N.H[0] * N.W[0];
        CK(cudaMemcpyAsync(N.x0, x, n0 * sizeof(float), cudaMemcpyHostToDevice, st));
        N.forward(st);
        if (z) CK(cudaMemcpyAsync(z, N.z0, n0 * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (t) {
            Arena tmp;
            float* td = tmp.alloc<float>(n0);
            CK(cudaMemcpyAsync(td, t, n0 * sizeof(float), cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(N.g, 0, LearnedNet::kParams * sizeof(float), st));
            N.loss(td, 1.f, st);
            N.backward(st);
            if (grad) CK(cudaMemcpyAsync(grad, N.g, LearnedNet::kParams * sizeof(float), cudaMemcpyDeviceToHost, st));
            double lt[2];
            CK(cudaMemcpyAsync(lt, N.lt, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (loss) *loss = lt[0];
        }
        CK(cudaStreamSynchronize(st));
        int h = 0;
        CK(cudaMemcpy(&h, N.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) return fail(ctx, VVM_GPU_ECUDA, "learned: an MMA completion wait gave up");
        return VVM_GPU_OK;
    });
}

// Training of the learned preconditioner. Pair sources: the caller's nb
// right-hand sides b_host (nb x NX*(NZ-1), reference ordering) followed by as
// many white-noise ones when given; otherwise half the model's own next steps
// and half white noise, or all white noise on stretched levels (no model
// steps there). Every pair is solved by the plain multigrid PCG; the model
// state is put back afterwards. The noise stands for the rough residuals
// flexible CG meets.
static int learned_train_impl(vvm_gpu_ctx* ctx, int npairs, int steps, int batch, double lr, int seed,
                       const double* b_host, double* loss_first, double* loss_last) {
    if (!ctx) return VVM_GPU_EINVAL;
    if (npairs < 1 || steps < 0 || batch < 1 || !(lr > 0))
        return fail(ctx, VVM_GPU_EINVAL, "learned_train: bad arguments");
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        ensure_learned(ctx);
        vvm_gpu_ctx* c = ctx;
        LearnedNet& N = *c->net;
        PCG<double>& P = *c->pcg64;
        cudaStream_t st = c->stream;
        const size_t n0 = (size_t)N.H[0] * N.W[0];
        Arena tmp;
        float* px = tmp.alloc<float>(n0 * npairs);
        float* pt = tmp.alloc<float>(n0 * npairs);
        // pairs (f, W) of the model's own steps, solved by the plain solver;
        // the state is put back afterwards
        Snapshot snap;
        snap.take(c);
        c->learned_collect = true;
        VecArgs<double> v = P.vargs();
        dim3 B = P.block(), G = P.grid(), g0(cdiv(P.NX, 64), cdiv(N.H[0], 4));
        int rc = VVM_GPU_OK;
        const int nmodel = b_host ? 0 : (npairs + 1) / 2;   // the rest: white noise
        const int nb = b_host ? npairs / 2 : 0;
        const size_t nun = (size_t)P.NX * P.NK;
        for (int i = 0; i < npairs && rc == VVM_GPU_OK; i++) {
            if (i < nb) {   // the caller's right-hand side, solved by the plain solver
                CK(cudaMemcpyAsync(c->staging, b_host + nun * i, nun * sizeof(double), cudaMemcpyHostToDevice, st));
                LAUNCH(&c->stats, VVM_K_POISSON_RHS, st, k_rhs_from_b<<<G, B, 0, st>>>(P.NX, P.NK, c->rwres, c->staging, c->Wf, P.pitch, c->wpartial));
                CKL();
                double rel = 0;
                P.solve(c->Wf, c->W, false, -1.0, 1e-10, 400, st, &rel);
            } else if (i < nmodel) {
                rc = c->mixed ? step_once<float>(c) : step_once<double>(c);
            } else {   // the residuals flexible CG meets are rough: noise, solved by the plain solver
                LAUNCH(&c->stats, VVM_K_LEARNED, st, k_white_noise<<<G, B, 0, st>>>(c->Wf, P.NX, P.NK, P.pitch, (unsigned)(seed * 7919 + i)));
                CKL();
                double rel = 0;
                P.solve(c->Wf, c->W, false, -1.0, 1e-10, 400, st, &rel);
            }
            // what the line solve leaves: input r1 = f - S L f, target
            // e1 = W - L f = S^{-1} r1, both over ||r1||
            P.mg.sweep(0, c->Wf, nullptr, nullptr, 0, 0, c->z64, 1.0, st);
            LAUNCH(&c->stats, VVM_K_CG, st, k_cg_residual<double><<<G, B, 0, st>>>(v, c->Wf, c->z64, c->r164, P.partial));
            CKL();
            LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_sdot<<<G, B, 0, st>>>(v, c->r164, N.dsc, P.partial));
            CKL();
            LAUNCH(&c->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, CG_SET_NRM));
            CKL();
            LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_in<<<g0, B, 0, st>>>(c->r164, nullptr, P.NX, P.NK, P.pitch, px + n0 * i, N.H[0], &P.sc->nrm, N.dsc));
            CKL();
            LAUNCH(&c->stats, VVM_K_LEARNED, st, k_net_in<<<g0, B, 0, st>>>(c->W, c->z64, P.NX, P.NK, P.pitch, pt + n0 * i, N.H[0], &P.sc->nrm, N.dsc_inv));
            CKL();
        }
        c->learned_collect = false;
        CK(cudaStreamSynchronize(st));
        snap.restore(c);
        c->drop_graphs();
        if (rc != VVM_GPU_OK) return rc;
        // Adam over random mini-batches of the pairs
        uint64_t s64 = 0x853C49E6748FEA9Bull ^ (uint64_t)(unsigned)seed;
        auto pick = [&]() {
            s64 ^= s64 << 13;
            s64 ^= s64 >> 7;
            s64 ^= s64 << 17;
            return (int)(s64 % (uint64_t)npairs);
        };
        double* hl = nullptr;
        CK(cudaMallocHost(&hl, 2 * sizeof(double)));
        const int probe = std::min(steps, 10);
        double first = 0, last = 0;
        for (int s = 0; s < steps; s++) {
            CK(cudaMemsetAsync(N.g, 0, LearnedNet::kParams * sizeof(float), st));
            double lsum = 0;
            const bool watch = (s < probe) || (s >= steps - probe);
            for (int b = 0; b < batch; b++) {
                const int i = pick();
                CK(cudaMemcpyAsync(N.x0, px + n0 * i, n0 * sizeof(float), cudaMemcpyDeviceToDevice, st));
                N.forward(st);
                N.loss(pt + n0 * i, 1.f / batch, st);
                N.backward(st);
                if (watch) {
                    CK(cudaMemcpyAsync(hl, N.lt, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    lsum += hl[0];
                }
            }
            N.adam((float)lr, st);
            if (s < probe) first += lsum / batch / probe;
            if (s >= steps - probe) last += lsum / batch / probe;
        }
        CK(cudaStreamSynchronize(st));
        cudaFreeHost(hl);
        if (loss_first) *loss_first = first;
        if (loss_last) *loss_last = last;
        int h = 0;
        CK(cudaMemcpy(&h, N.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) return fail(ctx, VVM_GPU_ECUDA, "learned: an MMA completion wait gave up");
        return VVM_GPU_OK;
    });
}


int vvm_gpu_learned_train(vvm_gpu_ctx* ctx, int npairs, int steps, int batch, double lr, int seed,
                          double* loss_first, double* loss_last) {
    return learned_train_impl(ctx, npairs, steps, batch, lr, seed, nullptr, loss_first, loss_last);
}

int vvm_gpu_learned_train_rhs(vvm_gpu_ctx* ctx, const double* b, int npairs, int steps, int batch, double lr,
                              int seed, double* loss_first, double* loss_last) {
    if (!b) return fail(ctx, VVM_GPU_EINVAL, "learned_train_rhs: b is NULL");
    if (npairs < 1) return fail(ctx, VVM_GPU_EINVAL, "learned_train_rhs: npairs < 1");
    return learned_train_impl(ctx, 2 * npairs, steps, batch, lr, seed, b, loss_first, loss_last);
}

int vvm_gpu_learned_time(vvm_gpu_ctx* ctx, int reps, double* ms_forward, double* ms_convs) {
    if (!ctx || reps < 1) return VVM_GPU_EINVAL;
    return guarded(ctx, [&]() -> int {
        if (int rc = need_state(ctx)) return rc;
        ensure_learned(ctx);
        LearnedNet& N = *ctx->net;
        PCG<double>& P = *ctx->pcg64;
        cudaStream_t st = ctx->stream;
        dim3 B = P.block(), G = P.grid(), g0(cdiv(P.NX, 64), cdiv(N.H[0], 4));
        // input: white noise over its norm, in the network's layout (work arrays only)
        LAUNCH(&ctx->stats, VVM_K_LEARNED, st, k_white_noise<<<G, B, 0, st>>>(ctx->r164, P.NX, P.NK, P.pitch, 12345u));
        CKL();
        LAUNCH(&ctx->stats, VVM_K_LEARNED, st, k_net_sdot<<<G, B, 0, st>>>(P.vargs(), ctx->r164, N.dsc, P.partial));
        CKL();
        LAUNCH(&ctx->stats, VVM_K_CG, st, k_cg_scalar<<<1, 1024, 0, st>>>(P.partial, P.npart, P.sc, CG_SET_NRM));
        CKL();
        LAUNCH(&ctx->stats, VVM_K_LEARNED, st, k_net_in<<<g0, B, 0, st>>>(ctx->r164, nullptr, P.NX, P.NK, P.pitch, N.x0, N.H[0], &P.sc->nrm, N.dsc));
        CKL();
        N.forward(st);   // warm-up, and valid activations for convs_only
        cudaEvent_t e[4];
        for (auto& x : e) CK(cudaEventCreate(&x));
        CK(cudaEventRecord(e[0], st));
        for (int r = 0; r < reps; r++) N.forward(st);
        CK(cudaEventRecord(e[1], st));
        CK(cudaEventRecord(e[2], st));
        for (int r = 0; r < reps; r++) N.convs_only(st);
        CK(cudaEventRecord(e[3], st));
        CK(cudaEventSynchronize(e[3]));
        float a = 0, b = 0;
        CK(cudaEventElapsedTime(&a, e[0], e[1]));
        CK(cudaEventElapsedTime(&b, e[2], e[3]));
        for (auto& x : e) cudaEventDestroy(x);
        if (ms_forward) *ms_forward = a / reps;
        if (ms_convs) *ms_convs = b / reps;
        int h = 0;
        CK(cudaMemcpy(&h, N.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) return fail(ctx, VVM_GPU_ECUDA, "learned: an MMA completion wait gave up");
        return VVM_GPU_OK;
    });
}

int vvm_gpu_learned_config(vvm_gpu_ctx* ctx, int mode, int cap) {
    if (!ctx) return VVM_GPU_EINVAL;
    if (mode < 0 || mode > 2 || cap < 1) return fail(ctx, VVM_GPU_EINVAL, "learned_config: bad arguments");
    return guarded(ctx, [&]() -> int {
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->learned_mode = mode;
        ctx->learned_cap = cap;
        ctx->drop_graphs();   // mode and cap are recorded into the graphs
        return VVM_GPU_OK;
    });
}

int vvm_gpu_learned_last(vvm_gpu_ctx* ctx, int* fcg_iters, int* fell_back) {
    if (!ctx) return VVM_GPU_EINVAL;
    return guarded(ctx, [&]() -> int {
        sync_graph_solve(ctx);
        if (fcg_iters) *fcg_iters = ctx->learned_iters;
        if (fell_back) *fell_back = ctx->learned_fallback;
        return VVM_GPU_OK;
    });
}

int vvm_gpu_set_tuning(vvm_gpu_ctx* ctx, int gs_tile_rows, int fft_threads) {
    if (!ctx) return VVM_GPU_EINVAL;
    if (!gs_schedule_ok(gs_tile_rows) || fft_threads < 0 || fft_threads > 1024)
        return fail(ctx, VVM_GPU_EINVAL, "set_tuning: knob out of range");
    return guarded(ctx, [&]() -> int {
        CK(cudaStreamSynchronize(ctx->stream));
        if (gs_tile_rows == kGSSchedCluster) ensure_gs_cluster(ctx);
        ctx->tune_gs_tr = gs_tile_rows;
        ctx->tune_fft = fft_threads;
        apply_tuning(ctx);
        ctx->drop_graphs();
        return VVM_GPU_OK;
    });
}

int vvm_gpu_get_tuning(vvm_gpu_ctx* ctx, int* gs_tile_rows_out, int* fft_threads) {
    if (!ctx) return VVM_GPU_EINVAL;
    if (gs_tile_rows_out) *gs_tile_rows_out = gs_tile_rows(ctx);   // kGSSchedCluster: the cluster schedule
    if (fft_threads) {
        *fft_threads = 0;
        if (ctx->spectral) {
            const int half = std::max(32, (ctx->d.nx - 2) / 2);
            *fft_threads = ctx->tune_fft > 0 ? std::max(32, std::min(ctx->tune_fft, std::min(half, 1024)))
                                             : std::min(half, 512);
        }
    }
    return VVM_GPU_OK;
}

int vvm_gpu_batch_create(const vvm_gpu_desc* descs, int ncases, int device, vvm_gpu_batch** out) {
    if (!descs || !out || ncases <= 0) return fail(nullptr, VVM_GPU_EINVAL, "batch_create: bad arguments");
    *out = nullptr;
    std::unique_ptr<vvm_gpu_batch> b(new vvm_gpu_batch());
    b->device = device;
    for (int i = 0; i < ncases; i++) {
        if (descs[i].flags & VVM_FLAG_STREAMFUNCTION)   // its solve reads its residual on the host
            return fail(nullptr, VVM_GPU_EINVAL, "batch_create: case " + std::to_string(i) +
                                                     ": the streamfunction formulation runs single contexts only");
        vvm_gpu_ctx* c = nullptr;
        int rc = vvm_gpu_create(&descs[i], device, &c);
        if (rc != VVM_GPU_OK) {
            g_create_error = "batch_create: case " + std::to_string(i) + ": " + g_create_error;
            return rc;
        }
        b->cases.push_back(c);
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&b->t0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->t1);
    b->joins.assign(ncases, nullptr);
    for (int i = 0; i < ncases && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(nullptr, VVM_GPU_ECUDA, std::string("batch_create: ") + cudaGetErrorString(e));
    *out = b.release();
    return VVM_GPU_OK;
}

int vvm_gpu_batch_destroy(vvm_gpu_batch* b) {
    if (!b) return VVM_GPU_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    cudaSetDevice(prev);
    return VVM_GPU_OK;
}

int vvm_gpu_batch_case(vvm_gpu_batch* b, int i, vvm_gpu_ctx** ctx) {
    if (!b || !ctx) return VVM_GPU_EINVAL;
    if (i < 0 || i >= (int)b->cases.size()) return batch_fail(b, VVM_GPU_EINVAL, "batch_case: index out of range");
    *ctx = b->cases[i];
    return VVM_GPU_OK;
}

int vvm_gpu_batch_step(vvm_gpu_batch* b, int nsteps) {
    if (!b) return VVM_GPU_EINVAL;
    if (nsteps < 0) return batch_fail(b, VVM_GPU_EINVAL, "batch_step: nsteps < 0");
    return batch_guarded(b, [&]() -> int {
        for (auto* c : b->cases)
            if (!c->has_state) return batch_fail(b, VVM_GPU_ESTATE, "batch_step: a case has no state uploaded");
        for (auto* c : b->cases)
            if (c->stretched) return batch_fail(b, VVM_GPU_EINVAL, "batch_step: a case has stretched levels");
        int rc = batch_step(b, nsteps);
        if (rc == VVM_GPU_ENOCONV) batch_fail(b, rc, "batch_step: a Poisson solve did not reach its tolerance");
        return rc;
    });
}

int vvm_gpu_batch_synchronize(vvm_gpu_batch* b) {
    return batch_guarded(b, [&]() -> int {
        CK(cudaStreamSynchronize(b->stream));
        for (size_t i = 0; i < b->cases.size(); i++) {
            vvm_gpu_ctx* c = b->cases[i];
            CK(cudaStreamSynchronize(c->stream));
            if (int rc = device_errors(c)) return batch_fail(b, rc, "case " + std::to_string(i) + ": " + c->err);
        }
        return VVM_GPU_OK;
    });
}

int vvm_gpu_batch_autotune(vvm_gpu_batch* b, int reps, int* ngroups) {
    if (!b) return VVM_GPU_EINVAL;
    return batch_guarded(b, [&]() -> int {
        for (auto* c : b->cases)
            if (!c->has_state) return batch_fail(b, VVM_GPU_ESTATE, "batch_autotune: a case has no state uploaded");
        return batch_autotune(b, reps > 0 ? reps : 3, ngroups);
    });
}

int vvm_gpu_batch_stream(vvm_gpu_batch* b, void** stream) {
    if (!b || !stream) return VVM_GPU_EINVAL;
    *stream = b->stream;
    return VVM_GPU_OK;
}

int vvm_gpu_batch_grouping(vvm_gpu_batch* b, int max_cases, int* groups) {
    return batch_guarded(b, [&]() -> int {
        if (max_cases >= 0 && max_cases != b->group_max) {
            CK(cudaStreamSynchronize(b->stream));
            b->group_max = max_cases;
            for (auto* c : b->cases) c->tune_group = 0;
            b->drop_graphs();
        }
        if (groups) *groups = b->last_groups;
        return VVM_GPU_OK;
    });
}

int vvm_gpu_batch_last_error(vvm_gpu_batch* b, char* buf, size_t len) {
    if (!b || !buf || len == 0) return VVM_GPU_EINVAL;
    std::snprintf(buf, len, "%s", b->err.c_str());
    return VVM_GPU_OK;
}

int vvm_gpu_last_solve(vvm_gpu_ctx* ctx, int* iters, double* relres) {
    if (!ctx) return VVM_GPU_EINVAL;
    return guarded(ctx, [&]() -> int {
        sync_graph_solve(ctx);
        if (iters) *iters = ctx->last_iters;
        if (relres) *relres = ctx->last_relres;
        return VVM_GPU_OK;
    });
}

}  // extern "C"
