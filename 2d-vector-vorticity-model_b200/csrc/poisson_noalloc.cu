// vvm_gpu_poisson_solve_noalloc: the cal_w elliptic solve without a context
// and without allocating device memory. It has no counterpart in the
// reference (whose solves allocate through Eigen or AMGX on every setup).
//
// The system is the one of vvm_gpu_poisson_solve_device: A W = b with the
// matrix of PoissonSolver::InitPoissonMatrix (src/PoissonSolver.cpp:760-796),
// unknown (k-2)*NX + (i-1), solved as S W = -b/rhow_k with
//   (S W) = (2 cx + ru + rd) W - cx (W[i-1] + W[i+1]) - ru W[k+1] - rd W[k-1],
//   cx = 1/rhow_k, ru = 1/rhou_k, rd = 1/rhou_{k-1},
// periodic in i and zero at k = 1 and k = nz-1. Method: FP64 conjugate
// gradients preconditioned by exact z-line solves (one Thomas pass per
// column; the z operator is the same in every column, so its factors are
// per-row), stopped on ||b - A W||_2 / ||b||_2 = ||rhow r||_2 / ||b||_2.
//
// Working memory is one file-scope __device__ array of fixed size. Its
// address is taken once per device with cudaGetSymbolAddress, on the first
// call made with that device current. Every word of it is written before it
// is read within one call, so nothing in it has to start at zero, and calls
// that overlap on one device share it and race.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vvm_gpu.h"
#include "vvm_common.cuh"

// Message of the last failed context-free call (vvm_gpu_last_error(NULL, ...)).
void vvm_set_context_free_error(const std::string& msg);

namespace {

constexpr int kMaxRows = VVM_NOALLOC_MAX_ROWS;          // NZ - 1
constexpr int kMaxUnknowns = VVM_NOALLOC_MAX_UNKNOWNS;  // NX * (NZ - 1)
constexpr int kMaxParts = 1024;                         // reduction partials
constexpr int kMaxDevices = 64;

// Scratch layout, in doubles: r, z, p, q (kMaxUnknowns each); per-row
// coefficients cx, ru, rd, rhow, c' and 1/pivot (kMaxRows each); partial
// sums; scalars.
constexpr size_t kOffZ = (size_t)kMaxUnknowns;
constexpr size_t kOffP = 2 * (size_t)kMaxUnknowns;
constexpr size_t kOffQ = 3 * (size_t)kMaxUnknowns;
constexpr size_t kOffRow = 4 * (size_t)kMaxUnknowns;
constexpr size_t kOffPart = kOffRow + 6 * (size_t)kMaxRows;
constexpr size_t kOffScal = kOffPart + kMaxParts;
constexpr size_t kScratchWords = kOffScal + 8;
static_assert(kScratchWords * sizeof(double) == VVM_NOALLOC_SCRATCH_BYTES, "scratch size");

__device__ __align__(256) double g_scratch[kScratchWords];

enum { S_BB = 0, S_RR, S_RZ, S_BETA, S_ALPHA };
enum { F_BB = 0, F_RZ_FIRST, F_RZ, F_PQ, F_RR };

struct Rows {   // per-row coefficients in scratch, kk = k - 2
    const double *cx, *ru, *rd, *rw, *cp, *inv;
};

// W = 0, r = -b / rhow_k; partial sums of b^2.
__global__ void k_na_init(int NX, int n, Rows R, const double* b, double* W, double* r, double* part) {
    __shared__ double sh[32];
    double v[1] = {0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double be = b[e];
        W[e] = 0.0;
        r[e] = -be / R.rw[e / NX];
        v[0] += be * be;
    }
    vvm::block_sum<1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// Sums the partials in a fixed order and updates the CG scalars.
__global__ void k_na_final(const double* part, int np, double* s, int mode) {
    __shared__ double sh[32];
    double v[1] = {0.0};
    for (int j = threadIdx.x; j < np; j += blockDim.x) v[0] += part[j];
    vvm::block_sum<1>(v, sh);
    if (threadIdx.x != 0) return;
    const double t = v[0];
    switch (mode) {
        case F_BB: s[S_BB] = t; s[S_RR] = t; break;       // rhow r = -b at W = 0
        case F_RZ_FIRST: s[S_RZ] = t; s[S_BETA] = 0.0; break;
        case F_RZ: s[S_BETA] = t / s[S_RZ]; s[S_RZ] = t; break;
        case F_PQ: s[S_ALPHA] = s[S_RZ] / t; break;
        default: s[S_RR] = t; break;
    }
}

// z = Dline^{-1} r (one thread per column, Thomas down and up the column);
// partial sums of r . z.
__global__ void k_na_precond(int NX, int NK, Rows R, const double* r, double* z, double* part) {
    __shared__ double sh[32];
    double v[1] = {0.0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < NX) {
        double y = 0.0;
        for (int kk = 0; kk < NK; kk++) {
            y = (r[(size_t)kk * NX + i] + R.rd[kk] * y) * R.inv[kk];
            z[(size_t)kk * NX + i] = y;
        }
        double next = 0.0;
        for (int kk = NK - 1; kk >= 0; kk--) {
            const size_t e = (size_t)kk * NX + i;
            next = z[e] - R.cp[kk] * next;
            z[e] = next;
            v[0] += r[e] * next;
        }
    }
    vvm::block_sum<1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// p = z + beta p (p = z on the first iteration: p's old contents are not read).
__global__ void k_na_dir(int n, const double* s, const double* z, double* p, int first) {
    const double beta = s[S_BETA];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        p[e] = first ? z[e] : z[e] + beta * p[e];
}

// q = S p; partial sums of p . q.
__global__ void k_na_spmv(int NX, int NK, Rows R, const double* p, double* q, double* part) {
    __shared__ double sh[32];
    double v[1] = {0.0};
    const int n = NX * NK;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int kk = e / NX, i = e - kk * NX;
        const int il = (i == 0) ? NX - 1 : i - 1, ir = (i == NX - 1) ? 0 : i + 1;
        const double c = R.cx[kk], ru = R.ru[kk], rd = R.rd[kk];
        const size_t row = (size_t)kk * NX;
        const double pc = p[e];
        double y = (2.0 * c + ru + rd) * pc - c * (p[row + il] + p[row + ir]);
        if (kk + 1 < NK) y -= ru * p[e + NX];
        if (kk > 0) y -= rd * p[e - NX];
        q[e] = y;
        v[0] += pc * y;
    }
    vvm::block_sum<1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// W += alpha p, r -= alpha q; partial sums of (rhow r)^2.
__global__ void k_na_update(int NX, int n, Rows R, const double* s, double* W, double* r, const double* p,
                            const double* q, double* part) {
    __shared__ double sh[32];
    double v[1] = {0.0};
    const double alpha = s[S_ALPHA];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        W[e] += alpha * p[e];
        const double re = r[e] - alpha * q[e];
        r[e] = re;
        const double t = R.rw[e / NX] * re;
        v[0] += t * t;
    }
    vvm::block_sum<1>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

struct Fail {
    int code;
    std::string msg;
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Fail{VVM_GPU_ECUDA, std::string("poisson_solve_noalloc: ") + what + ": " +
                                                        cudaGetErrorString(e)};
}

std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device. The first call
// on a device looks it up (which may load the module onto the device); later
// calls look it up again unless `st` is capturing, so a caller that reset the
// device (cudaDeviceReset, which reloads the module and may move the array)
// gets the new address. Under capture the address from the last call outside
// capture is used.
double* scratch_on(int dev, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(g_mu);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ck(cudaStreamIsCapturing(st, &cap), "cudaStreamIsCapturing");
    if (!g_addr[dev] || cap == cudaStreamCaptureStatusNone) {
        if (cap != cudaStreamCaptureStatusNone)
            throw Fail{VVM_GPU_ESTATE, "poisson_solve_noalloc: the first call on a device may not be captured"};
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress");
        g_addr[dev] = static_cast<double*>(p);
    }
    return g_addr[dev];
}

void check_device_buffer(const void* ptr, int dev, const char* name) {
    cudaPointerAttributes a{};
    ck(cudaPointerGetAttributes(&a, ptr), "cudaPointerGetAttributes");
    const bool ok = (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
    if (!ok)
        throw Fail{VVM_GPU_EINVAL, std::string("poisson_solve_noalloc: ") + name +
                                       " is not device memory of the current device"};
}

int solve(int NX, int NZ, const double* rhou, const double* rhow, const double* d_b, double* d_W, double tol,
          int maxit, void* stream, int* iters, double* relres) {
    if (!rhou || !rhow || !d_b || !d_W) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: NULL argument"};
    if (NX < 3 || NZ < 4) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: NX must be >= 3 and NZ >= 4"};
    const int NK = NZ - 1;
    const long long n = (long long)NX * NK;
    if (NK > kMaxRows || n > kMaxUnknowns)
        throw Fail{VVM_GPU_EINVAL,
                   "poisson_solve_noalloc: NX*(NZ-1) = " + std::to_string(n) + " unknowns in " +
                       std::to_string(NK) + " rows exceeds its static scratch (at most " +
                       std::to_string(kMaxUnknowns) + " unknowns and " + std::to_string(kMaxRows) +
                       " rows); use vvm_gpu_poisson_solve_device"};
    if (!(tol > 0.0)) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: tol must be > 0"};
    if (maxit <= 0) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: maxit must be > 0"};
    // per-row coefficients and the column Thomas factors (host, FP64)
    std::vector<double> row(6 * (size_t)kMaxRows, 0.0);
    double* cx = row.data();
    double* ru = cx + kMaxRows;
    double* rd = ru + kMaxRows;
    double* rw = rd + kMaxRows;
    double* cp = rw + kMaxRows;
    double* inv = cp + kMaxRows;
    double cprev = 0.0;
    for (int kk = 0; kk < NK; kk++) {
        const int k = kk + 2;
        if (!(rhow[k] > 0.0) || !(rhou[k] > 0.0) || !(rhou[k - 1] > 0.0))
            throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: rhou and rhow must be positive"};
        cx[kk] = 1.0 / rhow[k];
        ru[kk] = 1.0 / rhou[k];   // the diagonal keeps ru and rd at the lid and the floor
        rd[kk] = 1.0 / rhou[k - 1];
        rw[kk] = rhow[k];
        const double lower = (kk > 0) ? rd[kk] : 0.0;                // coupling to kk-1 is -rd
        const double piv = 2.0 * cx[kk] + ru[kk] + rd[kk] - lower * cprev;
        inv[kk] = 1.0 / piv;
        cp[kk] = (kk + 1 < NK) ? -ru[kk] / piv : 0.0;              // coupling to kk+1 is -ru
        cprev = -cp[kk];
    }
    // The elimination above writes y_k = (r_k + rd_k y_{k-1}) / piv_k and
    // z_k = y_k - cp_k z_{k+1}; rd of row 0 multiplies y_{-1} = 0.
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: device index too large"};
    check_device_buffer(d_b, dev, "b");
    check_device_buffer(d_W, dev, "W");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* S = scratch_on(dev, st);
    ck(cudaMemcpyAsync(S + kOffRow, row.data(), row.size() * sizeof(double), cudaMemcpyHostToDevice, st),
       "copy of the row coefficients");
    Rows R{S + kOffRow, S + kOffRow + kMaxRows, S + kOffRow + 2 * kMaxRows, S + kOffRow + 3 * kMaxRows,
           S + kOffRow + 4 * kMaxRows, S + kOffRow + 5 * kMaxRows};
    double *r = S, *z = S + kOffZ, *p = S + kOffP, *q = S + kOffQ, *part = S + kOffPart, *sc = S + kOffScal;
    const int T = 256;
    const int G = (int)std::min<long long>((n + T - 1) / T, kMaxParts);
    const int Gc = (NX + 127) / 128;   // <= kMaxParts since NX <= kMaxUnknowns / 3
    auto read = [&](int idx) {
        double h = 0.0;
        ck(cudaMemcpyAsync(&h, sc + idx, sizeof(double), cudaMemcpyDeviceToHost, st), "read of a CG scalar");
        ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        return h;
    };
    auto launched = [&](const char* what) { ck(cudaGetLastError(), what); };

    k_na_init<<<G, T, 0, st>>>(NX, (int)n, R, d_b, d_W, r, part);
    launched("k_na_init");
    k_na_final<<<1, 1024, 0, st>>>(part, G, sc, F_BB);
    launched("k_na_final");
    const double bb = read(S_BB);
    if (!std::isfinite(bb)) throw Fail{VVM_GPU_EINVAL, "poisson_solve_noalloc: b is not finite"};
    if (bb == 0.0) {   // W = 0 is exact
        if (iters) *iters = 0;
        if (relres) *relres = 0.0;
        return VVM_GPU_OK;
    }
    const double stop2 = tol * tol * bb;
    double rr = bb;
    int it = 0;
    while (it < maxit && rr > stop2) {
        it++;
        k_na_precond<<<Gc, 128, 0, st>>>(NX, NK, R, r, z, part);
        launched("k_na_precond");
        k_na_final<<<1, 1024, 0, st>>>(part, Gc, sc, it == 1 ? F_RZ_FIRST : F_RZ);
        launched("k_na_final");
        k_na_dir<<<G, T, 0, st>>>((int)n, sc, z, p, it == 1);
        launched("k_na_dir");
        k_na_spmv<<<G, T, 0, st>>>(NX, NK, R, p, q, part);
        launched("k_na_spmv");
        k_na_final<<<1, 1024, 0, st>>>(part, G, sc, F_PQ);
        launched("k_na_final");
        k_na_update<<<G, T, 0, st>>>(NX, (int)n, R, sc, d_W, r, p, q, part);
        launched("k_na_update");
        k_na_final<<<1, 1024, 0, st>>>(part, G, sc, F_RR);
        launched("k_na_final");
        rr = read(S_RR);
        if (!std::isfinite(rr)) break;
    }
    if (iters) *iters = it;
    if (relres) *relres = std::sqrt(rr / bb);
    if (!(rr <= stop2))
        throw Fail{VVM_GPU_ENOCONV, "poisson_solve_noalloc: tolerance not reached in " + std::to_string(it) +
                                        " iterations (relative residual " + std::to_string(std::sqrt(rr / bb)) +
                                        ")"};
    return VVM_GPU_OK;
}

}  // namespace

extern "C" int vvm_gpu_poisson_solve_noalloc(int NX, int NZ, const double* rhou, const double* rhow,
                                             const double* d_b, double* d_W, double tol, int maxit, void* stream,
                                             int* iters, double* relres) {
    try {
        return solve(NX, NZ, rhou, rhow, d_b, d_W, tol, maxit, stream, iters, relres);
    } catch (const Fail& f) {
        vvm_set_context_free_error(f.msg);
        return f.code;
    }
}
