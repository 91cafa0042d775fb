// Kernels of the cal_w elliptic solve (PoissonSolver::cal_w,
// src/PoissonSolver.cpp:439-479 with the matrix of :760-796).
//
// The reference assembles A, row (k, i) for k = 2..nz-2, i = 1..nx-2:
//   W[i-1] + W[i+1] - (2 + rhow_k/rhou_k + rhow_k/rhou_{k-1}) W
//     + (rhow_k/rhou_k) W[k+1] + (rhow_k/rhou_{k-1}) W[k-1]
// periodic in i, W = 0 at k = 1 and k = nz-1. A = diag(rhow_k) L with L
// symmetric negative definite, so A W = b is solved as S W = f with
//   S = -L,  f = -b / rhow_k,
// whose rows are
//   (S W) = (2 cx + ru + rd) W - cx (W[i-1] + W[i+1]) - ru W[k+1] - rd W[k-1],
//   cx = 1/rhow_k, ru = 1/rhou_k, rd = 1/rhou_{k-1}.
// The residual the reference's tolerance refers to is b - A W = -D (f - S W),
// so ||b - A W|| is the rhow-weighted norm of the CG residual.
//
// Unknowns live in an [NK][pitch] array (NK = nz-3 rows, kk = k-2; column
// ii = i-1, pitch a multiple of 32), periodic in ii without ghost columns.
//
// Preconditioner: geometric multigrid with semicoarsening in x (NX -> NX/2;
// the x coupling of level l is cx/4^l, rows unchanged), one damped z-line
// Jacobi sweep (omega = 2/3) before and after the coarse correction, each
// column's tridiagonal z operator solved exactly by a partitioned solver,
// full-weighting restriction, linear interpolation, and an exact solve of the
// one-column coarsest level. With the same damped sweep before and after and
// P = 2 R^T the V-cycle is a symmetric positive definite preconditioner.
#pragma once

#include "vvm_common.cuh"

namespace vvm {

struct ZOps {          // per-row z coefficients, [NK] doubles
    const double *ru, *rd;
    int NK;
};

template <typename P>
__device__ __forceinline__ P s_apply(const P* x, int pitch, int nxl, int NK, const ZOps& z,
                                     const double* cx, int kk, int i) {
    const int il = (i == 0) ? nxl - 1 : i - 1, ir = (i == nxl - 1) ? 0 : i + 1;
    const P c = P(cx[kk]), ru = P(z.ru[kk]), rd = P(z.rd[kk]);
    const size_t row = (size_t)kk * pitch;
    P xc = x[row + i];
    P y = (P(2) * c + ru + rd) * xc - c * (x[row + il] + x[row + ir]);
    if (kk + 1 < NK) y -= ru * x[row + pitch + i];
    if (kk > 0) y -= rd * x[row - pitch + i];
    return y;
}

// Linear interpolation of coarse column values onto fine column i.
template <typename P>
__device__ __forceinline__ P prolong_at(const P* xc, int pitch_c, int nc, int kk, int i) {
    const size_t row = (size_t)kk * pitch_c;
    if ((i & 1) == 0) return xc[row + (i >> 1)];
    int j0 = i >> 1, j1 = (j0 + 1 == nc) ? 0 : j0 + 1;
    return P(0.5) * (xc[row + j0] + xc[row + j1]);
}

// ---------------------------------------------------------------------------
// Partitioned (spike) solve of the z-line operator of one level.
//
// Every column of a level has the same tridiagonal z operator, so all its
// factors are precomputed on the host: the column's NK rows are cut into S
// segments (segment s = rows [s*NK/S, (s+1)*NK/S)); within a segment
// x = y - gL x[a-1] - gR x[b] where y solves the segment's own block and the
// spikes gL, gR its couplings; the 2S segment-end unknowns satisfy a small
// system whose inverse Minv (2S x 2S) is also precomputed. A block of
// 32 x S threads owns 32 adjacent columns (lanes: coalesced rows) and all S
// segments (warps); the only serial chain is the segment's own Thomas pass.

constexpr int kMaxSeg = 32;

struct LineLevel {
    int nxl, pitch, NK, S;
    const double* cx;                 // x coupling of the level, [NK]
    const double *lo, *inv, *cp;      // segment-local Thomas factors, [NK]
    const double *gL, *gR;            // spikes, [NK]
    const double* Minv;               // [2S][2S]
};

// y = (segment-local) T^{-1} r for rows [a, a+len), in registers.
template <typename P, int LS>
__device__ __forceinline__ void seg_thomas(const LineLevel& L, int a, int len, P (&r)[LS]) {
    P prev = P(0);
#pragma unroll
    for (int j = 0; j < LS; j++) {
        if (j < len) {
            prev = (r[j] - P(L.lo[a + j]) * prev) * P(L.inv[a + j]);
            r[j] = prev;
        }
    }
    P next = P(0);
#pragma unroll
    for (int j = LS - 1; j >= 0; j--) {
        if (j < len) {
            next = r[j] - P(L.cp[a + j]) * next;
            r[j] = next;
        }
    }
}

// One damped line-Jacobi sweep (or, with xin = xc = null and omega = 1, an
// exact line solve) for the 32-column strip starting at col0:
//   out = X + omega * Dline^{-1} (f - S X),  X = xin + P xc.
// shY: shared [2*kMaxSeg][32] of P. Every thread of the block must call it.
template <typename P, int LS>
__device__ __forceinline__ void line_sweep(const LineLevel& L, const ZOps& z, int col0, const P* f,
                                           const P* xin, const P* xc, int pitch_c, int nc, P* out, P omega,
                                           P* shY) {
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const int i = col0 + lane;
    const bool act = (i < L.nxl) && (s < L.S);
    const int a = (s * L.NK) / L.S, b = ((s + 1) * L.NK) / L.S, len = b - a;
    const bool has_x = (xin != nullptr) || (xc != nullptr);
    P y[LS], X[LS];
    if (act) {
        const int il = (i == 0) ? L.nxl - 1 : i - 1, ir = (i == L.nxl - 1) ? 0 : i + 1;
        auto Xat = [&](int kk, int col) -> P {
            P v = xin ? xin[(size_t)kk * L.pitch + col] : P(0);
            if (xc) v += prolong_at(xc, pitch_c, nc, kk, col);
            return v;
        };
#pragma unroll
        for (int j = 0; j < LS; j++) {
            X[j] = P(0);
            y[j] = P(0);
            if (j < len) {
                const int kk = a + j;
                P r = f[(size_t)kk * L.pitch + i];
                if (has_x) {
                    const P c = P(L.cx[kk]), ru = P(z.ru[kk]), rd = P(z.rd[kk]);
                    P x0 = Xat(kk, i);
                    P sx = (P(2) * c + ru + rd) * x0 - c * (Xat(kk, il) + Xat(kk, ir));
                    if (kk + 1 < L.NK) sx -= ru * Xat(kk + 1, i);
                    if (kk > 0) sx -= rd * Xat(kk - 1, i);
                    r -= sx;
                    X[j] = x0;
                }
                y[j] = r;
            }
        }
        seg_thomas<P, LS>(L, a, len, y);
        P ylast = y[0];
#pragma unroll
        for (int j = 0; j < LS; j++)
            if (j == len - 1) ylast = y[j];
        shY[(2 * s) * 32 + lane] = y[0];
        shY[(2 * s + 1) * 32 + lane] = ylast;
    }
    __syncthreads();
    if (act) {
        const int S2 = 2 * L.S;
        P XL = P(0), XR = P(0);
        if (s > 0) {
            const double* m = L.Minv + (size_t)(2 * (s - 1) + 1) * S2;
            for (int q = 0; q < S2; q++) XL += P(m[q]) * shY[q * 32 + lane];
        }
        if (s + 1 < L.S) {
            const double* m = L.Minv + (size_t)(2 * (s + 1)) * S2;
            for (int q = 0; q < S2; q++) XR += P(m[q]) * shY[q * 32 + lane];
        }
#pragma unroll
        for (int j = 0; j < LS; j++) {
            if (j < len) {
                const int kk = a + j;
                P e = y[j] - P(L.gL[kk]) * XL - P(L.gR[kk]) * XR;
                out[(size_t)kk * L.pitch + i] = X[j] + omega * e;
            }
        }
    }
    __syncthreads();
}

template <typename P>
struct SweepArgs {
    LineLevel L;
    ZOps z;
    const P *f, *xin, *xc;
    int pitch_c, nc;
    P* out;
    P omega;
};

template <typename P, int LS>
__global__ void __launch_bounds__(32 * kMaxSeg) k_line_sweep(SweepArgs<P> a) {
    __shared__ P shY[2 * kMaxSeg * 32];
    line_sweep<P, LS>(a.L, a.z, blockIdx.x * 32, a.f, a.xin, a.xc, a.pitch_c, a.nc, a.out, a.omega, shY);
}

template <typename P>
struct RestrictArgs {
    int nxl, pitch, NK;   // fine level
    ZOps z;
    const double* cx;
    const P *f, *x;
    P* fc;                // coarse rhs, [NK][pitch_c]
    int pitch_c;
};

// fc[j] = 1/4 r[2j-1] + 1/2 r[2j] + 1/4 r[2j+1], r = f - S x (periodic).
template <typename P>
__device__ __forceinline__ void restrict_point(const RestrictArgs<P>& a, int j, int kk) {
    const int i0 = 2 * j, im = (i0 == 0) ? a.nxl - 1 : i0 - 1, ip = i0 + 1;
    const size_t row = (size_t)kk * a.pitch;
    P r0 = a.f[row + i0] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, i0);
    P rm = a.f[row + im] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, im);
    P rp = a.f[row + ip] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, ip);
    a.fc[(size_t)kk * a.pitch_c + j] = P(0.25) * rm + P(0.5) * r0 + P(0.25) * rp;
}

template <typename P>
__global__ void k_mg_restrict(RestrictArgs<P> a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= (a.nxl >> 1) || kk >= a.NK) return;
    restrict_point(a, j, kk);
}

// The coarse end of the V-cycle in one block, with block barriers between
// phases. Levels wider than 32 columns are swept strip by strip. When NX is a
// power of two the last level has one column, its operator has no x part,
// and one exact line solve (omega = 1) finishes it; otherwise the last level
// has an odd column count and gets coarse_sweeps damped sweeps from zero.
constexpr int kMaxCoarseLevels = 8;

template <typename P>
struct CoarseCycleArgs {
    int nlev;                          // levels handled by the block (>= 1)
    LineLevel L[kMaxCoarseLevels];
    ZOps z;
    const P* f0;                       // rhs of its first level
    P* f[kMaxCoarseLevels];            // rhs of the following levels
    P* x[kMaxCoarseLevels];            // pre-smoothed iterates; coarsest solution
    P* y[kMaxCoarseLevels];            // post-smoothed results (y[0] = output)
    P omega;
    int coarse_sweeps;                 // 1 = exact solve of a single column
};

template <typename P, int LS>
__device__ __forceinline__ void sweep_all(const LineLevel& L, const ZOps& z, const P* f, const P* xin,
                                          const P* xc, int pitch_c, int nc, P* out, P omega, P* shY) {
    for (int c0 = 0; c0 < L.nxl; c0 += 32) line_sweep<P, LS>(L, z, c0, f, xin, xc, pitch_c, nc, out, omega, shY);
}

template <typename P, int LS>
__global__ void __launch_bounds__(32 * kMaxSeg) k_mg_coarse_cycle(CoarseCycleArgs<P> a) {
    __shared__ P shY[2 * kMaxSeg * 32];
    const int n = a.nlev;
    for (int l = 0; l < n - 1; l++) {
        const P* fl = (l == 0) ? a.f0 : a.f[l];
        sweep_all<P, LS>(a.L[l], a.z, fl, nullptr, nullptr, 0, 0, a.x[l], a.omega, shY);
        RestrictArgs<P> ra{a.L[l].nxl, a.L[l].pitch, a.L[l].NK, a.z, a.L[l].cx, fl, a.x[l], a.f[l + 1],
                           a.L[l + 1].pitch};
        const int nc = a.L[l].nxl >> 1, tot = nc * a.L[l].NK;
        for (int t = threadIdx.x; t < tot; t += blockDim.x) restrict_point(ra, t % nc, t / nc);
        __syncthreads();
    }
    {
        const int c = n - 1;
        const P* fl = (n == 1) ? a.f0 : a.f[c];
        P* target = (n == 1) ? a.y[0] : a.x[c];
        P* other = (n == 1) ? a.x[0] : a.y[c];
        const int K = a.coarse_sweeps;
        if (K <= 1) {
            sweep_all<P, LS>(a.L[c], a.z, fl, nullptr, nullptr, 0, 0, target, P(1), shY);
        } else {
            P* dst = (K & 1) ? target : other;
            const P* cur = nullptr;
            for (int it = 0; it < K; it++) {
                sweep_all<P, LS>(a.L[c], a.z, fl, cur, nullptr, 0, 0, dst, a.omega, shY);
                cur = dst;
                dst = (dst == target) ? other : target;
            }
        }
    }
    for (int l = n - 2; l >= 0; l--) {
        const P* fl = (l == 0) ? a.f0 : a.f[l];
        const P* coarse = (l + 1 == n - 1) ? a.x[n - 1] : a.y[l + 1];
        sweep_all<P, LS>(a.L[l], a.z, fl, a.x[l], coarse, a.L[l + 1].pitch, a.L[l + 1].nxl, a.y[l], a.omega,
                         shY);
    }
}

// ---------------------------------------------------------------------------
// CG vector kernels on the finest level. Partial sums go to
// partial[block] and are finished by k_cg_scalar in a fixed order.

struct CGScalars {     // device-resident scalars of one solve
    double rz, pq, rr, bb, alpha, beta, rz_new, pad;
};

template <typename P>
struct VecArgs {
    int nx, pitch, NK;
    ZOps z;
    const double* cx;
    const double* rhow_k;   // [NK] rhow at k = kk+2 (residual weights)
};

// q = S p and partial <p, q>.
template <typename P>
__global__ void k_cg_spmv(VecArgs<P> v, const P* p, P* q, double* partial) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        P y = s_apply(p, v.pitch, v.nx, v.NK, v.z, v.cx, kk, i);
        size_t id = (size_t)kk * v.pitch + i;
        q[id] = y;
        s[0] = (double)p[id] * (double)y;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// x += alpha p; r -= alpha q; partial ||rhow r||^2.
template <typename P>
__global__ void k_cg_update(VecArgs<P> v, const CGScalars* sc, P* x, P* r, const P* p, const P* q,
                            double* partial) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        const double al = sc->alpha;
        size_t id = (size_t)kk * v.pitch + i;
        x[id] = P((double)x[id] + al * (double)p[id]);
        P rn = P((double)r[id] - al * (double)q[id]);
        r[id] = rn;
        double wr = v.rhow_k[kk] * (double)rn;
        s[0] = wr * wr;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// partial <r, z>.
template <typename P>
__global__ void k_cg_dot(VecArgs<P> v, const P* r, const P* z, double* partial) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        size_t id = (size_t)kk * v.pitch + i;
        s[0] = (double)r[id] * (double)z[id];
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

// p = z + beta p (beta = 0 on the first iteration).
template <typename P>
__global__ void k_cg_dir(VecArgs<P> v, const CGScalars* sc, const P* z, P* p, int first) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < v.nx && kk < v.NK) {
        size_t id = (size_t)kk * v.pitch + i;
        p[id] = first ? z[id] : P((double)z[id] + sc->beta * (double)p[id]);
    }
}

// r = f - S x and partial ||rhow r||^2 (initial residual of a warm start).
template <typename P>
__global__ void k_cg_residual(VecArgs<P> v, const P* f, const P* x, P* r, double* partial) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        size_t id = (size_t)kk * v.pitch + i;
        P rv = f[id] - s_apply(x, v.pitch, v.nx, v.NK, v.z, v.cx, kk, i);
        r[id] = rv;
        double wr = v.rhow_k[kk] * (double)rv;
        s[0] = wr * wr;
    }
    block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
}

enum : int { CG_SET_BB = 0, CG_SET_RR, CG_SET_RZ, CG_PQ_ALPHA, CG_RZ_BETA };

// Finishes a partial-sum array (fixed order) and updates the CG scalars.
__global__ void k_cg_scalar(const double* partial, int n, CGScalars* sc, int mode);

}  // namespace vvm
