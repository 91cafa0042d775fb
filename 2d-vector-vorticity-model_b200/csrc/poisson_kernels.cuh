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
// pentadiagonal system whose banded LU is also precomputed. A block of
// 32 x S threads owns 32 adjacent columns (lanes: coalesced rows) and all S
// segments (warps); the serial chains are the segment's own Thomas pass and
// warp 0's banded solve of the 2S segment ends (one lane per column).

constexpr int kMaxSeg = 32;

struct LineLevel {
    int nxl, pitch, NK, S;
    const double* cx;                 // x coupling of the level, [NK]
    const double *lo, *inv, *cp;      // segment-local Thomas factors, [NK]
    const double *gL, *gR;            // spikes, [NK]
    const double* band;               // banded LU of the reduced system, [5][2S]
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

// Solves the pentadiagonal reduced system of the segment ends in place in
// sh[i*32 + lane] (i = 0..n-1): forward with the unit-lower band (l1, l2),
// backward with the upper band (u1, u2) and 1/diag. Coefficient e of row i is
// band[(e*n + i)*bstride], read from shared memory: the 2n-step recurrence
// is a serial chain, so each step must not wait on a global load.
// One lane per column; only one warp calls it.
template <typename P>
__device__ __forceinline__ void reduced_solve(const P* band, int bstride, int n, P* sh, int lane) {
    P z1 = P(0), z2 = P(0);
    for (int i = 0; i < n; i++) {
        P z = sh[i * 32 + lane] - band[(0 * n + i) * bstride] * z1 - band[(1 * n + i) * bstride] * z2;
        sh[i * 32 + lane] = z;
        z2 = z1;
        z1 = z;
    }
    P x1 = P(0), x2 = P(0);
    for (int i = n - 1; i >= 0; i--) {
        P x = (sh[i * 32 + lane] - band[(2 * n + i) * bstride] * x1 - band[(3 * n + i) * bstride] * x2) *
              band[(4 * n + i) * bstride];
        sh[i * 32 + lane] = x;
        x2 = x1;
        x1 = x;
    }
}

// Copies count band coefficients to shared memory (all threads of the block;
// ordered before their use by the first barrier of segment_couplings).
template <typename P>
__device__ __forceinline__ void stage_band(const double* g, int count, P* sh) {
    for (int t = threadIdx.x; t < count; t += blockDim.x) sh[t] = P(g[t]);
}

// Shared scratch of a line-solve block: segment ends, then the staged band.
constexpr int kShY = 2 * kMaxSeg * 32;
constexpr int kShBand = 10 * kMaxSeg;

// After each warp parked its segment's first/last y in shY: solves for the
// segment-end unknowns (warp 0) and returns this thread's couplings
// x[a-1] (XL) and x[b] (XR). Contains two block barriers.
template <typename P>
__device__ __forceinline__ void segment_couplings(const P* band, int bstride, int S, P* shY, int lane, int s,
                                                  bool lane_ok, P& XL, P& XR) {
    __syncthreads();
    if (s == 0 && lane_ok) reduced_solve(band, bstride, 2 * S, shY, lane);
    __syncthreads();
    XL = (s > 0 && s < S) ? shY[(2 * s - 1) * 32 + lane] : P(0);
    XR = (s + 1 < S) ? shY[(2 * s + 2) * 32 + lane] : P(0);
}

// One damped line-Jacobi sweep (or, with xin = xc = null and omega = 1, an
// exact line solve) for the 32-column strip starting at col0:
//   out = X + omega * Dline^{-1} (f - S X),  X = xin + P xc.
// Each thread loads its column's segment rows (and one row above and below)
// once; x neighbours come from the adjacent lanes by shuffle, and only the
// strip's edge lanes load a halo column. shY: shared [kShY + kShBand] of P.
// Every thread of the block must call it.
template <typename P, int LS>
__device__ __forceinline__ void line_sweep(const LineLevel& L, const ZOps& z, int col0, const P* f,
                                           const P* xin, const P* xc, int pitch_c, int nc, P* out, P omega,
                                           P* shY) {
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const int i = col0 + lane;
    const bool wact = (s < L.S);                 // warp has a segment
    P* shB = shY + kShY;
    stage_band(L.band, 10 * L.S, shB);
    const bool act = wact && (i < L.nxl);
    const int a = wact ? (s * L.NK) / L.S : 0, b = wact ? ((s + 1) * L.NK) / L.S : 0, len = b - a;
    const bool has_x = (xin != nullptr) || (xc != nullptr);
    auto Xat = [&](int kk, int col) -> P {
        P v = xin ? xin[(size_t)kk * L.pitch + col] : P(0);
        if (xc) v += prolong_at(xc, pitch_c, nc, kk, col);
        return v;
    };
    P y[LS], X[LS];
    if (wact) {
        const int il = (i == 0) ? L.nxl - 1 : i - 1, ir = (i >= L.nxl - 1) ? 0 : i + 1;
        const bool own_l = (lane > 0), own_r = (lane < 31) && (i + 1 < L.nxl);
        P Xv[LS + 2];
        P fv[LS];
#pragma unroll
        for (int j = 0; j < LS + 2; j++) {
            const int kk = a - 1 + j;
            Xv[j] = (has_x && act && j <= len + 1 && kk >= 0 && kk < L.NK) ? Xat(kk, i) : P(0);
        }
#pragma unroll
        for (int j = 0; j < LS; j++) fv[j] = (act && j < len) ? f[(size_t)(a + j) * L.pitch + i] : P(0);
#pragma unroll
        for (int j = 0; j < LS; j++) {
            P xl = P(0), xr = P(0);
            if (has_x) {
                xl = __shfl_up_sync(0xffffffffu, Xv[j + 1], 1);
                xr = __shfl_down_sync(0xffffffffu, Xv[j + 1], 1);
                if (act && j < len) {
                    if (!own_l) xl = Xat(a + j, il);
                    if (!own_r) xr = Xat(a + j, ir);
                }
            }
            X[j] = Xv[j + 1];
            P r = fv[j];
            if (has_x && act && j < len) {
                const int kk = a + j;
                const P c = P(L.cx[kk]), ru = P(z.ru[kk]), rd = P(z.rd[kk]);
                r -= (P(2) * c + ru + rd) * Xv[j + 1] - c * (xl + xr) - ru * Xv[j + 2] - rd * Xv[j];
            }
            y[j] = r;
        }
        if (act) {
            seg_thomas<P, LS>(L, a, len, y);
            P ylast = y[0];
#pragma unroll
            for (int j = 0; j < LS; j++)
                if (j == len - 1) ylast = y[j];
            shY[(2 * s) * 32 + lane] = y[0];
            shY[(2 * s + 1) * 32 + lane] = ylast;
        }
    }
    P XL, XR;
    segment_couplings(shB, 1, L.S, shY, lane, s, col0 + lane < L.nxl, XL, XR);
    if (act) {
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
    __shared__ P shY[kShY + kShBand];
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

// Pre-smoothing from a zero iterate fused with the restriction of the new
// residual: x = omega * Dline^{-1} f (no neighbour values needed), then
// r = f - S x and fc = full weighting of r. A block's 32 lanes cover fine
// columns c0-2 .. c0+29 (periodic) and own c0 .. c0+27: it stores x there,
// forms r on lanes 1..30 and the 14 coarse values whose three fine residuals
// it holds. Neighbouring blocks recompute the 4 overlap columns.
constexpr int kOwned = 28;

template <typename P, int LS>
__global__ void __launch_bounds__(32 * kMaxSeg) k_presmooth_restrict(LineLevel L, ZOps z, const P* f, P* xout,
                                                                      P* fc, int pitch_c, P omega) {
    __shared__ P shY[kShY + kShBand];
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const int c0 = blockIdx.x * kOwned;
    const int col = (c0 - 2 + lane + L.nxl) % L.nxl;
    const bool wact = (s < L.S);
    const int a = wact ? (s * L.NK) / L.S : 0, b = wact ? ((s + 1) * L.NK) / L.S : 0, len = b - a;
    const bool owned = (lane >= 2) && (lane < 2 + kOwned) && (c0 + lane - 2 < L.nxl);
    P* shB = shY + kShY;
    stage_band(L.band, 10 * L.S, shB);
    P y[LS], fv[LS];
    if (wact) {
#pragma unroll
        for (int j = 0; j < LS; j++) {
            fv[j] = (j < len) ? f[(size_t)(a + j) * L.pitch + col] : P(0);
            y[j] = fv[j];
        }
        seg_thomas<P, LS>(L, a, len, y);
        P ylast = y[0];
#pragma unroll
        for (int j = 0; j < LS; j++)
            if (j == len - 1) ylast = y[j];
        shY[(2 * s) * 32 + lane] = y[0];
        shY[(2 * s + 1) * 32 + lane] = ylast;
    }
    P XL, XR;
    segment_couplings(shB, 1, L.S, shY, lane, s, true, XL, XR);
    __syncthreads();   // every warp has read its couplings before shY is reused
    P x[LS];
    if (wact) {
#pragma unroll
        for (int j = 0; j < LS; j++) {
            x[j] = P(0);
            if (j < len) {
                const int kk = a + j;
                x[j] = omega * (y[j] - P(L.gL[kk]) * XL - P(L.gR[kk]) * XR);
                if (owned) xout[(size_t)kk * L.pitch + col] = x[j];
            }
        }
        // segment ends of x for the z neighbours of the residual
        P xlast = x[0];
#pragma unroll
        for (int j = 0; j < LS; j++)
            if (j == len - 1) xlast = x[j];
        shY[(2 * s) * 32 + lane] = x[0];
        shY[(2 * s + 1) * 32 + lane] = xlast;
    }
    __syncthreads();
    if (wact) {
        const P xbelow = (s > 0) ? shY[(2 * s - 1) * 32 + lane] : P(0);     // x at row a-1
        const P xabove = (s + 1 < L.S) ? shY[(2 * s + 2) * 32 + lane] : P(0);  // x at row b
#pragma unroll
        for (int j = 0; j < LS; j++) {
            const P xl = __shfl_up_sync(0xffffffffu, x[j], 1);
            const P xr = __shfl_down_sync(0xffffffffu, x[j], 1);
            P r = P(0);
            if (j < len) {
                const int kk = a + j;
                const P c = P(L.cx[kk]), ru = P(z.ru[kk]), rd = P(z.rd[kk]);
                P xd = (j == 0) ? xbelow : x[(j > 0) ? j - 1 : 0];
                P xu = (j == len - 1) ? xabove : x[(j + 1 < LS) ? j + 1 : LS - 1];
                r = fv[j] - ((P(2) * c + ru + rd) * x[j] - c * (xl + xr) - ru * xu - rd * xd);
            }
            const P rm = __shfl_up_sync(0xffffffffu, r, 1);
            const P rp = __shfl_down_sync(0xffffffffu, r, 1);
            if (j < len && owned && (lane & 1) == 0)
                fc[(size_t)(a + j) * pitch_c + (col >> 1)] = P(0.25) * rm + P(0.5) * r + P(0.25) * rp;
        }
    }
}

// Exact solve on a level of nc <= 32 columns. The operator is separable (x
// coefficients depend on the row only, periodic in x), so a real orthonormal
// Fourier basis Q (nc x nc) diagonalises its x part: mode m needs the
// tridiagonal z solve of (cx mu_m + ru + rd, -ru, -rd), mu_m the eigenvalue
// of the periodic [-1 2 -1]. One block: f and Q are staged in shared memory,
// each (mode lane, segment warp) transforms its rows and runs the partitioned
// solve with that mode's precomputed factors (warp 0 solving every mode's
// reduced system), and the inverse transform writes x.
struct ModeSolve {
    int nc, pitch, NK, S;
    const double* Q;                  // [nc][nc], Q[col*nc + m]
    const double *lo, *inv, *cp, *gL, *gR;   // [NK][nc]: mode fastest (coalesced)
    const double* band;               // [5][2S][nc]
};

// Segment Thomas pass of one mode (factors interleaved by mode, stride nc).
template <typename P, int LS>
__device__ __forceinline__ void seg_thomas_modes(const ModeSolve& M, int m, int a, int len, P (&r)[LS]) {
    const int nc = M.nc;
    P prev = P(0);
#pragma unroll
    for (int j = 0; j < LS; j++) {
        if (j < len) {
            const size_t e = (size_t)(a + j) * nc + m;
            prev = (r[j] - P(M.lo[e]) * prev) * P(M.inv[e]);
            r[j] = prev;
        }
    }
    P next = P(0);
#pragma unroll
    for (int j = LS - 1; j >= 0; j--) {
        if (j < len) {
            next = r[j] - P(M.cp[(size_t)(a + j) * nc + m]) * next;
            r[j] = next;
        }
    }
}

template <typename P, int LS>
__global__ void __launch_bounds__(32 * kMaxSeg) k_coarse_modes(ModeSolve M, const P* f, P* x) {
    extern __shared__ unsigned char smem_raw[];
    P* fs = reinterpret_cast<P*>(smem_raw);             // [NK][nc]: f, later the mode solution
    P* xh = fs;                                         // (f is dead after the first barrier)
    P* bs = fs + (size_t)M.NK * M.nc;                   // [5][2S][nc] band
    __shared__ P shY[2 * kMaxSeg * 32];
    __shared__ P Qs[32 * 32];    // Q[col][m]: forward transform, lanes = m
    __shared__ P QT[32 * 32];    // Q[col][m] at [m][col]: inverse, lanes = col
    const int nc = M.nc, NK = M.NK, S = M.S;
    for (int t = threadIdx.x; t < NK * nc; t += blockDim.x) {
        int kk = t / nc, c = t % nc;
        fs[t] = f[(size_t)kk * M.pitch + c];
    }
    stage_band(M.band, 10 * S * nc, bs);
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
        Qs[t] = P(M.Q[t]);
        QT[(t % nc) * nc + t / nc] = P(M.Q[t]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const bool act = (s < S) && (lane < nc);
    const int a = (s < S) ? (s * NK) / S : 0, b = (s < S) ? ((s + 1) * NK) / S : 0, len = b - a;
    const int m = lane;
    P y[LS];
    if (act) {
#pragma unroll
        for (int j = 0; j < LS; j++) {
            P v = P(0);
            if (j < len) {
                const P* row = fs + (size_t)(a + j) * nc;
#pragma unroll 8
                for (int c = 0; c < nc; c++) v += Qs[c * nc + m] * row[c];
            }
            y[j] = v;
        }
        seg_thomas_modes<P, LS>(M, m, a, len, y);
        P ylast = y[0];
#pragma unroll
        for (int j = 0; j < LS; j++)
            if (j == len - 1) ylast = y[j];
        shY[(2 * s) * 32 + lane] = y[0];
        shY[(2 * s + 1) * 32 + lane] = ylast;
    }
    P XL, XR;
    segment_couplings(bs + m, nc, S, shY, lane, s, lane < nc, XL, XR);
    if (act) {
#pragma unroll
        for (int j = 0; j < LS; j++) {
            if (j < len) {
                const int kk = a + j;
                xh[(size_t)kk * nc + m] = y[j] - P(M.gL[(size_t)kk * nc + m]) * XL - P(M.gR[(size_t)kk * nc + m]) * XR;
            }
        }
    }
    __syncthreads();
    if (act) {   // lane = output column
        const int cc = lane;
        for (int j = 0; j < len; j++) {
            const int kk = a + j;
            const P* row = xh + (size_t)kk * nc;
            P v = P(0);
#pragma unroll 8
            for (int q = 0; q < nc; q++) v += QT[q * nc + cc] * row[q];
            x[(size_t)kk * M.pitch + cc] = v;
        }
    }
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
    __shared__ P shY[kShY + kShBand];
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
    double rz, pq, rr, bb, alpha, beta, rz_new;
    double nrm;           // ||r1||^2 scaling the learned preconditioner's input
    double dsd, gam;      // (d, S d) and the Galerkin step (d, r1) / (d, S d) of its correction d
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
__device__ __forceinline__ void k_cg_spmv_body(const VecArgs<P>& v, const P* p, P* q, double* partial) {
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
template <typename P>
__global__ void k_cg_spmv(VecArgs<P> v, const P* p, P* q, double* partial) { k_cg_spmv_body<P>(v, p, q, partial); }

// x += alpha p; r -= alpha q; partial ||rhow r||^2.
template <typename P>
__device__ __forceinline__ void k_cg_update_body(const VecArgs<P>& v, const CGScalars* sc, P* x, P* r, const P* p, const P* q,
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
template <typename P>
__global__ void k_cg_update(VecArgs<P> v, const CGScalars* sc, P* x, P* r, const P* p, const P* q,
                            double* partial) { k_cg_update_body<P>(v, sc, x, r, p, q, partial); }

// partial <r, z>.
template <typename P>
__device__ __forceinline__ void k_cg_dot_body(const VecArgs<P>& v, const P* r, const P* z, double* partial) {
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
template <typename P>
__global__ void k_cg_dot(VecArgs<P> v, const P* r, const P* z, double* partial) { k_cg_dot_body<P>(v, r, z, partial); }

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

enum : int { CG_SET_BB = 0, CG_SET_RR, CG_SET_RZ, CG_PQ_ALPHA, CG_RZ_BETA, CG_SET_NRM, CG_FCG_BETA, CG_NET_DSD,
             CG_NET_GAMMA };

// Device-side loop state of a graph-captured solve.
struct CGCtl {
    int it;          // CG iterations of the current (inner) solve
    int total;       // CG iterations summed over refinement passes
    int outer;       // refinement passes
    int more;        // the loop's last decision (1: another iteration), for grouped launches
    double rr0;      // squared initial residual of the inner solve
    double relres;   // final ||b - A W|| / ||b||
};

// Finishes a partial-sum array (fixed order) and updates the CG scalars.
// CG_RZ_BETA with ctl != null takes beta = 0 on the first iteration.
__global__ void k_cg_scalar(const double* partial, int n, CGScalars* sc, int mode);
__global__ void k_cg_scalar_it(const double* partial, int n, CGScalars* sc, const CGCtl* ctl);

// p = z (first iteration of ctl) or z + beta p.
template <typename P>
__device__ __forceinline__ void k_cg_dir_it_body(const VecArgs<P>& v, const CGScalars* sc, const CGCtl* ctl, const P* z, P* p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < v.nx && kk < v.NK) {
        size_t id = (size_t)kk * v.pitch + i;
        p[id] = (ctl->it == 0) ? z[id] : P((double)z[id] + sc->beta * (double)p[id]);
    }
}
template <typename P>
__global__ void k_cg_dir_it(VecArgs<P> v, const CGScalars* sc, const CGCtl* ctl, const P* z, P* p) { k_cg_dir_it_body<P>(v, sc, ctl, z, p); }

// W = 0 when ||b|| = 0 (the solution of A W = 0), read on the device.
__global__ void k_zero_if_b0(int NX, int NK, int pitch, const CGScalars* sc, double* W);

// Loop conditions of graph-captured solves (one thread). `init` starts a
// loop, otherwise one iteration has finished and `body_kernels` kernels of
// its body ran (added to *exec, the context's count of executed kernels).
//   plain  : continue while ||rhow r||^2 > tol^2 ||b||^2, it < maxit
//   inner  : continue while ||rhow r||^2 > rtol^2 rr0, it < maxit
//   outer  : continue while the FP64 residual is above tol and the inner
//            iterations so far are below maxit
__global__ void k_loop_plain(const CGScalars* sc, CGCtl* ctl, cudaGraphConditionalHandle h, double tol2,
                             int maxit, int init, long long* exec, int body_kernels);
__global__ void k_loop_inner(const CGScalars* sc, CGCtl* ctl, cudaGraphConditionalHandle h, double rtol2,
                             int maxit, int init, long long* exec, int body_kernels);
__global__ void k_loop_outer(const CGScalars* sc64, CGCtl* ctl, const CGCtl* inner,
                             cudaGraphConditionalHandle h, double tol2, int maxit, int init, long long* exec,
                             int body_kernels);

// The check that opens a graph-recorded solve, in one launch (what
// k_zero_if_b0, k_cg_residual, k_cg_scalar and k_loop_plain do in turn):
// W = 0 when ||b|| = 0 (r = f then, and W is not read), r = f - S W and
// ||rhow r||^2 in per-block partials; the block that arrives last
// (arrive_last) totals them in a fixed order into sc->rr, starts the loop
// state (ctl) and sets the condition of the WHILE node that follows:
// continue while ||rhow r||^2 > tol^2 ||b||^2 and maxit > 0.
template <typename P>
__device__ __forceinline__ void k_cg_check_body(const VecArgs<P>& v, const P* f, P* x, P* r, double* partial, CGScalars* sc, CGCtl* ctl,
                           unsigned* arrive, cudaGraphConditionalHandle h, double tol2, int maxit) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    const bool zero = (sc->bb == 0.0);
    double s[1] = {0};
    if (i < v.nx && kk < v.NK) {
        const size_t id = (size_t)kk * v.pitch + i;
        P rv;
        if (zero) {
            x[id] = P(0);
            rv = f[id];
        } else {
            rv = f[id] - s_apply(x, v.pitch, v.nx, v.NK, v.z, v.cx, kk, i);
        }
        r[id] = rv;
        const double wr = v.rhow_k[kk] * (double)rv;
        s[0] = wr * wr;
    }
    block_sum(s, sh);
    const unsigned nb = gridDim.x * gridDim.y;
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = s[0];
    if (!arrive_last(arrive, nb)) return;
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.x + blockDim.x * threadIdx.y;
    double t[1] = {0};
    for (int b = tid; b < (int)nb; b += nt) t[0] += __ldcg(partial + b);
    block_sum(t, sh);
    if (tid == 0) {
        const double rr = t[0], bb = sc->bb;
        sc->rr = rr;
        ctl->it = 0;
        ctl->total = 0;
        ctl->relres = (bb > 0.0) ? sqrt(rr / bb) : 0.0;
        const bool more = (bb > 0.0) && (rr > tol2 * bb) && (maxit > 0) && isfinite(rr);
        ctl->more = more ? 1 : 0;
        if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
    }
}
template <typename P>
__global__ void k_cg_check(VecArgs<P> v, const P* f, P* x, P* r, double* partial, CGScalars* sc, CGCtl* ctl,
                           unsigned* arrive, cudaGraphConditionalHandle h, double tol2, int maxit) { k_cg_check_body<P>(v, f, x, r, partial, sc, ctl, arrive, h, tol2, maxit); }

}  // namespace vvm
