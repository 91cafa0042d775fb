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
// Jacobi sweep before and after the coarse correction (each column's
// tridiagonal z operator solved exactly, Thomas with per-level factors),
// full-weighting restriction, linear interpolation, and an exact solve on the
// coarsest level (real Fourier modes in x, one tridiagonal solve per mode).
// With the same damped sweep before and after and P = 2 R^T the V-cycle is a
// symmetric positive definite preconditioner.
#pragma once

#include "vvm_common.cuh"

namespace vvm {

struct ZOps {          // per-row z coefficients, [NK] doubles
    const double *ru, *rd;
    int NK;
};

struct LineFactors {   // Thomas factors of one level's line operator, [NK]
    const double *lo, *inv, *cp;
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

template <typename P>
struct SmoothArgs {
    int nxl, pitch, NK;
    ZOps z;
    const double* cx;
    LineFactors lf;
    const P* f;        // right-hand side of this level
    const P* xin;      // current iterate (null = zero)
    const P* xc;       // coarse correction to add first (null = none)
    int pitch_c, nc;
    P* out;            // xin + Pxc + omega * Dline^{-1} (f - S (xin + Pxc))
    P omega;
};

// Value of the iterate X = xin + P xc at (kk, i).
template <typename P>
__device__ __forceinline__ P smooth_X(const SmoothArgs<P>& a, int kk, int i) {
    P v = a.xin ? a.xin[(size_t)kk * a.pitch + i] : P(0);
    if (a.xc) v += prolong_at(a.xc, a.pitch_c, a.nc, kk, i);
    return v;
}

// One damped z-line Jacobi sweep; one thread per column.
template <typename P>
__global__ void k_mg_smooth(SmoothArgs<P> a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nxl) return;
    const int NK = a.NK;
    const bool has_x = (a.xin != nullptr) || (a.xc != nullptr);
    const int il = (i == 0) ? a.nxl - 1 : i - 1, ir = (i == a.nxl - 1) ? 0 : i + 1;
    // forward elimination; y_k parked in out
    P yprev = P(0);
    P xm = P(0), x0 = has_x ? smooth_X(a, 0, i) : P(0);
    for (int kk = 0; kk < NK; kk++) {
        P r = a.f[(size_t)kk * a.pitch + i];
        P xp = P(0);
        if (has_x) {
            xp = (kk + 1 < NK) ? smooth_X(a, kk + 1, i) : P(0);
            const P c = P(a.cx[kk]), ru = P(a.z.ru[kk]), rd = P(a.z.rd[kk]);
            P sx = (P(2) * c + ru + rd) * x0 - c * (smooth_X(a, kk, il) + smooth_X(a, kk, ir)) - ru * xp - rd * xm;
            r -= sx;
        }
        P y = (r - P(a.lf.lo[kk]) * yprev) * P(a.lf.inv[kk]);
        a.out[(size_t)kk * a.pitch + i] = y;
        yprev = y;
        xm = x0;
        x0 = xp;
    }
    // back substitution
    P xnext = P(0);
    for (int kk = NK - 1; kk >= 0; kk--) {
        size_t id = (size_t)kk * a.pitch + i;
        P e = a.out[id] - P(a.lf.cp[kk]) * xnext;
        xnext = e;
        P base = has_x ? smooth_X(a, kk, i) : P(0);
        a.out[id] = base + a.omega * e;
    }
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
__global__ void k_mg_restrict(RestrictArgs<P> a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = blockIdx.y * blockDim.y + threadIdx.y;
    const int nc = a.nxl >> 1;
    if (j >= nc || kk >= a.NK) return;
    const int i0 = 2 * j, im = (i0 == 0) ? a.nxl - 1 : i0 - 1, ip = i0 + 1;
    const size_t row = (size_t)kk * a.pitch;
    P r0 = a.f[row + i0] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, i0);
    P rm = a.f[row + im] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, im);
    P rp = a.f[row + ip] - s_apply(a.x, a.pitch, a.nxl, a.NK, a.z, a.cx, kk, ip);
    a.fc[(size_t)kk * a.pitch_c + j] = P(0.25) * rm + P(0.5) * r0 + P(0.25) * rp;
}

template <typename P>
struct CoarseArgs {
    int nc, pitch, NK;
    const double* Q;      // [nc][nc] orthonormal real Fourier basis, Q[j*nc + m]
    const double *lo, *inv, *cp;   // per mode factors, [nc][NK]
    const P* f;
    P* x;
    double* xh;           // scratch [NK][nc]
};

// Exact coarsest-level solve: x = Q (per-mode tridiagonal)^{-1} Q^T f.
template <typename P>
__global__ void k_mg_coarse(CoarseArgs<P> a) {
    const int m = threadIdx.x;
    const int nc = a.nc, NK = a.NK;
    if (m < nc) {
        const double* lo = a.lo + (size_t)m * NK;
        const double* inv = a.inv + (size_t)m * NK;
        const double* cp = a.cp + (size_t)m * NK;
        double yprev = 0;
        for (int kk = 0; kk < NK; kk++) {
            double fh = 0;
            for (int j = 0; j < nc; j++) fh += a.Q[j * nc + m] * (double)a.f[(size_t)kk * a.pitch + j];
            double y = (fh - lo[kk] * yprev) * inv[kk];
            a.xh[(size_t)kk * nc + m] = y;
            yprev = y;
        }
        double xnext = 0;
        for (int kk = NK - 1; kk >= 0; kk--) {
            double e = a.xh[(size_t)kk * nc + m] - cp[kk] * xnext;
            a.xh[(size_t)kk * nc + m] = e;
            xnext = e;
        }
    }
    __syncthreads();
    if (m < nc) {
        for (int kk = 0; kk < NK; kk++) {
            double v = 0;
            for (int q = 0; q < nc; q++) v += a.Q[m * nc + q] * a.xh[(size_t)kk * nc + q];
            a.x[(size_t)kk * a.pitch + m] = P(v);
        }
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
