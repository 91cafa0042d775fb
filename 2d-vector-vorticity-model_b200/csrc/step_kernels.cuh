// Physics kernels of the VVM step (everything except the elliptic solves).
//
// T is the storage and stencil arithmetic type: double for the plain FP64
// step, float for the mixed-precision step. Profiles stay double and are
// rounded to T on load. Domain-wide sums always accumulate in double.
//
// Each kernel restates one or more reference routines and keeps their index
// ranges, boundary treatment and expression order; the file:line citations
// name the reference code. Halo fills are fused into the producing kernel
// (store_center / store_westdown write every ghost image of a cell).
#pragma once

#include <cooperative_groups.h>

#include <type_traits>

#include "vvm_common.cuh"

namespace vvm {

// Per-level coefficient profiles precomputed on the host (double, [nz]),
// each formed with the reference's own expression.
struct Profiles {
    const double *rhou, *rhow, *thvb, *thb_init, *qvb0, *pib, *pb, *lambda2;
    const double *vt_c1;      // (1E-3*rhow[k])*0.5            Advection.cpp:165
    const double *vt_fac;     // pow(rhow[k]/rhow[1], -0.5)    Advection.cpp:165
    const double *pc;         // 380/(pow(pib,Cp/Rd)*P0)       MicroPhysics.cpp:10,82
    const double *dtcgr_th;   // dt*CGR of Nudge_theta (0 below k_start)
    const double *dtcgr_zeta; // dt*CGR of Nudge_zeta (0 below k_start or case 2)
    const double *q1ls, *q2ls;  // large-scale forcing profiles (may be all zero)
    double pf1, pf2;          // 1E-3*rhou[1], pow(rhou[1]/rhow[1], -0.5)  Iteration.cpp:115
    // Mixed step only: th and qv are stored as perturbations from the
    // reference profiles ref[0] = th0 (thb_init) and ref[1] = qv0 (qvb0).
    // For each: d0[k] = ref[k] - ref[k-1], s0[k] = ref[k] + ref[k-1],
    // g0[k] = ref[k+1] - ref[k-1], dn[k] = ref[k] - (nudging target)[k].
    const double *ref[2], *d0[2], *s0[2], *g0[2], *dn[2];
    // Vertical level metric (the reference's constants on uniform levels,
    // exactly; see upload_profiles): flux divergences at centres (r2dzc =
    // 1/(2 dc)) and faces (r2dzw = 1/(2 dw)), the w gradient across a centre
    // (rdzc = 1/dc), gradients across two centres (r2dzcc = 1/(z[k+1]-z[k-1])),
    // the eddy-coefficient cap (kmax = 0.8 dx dc / dt), the Gauss-Seidel
    // vertical factors of Mparam (gsM_*) and Hparam (gsS_*): cz = rdz2_k dt /
    // rho and the down term's density times its spacing ratio, and cal_u's
    // centre-to-centre spacing (dzw) and top factor (hfac = dx / dc_top, 1 on
    // uniform levels as the reference has it); pubarTop's top spacings.
    const double *r2dzc, *r2dzw, *rdzc, *r2dzcc, *kmax, *gsM_cz, *gsM_rhod, *gsS_cz, *gsS_rhod, *dzw;
    double rdz_up, rdz_dn, rdz_c, hfac;
};

// True for the mixed step, whose th and qv arrays hold perturbations.
template <typename T>
constexpr bool kPert = std::is_same<T, float>::value;

// AB2 bookkeeping shared by every prognostic tendency
// (e.g. Advection.cpp:69-71): slot (step+1)%2 receives the new tendency,
// slot step%2 holds the previous one, and on step 0 both become the new one.
struct AB2 {
    int sn, so, first;
    __host__ __device__ static AB2 of(int step) { return AB2{(step + 1) & 1, step & 1, step == 0}; }
};

template <typename T>
__device__ __forceinline__ T ab2_push(T* hn, T* ho, size_t idx, T tend, const AB2& s) {
    T old = s.first ? tend : ho[idx];
    hn[idx] = tend;
    if (s.first) ho[idx] = tend;
    return old;
}

// cp.async helpers: 16-byte global -> shared copies, grouped per row.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One element global -> shared, asynchronous (cp.async, 4 or 8 bytes).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// ---------------------------------------------------------------------------
// Vorticity advection + buoyancy + westdown halo of zetap
// (Iteration::pzeta_pt: Advection.cpp:84-149, Buoyancy.cpp:11-58,
// Boundary.cpp:21-30). One thread per interior zeta point (i, k),
// i = 1..nx-2, k = 2..nz-2.

template <typename T>
struct PZetaArgs {
    Dims d;
    Consts c;
    Profiles p;
    const T *zeta, *u, *w, *th, *qv, *qc, *qr;
    T* zetap;
    T *hz_n, *hz_o, *hb_n, *hb_o;  // dzeta_advect, dth_buoyancy slots
    AB2 ab;
};

// x-face mass flux Uw of Advection_zeta (Advection.cpp:90) from global
// memory: the halo face of k_pzeta's first tile.
template <typename T>
__device__ __forceinline__ T zeta_Uw(const PZetaArgs<T>& a, int i, int k) {
    const Dims& d = a.d;
    return T(0.25) * (T(a.p.rhou[k]) * (a.u[d.at(i + 1, k)] + a.u[d.at(i, k)]) +
                      T(a.p.rhou[k - 1]) * (a.u[d.at(i + 1, k - 1)] + a.u[d.at(i, k - 1)]));
}

// Tile of k_pzeta: 32 x 8 zeta points a block of 32 x 8 threads. zeta, u, w,
// th, qv, qc and qr are staged into shared memory (cp.async); the staggered
// mass fluxes Uw, Wu (Advection.cpp:90-91) are formed once a face point, the
// x and z fluxes once a face, and each point then differences its four
// fluxes and forms its buoyancy from the staged values.
constexpr int kPZBX = 32, kPZBZ = 8;

template <typename T>
struct PZetaShared {
    static constexpr int BX = kPZBX, BZ = kPZBZ;
    T z[BZ + 4][BX + 4];      // zeta: rows k0-2.., columns i0-2..
    T u[BZ + 1][BX + 4];      // u: rows k0-1.., columns i0-2..
    T w[BZ + 4][BX + 1];      // w: rows k0-2.., columns i0-1..
    T q[4][BZ + 1][BX + 1];   // th, qv, qc, qr: rows k0-1.., columns i0-1..
    T U[BZ][BX + 3];          // Uw at x faces fi = i0-2.., rows k0..
    T W[BZ + 3][BX];          // Wu at z faces fk = k0-2.., columns i0..
    T fu[BZ][BX + 1];         // flux_u at fi = i0-1..
    T fw[BZ + 1][BX];         // flux_w at fk = k0-1..
};

template <typename T>
__device__ __forceinline__ void k_pzeta_body(const PZetaArgs<T>& a) {
    constexpr int BX = kPZBX, BZ = kPZBZ, NT = BX * BZ;
    __shared__ PZetaShared<T> S;
    const Dims& d = a.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + BX * ty;
    const int i0 = 1 + blockIdx.x * BX, k0 = 2 + blockIdx.y * BZ;
    const int i = i0 + tx, k = k0 + ty;
    const bool act = (i <= d.nx - 2 && k <= d.nz - 2);

    // Stage: points outside the array are skipped; none of them is read (a
    // flux reads its outer neighbours only where the third-order bracket
    // applies, 2 <= index <= n-3).
    auto stage = [&](T* dst, const T* src, int rows, int cols, int kb, int ib) {
        for (int t = tid; t < rows * cols; t += NT) {
            const int r = t / cols, c = t - r * cols;
            const int kk = kb + r, ii = ib + c;
            if (kk >= 0 && kk <= d.nz - 1 && ii >= 0 && ii <= d.nx - 1) cp_async_elem(dst + t, src + d.at(ii, kk));
        }
    };
    stage(&S.z[0][0], a.zeta, BZ + 4, BX + 4, k0 - 2, i0 - 2);
    stage(&S.u[0][0], a.u, BZ + 1, BX + 4, k0 - 1, i0 - 2);
    stage(&S.w[0][0], a.w, BZ + 4, BX + 1, k0 - 2, i0 - 1);
    const T* qs[4] = {a.th, a.qv, a.qc, a.qr};
#pragma unroll
    for (int f = 0; f < 4; f++) stage(&S.q[f][0][0], qs[f], BZ + 1, BX + 1, k0 - 1, i0 - 1);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    // Uw(fi, k), fi = 0..nx-2, and Wu(i, fk), fk = 1..nz-2 (Advection.cpp:90-91)
    for (int t = tid; t < BZ * (BX + 3); t += NT) {
        const int r = t / (BX + 3), c = t - r * (BX + 3);
        const int fi = i0 - 2 + c, kk = k0 + r;
        if (fi >= 0 && fi <= d.nx - 2 && kk <= d.nz - 2) {
            const int uc = c, ur = r + 1;   // u at (fi, kk) in the staged tile
            S.U[r][c] = T(0.25) * (T(a.p.rhou[kk]) * (S.u[ur][uc + 1] + S.u[ur][uc]) +
                                   T(a.p.rhou[kk - 1]) * (S.u[ur - 1][uc + 1] + S.u[ur - 1][uc]));
        }
    }
    for (int t = tid; t < (BZ + 3) * BX; t += NT) {
        const int r = t / BX, c = t - r * BX;
        const int fk = k0 - 2 + r, ii = i0 + c;
        if (fk >= 1 && fk <= d.nz - 2 && ii <= d.nx - 2) {
            const int wc = c + 1, wr = r;   // w at (ii, fk)
            S.W[r][c] = T(0.25) * (T(a.p.rhow[fk + 1]) * (S.w[wr + 1][wc] + S.w[wr + 1][wc - 1]) +
                                   T(a.p.rhow[fk]) * (S.w[wr][wc] + S.w[wr][wc - 1]));
        }
    }
    __syncthreads();

    // x flux at face (fi+1/2, k), fi = 1..nx-2 (Advection.cpp:107,111-114);
    // the west face of point 1 is the halo copy of face nx-2 (Advection.cpp:123)
    for (int t = tid; t < BZ * (BX + 1); t += NT) {
        const int r = t / (BX + 1), c = t - r * (BX + 1);
        const int fi = i0 - 1 + c, kk = k0 + r;
        if (kk > d.nz - 2 || fi > d.nx - 2) continue;
        T f;
        if (fi == 0) {
            const int e = d.nx - 2;   // no bracket at nx-2
            f = zeta_Uw(a, e, kk) * (a.zeta[d.at(e + 1, kk)] + a.zeta[d.at(e, kk)]);
        } else {
            const T U = S.U[r][c + 1];
            const T* zr = &S.z[r + 2][c];   // zeta at fi-1 .. fi+2
            f = U * (zr[2] + zr[1]);
            if (fi >= 2 && fi <= d.nx - 3 && kk >= 2 && kk <= d.nz - 3) {
                const T Um = S.U[r][c], Up = S.U[r][c + 2];
                const T z0 = zr[0], z1 = zr[1], z2 = zr[2], z3 = zr[3];
                f += T(-1. / 3.) * (plus_part(U) * (z2 - z1) - sqrt(plus_part(U) * plus_part(Um)) * (z1 - z0) -
                                    minus_part(U) * (z2 - z1) - sqrt(fabs(minus_part(U) * minus_part(Up))) * (z3 - z2));
            }
        }
        S.fu[r][c] = f;
    }
    // z flux at face (i, fk+1/2), fk = 1..nz-2 (Advection.cpp:108,115-118)
    for (int t = tid; t < (BZ + 1) * BX; t += NT) {
        const int r = t / BX, c = t - r * BX;
        const int fk = k0 - 1 + r, ii = i0 + c;
        if (fk > d.nz - 2 || ii > d.nx - 2) continue;
        const T W = S.W[r + 1][c];
        const int zc = c + 2, zr = r + 1;   // zeta (ii, fk) in the staged tile
        T f = W * (S.z[zr + 1][zc] + S.z[zr][zc]);
        if (ii >= 2 && ii <= d.nx - 3 && fk >= 2 && fk <= d.nz - 3) {
            const T Wm = S.W[r][c], Wp = S.W[r + 2][c];
            const T z0 = S.z[zr - 1][zc], z1 = S.z[zr][zc], z2 = S.z[zr + 1][zc], z3 = S.z[zr + 2][zc];
            f += T(-1. / 3.) * (plus_part(W) * (z2 - z1) - sqrt(plus_part(W) * plus_part(Wm)) * (z1 - z0) -
                                minus_part(W) * (z2 - z1) - sqrt(fabs(minus_part(W) * minus_part(Wp))) * (z3 - z2));
        }
        S.fw[r][c] = f;
    }
    __syncthreads();
    if (!act) return;

    const size_t id = d.at(i, k);
    const T dt15 = T(1.5 * a.c.dt), dt05 = T(0.5 * a.c.dt);
    const T fu_i = S.fu[ty][tx + 1], fu_m = S.fu[ty][tx];
    const T fw_k = S.fw[ty + 1][tx], fw_m = S.fw[ty][tx];
    T rw = T(a.p.rhow[k]);
    T px = (fu_i - fu_m) * T(a.c.r2dx) / rw;
    T pz = (fw_k - fw_m) * T(a.p.r2dzw[k]) / rw;
    T tz = -px - pz;
    T oz = ab2_push(a.hz_n, a.hz_o, id, tz, a.ab);
    T zp = S.z[ty + 2][tx + 2] + dt15 * tz - dt05 * oz;
    // Bouyancy (Buoyancy.cpp:25-48); staged q[f][r][c] is (i0-1+c, k0-1+r)
    const int r1 = ty + 1, r0 = ty, c1 = tx + 1, c0 = tx;
    auto Q = [&](int f, int r, int c) { return S.q[f][r][c]; };
    T g_rw = T(a.c.gravity) / rw;
    T b;
    if constexpr (!kPert<T>) {
        auto thv = [&](int r, int c) { return Q(0, r, c) * (T(1) + T(0.608) * Q(1, r, c)); };   // Buoyancy.cpp:3-9
        b = g_rw * T(0.5) *
            ((thv(r1, c1) - thv(r1, c0)) / T(a.p.thvb[k]) + (thv(r0, c1) - thv(r0, c0)) / T(a.p.thvb[k - 1])) *
            T(a.c.rdx);
    } else {
        // thv(i) - thv(i-1) from perturbations th', qv' about th0(k), qv0(k):
        // dth' + 0.608 (th0 dqv' + qv0 dth' + (th'q')_i - (th'q')_{i-1}); the
        // large reference values never enter a difference
        auto thv_dx = [&](int r, int kk) {
            T t1 = Q(0, r, c1), t0 = Q(0, r, c0), q1 = Q(1, r, c1), q0 = Q(1, r, c0);
            T dt = t1 - t0, dq = q1 - q0;
            return dt + T(0.608) * (T(a.p.ref[0][kk]) * dq + T(a.p.ref[1][kk]) * dt + (t1 * q1 - t0 * q0));
        };
        b = g_rw * T(0.5) * (thv_dx(r1, k) / T(a.p.thvb[k]) + thv_dx(r0, k - 1) / T(a.p.thvb[k - 1])) * T(a.c.rdx);
    }
    T bc = g_rw * (T(0.5) * (Q(2, r1, c1) + Q(2, r0, c1)) - T(0.5) * (Q(2, r1, c0) + Q(2, r0, c0))) * T(a.c.rdx);
    T br = g_rw * (T(0.5) * (Q(3, r1, c1) + Q(3, r0, c1)) - T(0.5) * (Q(3, r1, c0) + Q(3, r0, c0))) * T(a.c.rdx);
    T tb = b + (-bc - br);
    T ob = ab2_push(a.hb_n, a.hb_o, id, tb, a.ab);
    zp += (dt15 * tb) - (dt05 * ob);
    store_westdown(a.zetap, d, i, k, zp);
}
template <typename T>
__global__ void __launch_bounds__(kPZBX * kPZBZ) k_pzeta(PZetaArgs<T> a) { k_pzeta_body<T>(a); }

// ---------------------------------------------------------------------------
// Scalar advection (Advection_thermo, Advection.cpp:25-81) of th, qv, qc, qr,
// rain sedimentation (Advection_qrVT, Advection.cpp:153-192), the surface
// precipitation diagnostic (Iteration.cpp:114-119) and the per-block partial
// sums of NegativeValueProcess (MicroPhysics.cpp:116-138). Writes the raw
// interior future values; k_apply finishes them. One thread per interior
// cell (i = 1..nx-2, k = 1..nz-2).

enum : int { F_TH = 1, F_QV = 2, F_QC = 4, F_QR = 8 };

template <typename T>
struct PAdvArgs {
    Dims d;
    Consts c;
    Profiles p;
    const T *u, *w;
    const T* now[4];   // th, qv, qc, qr
    T* fut[4];         // thp, qvp, qcp, qrp
    T* hn[4];          // d*_advect new slot
    T* ho[4];          // d*_advect old slot
    T *hvt_n, *hvt_o;  // dqr_VT
    T* precip;         // [nx]
    double* partial;   // [gridDim.x*gridDim.y][6]: (pos, neg) of qv, qc, qr
    int* err;          // device error word (kStageErrWait), may be null
    int mask;          // F_* fields to advect
    int nvp_mask;      // F_* fields whose NVP sums are wanted
    int do_vt;         // sedimentation of qr (with F_QR)
    int do_precip;     // surface rain diagnostic
    AB2 ab;
};

// The velocity part of one face's flux, shared by every advected field:
// flux = base (v0 + vm) - 1/3 (c1 (v0 - vm) - c2 (vm - vmm) - c3 (v0 - vm)
// - c4 (vp - v0)), the bracket only away from the boundaries (hi = 0 there).
// Each coefficient is formed exactly as the per-field expressions of
// Advection.cpp:40-50 form it.
template <typename T>
struct Face {
    T base, c1, c2, c3, c4;
    bool hi;
};

// x face (i-1/2, k), i = 1..nx-2 (Advection.cpp:36,40-44).
template <typename T>
__device__ __forceinline__ Face<T> face_u(const PAdvArgs<T>& a, int i, int k) {
    const Dims& d = a.d;
    Face<T> F;
    const T ru = T(a.p.rhou[k]);
    const T ui = a.u[d.at(i, k)];
    F.base = ru * ui;
    F.hi = (i >= 2 && i <= d.nx - 3 && k >= 2 && k <= d.nz - 3);
    F.c1 = F.c2 = F.c3 = F.c4 = T(0);
    if (F.hi) {
        const T um = a.u[d.at(i - 1, k)], up = a.u[d.at(i + 1, k)];
        F.c1 = ru * plus_part(ui);
        F.c2 = sqrt(ru * plus_part(ui) * ru * plus_part(um));
        F.c3 = ru * minus_part(ui);
        F.c4 = sqrt(fabs(ru * minus_part(ui) * ru * minus_part(up)));
    }
    return F;
}

// z face (i, k-1/2), k = 1..nz-2 (Advection.cpp:37,46-50).
template <typename T>
__device__ __forceinline__ Face<T> face_w(const PAdvArgs<T>& a, int i, int k) {
    const Dims& d = a.d;
    Face<T> F;
    const T rk = T(a.p.rhow[k]);
    const T wk = a.w[d.at(i, k)];
    F.base = rk * wk;
    F.hi = (i >= 2 && i <= d.nx - 3 && k >= 2 && k <= d.nz - 3);
    F.c1 = F.c2 = F.c3 = F.c4 = T(0);
    if (F.hi) {
        const T rkm = T(a.p.rhow[k - 1]), rkp = T(a.p.rhow[k + 1]);
        const T wm = a.w[d.at(i, k - 1)], wp = a.w[d.at(i, k + 1)];
        F.c1 = rk * plus_part(wk);
        F.c2 = sqrt(rk * plus_part(wk) * rkm * plus_part(wm));
        F.c3 = rk * minus_part(wk);
        F.c4 = sqrt(fabs(rk * minus_part(wk) * rkp * minus_part(wp)));
    }
    return F;
}

// Flux through a face from the field values vmm, vm | v0, vp across it.
template <typename T>
__device__ __forceinline__ T face_flux(const Face<T>& F, T vmm, T vm, T v0, T vp) {
    T f = F.base * (v0 + vm);
    if (F.hi) f += T(-1. / 3.) * (F.c1 * (v0 - vm) - F.c2 * (vm - vmm) - F.c3 * (v0 - vm) - F.c4 * (vp - v0));
    return f;
}

// The same with the third-order differences of a perturbation v' about a
// profile: dk = (v0 - vm) + d0[k] etc. (mixed step, z faces of th and qv).
template <typename T>
__device__ __forceinline__ T face_flux_pert(const Face<T>& F, T vmm, T vm, T v0, T vp, T dkm0, T dk0, T dkp0) {
    T f = F.base * (v0 + vm);
    if (F.hi) {
        const T dk = (v0 - vm) + dk0, dkm = (vm - vmm) + dkm0, dkp = (vp - v0) + dkp0;
        f += T(-1. / 3.) * (F.c1 * dk - F.c2 * dkm - F.c3 * dk - F.c4 * dkp);
    }
    return f;
}

// Sedimentation flux at (i, k-1/2), k = 1..nz-2 (Advection.cpp:165-166).
template <typename T>
__device__ __forceinline__ T vt_flux(const PAdvArgs<T>& a, const T* qr, int i, int k) {
    T s = qr[a.d.at(i, k)] + qr[a.d.at(i, k - 1)];
    T VT = T(1E-2) * (T(3634) * pow(T(a.p.vt_c1[k]) * s, T(0.1346)) * T(a.p.vt_fac[k]));
    return T(a.p.rhow[k]) * VT * s;
}

// Final sums of NegativeValueProcess and its rescaling factor
// (MicroPhysics.cpp:125-127): nvp[2f] = 1 if positives are rescaled,
// nvp[2f+1] = 1 - |neg/pos|. One block (k_nvp_final); fixed summation
// order. `sh`: 32 * 6 doubles. (Finishing the sums in the producer's last
// block instead costs every block of the producer a fence and an atomic
// before it retires, more than this launch.)
__device__ __forceinline__ void nvp_finish(const double* partial, int nblocks, double* nvp, double* sh) {
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.x + blockDim.x * threadIdx.y;
    double s[6] = {0, 0, 0, 0, 0, 0};
    // four partials a round in flight (a few round trips to L2, not one a partial)
    int b = tid;
    for (; b + 3 * nt < nblocks; b += 4 * nt) {
        double x[4][6];
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int j = 0; j < 6; j++) x[q][j] = __ldcg(partial + (size_t)(b + q * nt) * 6 + j);
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int j = 0; j < 6; j++) s[j] += x[q][j];
    }
    for (; b < nblocks; b += nt)
#pragma unroll
        for (int j = 0; j < 6; j++) s[j] += __ldcg(partial + (size_t)b * 6 + j);
    block_sum(s, sh);
    if (tid == 0) {
        for (int f = 0; f < 3; f++) {
            const double pos = s[2 * f], neg = s[2 * f + 1];
            const bool skip = (pos == 0. || fabs(neg) > pos);
            nvp[2 * f] = skip ? 0.0 : 1.0;
            nvp[2 * f + 1] = skip ? 1.0 : 1. - fabs(neg / pos);
        }
    }
}

__global__ void k_nvp_final(const double* partial, int nblocks, double* nvp);

// Tile of k_padv: 32 x 8 cells a block of 32 x 8 threads. The four fields
// are staged into shared memory with two halo cells a side (one TMA box a
// field, issued first); every face of the tile (33 x 8 x-faces, 32 x 9 z-faces) is then
// evaluated once, by one thread: its velocity part (in registers) once for
// all fields, its flux once per field and, for qr, its sedimentation flux,
// into shared memory; a cell differences the four fluxes around it. The expressions are the per-cell ones of
// Advection.cpp:36-58, so each cell's tendency is what a thread computing
// its own four faces would get, at about half the arithmetic (two square
// roots a face, one pow a sedimentation face) and with every stencil read
// from shared memory.
constexpr int kPAdvBX = 32, kPAdvBZ = 8;
constexpr int kStageErrWait = 4;   // device error word: a stencil's TMA staging wait gave up

// The staged box of one field: rows k0-2 .. k0+BZ+1 and 40 columns from x0,
// the halo's first column i0-2 rounded down to a 16-byte boundary (TMA
// requires x * element size to be a multiple of 16): x0 = i0-2 - kPAdvOff.
constexpr int kPAdvVX = 40, kPAdvVZ = kPAdvBZ + 4;
template <typename T>
constexpr int kPAdvOff = sizeof(T) == 8 ? 1 : 3;

template <typename T>
struct PAdvShared {
    static constexpr int BX = kPAdvBX, BZ = kPAdvBZ, VX = kPAdvVX, VZ = kPAdvVZ;
    T v[4][VZ][VX];           // th, qv, qc, qr: rows k0-2.., columns x0.. (each box a multiple of 128 bytes)
    T fx[4][BZ][BX + 1];      // x fluxes of each field
    T fz[4][BZ + 1][BX];      // z fluxes of each field
    T gz[BZ + 1][BX];         // sedimentation fluxes of qr
    double red[32 * 6];       // block_sum scratch
};

// Sedimentation flux from s = qr(k) + qr(k-1) at (i, k-1/2) (vt_flux's expression).
template <typename T>
__device__ __forceinline__ T vt_flux_s(const PAdvArgs<T>& a, T s, int k) {
    T VT = T(1E-2) * (T(3634) * pow(T(a.p.vt_c1[k]) * s, T(0.1346)) * T(a.p.vt_fac[k]));
    return T(a.p.rhow[k]) * VT * s;
}

// Dynamic shared memory: sizeof(PAdvShared<T>) (about 36 KB FP64, 19 KB
// mixed). At most 64 registers a thread, four blocks a SM (neither step
// spills). map[f]: the tensor map of a.now[f], box {kPAdvVX, kPAdvVZ}.
// The maps are read where they lie (a kernel parameter, or global memory
// for a grouped launch): TMA takes their addresses.
template <typename T>
__device__ __forceinline__ void k_padv_body(const CUtensorMap* m0, const CUtensorMap* m1, const CUtensorMap* m2,
                                            const CUtensorMap* m3, const PAdvArgs<T>& a) {
    constexpr int BX = kPAdvBX, BZ = kPAdvBZ, VX = kPAdvVX, VZ = kPAdvVZ, OFF = kPAdvOff<T>;
    extern __shared__ __align__(128) unsigned char padv_smem[];
    __shared__ uint64_t stage_bar;
    PAdvShared<T>& S = *reinterpret_cast<PAdvShared<T>*>(padv_smem);
    const Dims& d = a.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + BX * ty;
    const int i0 = 1 + blockIdx.x * BX, k0 = 1 + blockIdx.y * BZ;
    const int i = i0 + tx, k = k0 + ty;
    const bool act = (i <= d.nx - 2 && k <= d.nz - 2);

    // Stage the fields, one TMA box each: points outside the array read as
    // zero and are never used, since a face reads its outer neighbours only
    // where the third-order bracket applies (2 <= index <= n-3).
    const uint32_t bar = smem_u32(&stage_bar);
    if (tid == 0) mbar_init1(bar);
    __syncthreads();
    if (tid == 0) {
        const CUtensorMap* maps[4] = {m0, m1, m2, m3};
        uint32_t bytes = 0;
        for (int f = 0; f < 4; f++)
            if (a.mask & (1 << f)) bytes += VZ * VX * sizeof(T);
        mbar_expect_tx(bar, bytes);
        for (int f = 0; f < 4; f++)
            if (a.mask & (1 << f)) tma_load_2d(smem_u32(&S.v[f][0][0]), maps[f], i0 - 2 - OFF, k0 - 2, bar);
    }

    // Faces: x face (r, c) is fi = i0 + c, between cells fi-1 and fi, on row
    // k0 + r; the east face of cell nx-2 is the halo copy of face 1
    // (BoundaryProcess2D_center on flux_u, Advection.cpp:55). z face (r, c) is
    // fk = k0 + r, between cells fk-1 and fk, in column i0 + c; face nz-1
    // carries no flux (Advection.cpp:57-58).
    auto xface_ok = [&](int r, int c) { return k0 + r <= d.nz - 2 && i0 + c <= d.nx - 1; };
    auto zface_ok = [&](int r, int c) { return k0 + r <= d.nz - 2 && i0 + c <= d.nx - 2; };
    auto zflux_ok = [&](int r, int c) { return k0 + r <= d.nz - 1 && i0 + c <= d.nx - 2; };
    auto xface_i = [&](int c) { int fi = i0 + c; return fi == d.nx - 1 ? 1 : fi; };

    // velocity parts of the thread's own faces, its cell's west and bottom
    // ones, while the copies are in flight
    const bool xo = xface_ok(ty, tx), zo = zface_ok(ty, tx), zfo = zflux_ok(ty, tx);
    Face<T> Fx{}, Fz{};
    if (xo) Fx = face_u(a, xface_i(tx), k0 + ty);
    if (zo) Fz = face_w(a, i0 + tx, k0 + ty);
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {   // the copies never landed: report and leave
        if (tid == 0 && a.err) atomicOr(a.err, kStageErrWait);
        mbar_wait_bounded(bar, 0);
        return;
    }

    // staged column of index ii: ii - (i0 - 2) + OFF
    auto xflux = [&](const Face<T>& F, int f, int r, int c) {
        if (i0 + c == d.nx - 1) {   // face 1 (no bracket), read where it lies
            const T* v = a.now[f];
            return face_flux(F, T(0), v[d.at(0, k0 + r)], v[d.at(1, k0 + r)], T(0));
        }
        const T* row = &S.v[f][r + 2][c + OFF];   // columns fi-2 .. fi+1
        return face_flux(F, F.hi ? row[0] : T(0), row[1], row[2], F.hi ? row[3] : T(0));
    };
    // th and qv of the mixed step take the perturbation form (third-order
    // differences with the profile's d0)
    auto zflux = [&](const Face<T>& F, int f, int r, int c) {
        const int fk = k0 + r;
        if (fk == d.nz - 1) return T(0);
        const T vmm = S.v[f][r][c + 2 + OFF], vm = S.v[f][r + 1][c + 2 + OFF], v0 = S.v[f][r + 2][c + 2 + OFF],
                vp = S.v[f][r + 3][c + 2 + OFF];   // rows fk-2 .. fk+1
        if (kPert<T> && f < 2 && F.hi) {
            const double* d0 = a.p.d0[f];
            return face_flux_pert(F, vmm, vm, v0, vp, T(d0[fk - 1]), T(d0[fk]), T(d0[fk + 1]));
        }
        return face_flux(F, F.hi ? vmm : T(0), vm, v0, F.hi ? vp : T(0));
    };
    auto gflux = [&](int r, int c) {
        const int fk = k0 + r;
        return fk == d.nz - 1 ? T(0) : vt_flux_s(a, S.v[3][r + 2][c + 2 + OFF] + S.v[3][r + 1][c + 2 + OFF], fk);
    };

    const bool vt = (a.mask & F_QR) && a.do_vt;
    for (int f = 0; f < 4; f++) {
        if (!(a.mask & (1 << f))) continue;
        if (xo) S.fx[f][ty][tx] = xflux(Fx, f, ty, tx);
        if (zfo) S.fz[f][ty][tx] = zflux(Fz, f, ty, tx);
    }
    if (vt && zfo) S.gz[ty][tx] = gflux(ty, tx);
    // the tile's east column of x faces (warp 0, lanes 0..7, one a row) and
    // its top row of z faces (warp 1)
    if (ty == 0 && tx < BZ && xface_ok(tx, BX)) {
        const Face<T> F = face_u(a, xface_i(BX), k0 + tx);
        for (int f = 0; f < 4; f++)
            if (a.mask & (1 << f)) S.fx[f][tx][BX] = xflux(F, f, tx, BX);
    }
    if (ty == 1 && zflux_ok(BZ, tx)) {
        Face<T> F{};
        if (zface_ok(BZ, tx)) F = face_w(a, i0 + tx, k0 + BZ);
        for (int f = 0; f < 4; f++)
            if (a.mask & (1 << f)) S.fz[f][BZ][tx] = zflux(F, f, BZ, tx);
        if (vt) S.gz[BZ][tx] = gflux(BZ, tx);
    }
    __syncthreads();

    double sums[6] = {0, 0, 0, 0, 0, 0};
    if (act) {
        const size_t id = d.at(i, k);
        const T dt15 = T(1.5 * a.c.dt), dt05 = T(0.5 * a.c.dt);
        const T ru = T(a.p.rhou[k]);
        // mixed step: one division for the cell's flux divergences (the FP64
        // step keeps the reference's (difference * r2d) / rhou per term)
        const T sx = kPert<T> ? T(a.c.r2dx) / ru : T(0), sz = kPert<T> ? T(a.p.r2dzc[k]) / ru : T(0);
        const int ip = (i == d.nx - 2) ? 1 : i + 1;
        const bool top = (k == d.nz - 2);
        for (int f = 0; f < 4; f++) {
            if (!(a.mask & (1 << f))) continue;
            const T fu_0 = S.fx[f][ty][tx], fu_p = S.fx[f][ty][tx + 1];
            const T fw_0 = S.fz[f][ty][tx], fw_p = S.fz[f][ty + 1][tx];
            T px, pz;
            if (!kPert<T> || f >= 2) {
                if constexpr (kPert<T>) {
                    px = (fu_p - fu_0) * sx;
                    pz = (fw_p - fw_0) * sz;
                } else {
                    px = (fu_p - fu_0) * T(a.c.r2dx) / ru;
                    pz = (fw_p - fw_0) * T(a.p.r2dzc[k]) / ru;
                }
            } else {
                // v = v0(k) + v': the v0 parts of both fluxes are added in
                // difference form, 2 v0 (u[i+1] - u[i]) in x and
                // s0[k+1] (m[k+1] - m[k]) + m[k] g0[k] in z, m = rhow w.
                T m0 = T(a.p.rhow[k]) * a.w[d.at(i, k)];
                T refz = top ? -m0 * T(a.p.s0[f][k])
                             : T(a.p.s0[f][k + 1]) * (T(a.p.rhow[k + 1]) * a.w[d.at(i, k + 1)] - m0) +
                                   m0 * T(a.p.g0[f][k]);
                T refx = T(2.0 * a.p.ref[f][k]) * (a.u[d.at(ip, k)] - a.u[d.at(i, k)]);
                px = (fu_p - fu_0) * sx + refx * T(a.c.r2dx);
                pz = (fw_p - fw_0 + refz) * sz;
            }
            T t = -px - pz;
            T o = ab2_push(a.hn[f], a.ho[f], id, t, a.ab);
            T out = S.v[f][ty + 2][tx + 2 + OFF] + dt15 * t - dt05 * o;
            if (f == 3 && vt) {
                const T gp = S.gz[ty + 1][tx], g0 = S.gz[ty][tx];
                T tv = kPert<T> ? (gp - g0) * sz : (gp - g0) * T(a.p.r2dzc[k]) / ru;
                T ov = ab2_push(a.hvt_n, a.hvt_o, id, tv, a.ab);
                out += dt15 * tv - dt05 * ov;
            }
            a.fut[f][id] = out;
            if (f >= 1 && (a.nvp_mask & (1 << f))) {
                double full = (double)out;
                if (kPert<T> && f == 1) full += a.p.ref[1][k];
                if (full >= 0.0) sums[2 * (f - 1)] += full;
                else sums[2 * (f - 1) + 1] += full;
            }
        }
        if (a.do_precip && k == 1) {
            const T* qr = a.now[3];
            T q1 = qr[d.at(i, 1)];
            T VT = T(1E-2) * (T(3634) * pow(T(a.p.pf1) * q1, T(0.1346)) * T(a.p.pf2));
            T rain = -T(a.p.rhou[1]) * (T(0.5) * (a.w[d.at(i, 2)] + T(0)) - VT) * q1;
            a.precip[i] = (rain < T(0)) ? T(0) : rain;
        }
    }
    if (a.nvp_mask) {
        block_sum(sums, S.red);
        if (tid == 0) {
            double* out = a.partial + (size_t)(blockIdx.x + gridDim.x * blockIdx.y) * 6;
#pragma unroll
            for (int j = 0; j < 6; j++) out[j] = sums[j];
        }
    }
}
template <typename T>
__global__ void __launch_bounds__(kPAdvBX * kPAdvBZ, 4)
    k_padv(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
           const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap m3, PAdvArgs<T> a) {
    k_padv_body<T>(&m0, &m1, &m2, &m3, a);
}

// ---------------------------------------------------------------------------
// Finishes th, qv, qc, qr after advection or microphysics: the rescaling of
// NegativeValueProcess, AddForcing (AddForcing.cpp:6-28) and the
// BoundaryProcess2D_center halo. One thread per interior cell.

template <typename T>
struct ApplyArgs {
    Dims d;
    Consts c;
    Profiles p;
    T* fut[4];               // thp, qvp, qcp, qrp (in place)
    const double* nvp;       // [6] from k_nvp_final
    const T* th_forcing;     // init_th_forcing (may be null)
    int mask;                // fields to finish
    int nvp_mask;            // fields to clip/rescale
    int forcing;             // add Q1LS/Q2LS
    int forcing_th;          // add dt*init_th_forcing (status_for_adding_forcing)
    int halo;                // write ghost images
};

template <typename T>
__device__ __forceinline__ T nvp_apply(T v, const double* nvp, int f) {
    if (!(v >= T(0))) return T(0);                        // MicroPhysics.cpp:121-122
    if (nvp[2 * f] != 0.0 && v > T(0)) return v * T(nvp[2 * f + 1]);   // MicroPhysics.cpp:130
    return v;
}

// What k_apply does to one value of field f at (id, row k): the rescaling of
// NegativeValueProcess, then AddForcing. Shared with the fused form at the
// top of k_kessler, so both give the same bits.
template <typename T>
struct AdvFinish {
    const double* nvp;       // [6] from k_nvp_final
    const T* th_forcing;     // init_th_forcing (may be null)
    int nvp_mask;            // fields to clip/rescale
    int forcing;             // add Q1LS/Q2LS
    int forcing_th;          // add dt*init_th_forcing
};

template <typename T>
__device__ __forceinline__ T finish_value(const AdvFinish<T>& a, const Profiles& p, T dt, int f, T v, int k,
                                          size_t id) {
    if (f >= 1 && (a.nvp_mask & (1 << f))) {
        if (kPert<T> && f == 1) {   // NegativeValueProcess acts on the full qv
            double full = p.ref[1][k] + (double)v;
            v = T(nvp_apply(full, a.nvp, 0) - p.ref[1][k]);
        } else {
            v = nvp_apply(v, a.nvp, f - 1);
        }
    }
    if (f == 0) {
        if (a.forcing) v += dt * T(p.q1ls[k]);
        if (a.forcing_th) v += dt * a.th_forcing[id];
    }
    if (f == 1 && a.forcing) v += dt * T(p.q2ls[k]);
    return v;
}

template <typename T>
__device__ __forceinline__ void k_apply_body(const ApplyArgs<T>& a) {
    const Dims& d = a.d;
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx - 2 || k > d.nz - 2) return;
    const size_t id = d.at(i, k);
    const T dt = T(a.c.dt);
    const AdvFinish<T> fin{a.nvp, a.th_forcing, a.nvp_mask, a.forcing, a.forcing_th};
    for (int f = 0; f < 4; f++) {
        if (!(a.mask & (1 << f))) continue;
        const T v = finish_value(fin, a.p, dt, f, a.fut[f][id], k, id);
        if (a.halo) store_center(a.fut[f], d, i, k, v);
        else a.fut[f][id] = v;
    }
}
template <typename T>
__global__ void k_apply(ApplyArgs<T> a) { k_apply_body<T>(a); }

// ---------------------------------------------------------------------------
// BoundaryProcess2D_all (Boundary.cpp:32-52) as a standalone pass.

template <typename T>
struct HaloArgs {
    Dims d;
    T *zetap, *w;        // westdown
    T* center[5];        // thp, u, qvp, qcp, qrp
};

template <typename T>
__global__ void k_halo_all(HaloArgs<T> a) {
    const Dims& d = a.d;
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx - 2 || k > d.nz - 2) return;
    const size_t id = d.at(i, k);
    if (k >= 2) {
        store_westdown(a.zetap, d, i, k, a.zetap[id]);
        store_westdown(a.w, d, i, k, a.w[id]);
    }
#pragma unroll
    for (int f = 0; f < 5; f++) store_center(a.center[f], d, i, k, a.center[f][id]);
}

// ---------------------------------------------------------------------------
// Kessler warm rain, applied cell by cell in the reference's order:
// autoconversion (MicroPhysics.cpp:29-51), accretion (:54-77), evaporation
// (:80-114), saturation adjustment (:7-26); then the NVP partial sums of qvp,
// qcp, qrp. One thread per interior cell.

template <typename T>
struct KesslerArgs {
    Dims d;
    Consts c;
    Profiles p;
    T *thp, *qvp, *qcp, *qrp;
    T *d_auto, *d_accr, *d_evap, *d_cond;  // diagnostics (may be null)
    double* partial;
    int nvp;  // accumulate NVP sums
    // The finish of the advection step (k_apply's rescaling and forcing of
    // th, qv, qc, qr) applied to each value as it is read, in place of a
    // k_apply launch whose halo images the apply after Kessler rewrites.
    AdvFinish<T> pre;
    int do_pre;
};

// One cell of Kessler warm rain in compute type C; writes the four rates.
template <typename C>
__device__ __forceinline__ void kessler_cell(C& th, C& qv, C& qc, C& qr, C dt, C lv, C cp, C pib, C rhou,
                                             C pc, C pb, C rates[4]) {
    {   // autoconversion
        C qcplus = smax(C(0), qc);
        C ar = C(0.001) * (qcplus - C(0.001));
        ar = smax(C(0), ar);
        C arcrdt = smin(ar * dt, qcplus);
        qc = qc - arcrdt;
        qr = qr + arcrdt;
        rates[0] = arcrdt;
    }
    {   // accretion
        C qcplus = smax(C(0), qc), qrplus = smax(C(0), qr);
        C cr = C(2.2) * qcplus * (pow(qrplus, C(0.875)));
        C arcrdt = smin(cr * dt, qcplus);
        qc = qc - arcrdt;
        qr = qr + arcrdt;
        rates[1] = arcrdt;
    }
    {   // evaporation of rain
        C qrplus = smax(C(0), qr), qvplus = smax(C(0), qv);
        C qvs = pc * exp(C(17.27) * (pib * th - C(273.)) / (pib * th - C(36.)));
        C deficit = smax((C(1.) - qvplus / qvs), C(0.));
        C coef = C(1.6) + C(124.9) * pow((C(1E-3) * rhou * qrplus), C(0.2046));
        C er = coef * deficit * (pow(C(1E-3) * rhou * qrplus, C(0.525))) /
               ((C(5.4E5) + C(2.55E6) / (C(1E-2) * pb * qvs)) * C(1E-3) * rhou);
        C erdt = smin(qrplus, smax(C(0.), er * dt));
        qr = qr - erdt;
        qv = qv + erdt;
        th = th - lv * erdt / (cp * pib);
        rates[2] = erdt;
    }
    {   // saturation adjustment
        C qvs = pc * exp(C(17.27) * (pib * th - C(273.)) / (pib * th - C(36.)));
        C tm = th * pib - C(36.);
        C phi = qvs * (C(17.27) * C(237.) * lv) / (cp * (tm * tm));
        C cnd = (qv - qvs) / (C(1) + phi);
        if (fabs(cnd) > qc && cnd < C(0)) cnd = -qc;
        qv = qv - cnd;
        qc = qc + cnd;
        th = th + lv / (cp * pib) * cnd;
        rates[3] = cnd;
    }
}

// The mixed step runs this kernel's arithmetic in FP64 on its FP32 storage:
// the saturation adjustment subtracts qvs from qv, which cancel to a few
// units of the FP32 epsilon near saturation.
template <typename T>
__device__ __forceinline__ void k_kessler_body(const KesslerArgs<T>& a) {
    using C = double;
    __shared__ double sh[32 * 6];
    const Dims& d = a.d;
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const bool act = (i <= d.nx - 2 && k <= d.nz - 2);
    double sums[6] = {0, 0, 0, 0, 0, 0};
    if (act) {
        const size_t id = d.at(i, k);
        const C th0 = kPert<T> ? a.p.ref[0][k] : 0.0, qv0 = kPert<T> ? a.p.ref[1][k] : 0.0;
        T tv = a.thp[id], qvv = a.qvp[id], qcv = a.qcp[id], qrv = a.qrp[id];
        if (a.do_pre) {
            const T dt = T(a.c.dt);
            tv = finish_value(a.pre, a.p, dt, 0, tv, k, id);
            qvv = finish_value(a.pre, a.p, dt, 1, qvv, k, id);
            qcv = finish_value(a.pre, a.p, dt, 2, qcv, k, id);
            qrv = finish_value(a.pre, a.p, dt, 3, qrv, k, id);
        }
        C th = th0 + (C)tv, qv = qv0 + (C)qvv, qc = qcv, qr = qrv;
        C rates[4];
        kessler_cell<C>(th, qv, qc, qr, a.c.dt, a.c.lv, a.c.cp, a.p.pib[k], a.p.rhou[k], a.p.pc[k], a.p.pb[k],
                        rates);
        if (a.d_auto) {
            a.d_auto[id] = T(rates[0]);
            a.d_accr[id] = T(rates[1]);
            a.d_evap[id] = T(rates[2]);
            a.d_cond[id] = T(rates[3]);
        }
        a.thp[id] = T(th - th0);
        a.qvp[id] = T(qv - qv0);
        a.qcp[id] = T(qc);
        a.qrp[id] = T(qr);
        if (a.nvp) {
            C q[3] = {qv, qc, qr};
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (q[f] >= C(0)) sums[2 * f] += (double)q[f];
                else sums[2 * f + 1] += (double)q[f];
            }
        }
    }
    if (a.nvp) {
        block_sum(sums, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            double* out = a.partial + (size_t)(blockIdx.x + gridDim.x * blockIdx.y) * 6;
#pragma unroll
            for (int j = 0; j < 6; j++) out[j] = sums[j];
        }
    }
}
template <typename T>
__global__ void k_kessler(KesslerArgs<T> a) { k_kessler_body<T>(a); }

// ---------------------------------------------------------------------------
// Eddy coefficients (Turbulence::RKM_RKH, Turbulent.cpp:5-45) with their
// center halo. One thread per interior cell.

template <typename T>
struct RKArgs {
    Dims d;
    Consts c;
    Profiles p;
    const T *u, *w, *thp;
    T *RKM, *RKH;
};

template <typename T>
__device__ __forceinline__ void k_rkm_rkh_body(const RKArgs<T>& a) {
    const Dims& d = a.d;
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx - 2 || k > d.nz - 2) return;
    const T* u = a.u;
    const T* w = a.w;
    T Rzeta = T(0.5) * ((w[d.at(i + 1, k + 1)] + w[d.at(i + 1, k)]) - (w[d.at(i - 1, k + 1)] + w[d.at(i - 1, k)])) * T(a.c.r2dx) +
              T(0.5) * ((u[d.at(i + 1, k + 1)] + u[d.at(i, k + 1)]) - (u[d.at(i + 1, k - 1)] + u[d.at(i, k - 1)])) * T(a.p.r2dzcc[k]);
    T rot = (u[d.at(i + 1, k)] - u[d.at(i, k)]) * T(a.c.rdx) + (w[d.at(i, k + 1)] - w[d.at(i, k)]) * T(a.p.rdzc[k]);
    T Rotat = rot * rot;
    T th0 = a.thp[d.at(i, k)];
    T dth = a.thp[d.at(i, k + 1)] - a.thp[d.at(i, k - 1)];
    if constexpr (kPert<T>) {       // perturbation storage: add the profile parts
        th0 += T(a.p.ref[0][k]);
        dth += T(a.p.g0[0][k]);
    }
    T def2 = Rzeta * Rzeta + T(2.) * Rotat;
    T Ri = (T(a.c.gravity) / th0 * dth * T(a.p.r2dzcc[k])) / def2;
    T lam = T(a.p.lambda2[k]);
    T km, kh;
    if (Ri < T(0)) {
        km = lam * sqrt(def2) * sqrt(T(1.) - T(16.) * Ri);
        kh = lam * sqrt(def2) * T(1.4) * sqrt(T(1.) - T(40.) * Ri);
    } else if (T(0) < Ri && Ri < T(0.25)) {
        km = lam * sqrt(def2) * pow(T(1.) - T(4.) * Ri, T(4));
        kh = lam * sqrt(def2) * T(1.4) * (T(1.) - T(1.2) * Ri) * pow(T(1.) - T(4.) * Ri, T(4));
    } else {
        km = T(0.);
        kh = T(0.);
    }
    const T kmax = T(a.p.kmax[k]);
    km = smax(km, T(10.));
    kh = smax(kh, T(10.));
    km = smin(km, kmax);
    kh = smin(kh, kmax);
    store_center(a.RKM, d, i, k, km);
    store_center(a.RKH, d, i, k, kh);
}
template <typename T>
__global__ void k_rkm_rkh(RKArgs<T> a) { k_rkm_rkh_body<T>(a); }

// ---------------------------------------------------------------------------
// In-place Gauss-Seidel diffusion (Turbulence::Mparam / Hparam,
// Turbulent.cpp:68-114), exact to round-off, with the top-layer nudging of
// theta and zeta fused in (NumericalProcess.cpp:60-85).
//
// The reference sweeps k outer, i inner and reads the already-updated left
// (i-1) and lower (k-1) neighbours, so cell (i, k) obeys
//   v'(i,k) = A0(i,k) + C(i,k) v'(i,k-1) + B(i,k) v'(i-1,k),
// where A0, C and B depend on old values only: B is the left-face
// coefficient, C the lower-face one, A0 collects the rest.
//
// The recurrence is lower triangular in (k, i): a cell depends on the cells
// left of it in its row and below it in its column. The padded rows are cut
// into tiles of tr rows (from k = 1) by 128 columns (from i = 0), one warp a
// tile, 4 cells a lane. A pass computes every tile at once from inflows left
// by the previous pass: the value left of each of its rows (the right outflow
// of the tile on its left) and the row below it (the top outflow of the tile
// below). Inside a tile each row is exact: a scan over the warp of the affine
// maps y_i = a_i + B_i y_{i-1}, a_i = A0 + C x (x the value below), the
// lanes' maps composed with shuffles, then applied cell by cell from the
// inflow.
//
// A tile's outputs are final once its inflows are, so the tiles of the d-th
// anti-diagonal (b + c = d) are final after pass d + 1, and nb + nc - 1 passes
// reproduce the sequential sweep over the tiles. The passes stop earlier, as
// soon as no outflow that another tile reads changed bit for bit from one
// pass to the next: the following pass would then read the same inflows and
// repeat every value, so that is the fixed point the full count reaches. With
// diffusion coefficients of a step (B, C ~ dt K / dx^2, 1e-3 for the minimum
// K = 10 m^2/s at dx = 100 m) an inflow error shrinks about a thousandfold a
// pass; three passes are typical.
//
// Pass 1 reads the old values: it forms A0 from them and stores it, takes
// its inflows from them (the guess), and writes no field, so every tile of it
// reads the old state. Passes 2 on read A0, form B and C from the eddy
// coefficients (which no pass changes) and write the field; at least two
// passes run.
//
// Buffers (parity q = pass & 1 written by a pass, q ^ 1 read):
//   right[q][f][b][c][r]   y at the tile's last column, rows r = 0..tr-1
//   top[q][f][b][c][col]   y of the tile's top row, col = 0..127
// The last block of a pass (a thread-fence and counter, no waiting) decides
// whether another pass follows, and sets the condition of the graph's WHILE
// node when the passes run in a graph; the last pass of a sweep resets the
// pass state for the next one (the host also clears it before each sweep). A
// later pass launched after the sweep converged returns at once, so a graph
// runs the typical count unconditionally and enters its WHILE node only when
// more passes are needed.

template <typename T>
struct GSArgs {
    Dims d;
    Consts c;
    Profiles p;
    T* v[5];          // zetap (Mparam, RKM), thp, qvp, qcp, qrp (Hparam, RKH)
    const T *RKM, *RKH;
    int mask;         // bit f: diffuse field f
    int nudge;        // fuse Nudge_theta (field 1) and Nudge_zeta (field 0)
    T* A0;            // per-cell constant term, [5][cells] (written by pass 1 / k_gs_coeffs)
    T *C, *B;         // per-cell lower and left coefficients (the cluster schedule only)
    int* err;         // device error word (kGSErrWait, the cluster schedule), may be null
};

constexpr int kGSMaxNX = 8192;
constexpr int kGSMaxPerThread = 8;      // cells a thread of the cal_u column integral

constexpr int kGTCols = 128;   // columns of a tile: 32 lanes x 4 cells
constexpr int kGTPer = 4;
// Rows of a tile: the autotuner's knob (the passes a sweep needs do not
// depend on it; taller tiles mean fewer, longer tiles a pass).
constexpr int kGSTileRowsMin = 4, kGSTileRowsMax = 32, kGSTileRowsDefault = 8;
constexpr int kGSRowVals = 9;   // scalars a tile row keeps in shared memory
inline bool gs_tile_rows_ok(int tr) { return tr == 4 || tr == 8 || tr == 16 || tr == 32; }
// Blocks a SM the tile kernel is compiled for: three in FP64 (up to 168
// registers a thread: pass 1 then keeps its rolling windows without spilling;
// the 1360 tiles of the 2048 x 256 default still fit in one wave), four in
// FP32.
template <typename T>
constexpr int kGSTileMinBlocks = sizeof(T) == 8 ? 3 : 4;

struct GSTileCtl {    // zeroed before a sweep
    int pass;         // passes of the sweep completed
    int changed[2];   // by parity of the pass that wrote an outflow differing from its previous one
    int done;         // blocks of the current pass that finished
    int more;         // another pass follows (read by the host loop)
    int passes;       // passes run by the last sweep
};

template <typename T>
struct GSTileArgs {
    int nb, nc, tr;   // bands of tr rows from k = 1, chunks of 128 columns from i = 0
    T* right;         // [2][5][nb][nc][tr]
    T* top;           // [2][5][nb][nc][128]
    GSTileCtl* ctl;
    long long* exec;  // kernels run inside graph loops (counted by the deciding block)
    __device__ __forceinline__ size_t ri(int q, int f, int b, int c) const {
        return ((((size_t)q * 5 + f) * nb + b) * nc + c) * tr;
    }
    __device__ __forceinline__ size_t ti(int q, int f, int b, int c) const {
        return ((((size_t)q * 5 + f) * nb + b) * nc + c) * kGTCols;
    }
};

// 4 consecutive cells of one row (16-byte aligned: i a multiple of 4, rows of
// a multiple of 32 cells).
template <typename T>
__device__ __forceinline__ void gs_ld4(const T* p, T (&x)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 u = __ldg(reinterpret_cast<const float4*>(p));
        x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w;
    } else {
        const double2 u = __ldg(reinterpret_cast<const double2*>(p)), w = __ldg(reinterpret_cast<const double2*>(p) + 1);
        x[0] = u.x, x[1] = u.y, x[2] = w.x, x[3] = w.y;
    }
}

// One pass over every tile: 4 warps (tiles) a block. Each lane keeps its
// cells' rows of K (k-1, k and, in pass 1, k+1) and, in pass 1, of the old
// field (k, k+1) in registers, rolled up a row at a time; the next row's
// loads are issued before the current row's scan. Left and right neighbours
// come from the adjacent lane by shuffle (the tile's edge lanes load theirs).
// B, C (and in pass 1 A0) follow Turbulent.cpp:83-88 for zeta and :107-112
// for the scalars term by term. The ghost i = 0 gets the constant map
// v'(0, k) = v(0, k) (never updated), cells beyond NX the identity map, so a
// row's scan needs no edge cases. Stores the nudged values (Nudge_zeta,
// Nudge_theta) of interior cells, carries the un-nudged ones.
// FIRST: pass 1 (launched on its own, before the loop of the later passes).
template <typename T, bool FIRST>
__device__ __forceinline__ void k_gs_tiles_body(const GSArgs<T>& a, const GSTileArgs<T>& t, cudaGraphConditionalHandle h) {
    __shared__ int any_changed;
    // per warp and row of its tile: cz, the czd and czu density factors,
    // nudging dn and tn, the inflow left of the row and its previous value,
    // and (pass 1, th' and qv') the profile differences at k and k+1
    __shared__ T rowv[4][kGSTileRowsMax][kGSRowVals];
    const Dims& d = a.d;
    const int NX = d.nx - 2, kend = d.nz - 2;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) any_changed = 0;
    __syncthreads();
    constexpr bool first = FIRST;
    // a pass launched after the sweep converged has nothing to do
    if (!FIRST && !*(volatile int*)&t.ctl->more) return;
    const int pass = FIRST ? 1 : t.ctl->pass + 1;
    const int q = pass & 1, qp = q ^ 1;
    const int tile = blockIdx.x * 4 + wid;
    const int ntiles = 5 * t.nb * t.nc;
    const int c = tile % t.nc, b = (tile / t.nc) % t.nb, f = tile / (t.nc * t.nb);
    if (tile < ntiles && (a.mask & (1 << f))) {   // uniform over the warp
        T* v = a.v[f];
        const bool mom = (f == 0);
        const T* K = mom ? a.RKM : a.RKH;
        T* A0s = a.A0 + (size_t)f * d.cells();
        const int i0 = c * kGTCols + lane * kGTPer;
        const bool act = i0 < d.pitch;   // pitch is a multiple of 32, so of kGTPer
        const int k0 = 1 + b * t.tr;
        const int rows = min(t.tr, kend - k0 + 1);
        const int ilast = c * kGTCols + kGTCols - 1;   // the tile's last column
        const bool edge_l = (lane == 0 && i0 >= 1);             // its left neighbour is in another tile
        const bool edge_r = (lane == 31 && act && i0 + 3 <= NX); // its right neighbour is needed
        const T cx = T(a.c.rdx2 * a.c.dt);
        const bool pert = kPert<T> && (f == 1 || f == 2);
        auto row4 = [&](const T* base, int k, T (&x)[4]) {
            if (act) gs_ld4(base + d.at(i0, k), x);
            else x[0] = x[1] = x[2] = x[3] = T(0);
        };
        bool diff = false;
        // the row below the tile: the old row 0 (never updated), or the top
        // outflow of the tile below (pass 1: the old values there)
        T below[kGTPer];
        if (b == 0 || first) {
            row4(v, k0 - 1, below);
            if (b == 0) {
#pragma unroll
                for (int e = 0; e < kGTPer; e++)
                    if (!(i0 + e >= 1 && i0 + e <= NX)) below[e] = T(0);
            }
        } else {
#pragma unroll
            for (int e = 0; e < kGTPer; e++) below[e] = t.top[t.ti(qp, f, b - 1, c) + lane * kGTPer + e];
        }
        // rolling windows: K rows k-1 (Kd), k (Kc), k+1 (Ku); old field rows k (v0), k+1 (vu)
        T Kd[4], Kc[4], Ku[4], v0[4], vu[4], An[4];
        row4(K, k0 - 1, Kd);
        row4(K, k0, Kc);
        if (first) {
            row4(K, k0 + 1, Ku);
            row4(v, k0, v0);
            row4(v, k0 + 1, vu);
        } else {
            row4(A0s, k0, An);
        }
        // the edge lanes' neighbours in the next tiles, a row ahead as well:
        // lane 0 K(i0-1, k) (and, rolled, K(i0-1, k-1)); lane 31 in pass 1
        // K(i0+4, k) and v(i0+4, k)
        T eKl = T(0), eKld = T(0), eKr = T(0), evr = T(0);
        if (edge_l) {
            eKl = K[d.at(i0 - 1, k0)];
            eKld = K[d.at(i0 - 1, k0 - 1)];
        }
        if (first && edge_r) {
            eKr = K[d.at(i0 + 4, k0)];
            evr = v[d.at(i0 + 4, k0)];
        }
        const T* rin = t.right + t.ri(qp, f, b, c - 1);   // read only when c > 0
        T* rout = t.right + t.ri(q, f, b, c);
        const T* rold = t.right + t.ri(qp, f, b, c);
        // the rows' scalars, one lane a row, all loads at once
        if (lane < rows) {
            const int k = k0 + lane;
            T* rv = rowv[wid][lane];
            if (mom) {
                rv[0] = T(a.p.gsM_cz[k]);
                rv[1] = T(a.p.gsM_rhod[k]);
                rv[2] = T(a.p.rhou[k]);
            } else {
                rv[0] = T(a.p.gsS_cz[k]);
                rv[1] = T(a.p.gsS_rhod[k]);
                rv[2] = T(a.p.rhow[k + 1]);
            }
            T dn = T(0), tn = T(0);   // nudging of row k: out = y - dn (y - tn)
            if (a.nudge && f == 0) dn = T(a.p.dtcgr_zeta[k]);
            if (a.nudge && f == 1) {
                dn = T(a.p.dtcgr_th[k]);
                tn = kPert<T> ? T(-a.p.dn[0][k]) : T(a.p.thb_init[k]);
            }
            rv[3] = dn;
            rv[4] = tn;
            rv[5] = (c > 0) ? (first ? v[d.at(c * kGTCols - 1, k)] : rin[lane]) : T(0);
            rv[6] = (c + 1 < t.nc) ? (first ? v[d.at(ilast, k)] : rold[lane]) : T(0);
            if (first && pert) {
                rv[7] = T(a.p.d0[f - 1][k]);
                rv[8] = T(a.p.d0[f - 1][k + 1]);
            }
        }
        __syncwarp();
        for (int r = 0; r < rows; r++) {
            const T* rv = rowv[wid][r];
            const int k = k0 + r;
            const bool more_rows = r + 1 < rows;
            // the next row's loads, in flight during this row's work
            T Kn[4], vn[4], An2[4];
            T eKl_n = T(0), eKr_n = T(0), evr_n = T(0);
            if (more_rows) {
                if (first) {
                    row4(K, k + 2, Kn);
                    row4(v, k + 2, vn);
                } else {
                    row4(K, k + 1, Kn);
                    row4(A0s, k + 1, An2);
                }
                if (edge_l) eKl_n = K[d.at(i0 - 1, k + 1)];
                if (first && edge_r) {
                    eKr_n = K[d.at(i0 + 4, k + 1)];
                    evr_n = v[d.at(i0 + 4, k + 1)];
                }
            }
            // neighbours across lanes (the edge lanes' from the next tiles)
            T Kl0 = __shfl_up_sync(0xffffffffu, Kc[3], 1);
            T Kld0 = __shfl_up_sync(0xffffffffu, Kd[3], 1);
            T Kr3 = __shfl_down_sync(0xffffffffu, Kc[0], 1);
            T vr3 = __shfl_down_sync(0xffffffffu, first ? v0[0] : T(0), 1);
            if (edge_l) {
                Kl0 = eKl;
                Kld0 = eKld;
            }
            if (first && edge_r) {
                Kr3 = eKr;
                vr3 = evr;
            }
            const T cz = rv[0], rhod = rv[1], rhou_ = rv[2];
            T aa[kGTPer], bb[kGTPer];
#pragma unroll
            for (int e = 0; e < kGTPer; e++) {
                const int i = i0 + e;
                T A0, B, C;
                if (!act || i > NX) {          // beyond NX: identity
                    A0 = T(0);
                    B = T(1);
                    C = T(0);
                } else if (i == 0) {           // the ghost: constant map
                    A0 = first ? v0[0] : An[0];
                    B = T(0);
                    C = T(0);
                } else {
                    const T Kl = (e == 0) ? Kl0 : Kc[e - 1];
                    T ax = T(0), bx, czu = T(0), czd;
                    if (mom) {
                        const T Kld = (e == 0) ? Kld0 : Kd[e - 1];
                        bx = T(0.5) * (Kl + Kld);
                        czd = rhod * T(0.5) * (Kd[e] + Kld);
                        if (first) {
                            ax = T(0.5) * (Kc[e] + Kd[e]);
                            czu = rhou_ * T(0.5) * (Kc[e] + Kl);
                        }
                    } else {
                        bx = T(0.5) * (Kc[e] + Kl);
                        czd = rhod * T(0.5) * (Kc[e] + Kd[e]);
                        if (first) {
                            const T Kr = (e == 3) ? Kr3 : Kc[e + 1];
                            ax = T(0.5) * (Kr + Kc[e]);
                            czu = rhou_ * T(0.5) * (Ku[e] + Kc[e]);
                        }
                    }
                    C = cz * czd;
                    B = cx * bx;
                    if (first) {
                        const T vc = v0[e], vr = (e == 3) ? vr3 : v0[e + 1];
                        T du = vu[e] - vc, dd = vc;
                        if (pert) {   // th', qv' about a profile
                            du += rv[8];
                            dd += rv[7];
                        }
                        // v + cx (ax (vr - v) - bx (v - v'[i-1])) + cz (czu du - czd (dd - v'below))
                        A0 = vc + cx * (ax * (vr - vc) - bx * vc) + cz * (czu * du - czd * dd);
                    } else {
                        A0 = An[e];
                    }
                }
                if (first && act) A0s[d.at(i0, k) + e] = A0;
                aa[e] = A0 + C * below[e];
                bb[e] = B;
            }
            // the lane's map over its cells: y_out = P + M y_in
            T P = T(0), M = T(1);
#pragma unroll
            for (int e = 0; e < kGTPer; e++) {
                P = aa[e] + bb[e] * P;
                M = bb[e] * M;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {   // inclusive scan: own map after the lower lanes'
                const T qP = __shfl_up_sync(0xffffffffu, P, o), qM = __shfl_up_sync(0xffffffffu, M, o);
                if (lane >= o) {
                    P = P + M * qP;
                    M = M * qM;
                }
            }
            // the inflow left of the row (chunk 0 starts at the ghost, B = 0)
            const T x = rv[5];
            const T eP = __shfl_up_sync(0xffffffffu, P, 1), eM = __shfl_up_sync(0xffffffffu, M, 1);
            T y = (lane == 0) ? x : eP + eM * x;
            const T dn = rv[3], tn = rv[4];
            T out[kGTPer];
#pragma unroll
            for (int e = 0; e < kGTPer; e++) {
                y = aa[e] + bb[e] * y;
                below[e] = y;
                out[e] = y - dn * (y - tn);
            }
            if (act && !first) {
                T* dst = v + d.at(i0, k);
                if (i0 >= 1 && i0 + kGTPer - 1 <= NX) {
                    if constexpr (sizeof(T) == 4) {
                        *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
                    } else {
                        *reinterpret_cast<double2*>(dst) = make_double2(out[0], out[1]);
                        *reinterpret_cast<double2*>(dst + 2) = make_double2(out[2], out[3]);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < kGTPer; e++)
                        if (i0 + e >= 1 && i0 + e <= NX) dst[e] = out[e];
                }
            }
            const T yr = __shfl_sync(0xffffffffu, y, 31);   // y at the tile's last column
            if (lane == 0) {
                rout[r] = yr;
                if (c + 1 < t.nc && !(yr == rv[6])) diff = true;   // read by the tile on the right
            }
            // roll the windows up a row
            if (more_rows) {
                eKld = eKl;
                eKl = eKl_n;
                eKr = eKr_n;
                evr = evr_n;
#pragma unroll
                for (int e = 0; e < kGTPer; e++) {
                    Kd[e] = Kc[e];
                    if (first) {
                        Kc[e] = Ku[e];
                        Ku[e] = Kn[e];
                        v0[e] = vu[e];
                        vu[e] = vn[e];
                    } else {
                        Kc[e] = Kn[e];
                        An[e] = An2[e];
                    }
                }
            }
        }
        T* tout = t.top + t.ti(q, f, b, c) + lane * kGTPer;
        const T* told = t.top + t.ti(qp, f, b, c) + lane * kGTPer;
        const int ktop = k0 + rows - 1;
#pragma unroll
        for (int e = 0; e < kGTPer; e++) {
            tout[e] = below[e];
            if (b + 1 < t.nb) {   // read by the tile above
                const T prev = first ? (act ? v[d.at(i0 + e, ktop)] : T(0)) : told[e];
                if (!(below[e] == prev)) diff = true;
            }
        }
        if (__any_sync(0xffffffffu, diff) && lane == 0) any_changed = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (any_changed) t.ctl->changed[q] = 1;
        __threadfence();
        const int prev = atomicAdd(&t.ctl->done, 1);
        if (prev == (int)gridDim.x - 1) {   // the last block of the pass decides
            __threadfence();
            const int ch = *(volatile int*)&t.ctl->changed[q];
            // pass 1 writes no field: a second pass always follows; every tile
            // is final after nb + nc - 1 passes
            const int more = (first || ch) && pass < max(2, t.nb + t.nc - 1);
            t.ctl->done = 0;
            t.ctl->passes = pass;
            t.ctl->more = more;
            if (more) {
                t.ctl->changed[qp] = 0;   // the next pass writes that parity
                t.ctl->pass = pass;
            } else {                      // ready for the next sweep
                t.ctl->changed[0] = t.ctl->changed[1] = 0;
                t.ctl->pass = 0;
            }
            if (t.exec) *t.exec += 1;
            if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
        }
    }
}
template <typename T, bool FIRST>
__global__ void __launch_bounds__(128, kGSTileMinBlocks<T>) k_gs_tiles(GSArgs<T> a, GSTileArgs<T> t, cudaGraphConditionalHandle h) { k_gs_tiles_body<T, FIRST>(a, t, h); }

// ---------------------------------------------------------------------------
// The second schedule of the same recurrence: one thread-block cluster a field.
// k_gs_coeffs forms A0, C, B for every cell of the five fields in parallel;
// k_gs_cluster then runs the recurrence, one cluster per field. Row k is a
// first-order linear recurrence along i (v'(0,k) the untouched ghost), solved
// as a scan of affine maps: each thread composes the maps of its PER
// contiguous cells and the warp scans those with shuffles; warps pass the
// carry along the row to the next warp, so consecutive warps work on
// consecutive rows at the same time (a wavefront across the cluster). One
// pass and no repeated arithmetic: the schedule for many cases stepping at
// once (a batch), where the GPU is busy with other cases while a cluster's
// chain runs; the tiles are for one case alone, where the chain is the
// step's critical path. Results agree with the tiles' to round-off (the
// carries associate differently).

// A0, C, B of cell (i, k) of field blockIdx.z, i = 0..pitch-1, k = 1..nz-2
// (Turbulent.cpp:83-88 for zeta, :107-112 for the scalars). The ghost i = 0
// gets the constant map v'(0, k) = v(0, k) (never updated), cells beyond
// NX the identity map, so a row's scan needs no edge cases.
template <typename T>
__global__ void k_gs_coeffs(GSArgs<T> a) {
    const int f = blockIdx.z;
    if (!(a.mask & (1 << f))) return;
    const Dims& d = a.d;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= d.pitch || k > d.nz - 2) return;
    const T* v = a.v[f];
    if (i == 0 || i > d.nx - 2) {
        const size_t e = (size_t)f * d.cells() + d.at(i, k);
        a.A0[e] = (i == 0) ? v[d.at(0, k)] : T(0);
        a.C[e] = T(0);
        a.B[e] = (i == 0) ? T(0) : T(1);
        return;
    }
    const bool mom = (f == 0);
    const T* K = mom ? a.RKM : a.RKH;
    const T cx = T(a.c.rdx2 * a.c.dt);
    const T cz = mom ? T(a.p.gsM_cz[k]) : T(a.p.gsS_cz[k]);
    T v0 = v[d.at(i, k)], vr = v[d.at(i + 1, k)], vu = v[d.at(i, k + 1)];
    T ax, bx, czu, czd;
    if (mom) {
        T Kc = K[d.at(i, k)], Kd = K[d.at(i, k - 1)], Kl = K[d.at(i - 1, k)], Kld = K[d.at(i - 1, k - 1)];
        ax = T(0.5) * (Kc + Kd);
        bx = T(0.5) * (Kl + Kld);
        czu = T(a.p.rhou[k]) * T(0.5) * (Kc + Kl);
        czd = T(a.p.gsM_rhod[k]) * T(0.5) * (Kd + Kld);
    } else {
        T Kc = K[d.at(i, k)], Kr = K[d.at(i + 1, k)], Kl = K[d.at(i - 1, k)];
        T Ku = K[d.at(i, k + 1)], Kd = K[d.at(i, k - 1)];
        ax = T(0.5) * (Kr + Kc);
        bx = T(0.5) * (Kc + Kl);
        czu = T(a.p.rhow[k + 1]) * T(0.5) * (Ku + Kc);
        czd = T(a.p.gsS_rhod[k]) * T(0.5) * (Kc + Kd);
    }
    T du = vu - v0, dd = v0;
    if (kPert<T> && (f == 1 || f == 2)) {   // th', qv' about a profile
        du += T(a.p.d0[f - 1][k + 1]);
        dd += T(a.p.d0[f - 1][k]);
    }
    // v + cx (ax (vr - v) - bx (v - v'[i-1])) + cz (czu du - czd (dd - v'below))
    const size_t e = (size_t)f * d.cells() + d.at(i, k);
    a.A0[e] = v0 + cx * (ax * (vr - v0) - bx * v0) + cz * (czu * du - czd * dd);
    a.C[e] = cz * czd;
    a.B[e] = cx * bx;
}

constexpr int kGSSpinLimit = 1 << 22;   // polls before a wait gives up
constexpr int kGSErrWait = 1;           // device error word: a Gauss-Seidel wait gave up
constexpr size_t kGSRingBytes = 200 * 1024;   // cp.async ring of coefficient rows
constexpr int kGSCarry = 64;            // inbox slots (rows) of a warp
constexpr int kGSAckEvery = 16;         // rows between acknowledgements

// Flags between CTAs of a cluster: acquire / release at cluster scope through
// generic addresses (local shared memory, or a peer CTA's mapped into the
// cluster window).
__device__ __forceinline__ int ld_acquire_cluster(const int* p) {
    int v;
    asm volatile("ld.acquire.cluster.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cluster(int* p, int v) {
    asm volatile("st.release.cluster.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_cluster_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.cluster.b64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_cluster_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.cluster.b64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// A carry travels as row-tagged 64-bit words: (row << 32) | 32 bits of the
// value (one word for float, two for double). A 64-bit store is seen whole,
// so a reader that finds its row in every word holds that row's value; no
// flag and no fence is needed.
template <typename T>
struct Tagged {
    static constexpr int kWords = sizeof(T) / 4;
    __device__ static void put(unsigned long long* w, T x, int row) {
        const unsigned long long tag = (unsigned long long)(unsigned)row << 32;
        if constexpr (sizeof(T) == 4) {
            st_relaxed_cluster_u64(w, tag | __float_as_uint(x));
        } else {
            const unsigned long long b = (unsigned long long)__double_as_longlong(x);
            st_relaxed_cluster_u64(w, tag | (b >> 32));
            st_relaxed_cluster_u64(w + 1, tag | (b & 0xffffffffull));
        }
    }
    // true and x set when every word carries `row`
    __device__ static bool get(const unsigned long long* w, int row, T& x) {
        const unsigned long long w0 = ld_relaxed_cluster_u64(w);
        if ((int)(w0 >> 32) != row) return false;
        if constexpr (sizeof(T) == 4) {
            x = __uint_as_float((unsigned)w0);
        } else {
            const unsigned long long w1 = ld_relaxed_cluster_u64(w + 1);
            if ((int)(w1 >> 32) != row) return false;
            x = __longlong_as_double((long long)((w0 << 32) | (w1 & 0xffffffffull)));
        }
        return true;
    }
};

// The recurrence of one field spread over a cluster of CS CTAs. The padded
// row is cut into chunks of 32*PER cells, one per warp; global warp g sits in
// CTA g / W as its warp g % W (W warps a CTA). Each warp walks the rows in
// order on its own: it waits for the carry-in that warp g-1 left, row-tagged,
// in its own inbox (written locally, or into this CTA's shared memory from
// the previous CTA through the cluster window), acknowledges every
// kGSAckEvery-th row in warp g-1's shared memory (a release store, so its
// reads of the inbox come first), and, once warp g+1 has acknowledged the row
// that last used the inbox slot it is about to reuse, writes its carry-out
// into warp g+1's inbox. Everything is polled in local shared memory. Cluster barriers open (all inboxes
// initialised before any peer writes) and close (no CTA exits while a peer may
// still write into it) the kernel. Each wait polls at most kGSSpinLimit
// times; a warp that gives up raises the abort flag of every CTA of the
// cluster and the device error word, so every wait ends. Coefficient rows are
// staged in shared memory by cp.async, D rows ahead (a thread reads back only
// what it copied); the rows' nudging scalars are tabulated in shared memory at
// the start. Dynamic shared memory: D * 3 * blockDim.x * PER values of T, then
// 2 * nz values of T.
constexpr int kGSClusterWarps = 10;   // warps a CTA at most (NX = 8192: 9)

// The carry of a row pair: two row-tagged values (the pair's first row as tag).
template <typename T>
struct Tagged2 {
    static constexpr int kWords = 2 * Tagged<T>::kWords;
    __device__ static void put(unsigned long long* w, T x0, T x1, int row) {
        Tagged<T>::put(w, x0, row);
        Tagged<T>::put(w + Tagged<T>::kWords, x1, row);
    }
    __device__ static bool get(const unsigned long long* w, int row, T& x0, T& x1) {
        return Tagged<T>::get(w, row, x0) && Tagged<T>::get(w + Tagged<T>::kWords, row, x1);
    }
};

// Two rows a step. With V_i = (v'(i, k), v'(i, k+1)) the pair obeys
// V_i = alpha_i + M_i V_{i-1}, M_i = [[B_k, 0], [C_{k+1} B_k, B_{k+1}]],
// alpha_i = (a_i, A0_{k+1} + C_{k+1} a_i), a_i = A0_k + C_k v'(i, k-1): one scan
// over the row advances both rows, so the serial chain has half as many
// steps, each with five values a shuffle round instead of two (the rounds'
// shuffles are independent and overlap). The cells are then applied with the
// scalar formulas, row k first. An odd last row runs as a pair whose second
// row is the identity and is not stored.
template <typename T, int PER, int D, int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(32 * kGSClusterWarps) k_gs_cluster(GSArgs<T> a) {
    static_assert(D % 2 == 0, "the ring holds whole row pairs");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int kW = Tagged2<T>::kWords;
    __shared__ unsigned long long inbox[kGSClusterWarps][kGSCarry][kW];
    __shared__ int ack_in[kGSClusterWarps], abort_flag;
    namespace cgx = cooperative_groups;
    cgx::cluster_group cl = cgx::this_cluster();
    const int crank = (int)cl.block_rank();
    const int f = blockIdx.x / CS;
    const Dims& d = a.d;
    const int NX = d.nx - 2, kend = d.nz - 2;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, W = blockDim.x >> 5;
    for (int j = tid; j < kGSClusterWarps * kGSCarry * kW; j += blockDim.x)
        (&inbox[0][0][0])[j] = 0ull;    // tag 0: no row
    if (tid < kGSClusterWarps) ack_in[tid] = 0;
    if (tid == 0) abort_flag = 0;
    // nudging of row k: out = x - dn[k] (x - tn[k]) (dn = 0: none)
    T* dn_tab = reinterpret_cast<T*>(smem_raw) + (size_t)D * 3 * blockDim.x * PER;
    T* tn_tab = dn_tab + d.nz;
    for (int k = tid; k < d.nz; k += blockDim.x) {
        T dn = T(0), tn = T(0);
        if (a.nudge && f == 0) dn = T(a.p.dtcgr_zeta[k]);                      // Nudge_zeta
        if (a.nudge && f == 1) {                                                 // Nudge_theta
            dn = T(a.p.dtcgr_th[k]);
            tn = kPert<T> ? T(-a.p.dn[0][k]) : T(a.p.thb_init[k]);
        }
        dn_tab[k] = dn;
        tn_tab[k] = tn;
    }
    cl.sync();
    const int gwn = (d.pitch + 32 * PER - 1) / (32 * PER);   // warps with cells
    const int g = crank * W + wid;
    const bool run = (a.mask & (1 << f)) && g < gwn;
    if (run) {
        T* v = a.v[f];
        const int i0 = (g * 32 + lane) * PER;
        const bool act = i0 < d.pitch;       // pitch is a multiple of PER
        const size_t fo = (size_t)f * d.cells();
        const T* gsrc[3] = {a.A0 + fo, a.C + fo, a.B + fo};
        T* ring = reinterpret_cast<T*>(smem_raw);
        constexpr int kVec = 16 / sizeof(T);
        auto slot = [&](int r, int arr) { return ring + ((size_t)(r * 3 + arr) * blockDim.x + tid) * PER; };
        auto issue = [&](int k, int r) {
            if (act && k <= kend) {
#pragma unroll
                for (int arr = 0; arr < 3; arr++) {
                    const T* src = gsrc[arr] + d.at(i0, k);
                    T* dst = slot(r, arr);
#pragma unroll
                    for (int q = 0; q < PER; q += kVec) cp_async16(dst + q, src + q);
                }
            }
            cp_async_commit();
        };
        // neighbours in the chain and their flags
        const bool has_pred = g > 0, has_succ = g + 1 < gwn;
        const int pc = (g - 1) / W, pw = (g - 1) % W, sc = (g + 1) / W, sw = (g + 1) % W;
        int* pred_ack = has_pred ? cl.map_shared_rank(&ack_in[pw], pc) : nullptr;
        unsigned long long* succ_box = has_succ ? cl.map_shared_rank(&inbox[sw][0][0], sc) : nullptr;
        auto give_up = [&]() {   // lane 0 of a warp whose wait ran out: stop the cluster
            for (int r = 0; r < CS; r++) *(volatile int*)cl.map_shared_rank(&abort_flag, r) = 1;
            if (a.err) atomicOr(a.err, kGSErrWait);
        };
        auto wait_carry = [&](int k, T& x0, T& x1) {   // all lanes; warp-uniform result
            bool okw = false;
            const unsigned long long* w = &inbox[wid][k % kGSCarry][0];
            for (int it = 0; it < kGSSpinLimit; it++) {
                if (Tagged2<T>::get(w, k, x0, x1)) {
                    okw = true;
                    break;
                }
                if (*(volatile int*)&abort_flag) break;
            }
            const bool all = __all_sync(0xffffffffu, okw);
            if (!all && lane == 0 && !*(volatile int*)&abort_flag) give_up();
            return all;
        };
        auto wait_ge = [&](const int* p, int target) {   // all lanes; warp-uniform result
            bool okw = false;
            for (int it = 0; it < kGSSpinLimit; it++) {
                if (ld_acquire_cluster(p) >= target) {
                    okw = true;
                    break;
                }
                if (*(volatile int*)&abort_flag) break;
            }
            const bool all = __all_sync(0xffffffffu, okw);
            if (!all && lane == 0 && !*(volatile int*)&abort_flag) give_up();
            return all;
        };
        T vdn[PER];
#pragma unroll
        for (int e = 0; e < PER; e++) {
            const int i = i0 + e;
            vdn[e] = (act && i >= 1 && i <= NX) ? v[d.at(i, 0)] : T(0);
        }
#pragma unroll
        for (int r = 0; r < D; r++) issue(1 + r, r);
        bool ok = true;
        int ack_seen = 0;   // last acknowledgement read from warp g+1
        auto pair = [&](int k, int r) {   // rows k and k+1 (k+1 may be past the last row)
            const bool two = k + 1 <= kend;
            const T dn0 = dn_tab[k], tn0 = tn_tab[k];
            const T dn1 = two ? dn_tab[k + 1] : T(0), tn1 = two ? tn_tab[k + 1] : T(0);
            const int s = k % kGSCarry;
            // read the carry-in early: when warp g-1 is ahead it is there
            T x0 = T(0), x1 = T(0);   // warp 0 starts at the ghost's constant map
            bool have = !has_pred || Tagged2<T>::get(&inbox[wid][s][0], k, x0, x1);
            cp_async_wait<D - 2>();
            T Aa[PER], Bk[PER], A2[PER], C2[PER], B2[PER];
            if (act) {
                const T* sa = slot(r, 0);
                const T* scc = slot(r, 1);
                const T* sb = slot(r, 2);
                const T* ta = slot(r + 1, 0);
                const T* tc = slot(r + 1, 1);
                const T* tb = slot(r + 1, 2);
#pragma unroll
                for (int e = 0; e < PER; e++) {
                    Aa[e] = sa[e] + scc[e] * vdn[e];
                    Bk[e] = sb[e];
                    A2[e] = two ? ta[e] : T(0);
                    C2[e] = two ? tc[e] : T(0);
                    B2[e] = two ? tb[e] : T(1);
                }
            } else {
#pragma unroll
                for (int e = 0; e < PER; e++) {
                    Aa[e] = T(0);
                    Bk[e] = T(1);
                    A2[e] = T(0);
                    C2[e] = T(0);
                    B2[e] = T(1);
                }
            }
            // the lane's map over its cells: (p0, p1) offsets, M = [[m00, 0], [m10, m11]]
            T p0 = T(0), p1 = T(0), m00 = T(1), m10 = T(0), m11 = T(1);
#pragma unroll
            for (int e = 0; e < PER; e++) {
                const T c0 = Aa[e], c1 = A2[e] + C2[e] * Aa[e];
                const T n00 = Bk[e], n10 = C2[e] * Bk[e], n11 = B2[e];
                p1 = c1 + n10 * p0 + n11 * p1;
                p0 = c0 + n00 * p0;
                m10 = n10 * m00 + n11 * m10;
                m00 = n00 * m00;
                m11 = n11 * m11;
            }
            issue(k + D, r);
            issue(k + 1 + D, r + 1);
            T s0 = p0, s1 = p1, s00 = m00, s10 = m10, s11 = m11;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T q0 = __shfl_up_sync(0xffffffffu, s0, o), q1 = __shfl_up_sync(0xffffffffu, s1, o);
                const T q00 = __shfl_up_sync(0xffffffffu, s00, o), q10 = __shfl_up_sync(0xffffffffu, s10, o);
                const T q11 = __shfl_up_sync(0xffffffffu, s11, o);
                if (lane >= o) {   // own map after the lower lanes'
                    s1 = s1 + s10 * q0 + s11 * q1;
                    s0 = s0 + s00 * q0;
                    s10 = s10 * q00 + s11 * q10;
                    s00 = s00 * q00;
                    s11 = s11 * q11;
                }
            }
            const T t0 = __shfl_sync(0xffffffffu, s0, 31), t1 = __shfl_sync(0xffffffffu, s1, 31);
            const T t00 = __shfl_sync(0xffffffffu, s00, 31), t10 = __shfl_sync(0xffffffffu, s10, 31);
            const T t11 = __shfl_sync(0xffffffffu, s11, 31);
            T e0 = __shfl_up_sync(0xffffffffu, s0, 1), e1 = __shfl_up_sync(0xffffffffu, s1, 1);
            T e00 = __shfl_up_sync(0xffffffffu, s00, 1), e10 = __shfl_up_sync(0xffffffffu, s10, 1);
            T e11 = __shfl_up_sync(0xffffffffu, s11, 1);
            if (lane == 0) {
                e0 = T(0);
                e1 = T(0);
                e00 = T(1);
                e10 = T(0);
                e11 = T(1);
            }
            if (has_pred) {
                if (!__all_sync(0xffffffffu, have)) ok = ok && wait_carry(k, x0, x1);
                if (((k - 1) >> 1) % (kGSAckEvery / 2) == 0) {   // every kGSAckEvery rows
                    __syncwarp();
                    if (lane == 0) st_release_cluster(pred_ack, k);
                }
            }
            if (has_succ) {
                // slot s last held the pair at row k - kGSCarry
                if (ack_seen < k - kGSCarry) {
                    ok = ok && wait_ge(&ack_in[wid], k - kGSCarry);
                    ack_seen = ld_acquire_cluster(&ack_in[wid]);
                }
                if (lane == 0) Tagged2<T>::put(succ_box + (size_t)s * kW, t0 + t00 * x0, t1 + t10 * x0 + t11 * x1, k);
            }
            T y0 = e0 + e00 * x0, y1 = e1 + e10 * x0 + e11 * x1;
            T out0[PER], out1[PER];
#pragma unroll
            for (int e = 0; e < PER; e++) {
                y0 = Aa[e] + Bk[e] * y0;
                y1 = (A2[e] + C2[e] * y0) + B2[e] * y1;
                vdn[e] = y1;
                out0[e] = y0 - dn0 * (y0 - tn0);
                out1[e] = y1 - dn1 * (y1 - tn1);
            }
            auto store = [&](int kk, const T (&out)[PER]) {
                T* dst = v + d.at(i0, kk);
                if (act && i0 >= 1 && i0 + PER - 1 <= NX) {
#pragma unroll
                    for (int q = 0; q < PER; q += kVec) {
                        if constexpr (sizeof(T) == 4)
                            *reinterpret_cast<float4*>(dst + q) = make_float4(out[q], out[q + 1], out[q + 2], out[q + 3]);
                        else
                            *reinterpret_cast<double2*>(dst + q) = make_double2(out[q], out[q + 1]);
                    }
                } else if (act) {
#pragma unroll
                    for (int e = 0; e < PER; e++)
                        if (i0 + e >= 1 && i0 + e <= NX) dst[e] = out[e];
                }
            };
            store(k, out0);
            if (two) store(k + 1, out1);
        };
        for (int k = 1; k <= kend && ok; k += D) {
#pragma unroll
            for (int r = 0; r < D; r += 2)
                if (k + r <= kend && ok) pair(k + r, r);
        }
        cp_async_wait<0>();
    }
    cl.sync();
}

// ---------------------------------------------------------------------------
// Top-layer nudging as standalone passes (NumericalProcess.cpp:60-96).

template <typename T>
struct NudgeArgs {
    Dims d;
    Consts c;
    Profiles p;
    T *thp, *zetap, *qvp;
    const T* qv;
    int do_th, do_zeta;
    double tau;       // moisture_nudge_time, 0 = off
};

template <typename T>
__device__ __forceinline__ void k_nudge_body(const NudgeArgs<T>& a) {
    const Dims& d = a.d;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= d.nx || k >= d.nz) return;
    const size_t id = d.at(i, k);
    const bool inner = (i >= 1 && i <= d.nx - 2 && k >= 1 && k <= d.nz - 2);
    if (inner && a.do_th) {
        T x = a.thp[id];
        T tref = kPert<T> ? T(-a.p.dn[0][k]) : T(a.p.thb_init[k]);
        a.thp[id] = x - T(a.p.dtcgr_th[k]) * (x - tref);
    }
    if (inner && a.do_zeta) {
        T x = a.zetap[id];
        a.zetap[id] = x - T(a.p.dtcgr_zeta[k]) * x;
    }
    if (a.tau != 0.0)  // every cell, ghosts included (NumericalProcess.cpp:90-94)
        a.qvp[id] = a.qvp[id] + T(a.c.dt) * ((kPert<T> ? T(-a.p.dn[1][k]) : T(a.p.qvb0[k])) - a.qv[id]) / T(a.tau);
}
template <typename T>
__global__ void k_nudge(NudgeArgs<T> a) { k_nudge_body<T>(a); }

// ---------------------------------------------------------------------------
// Horizontal means (Iteration::updateMean, Iteration.cpp:42-86): thb, qvb and
// thvb = thb (1 + 0.608 qvb) per level with their 1D halos. One block per
// interior level. Optionally rotates ubarTop (nextTimeStep, :166-167).

template <typename T>
struct MeanArgs {
    Dims d;
    const double *ref_th, *ref_qv;   // perturbation profiles (null in the FP64 step)
    const T *thp, *qvp;
    double *thb, *qvb, *thvb;
    double* ubar;   // [0] ubarTop, [1] ubarTopp
    int rotate_ubar;
};

template <typename T>
__device__ __forceinline__ void k_update_mean_body(const MeanArgs<T>& a) {
    __shared__ double sh[32 * 2];
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x;
    double s[2] = {0, 0};
    for (int i = 1 + threadIdx.x; i <= d.nx - 2; i += blockDim.x) {
        s[0] += (double)a.thp[d.at(i, k)];
        s[1] += (double)a.qvp[d.at(i, k)];
    }
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        double n = (double)(d.nx - 2.);
        double tb = s[0] / n, qb = s[1] / n;
        if (a.ref_th) { tb += a.ref_th[k]; qb += a.ref_qv[k]; }
        double tv = tb * (1 + 0.608 * qb);
        a.thb[k] = tb;
        a.qvb[k] = qb;
        a.thvb[k] = tv;
        if (k == 1) { a.thb[0] = tb; a.qvb[0] = qb; a.thvb[0] = tv; }
        if (k == d.nz - 2) { a.thb[d.nz - 1] = tb; a.qvb[d.nz - 1] = qb; a.thvb[d.nz - 1] = tv; }
        if (k == 1 && a.rotate_ubar) a.ubar[0] = a.ubar[1];
    }
}
template <typename T>
__global__ void k_update_mean(MeanArgs<T> a) { k_update_mean_body<T>(a); }

// ---------------------------------------------------------------------------
// Domain-mean top wind tendency (PoissonSolver::pubarTop_pt,
// PoissonSolver.cpp:655-676). One block.

template <typename T>
struct PubarArgs {
    Dims d;
    Consts c;
    Profiles p;
    const T *u, *w, *RKM;
    double* ubar;     // [0] ubarTop, [1] ubarTopp
    double* dubar;    // dubarTop_advect[2]
    AB2 ab;
};

template <typename T>
__device__ __forceinline__ void k_pubartop_body(const PubarArgs<T>& a) {
    __shared__ double sh[32 * 3];
    const Dims& d = a.d;
    const int t = d.nz - 2, b = d.nz - 3, top = d.nz - 1;
    const double* rhou = a.p.rhou;
    const double* rhow = a.p.rhow;
    double s[3] = {0, 0, 0};
    for (int i = 1 + threadIdx.x; i < d.nx - 1; i += blockDim.x) {
        double ut = a.u[d.at(i, t)], ub = a.u[d.at(i, b)], utop = a.u[d.at(i, top)];
        double wt = a.w[d.at(i, t)], wtm = a.w[d.at(i - 1, t)];
        const T* K = a.RKM;
        s[0] += 0.25 * (rhou[t] * ut + rhou[b] * ub) * (wt + wtm);
        s[1] += rhow[top] * 0.25 * ((double)K[d.at(i, top)] + K[d.at(i, t)] + K[d.at(i - 1, top)] + K[d.at(i - 1, t)]) *
                (a.p.rdz_up * (utop - ut));
        s[2] += rhow[t] * 0.25 * ((double)K[d.at(i, t)] + K[d.at(i, b)] + K[d.at(i - 1, t)] + K[d.at(i - 1, b)]) *
                (a.c.rdx * (wt - wtm) + a.p.rdz_dn * (ut - ub));
    }
    block_sum(s, sh);
    if (threadIdx.x == 0) {
        double n = (double)(d.nx - 2.);
        double down = s[0] / n, kup = s[1] / n, kdown = s[2] / n;
        double pa = (-down) * a.p.rdz_c / rhou[t];
        double pb = (kup - kdown) * a.p.rdz_c / rhou[t];
        double tend = -pa + pb;
        double old = a.ab.first ? tend : a.dubar[a.ab.so];
        a.dubar[a.ab.sn] = tend;
        if (a.ab.first) a.dubar[a.ab.so] = tend;
        a.ubar[1] = a.ubar[0] + 1.5 * a.c.dt * tend - 0.5 * a.c.dt * old;
    }
}
template <typename T>
__global__ void k_pubartop(PubarArgs<T> a) { k_pubartop_body<T>(a); }

// ---------------------------------------------------------------------------
// cal_u (PoissonSolver.cpp:580-653): the top-row wind from the periodic chi
// problem and the column integral below it.
//
// Top row: chi[i-1] - 2 chi[i] + chi[i+1] = h[i] only enters through
// uxi = (chi[i] - chi[i-1])/dx with its mean removed. The differences satisfy
// d[i+1] - d[i] = h[i], so uxi is an exclusive prefix sum of h (any constant
// cancels in the mean removal); the reference reaches the same values with
// CG to 1e-12. Every block of the column kernel computes the whole top row
// (one block's worth of work, the same arithmetic in every block) and keeps
// its own 32 columns: no second launch waits for a one-block kernel.

template <typename T>
struct CalUArgs {
    Dims d;
    Consts c;
    Profiles p;
    T* u;
    const T *w, *zetap;
    const double* ubar;   // [1] = ubarTopp
};

constexpr int kCalUThreads = 1024;

// The top-row u of columns own_lo .. own_lo+31 into own[] (kCalUThreads
// threads, one block).
template <typename T>
__device__ __forceinline__ void cal_u_top_row(const CalUArgs<T>& a, T* own, int own_lo) {
    __shared__ double sh[32 * 1];
    __shared__ double scan[32];
    const Dims& d = a.d;
    const int NX = d.nx - 2, t = d.nz - 2;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = (NX + kCalUThreads - 1) / kCalUThreads;
    const int i0 = 1 + tid * per;
    const double c = a.p.rhow[t] / a.p.rhou[t];
    double h[kGSMaxPerThread];
    double s[1] = {0};
#pragma unroll
    for (int e = 0; e < kGSMaxPerThread; e++) {
        int i = i0 + e;
        h[e] = 0;
        if (e < per && i <= NX) {
            h[e] = -(0. - a.p.rhow[t] * (double)a.w[d.at(i, t)]) / a.p.rhou[t] * a.c.dx * a.p.hfac;
            s[0] += h[e];
        }
    }
    (void)c;
    block_sum(s, sh);
    const double hmean = s[0] / NX;
    double loc = 0;
#pragma unroll
    for (int e = 0; e < kGSMaxPerThread; e++) {
        int i = i0 + e;
        if (e < per && i <= NX) { h[e] = h[e] - hmean; loc += h[e]; }
    }
    // exclusive scan of the chunk totals
    double incl = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double p = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += p;
    }
    if (lane == 31) scan[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        double x = scan[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double p = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += p;
        }
        scan[lane] = x;
    }
    __syncthreads();
    double run = incl - loc + (wid > 0 ? scan[wid - 1] : 0.0);
    double ux[kGSMaxPerThread];
    double s2[1] = {0};
#pragma unroll
    for (int e = 0; e < kGSMaxPerThread; e++) {
        int i = i0 + e;
        ux[e] = 0;
        if (e < per && i <= NX) {
            ux[e] = run * a.c.rdx;
            run += h[e];
            s2[0] += ux[e];
        }
    }
    block_sum(s2, sh);
    const double umean = s2[0] / NX;
    const double ubarp = a.ubar[1];
#pragma unroll
    for (int e = 0; e < kGSMaxPerThread; e++) {
        int i = i0 + e;
        if (e < per && i <= NX && i >= own_lo && i < own_lo + 32) own[i - own_lo] = T((ux[e] - umean) + ubarp);
    }
}

// Column integral u(i, k) = u(i, nz-2) + sum_{m=k}^{nz-3} (dw/dx - rhow zeta)(-dz)
// from the top down (PoissonSolver.cpp:644-651), with the center halo of u;
// u(i, nz-2), the top row, comes from cal_u_top_row in the same block.
// A block owns 32 columns (lanes) and kColSeg z-segments (warps): each thread
// sums its segment, the segment totals are scanned from the top in shared
// memory, then each thread writes its rows. Thirty-two segments give the 64
// blocks of a 2048-column grid 32 warps each (about 8 rows a thread at
// NZ = 256), so the short chains, not a few long ones, set the time.
constexpr int kColSeg = 32;

template <typename T>
__device__ __forceinline__ void k_cal_u_columns_body(const CalUArgs<T>& a) {
    static_assert(32 * kColSeg == kCalUThreads, "the top row takes the column kernel's block");
    __shared__ T tot[kColSeg][32];
    __shared__ T utop_sh[32];
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const int i = 1 + blockIdx.x * 32 + lane;
    const bool act = (i <= d.nx - 2);
    const int t = d.nz - 2, nrow = d.nz - 3;               // rows k = 1..nz-3
    // segment s covers rows from the top: k in (khi - len, khi]
    const int r0 = (s * nrow) / kColSeg, r1 = ((s + 1) * nrow) / kColSeg;
    const T rdx = T(a.c.rdx);
    auto term = [&](int k) -> T {
        return ((a.w[d.at(i, k + 1)] - a.w[d.at(i - 1, k + 1)]) * rdx - T(a.p.rhow[k + 1]) * a.zetap[d.at(i, k + 1)]) *
               T(-a.p.dzw[k + 1]);
    };
    cal_u_top_row(a, utop_sh, 1 + blockIdx.x * 32);
    T sum = T(0);
    if (act)
        for (int r = r0; r < r1; r++) sum += term(t - 1 - r);
    tot[s][lane] = sum;
    __syncthreads();
    if (!act) return;
    const T utop = utop_sh[lane];
    T area = T(0);
    for (int q = 0; q < s; q++) area += tot[q][lane];
    if (s == 0) store_center(a.u, d, i, t, utop);
    for (int r = r0; r < r1; r++) {
        int k = t - 1 - r;
        area += term(k);
        store_center(a.u, d, i, k, area + utop);
    }
}
template <typename T>
__global__ void __launch_bounds__(32 * kColSeg) k_cal_u_columns(CalUArgs<T> a) { k_cal_u_columns_body<T>(a); }

}  // namespace vvm
