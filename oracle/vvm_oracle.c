/* CPU restatement of the reference VVM time step; see vvm_oracle.h.
 *
 * Test infrastructure only (the checker for the GPU path). Each routine cites
 * the reference code it restates; expressions keep the reference's operand
 * order so that results agree bit for bit where the algorithm is the same.
 */
#include "vvm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The threaded CPU baseline (Makefile target _build/libvvmoracle_mt.so) is
 * this file built with -fopenmp -DORC_FAST_SOLVE: loops over rows split
 * across threads (every temporary is local to its iteration, so no thread
 * writes what another reads), the five Gauss-Seidel sweeps run concurrently
 * (each is serial within its field, as the reference's in-place update
 * requires), domain sums reduce per thread, and cal_w's Fourier transforms
 * are radix-2 FFTs when NX is a power of two. The serial build (the checker
 * pinned to the reference) compiles none of that: ORC_PAR is empty there. */
#ifdef _OPENMP
#define ORC_PAR _Pragma("omp parallel for schedule(static)")
#else
#define ORC_PAR
#endif

#define F2(a, i, k) ((a)[(size_t)(i) * m->nz + (k)])
#define H3(a, i, k, s) ((a)[((size_t)(i) * m->nz + (k)) * 2 + (s)])

struct orc_model {
    int nx, nz, step, CASE, status_for_adding_forcing, streamfunction;
    double dx, dz, dt, d2t, rdx, r2dx, rdz, r2dz, rdx2, rdz2;
    double GRAVITY, Cp, Cv, Rd, Lv, P0, PSURF, CRAD, addforcingtime, moisture_nudge_time;
    double ubarTopp, ubarTop, ubarTopm, dubarTop_advect[2];
    /* 2D */
    double *zeta, *zetam, *zetap, *th, *thm, *thp, *u, *w, *qv, *qvm, *qvp, *qc, *qcm, *qcp;
    double *qr, *qrm, *qrp, *RKM, *RKH, *U_w, *W_u, *init_th_forcing;
    double *evaporation, *accretion, *autoconversion, *condensation, *psi;
    /* AB2 */
    double *dth_advect, *dth_buoyancy, *dzeta_advect, *dqv_advect, *dqc_advect, *dqr_advect, *dqr_VT;
    /* 1D */
    double *thb, *thbm, *thb_zeta, *thb_init, *rhou, *rhow, *pib, *qvb, *qvb0, *pb, *thvb, *thvbm;
    double *z, *z_zeta, *lambda2, *xi, *uxi, *precip, *Q1LS, *Q2LS;
    /* scratch */
    double *flux_u, *flux_w, *work;
    /* vertical level metric (levels()): per-level factors that equal the
     * reference's constants on uniform levels */
    int stretched, lv_ks;
    double *lv_r2dzc, *lv_r2dzw, *lv_rdzc, *lv_r2dzcc, *lv_kmax, *lv_rdz2M, *lv_rdM, *lv_rdz2S, *lv_rdS,
        *lv_dzw, *lv_wa, *lv_wh;
    double lv_rdz_up, lv_rdz_dn, lv_rdz_c, lv_hfac;
};

static double* alloc0(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

orc_model* orc_create(int NX, int NZ, double dx, double dz, double dt, int CASE,
                      double moisture_nudge_time, double addforcingtime) {
    orc_model* m = (orc_model*)calloc(1, sizeof(orc_model));
    /* src/Declare.hpp:78-96 (constructor), main.cpp:68-72 (constants) */
    m->nx = NX + 2;
    m->nz = NZ + 2;
    m->dx = dx; m->dz = dz; m->dt = dt; m->d2t = 2.0 * dt;
    m->rdx = 1.0 / dx; m->r2dx = m->rdx / 2.0; m->rdz = 1.0 / dz; m->r2dz = m->rdz / 2.0;
    m->rdx2 = m->rdx * m->rdx; m->rdz2 = m->rdz * m->rdz;
    m->GRAVITY = 9.80665; m->Cp = 1003.5; m->Cv = 716.5; m->Rd = 287.; m->Lv = 2.5E6;
    m->P0 = 1E5; m->PSURF = 96500.; m->CRAD = 1. / 3600.;
    m->CASE = CASE; m->moisture_nudge_time = moisture_nudge_time;
    m->addforcingtime = addforcingtime; m->status_for_adding_forcing = 1;
    size_t n2 = (size_t)m->nx * m->nz, nz = m->nz, nx = m->nx;
    double** two[] = {&m->zeta, &m->zetam, &m->zetap, &m->th, &m->thm, &m->thp, &m->u, &m->w,
                      &m->qv, &m->qvm, &m->qvp, &m->qc, &m->qcm, &m->qcp, &m->qr, &m->qrm,
                      &m->qrp, &m->RKM, &m->RKH, &m->U_w, &m->W_u, &m->init_th_forcing,
                      &m->evaporation, &m->accretion, &m->autoconversion, &m->condensation,
                      &m->flux_u, &m->flux_w, &m->psi};
    for (size_t j = 0; j < sizeof(two) / sizeof(two[0]); j++) *two[j] = alloc0(n2);
    double** hist[] = {&m->dth_advect, &m->dth_buoyancy, &m->dzeta_advect, &m->dqv_advect,
                       &m->dqc_advect, &m->dqr_advect, &m->dqr_VT};
    for (size_t j = 0; j < sizeof(hist) / sizeof(hist[0]); j++) *hist[j] = alloc0(2 * n2);
    double** one[] = {&m->thb, &m->thbm, &m->thb_zeta, &m->thb_init, &m->rhou, &m->rhow,
                      &m->pib, &m->qvb, &m->qvb0, &m->pb, &m->thvb, &m->thvbm, &m->z,
                      &m->z_zeta, &m->lambda2, &m->Q1LS, &m->Q2LS};
    for (size_t j = 0; j < sizeof(one) / sizeof(one[0]); j++) *one[j] = alloc0(nz);
    m->xi = alloc0(nx); m->uxi = alloc0(nx); m->precip = alloc0(nx);
    double** lv[] = {&m->lv_r2dzc, &m->lv_r2dzw, &m->lv_rdzc, &m->lv_r2dzcc, &m->lv_kmax, &m->lv_rdz2M,
                     &m->lv_rdM, &m->lv_rdz2S, &m->lv_rdS, &m->lv_dzw, &m->lv_wa, &m->lv_wh};
    for (size_t j = 0; j < sizeof(lv) / sizeof(lv[0]); j++) *lv[j] = alloc0(nz);
    m->work = alloc0(4 * n2 + 8 * (nx + nz));
    return m;
}

void orc_destroy(orc_model* m) {
    if (!m) return;
    double* all[] = {m->zeta, m->zetam, m->zetap, m->th, m->thm, m->thp, m->u, m->w, m->qv,
                     m->qvm, m->qvp, m->qc, m->qcm, m->qcp, m->qr, m->qrm, m->qrp, m->RKM,
                     m->RKH, m->U_w, m->W_u, m->init_th_forcing, m->evaporation, m->accretion,
                     m->autoconversion, m->condensation, m->flux_u, m->flux_w, m->dth_advect,
                     m->dth_buoyancy, m->dzeta_advect, m->dqv_advect, m->dqc_advect,
                     m->dqr_advect, m->dqr_VT, m->thb, m->thbm, m->thb_zeta, m->thb_init,
                     m->rhou, m->rhow, m->pib, m->qvb, m->qvb0, m->pb, m->thvb, m->thvbm, m->z,
                     m->z_zeta, m->lambda2, m->Q1LS, m->Q2LS, m->xi, m->uxi, m->precip, m->work, m->psi,
                     m->lv_r2dzc, m->lv_r2dzw, m->lv_rdzc, m->lv_r2dzcc, m->lv_kmax, m->lv_rdz2M, m->lv_rdM,
                     m->lv_rdz2S, m->lv_rdS, m->lv_dzw, m->lv_wa, m->lv_wh};
    for (size_t j = 0; j < sizeof(all) / sizeof(all[0]); j++) free(all[j]);
    free(m);
}

void orc_dims(orc_model* m, int* nx, int* nz) { *nx = m->nx; *nz = m->nz; }

double* orc_field(orc_model* m, const char* n) {
    struct { const char* n; double* p; } t[] = {
        {"zeta", m->zeta}, {"zetam", m->zetam}, {"zetap", m->zetap}, {"th", m->th},
        {"thm", m->thm}, {"thp", m->thp}, {"u", m->u}, {"w", m->w}, {"qv", m->qv},
        {"qvm", m->qvm}, {"qvp", m->qvp}, {"qc", m->qc}, {"qcm", m->qcm}, {"qcp", m->qcp},
        {"qr", m->qr}, {"qrm", m->qrm}, {"qrp", m->qrp}, {"RKM", m->RKM}, {"RKH", m->RKH},
        {"U_w", m->U_w}, {"W_u", m->W_u}, {"init_th_forcing", m->init_th_forcing},
        {"evaporation", m->evaporation}, {"accretion", m->accretion},
        {"autoconversion", m->autoconversion}, {"condensation", m->condensation}, {"psi", m->psi}};
    for (size_t j = 0; j < sizeof(t) / sizeof(t[0]); j++) if (!strcmp(t[j].n, n)) return t[j].p;
    return NULL;
}

double* orc_hist(orc_model* m, const char* n) {
    struct { const char* n; double* p; } t[] = {
        {"dth_advect", m->dth_advect}, {"dth_buoyancy", m->dth_buoyancy},
        {"dzeta_advect", m->dzeta_advect}, {"dqv_advect", m->dqv_advect},
        {"dqc_advect", m->dqc_advect}, {"dqr_advect", m->dqr_advect}, {"dqr_VT", m->dqr_VT}};
    for (size_t j = 0; j < sizeof(t) / sizeof(t[0]); j++) if (!strcmp(t[j].n, n)) return t[j].p;
    return NULL;
}

double* orc_prof(orc_model* m, const char* n) {
    struct { const char* n; double* p; } t[] = {
        {"thb", m->thb}, {"thbm", m->thbm}, {"thb_zeta", m->thb_zeta}, {"thb_init", m->thb_init},
        {"rhou", m->rhou}, {"rhow", m->rhow}, {"pib", m->pib}, {"qvb", m->qvb},
        {"qvb0", m->qvb0}, {"pb", m->pb}, {"thvb", m->thvb}, {"thvbm", m->thvbm}, {"z", m->z},
        {"z_zeta", m->z_zeta}, {"lambda2", m->lambda2}, {"xi", m->xi}, {"uxi", m->uxi},
        {"precip", m->precip}, {"Q1LS", m->Q1LS}, {"Q2LS", m->Q2LS}};
    for (size_t j = 0; j < sizeof(t) / sizeof(t[0]); j++) if (!strcmp(t[j].n, n)) return t[j].p;
    return NULL;
}

double* orc_scalar(orc_model* m, const char* n) {
    if (!strcmp(n, "ubarTopp")) return &m->ubarTopp;
    if (!strcmp(n, "ubarTop")) return &m->ubarTop;
    if (!strcmp(n, "ubarTopm")) return &m->ubarTopm;
    if (!strcmp(n, "dubarTop_advect")) return m->dubarTop_advect;
    if (!strcmp(n, "CRAD")) return &m->CRAD;
    return NULL;
}

int* orc_step_ptr(orc_model* m) { return &m->step; }

/* ---------------------------------------------------------------- levels */

/* The vertical metric of the column. The reference's levels are uniform
 * (src/Init.cpp:125-129) and its operators assume one spacing dz (and, in
 * cal_w and cal_u, dx = dz). On levels with face heights z_zeta[k] and centre
 * heights z[k] midway between faces, with
 *   dc[k] = 2 (z[k] - z_zeta[k])     the thickness of centre cell k,
 *   dw[k] = z[k] - z[k-1]            the distance between the centres around face k
 *                                    (mirror centres below the surface and above the top
 *                                    face: dw[1] = dc[1], dw[nz-1] = dc[nz-2]),
 * each vertical difference is divided by the spacing it spans: a flux
 * divergence at a centre by dc, at a face by dw; a gradient across two
 * centres by z[k+1] - z[k-1]. The Gauss-Seidel diffusion's down-gradient
 * is scaled by the ratio of its spacing to the up-gradient's (lv_rdM,
 * lv_rdS) so that one factor (lv_rdz2M, lv_rdz2S) multiplies the bracket
 * as in the reference. cal_w takes the stretched matrix of
 * oracle/stretched_poisson.py; cal_u integrates over dw and takes the
 * top divergence over dc (lv_hfac = dx / dc[nz-2], where the reference's
 * dx stands for dz). When every spacing is within 1e-9 dz of dz the factors
 * are the reference's constants (and the down ratios exactly 1), so the
 * routines reproduce the reference bit for bit. Nudging starts at the last
 * face at or below 12 km (the reference's 12000 / dz + 1 on uniform levels). */
static void levels(orc_model* m) {
    int nz = m->nz;
    double *z = m->z, *zz = m->z_zeta;
    int uniform = 1;
    for (int k = 1; k <= nz - 2; k++)
        if (fabs(2.0 * (z[k] - zz[k]) - m->dz) > 1e-9 * m->dz) uniform = 0;
    for (int k = 2; k <= nz - 2; k++)
        if (fabs((z[k] - z[k - 1]) - m->dz) > 1e-9 * m->dz) uniform = 0;
    m->stretched = !uniform;
    if (uniform) {
        for (int k = 0; k < nz; k++) {
            m->lv_r2dzc[k] = m->r2dz; m->lv_r2dzw[k] = m->r2dz; m->lv_rdzc[k] = m->rdz;
            m->lv_r2dzcc[k] = m->r2dz; m->lv_kmax[k] = 0.8 * m->dx * m->dz / m->dt;
            m->lv_rdz2M[k] = m->rdz2; m->lv_rdM[k] = 1.0; m->lv_rdz2S[k] = m->rdz2; m->lv_rdS[k] = 1.0;
            m->lv_dzw[k] = m->dz; m->lv_wa[k] = 1.0; m->lv_wh[k] = 1.0;
        }
        m->lv_rdz_up = m->lv_rdz_dn = m->lv_rdz_c = m->rdz;
        m->lv_hfac = 1.0;
        m->lv_ks = 12000. / m->dz + 1;
        return;
    }
    double* dw = m->lv_dzw;
    double* tmp = (double*)malloc(sizeof(double) * nz);
    for (int k = 1; k <= nz - 2; k++) tmp[k] = 2.0 * (z[k] - zz[k]);
    tmp[0] = tmp[1]; tmp[nz - 1] = tmp[nz - 2];
    for (int k = 2; k <= nz - 2; k++) dw[k] = z[k] - z[k - 1];
    dw[1] = tmp[1]; dw[0] = tmp[1]; dw[nz - 1] = tmp[nz - 2];
    for (int k = 0; k < nz; k++) {
        m->lv_r2dzc[k] = (1.0 / tmp[k]) / 2.0;
        m->lv_r2dzw[k] = (1.0 / dw[k]) / 2.0;
        m->lv_rdzc[k] = 1.0 / tmp[k];
        m->lv_kmax[k] = 0.8 * m->dx * tmp[k] / m->dt;
    }
    for (int k = 1; k <= nz - 2; k++) {
        double zm = (k == 1) ? z[1] - tmp[1] : z[k - 1];          /* mirror centre below the surface */
        double zp = (k == nz - 2) ? z[nz - 2] + tmp[nz - 2] : z[k + 1];   /* and above the top face */
        m->lv_r2dzcc[k] = 1.0 / (zp - zm);
        /* Mparam (zeta at face k): bracket over dw[k]; up difference over dc[k], down over dc[k-1] */
        m->lv_rdz2M[k] = (1.0 / dw[k]) * (1.0 / tmp[k]);
        m->lv_rdM[k] = tmp[k] / tmp[k - 1];
        /* Hparam (centre k): bracket over dc[k]; up difference over dw[k+1], down over dw[k] */
        m->lv_rdz2S[k] = (1.0 / tmp[k]) * (1.0 / dw[k + 1]);
        m->lv_rdS[k] = dw[k + 1] / dw[k];
    }
    m->lv_rdz_up = 1.0 / dw[nz - 1];
    m->lv_rdz_dn = 1.0 / dw[nz - 2];
    m->lv_rdz_c = 1.0 / tmp[nz - 2];
    m->lv_hfac = m->dx / tmp[nz - 2];
    /* cal_w's metric (oracle/stretched_poisson.py): a_k = dw[k] / dx, h_k = dx / dc[k] */
    for (int k = 0; k < nz; k++) { m->lv_wa[k] = 1.0; m->lv_wh[k] = 1.0; }
    for (int k = 2; k <= nz - 2; k++) m->lv_wa[k] = (z[k] - z[k - 1]) / m->dx;
    for (int k = 1; k <= nz - 2; k++) m->lv_wh[k] = m->dx / (2.0 * (z[k] - zz[k]));
    int ks = 1;
    for (int k = 1; k <= nz - 1; k++) if (zz[k] <= 12000.) ks = k;
    m->lv_ks = ks;
    free(tmp);
}

/* ---------------------------------------------------------------- halos */

/* src/Boundary.cpp:3-7 */
static void bc1d_center(double* v, int nz) { v[0] = v[1]; v[nz - 1] = v[nz - 2]; }

/* src/Boundary.cpp:9-19: periodic in x on rows 1..nz-2, then zero gradient
 * in z over every column (ghost columns included). */
static void bc2d_center(orc_model* m, double* v) {
    int nx = m->nx, nz = m->nz;
    for (int k = 1; k <= nz - 2; k++) { F2(v, 0, k) = F2(v, nx - 2, k); F2(v, nx - 1, k) = F2(v, 1, k); }
    for (int i = 0; i <= nx - 1; i++) { F2(v, i, 0) = F2(v, i, 1); F2(v, i, nz - 1) = F2(v, i, nz - 2); }
}

/* src/Boundary.cpp:21-30: periodic in x, zero on rows 0, 1 and nz-1. */
static void bc2d_westdown(orc_model* m, double* v) {
    int nx = m->nx, nz = m->nz;
    for (int k = 1; k <= nz - 2; k++) { F2(v, 0, k) = F2(v, nx - 2, k); F2(v, nx - 1, k) = F2(v, 1, k); }
    for (int i = 0; i <= nx - 1; i++) { F2(v, i, 0) = 0.; F2(v, i, 1) = 0.; F2(v, i, nz - 1) = 0.; }
}

/* src/Boundary.cpp:32-52 (WATER, no P3) */
static void bc_all(orc_model* m) {
    bc2d_westdown(m, m->zetap);
    bc2d_center(m, m->thp);
    bc2d_westdown(m, m->w);
    bc2d_center(m, m->u);
    bc2d_center(m, m->qvp);
    bc2d_center(m, m->qcp);
    bc2d_center(m, m->qrp);
}

/* ------------------------------------------------------------ advection */

/* std::max / std::min semantics (first argument wins ties and NaN), which
 * the reference's std::max/std::min calls follow. */
static double maxd(double a, double b) { return (a < b) ? b : a; }
static double mind(double a, double b) { return (b < a) ? b : a; }

static double plus_part(double v) { return 0.5 * (v + fabs(v)); }   /* src/Advection.cpp:17-19 */
static double minus_part(double v) { return 0.5 * (v - fabs(v)); }  /* src/Advection.cpp:21-23 */

/* Flux-form advection of a scalar at cell centres with the 3rd-order
 * upwind-biased correction on i in [2, nx-3], k in [2, nz-3], then AB2
 * (src/Advection.cpp:25-81). */
static void advect_scalar(orc_model* m, const double* now, double* future, double* dvar) {
    int nx = m->nx, nz = m->nz;
    double *fu = m->flux_u, *fw = m->flux_w, *u = m->u, *w = m->w, *rhou = m->rhou, *rhow = m->rhow;
    memset(fu, 0, sizeof(double) * nx * nz);
    memset(fw, 0, sizeof(double) * nx * nz);
    ORC_PAR
    for (int k = 1; k <= nz - 1; k++) {
        for (int i = 1; i <= nx - 1; i++) {
            F2(fu, i, k) = rhou[k] * F2(u, i, k) * (F2(now, i, k) + F2(now, i - 1, k));
            F2(fw, i, k) = rhow[k] * F2(w, i, k) * (F2(now, i, k) + F2(now, i, k - 1));
            if (i >= 2 && i <= nx - 3 && k >= 2 && k <= nz - 3) {
                F2(fu, i, k) += -1. / 3. *
                    (rhou[k] * plus_part(F2(u, i, k)) * (F2(now, i, k) - F2(now, i - 1, k))
                     - sqrt(rhou[k] * plus_part(F2(u, i, k)) * rhou[k] * plus_part(F2(u, i - 1, k))) * (F2(now, i - 1, k) - F2(now, i - 2, k))
                     - rhou[k] * minus_part(F2(u, i, k)) * (F2(now, i, k) - F2(now, i - 1, k))
                     - sqrt(fabs(rhou[k] * minus_part(F2(u, i, k)) * rhou[k] * minus_part(F2(u, i + 1, k)))) * (F2(now, i + 1, k) - F2(now, i, k)));
                F2(fw, i, k) += -1. / 3. *
                    (rhow[k] * plus_part(F2(w, i, k)) * (F2(now, i, k) - F2(now, i, k - 1))
                     - sqrt(rhow[k] * plus_part(F2(w, i, k)) * rhow[k - 1] * plus_part(F2(w, i, k - 1))) * (F2(now, i, k - 1) - F2(now, i, k - 2))
                     - rhow[k] * minus_part(F2(w, i, k)) * (F2(now, i, k) - F2(now, i, k - 1))
                     - sqrt(fabs(rhow[k] * minus_part(F2(w, i, k)) * rhow[k + 1] * minus_part(F2(w, i, k + 1)))) * (F2(now, i, k + 1) - F2(now, i, k)));
            }
        }
    }
    bc2d_center(m, fu);
    bc2d_center(m, fw);
    for (int i = 0; i < nx; i++) { F2(fw, i, 0) = 0.; F2(fw, i, nz - 1) = 0.; }
    int sn = (m->step + 1) % 2, so = m->step % 2;
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++) {
        for (int i = 1; i <= nx - 2; i++) {
            double px = (F2(fu, i + 1, k) - F2(fu, i, k)) * m->r2dx / rhou[k];
            double pz = (F2(fw, i, k + 1) - F2(fw, i, k)) * m->lv_r2dzc[k] / rhou[k];
            H3(dvar, i, k, sn) = -px - pz;
            if (m->step == 0) H3(dvar, i, k, 0) = H3(dvar, i, k, 1);
            F2(future, i, k) = F2(now, i, k) + 1.5 * m->dt * H3(dvar, i, k, sn) - 0.5 * m->dt * H3(dvar, i, k, so);
        }
    }
}

/* Vorticity advection at zeta points (src/Advection.cpp:84-149). */
static void advect_zeta(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double *Uw = m->U_w, *Wu = m->W_u, *u = m->u, *w = m->w, *z = m->zeta;
    double *rhou = m->rhou, *rhow = m->rhow, *fu = m->flux_u, *fw = m->flux_w;
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++) {
        for (int i = 1; i <= nx - 2; i++) {
            F2(Uw, i, k) = 0.25 * (rhou[k] * (F2(u, i + 1, k) + F2(u, i, k)) + rhou[k - 1] * (F2(u, i + 1, k - 1) + F2(u, i, k - 1)));
            F2(Wu, i, k) = 0.25 * (rhow[k + 1] * (F2(w, i, k + 1) + F2(w, i - 1, k + 1)) + rhow[k] * (F2(w, i, k) + F2(w, i - 1, k)));
        }
    }
    bc2d_center(m, Uw);
    bc2d_center(m, Wu);
    for (int i = 0; i < nx; i++) { F2(Wu, i, 0) = 0.; F2(Wu, i, nz - 1) = 0.; }
    memset(fu, 0, sizeof(double) * nx * nz);
    memset(fw, 0, sizeof(double) * nx * nz);
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++) {
        for (int i = 0; i <= nx - 2; i++) {
            F2(fu, i, k) = F2(Uw, i, k) * (F2(z, i + 1, k) + F2(z, i, k));
            F2(fw, i, k) = F2(Wu, i, k) * (F2(z, i, k + 1) + F2(z, i, k));
            if (i >= 2 && i <= nx - 3 && k >= 2 && k <= nz - 3) {
                F2(fu, i, k) += -1. / 3. * (plus_part(F2(Uw, i, k)) * (F2(z, i + 1, k) - F2(z, i, k))
                    - sqrt(plus_part(F2(Uw, i, k)) * plus_part(F2(Uw, i - 1, k))) * (F2(z, i, k) - F2(z, i - 1, k))
                    - minus_part(F2(Uw, i, k)) * (F2(z, i + 1, k) - F2(z, i, k))
                    - sqrt(fabs(minus_part(F2(Uw, i, k)) * minus_part(F2(Uw, i + 1, k)))) * (F2(z, i + 2, k) - F2(z, i + 1, k)));
                F2(fw, i, k) += -1. / 3. * (plus_part(F2(Wu, i, k)) * (F2(z, i, k + 1) - F2(z, i, k))
                    - sqrt(plus_part(F2(Wu, i, k)) * plus_part(F2(Wu, i, k - 1))) * (F2(z, i, k) - F2(z, i, k - 1))
                    - minus_part(F2(Wu, i, k)) * (F2(z, i, k + 1) - F2(z, i, k))
                    - sqrt(fabs(minus_part(F2(Wu, i, k)) * minus_part(F2(Wu, i, k + 1)))) * (F2(z, i, k + 2) - F2(z, i, k + 1)));
            }
        }
    }
    bc2d_center(m, fu);
    bc2d_center(m, fw);
    for (int i = 0; i < nx; i++) { F2(fw, i, 0) = 0.; F2(fw, i, nz - 1) = 0.; }
    int sn = (m->step + 1) % 2, so = m->step % 2;
    ORC_PAR
    for (int k = 2; k <= nz - 2; k++) {
        for (int i = 1; i <= nx - 2; i++) {
            double px = (F2(fu, i, k) - F2(fu, i - 1, k)) * m->r2dx / rhow[k];
            double pz = (F2(fw, i, k) - F2(fw, i, k - 1)) * m->lv_r2dzw[k] / rhow[k];
            H3(m->dzeta_advect, i, k, sn) = -px - pz;
            if (m->step == 0) H3(m->dzeta_advect, i, k, 0) = H3(m->dzeta_advect, i, k, 1);
            F2(m->zetap, i, k) = F2(z, i, k) + 1.5 * m->dt * H3(m->dzeta_advect, i, k, sn) - 0.5 * m->dt * H3(m->dzeta_advect, i, k, so);
        }
    }
}

/* Rain sedimentation (src/Advection.cpp:153-192). */
static void advect_qr_vt(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double *fw = m->flux_w, *qr = m->qr, *rhow = m->rhow, *rhou = m->rhou;
    memset(fw, 0, sizeof(double) * nx * nz);
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++) {
        for (int i = 1; i <= nx - 2; i++) {
            double VT = 1E-2 * (3634 * pow(1E-3 * rhow[k] * 0.5 * (F2(qr, i, k) + F2(qr, i, k - 1)), 0.1346) * pow(rhow[k] / rhow[1], -0.5));
            F2(fw, i, k) = rhow[k] * VT * (F2(qr, i, k) + F2(qr, i, k - 1));
        }
    }
    bc2d_center(m, fw);
    for (int i = 0; i < nx; i++) { F2(fw, i, 0) = 0.; F2(fw, i, nz - 1) = 0.; }
    int sn = (m->step + 1) % 2, so = m->step % 2;
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++) {
        for (int i = 1; i <= nx - 2; i++) {
            double p = (F2(fw, i, k + 1) - F2(fw, i, k)) * m->lv_r2dzc[k] / rhou[k];
            H3(m->dqr_VT, i, k, sn) = p;
            if (m->step == 0) H3(m->dqr_VT, i, k, 0) = H3(m->dqr_VT, i, k, 1);
            F2(m->qrp, i, k) += 1.5 * m->dt * H3(m->dqr_VT, i, k, sn) - 0.5 * m->dt * H3(m->dqr_VT, i, k, so);
        }
    }
}

/* ------------------------------------------------------------- buoyancy */

static double thv(orc_model* m, int i, int k) {  /* src/Buoyancy.cpp:3-9 */
    return F2(m->th, i, k) * (1 + 0.608 * F2(m->qv, i, k));
}

/* src/Buoyancy.cpp:11-58 (WATER, AB2) */
static void buoyancy(orc_model* m) {
    int nx = m->nx, nz = m->nz, sn = (m->step + 1) % 2, so = m->step % 2;
    double *rhow = m->rhow, *thvb = m->thvb, *qc = m->qc, *qr = m->qr, g = m->GRAVITY;
    ORC_PAR
    for (int k = 2; k < nz - 1; k++) {
        for (int i = 1; i < nx - 1; i++) {
            double b = g / rhow[k] * 0.5 * ((thv(m, i, k) - thv(m, i - 1, k)) / thvb[k] + (thv(m, i, k - 1) - thv(m, i - 1, k - 1)) / thvb[k - 1]) * m->rdx;
            H3(m->dth_buoyancy, i, k, sn) = b;
            if (m->step == 0) H3(m->dth_buoyancy, i, k, 0) = H3(m->dth_buoyancy, i, k, 1);
            double bc = g / rhow[k] * (0.5 * (F2(qc, i, k) + F2(qc, i, k - 1)) - 0.5 * (F2(qc, i - 1, k) + F2(qc, i - 1, k - 1))) * m->rdx;
            double br = g / rhow[k] * (0.5 * (F2(qr, i, k) + F2(qr, i, k - 1)) - 0.5 * (F2(qr, i - 1, k) + F2(qr, i - 1, k - 1))) * m->rdx;
            H3(m->dth_buoyancy, i, k, sn) += -bc - br;
            if (m->step == 0) H3(m->dth_buoyancy, i, k, 0) = H3(m->dth_buoyancy, i, k, 1);
            F2(m->zetap, i, k) += (1.5 * m->dt * H3(m->dth_buoyancy, i, k, sn)) - (0.5 * m->dt * H3(m->dth_buoyancy, i, k, so));
        }
    }
}

/* --------------------------------------------------------- microphysics */

/* src/MicroPhysics.cpp:116-138: clip negatives, rescale positives so the
 * domain total is conserved (two domain-wide sums). */
static void negative_value_process(orc_model* m, double* v) {
    int nx = m->nx, nz = m->nz;
    double pos = 0., neg = 0.;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+ : pos, neg)
#endif
    for (int k = 1; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++) {
            if (F2(v, i, k) >= 0.) pos += F2(v, i, k);
            else { neg += F2(v, i, k); F2(v, i, k) = 0.; }
        }
    if (pos == 0. || fabs(neg) > pos) return;
    double ratio = 1. - fabs(neg / pos);
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++)
            if (F2(v, i, k) > 0) F2(v, i, k) = F2(v, i, k) * ratio;
}

/* src/MicroPhysics.cpp:29-51 */
static void autoconversion(orc_model* m) {
    double autort = 0.001, autotr = 0.001;
    ORC_PAR
    for (int k = 1; k <= m->nz - 2; k++)
        for (int i = 1; i <= m->nx - 2; i++) {
            double qcplus = maxd(0., F2(m->qcp, i, k));
            double ar = autort * (qcplus - autotr);
            ar = maxd(0., ar);
            double arcrdt = mind(ar * m->dt, qcplus);
            F2(m->qcp, i, k) = F2(m->qcp, i, k) - arcrdt;
            F2(m->qrp, i, k) = F2(m->qrp, i, k) + arcrdt;
            F2(m->autoconversion, i, k) = arcrdt;
        }
}

/* src/MicroPhysics.cpp:54-77 */
static void accretion(orc_model* m) {
    double accrrt = 2.2;
    ORC_PAR
    for (int k = 1; k <= m->nz - 2; k++)
        for (int i = 1; i <= m->nx - 2; i++) {
            double qcplus = maxd(0., F2(m->qcp, i, k));
            double qrplus = maxd(0., F2(m->qrp, i, k));
            double cr = accrrt * qcplus * (pow(qrplus, 0.875));
            double arcrdt = mind(cr * m->dt, qcplus);
            F2(m->qcp, i, k) = F2(m->qcp, i, k) - arcrdt;
            F2(m->qrp, i, k) = F2(m->qrp, i, k) + arcrdt;
            F2(m->accretion, i, k) = arcrdt;
        }
}

/* src/MicroPhysics.cpp:80-114 */
static void evaporation(orc_model* m) {
    ORC_PAR
    for (int k = 1; k <= m->nz - 2; k++) {
        double pc = 380. / (pow(m->pib[k], m->Cp / m->Rd) * m->P0);
        for (int i = 1; i <= m->nx - 2; i++) {
            double qrplus = maxd(0., F2(m->qrp, i, k));
            double qvplus = maxd(0., F2(m->qvp, i, k));
            double qvs = pc * exp(17.27 * (m->pib[k] * F2(m->thp, i, k) - 273.) / (m->pib[k] * F2(m->thp, i, k) - 36.));
            double deficit = maxd((1. - qvplus / qvs), 0.);
            double coef = 1.6 + 124.9 * pow((1E-3 * m->rhou[k] * qrplus), 0.2046);
            double er = coef * deficit * (pow(1E-3 * m->rhou[k] * qrplus, 0.525)) / ((5.4E5 + 2.55E6 / (1E-2 * m->pb[k] * qvs)) * 1E-3 * m->rhou[k]);
            double erdt = mind(qrplus, maxd(0., er * m->dt));
            F2(m->qrp, i, k) = F2(m->qrp, i, k) - erdt;
            F2(m->qvp, i, k) = F2(m->qvp, i, k) + erdt;
            F2(m->thp, i, k) = F2(m->thp, i, k) - m->Lv * erdt / (m->Cp * m->pib[k]);
            F2(m->evaporation, i, k) = erdt;
        }
    }
}

/* Saturation adjustment (src/MicroPhysics.cpp:7-26). */
static void condensation(orc_model* m) {
    ORC_PAR
    for (int k = 1; k <= m->nz - 2; k++) {
        double pc = 380. / (pow(m->pib[k], m->Cp / m->Rd) * m->P0);
        for (int i = 1; i <= m->nx - 2; i++) {
            double qvs = pc * exp(17.27 * (m->pib[k] * F2(m->thp, i, k) - 273.) / (m->pib[k] * F2(m->thp, i, k) - 36.));
            double phi = qvs * (17.27 * 237. * m->Lv) / (m->Cp * pow(F2(m->thp, i, k) * m->pib[k] - 36., 2));
            double C = (F2(m->qvp, i, k) - qvs) / (1 + phi);
            if (fabs(C) > F2(m->qcp, i, k) && C < 0) C = -F2(m->qcp, i, k);
            F2(m->qvp, i, k) = F2(m->qvp, i, k) - C;
            F2(m->qcp, i, k) = F2(m->qcp, i, k) + C;
            F2(m->thp, i, k) = F2(m->thp, i, k) + m->Lv / (m->Cp * m->pib[k]) * C;
            F2(m->condensation, i, k) = C;
        }
    }
}

/* Surface rain diagnostic (src/Iteration.cpp:114-119). */
static void precip_diag(orc_model* m) {
    for (int i = 1; i <= m->nx - 2; i++) {
        double VT = 1E-2 * (3634 * pow(1E-3 * m->rhou[1] * F2(m->qr, i, 1), 0.1346) * pow(m->rhou[1] / m->rhow[1], -0.5));
        double rain = -m->rhou[1] * (0.5 * (F2(m->w, i, 2) + 0.) - VT) * F2(m->qr, i, 1);
        m->precip[i] = rain < 0 ? 0. : rain;
    }
}

/* src/AddForcing.cpp:6-28 as built for the Kessler configuration: the
 * large-scale Q1/Q2 terms (TROPICALFORCING) are carried as optional profiles
 * that are zero unless a caller sets them; the random th forcing is added
 * while status_for_adding_forcing holds. */
static void add_forcing(orc_model* m) {
    ORC_PAR
    for (int k = 1; k <= m->nz - 2; k++)
        for (int i = 1; i <= m->nx - 2; i++) {
            double dt = m->dt;
            F2(m->thp, i, k) += dt * m->Q1LS[k];
            F2(m->qvp, i, k) += dt * m->Q2LS[k];
            if (m->status_for_adding_forcing) F2(m->thp, i, k) += dt * F2(m->init_th_forcing, i, k);
        }
}

/* ------------------------------------------------------------ elliptic */

/* Exact solve of the cal_w system A x = b (matrix: src/PoissonSolver.cpp:760-796).
 * Row (k, i), k = 2..nz-2, i = 1..nx-2:
 *   x[i-1] + x[i+1] - (2 + rhow_k/rhou_k + rhow_k/rhou_{k-1}) x
 *     + (rhow_k/rhou_k) x[k+1] + (rhow_k/rhou_{k-1}) x[k-1] = b,
 * periodic in i, x = 0 beyond k = 2 and k = nz-2. A real DFT in i turns the
 * x-part of mode p into -4 sin^2(pi p / NX); each mode then needs one
 * tridiagonal solve in k. */
/* Row (kk, j) of a separable operator with level coefficients cx, ru, rd:
 *   cx[kk] (x[j-1] + x[j+1] - 2 x) + ru[kk] (x[kk+1] - x) + rd[kk] (x[kk-1] - x) = b,
 * periodic in j, x = 0 beyond the first and last rows; solved exactly. */
static void solve_separable(int NX, int NK, const double* cxk, const double* ruk, const double* rdk,
                            const double* b, double* x);

void orc_solve_A(orc_model* m, const double* b, double* x) {
    int NK = m->nz - 3;
    double* cf = (double*)malloc(sizeof(double) * 3 * NK);
    for (int kk = 0; kk < NK; kk++) {
        int k = kk + 2;
        cf[kk] = 1.0;
        cf[NK + kk] = m->rhow[k] / m->rhou[k];
        cf[2 * NK + kk] = m->rhow[k] / m->rhou[k - 1];
    }
    solve_separable(m->nx - 2, NK, cf, cf + NK, cf + 2 * NK, b, x);
    free(cf);
}

#ifdef ORC_FAST_SOLVE
/* In-place iterative radix-2 FFT of n = 2^q complex values (Cooley-Tukey,
 * decimation in time): bit-reversal permutation, then log2(n) butterfly
 * stages; sign -1 forward, +1 backward (unscaled). Twiddles come from a
 * table of cos / sin(2 pi j / n), j < n/2. */
static void fft_radix2(double* re, double* im, int n, const double* tc, const double* ts, int sign) {
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, stride = n / len;
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < half; k++) {
                const double wr = tc[k * stride], wi = sign * ts[k * stride];
                const int a = i + k, b = a + half;
                const double vr = re[b] * wr - im[b] * wi, vi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - vr; im[b] = im[a] - vi;
                re[a] += vr; im[a] += vi;
            }
    }
}

/* solve_separable for NX a power of two: FFT each row, one real tridiagonal
 * solve per mode applied to the real and imaginary parts, inverse FFT. */
static void solve_separable_fft(int NX, int NK, const double* cxk, const double* ruk, const double* rdk,
                                const double* b, double* x) {
    const double twopi = 6.283185307179586476925286766559;
    double* tc = (double*)malloc(sizeof(double) * (NX / 2 + 1));
    double* ts = (double*)malloc(sizeof(double) * (NX / 2 + 1));
    for (int j = 0; j < NX / 2; j++) { tc[j] = cos(twopi * j / NX); ts[j] = sin(twopi * j / NX); }
    double* hr = (double*)malloc(sizeof(double) * (size_t)NX * NK);
    double* hi = (double*)malloc(sizeof(double) * (size_t)NX * NK);
    ORC_PAR
    for (int kk = 0; kk < NK; kk++) {
        double* r = hr + (size_t)kk * NX;
        double* q = hi + (size_t)kk * NX;
        for (int j = 0; j < NX; j++) { r[j] = b[(size_t)kk * NX + j]; q[j] = 0.; }
        fft_radix2(r, q, NX, tc, ts, -1);
    }
    ORC_PAR
    for (int p = 0; p < NX; p++) {
        double* cp = (double*)malloc(sizeof(double) * NK);
        const int pm = p <= NX / 2 ? p : NX - p;
        const double lam = -4.0 * pow(sin(3.14159265358979323846264338327950 * pm / NX), 2);
        double den0 = cxk[0] * lam - (ruk[0] + rdk[0]);
        cp[0] = (NK > 1 ? ruk[0] : 0.) / den0;
        hr[p] /= den0;
        hi[p] /= den0;
        for (int kk = 1; kk < NK; kk++) {
            const double up = kk < NK - 1 ? ruk[kk] : 0., lw = rdk[kk];
            const double den = cxk[kk] * lam - (ruk[kk] + rdk[kk]) - lw * cp[kk - 1];
            cp[kk] = up / den;
            hr[(size_t)kk * NX + p] = (hr[(size_t)kk * NX + p] - lw * hr[(size_t)(kk - 1) * NX + p]) / den;
            hi[(size_t)kk * NX + p] = (hi[(size_t)kk * NX + p] - lw * hi[(size_t)(kk - 1) * NX + p]) / den;
        }
        for (int kk = NK - 2; kk >= 0; kk--) {
            hr[(size_t)kk * NX + p] -= cp[kk] * hr[(size_t)(kk + 1) * NX + p];
            hi[(size_t)kk * NX + p] -= cp[kk] * hi[(size_t)(kk + 1) * NX + p];
        }
        free(cp);
    }
    ORC_PAR
    for (int kk = 0; kk < NK; kk++) {
        double* r = hr + (size_t)kk * NX;
        double* q = hi + (size_t)kk * NX;
        fft_radix2(r, q, NX, tc, ts, +1);
        for (int j = 0; j < NX; j++) x[(size_t)kk * NX + j] = r[j] / NX;
    }
    free(tc); free(ts); free(hr); free(hi);
}
#endif

static void solve_separable(int NX, int NK, const double* cxk, const double* ruk, const double* rdk,
                            const double* b, double* x) {
#ifdef ORC_FAST_SOLVE
    if (NX >= 2 && (NX & (NX - 1)) == 0) {
        solve_separable_fft(NX, NK, cxk, ruk, rdk, b, x);
        return;
    }
#endif
    double* c = (double*)malloc(sizeof(double) * NX);
    double* s = (double*)malloc(sizeof(double) * NX);
    double* hat = (double*)calloc((size_t)NX * NK, sizeof(double));
    double* sol = (double*)calloc((size_t)NX * NK, sizeof(double));
    double *lo = (double*)malloc(sizeof(double) * NK), *di = (double*)malloc(sizeof(double) * NK),
           *up = (double*)malloc(sizeof(double) * NK), *cp = (double*)malloc(sizeof(double) * NK),
           *dp = (double*)malloc(sizeof(double) * NK);
    const double twopi = 6.283185307179586476925286766559;
    for (int j = 0; j < NX; j++) { c[j] = cos(twopi * j / NX); s[j] = sin(twopi * j / NX); }
    /* forward: coefficients of cos and sin for modes p = 0..NX/2 */
    int P = NX / 2;
    for (int kk = 0; kk < NK; kk++) {
        const double* row = b + (size_t)kk * NX;
        for (int p = 0; p <= P; p++) {
            double a = 0., bs = 0.;
            for (int j = 0; j < NX; j++) {
                int t = (int)(((long long)p * j) % NX);
                a += row[j] * c[t];
                bs += row[j] * s[t];
            }
            hat[(size_t)kk * NX + p] = a;
            if (p > 0 && !(NX % 2 == 0 && p == P)) hat[(size_t)kk * NX + NX - p] = bs;
        }
    }
    /* one tridiagonal solve per coefficient column */
    for (int col = 0; col < NX; col++) {
        int p = col <= P ? col : NX - col;
        double lam = -4.0 * pow(sin(3.14159265358979323846264338327950 * p / NX), 2);
        for (int kk = 0; kk < NK; kk++) {
            double ru = ruk[kk], rd = rdk[kk];
            di[kk] = cxk[kk] * lam - (ru + rd);
            up[kk] = kk < NK - 1 ? ru : 0.;
            lo[kk] = kk > 0 ? rd : 0.;
        }
        cp[0] = up[0] / di[0];
        dp[0] = hat[col] / di[0];
        for (int kk = 1; kk < NK; kk++) {
            double den = di[kk] - lo[kk] * cp[kk - 1];
            cp[kk] = up[kk] / den;
            dp[kk] = (hat[(size_t)kk * NX + col] - lo[kk] * dp[kk - 1]) / den;
        }
        sol[(size_t)(NK - 1) * NX + col] = dp[NK - 1];
        for (int kk = NK - 2; kk >= 0; kk--)
            sol[(size_t)kk * NX + col] = dp[kk] - cp[kk] * sol[(size_t)(kk + 1) * NX + col];
    }
    /* inverse */
    for (int kk = 0; kk < NK; kk++) {
        const double* h = sol + (size_t)kk * NX;
        for (int j = 0; j < NX; j++) {
            double v = h[0];
            for (int p = 1; p <= P; p++) {
                int t = (int)(((long long)p * j) % NX);
                if (NX % 2 == 0 && p == P) v += h[p] * c[t];
                else v += 2.0 * (h[p] * c[t] + h[NX - p] * s[t]);
            }
            x[(size_t)kk * NX + j] = v / NX;
        }
    }
    free(c); free(s); free(hat); free(sol); free(lo); free(di); free(up); free(cp); free(dp);
}

/* The cal_w system on stretched levels (oracle/stretched_poisson.py): row
 * (k, i) as orc_solve_A's with ru_k = rhow_k h_k / (a_k rhou_k) and
 * rd_k = rhow_k h_{k-1} / (a_k rhou_{k-1}), a and h from levels(). */
void orc_solve_W(orc_model* m, const double* b, double* x) {
    int NK = m->nz - 3;
    levels(m);
    double* cf = (double*)malloc(sizeof(double) * 3 * NK);
    for (int kk = 0; kk < NK; kk++) {
        int k = kk + 2;
        double a = m->lv_wa[k];
        cf[kk] = 1.0;
        cf[NK + kk] = m->rhow[k] * m->lv_wh[k] / (a * m->rhou[k]);
        cf[2 * NK + kk] = m->rhow[k] * m->lv_wh[k - 1] / (a * m->rhou[k - 1]);
    }
    solve_separable(m->nx - 2, NK, cf, cf + NK, cf + 2 * NK, b, x);
    free(cf);
}

void orc_apply_A(orc_model* m, const double* x, double* y) {
    int NX = m->nx - 2, NK = m->nz - 3;
    for (int kk = 0; kk < NK; kk++) {
        int k = kk + 2;
        double ru = m->rhow[k] / m->rhou[k], rd = m->rhow[k] / m->rhou[k - 1];
        for (int j = 0; j < NX; j++) {
            double xc = x[(size_t)kk * NX + j];
            double v = -(2. + ru + rd) * xc + x[(size_t)kk * NX + (j + NX - 1) % NX] + x[(size_t)kk * NX + (j + 1) % NX];
            if (kk + 1 < NK) v += ru * x[(size_t)(kk + 1) * NX + j];
            if (kk > 0) v += rd * x[(size_t)(kk - 1) * NX + j];
            y[(size_t)kk * NX + j] = v;
        }
    }
}

/* src/PoissonSolver.cpp:439-479 (Eigen branch) with an exact solve. */
static void cal_w(orc_model* m) {
    int nx = m->nx, nz = m->nz, NX = nx - 2;
    double* b = m->work;
    double* x = m->work + (size_t)nx * nz;
    int cnt = 0;
    for (int k = 2; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++)
            b[cnt++] = m->rhow[k] * m->rhow[k] * (F2(m->zetap, i + 1, k) - F2(m->zetap, i, k)) * m->dx;
    if (m->stretched) orc_solve_W(m, b, x);
    else orc_solve_A(m, b, x);
    cnt = 0;
    for (int k = 2; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++) F2(m->w, i, k) = x[cnt++] / m->rhow[k];
    (void)NX;
    bc2d_westdown(m, m->w);
}

/* The streamfunction formulation (STREAMFUNCTION), which the reference ships
 * switched off and unfinished (src/Config.hpp:8). Its matrix
 * (src/PoissonSolver.cpp:726-756), row (k, i), k = 2..nz-2, i = 1..nx-2:
 *   (x[i-1] + x[i+1]) / rhow_k + x[k+1] / rhou_k + x[k-1] / rhou_{k-1}
 *     - (2 / rhow_k + 1 / rhou_k + 1 / rhou_{k-1} - POISSONPARAM) x = b,
 * periodic in i, with POISSONPARAM = 0 (the reference defines it nowhere). */
void orc_apply_psi(orc_model* m, const double* x, double* y) {
    int NX = m->nx - 2, NK = m->nz - 3;
    for (int kk = 0; kk < NK; kk++) {
        int k = kk + 2;
        double cx = 1. / m->rhow[k], ru = 1. / m->rhou[k], rd = 1. / m->rhou[k - 1];
        for (int j = 0; j < NX; j++) {
            double xc = x[(size_t)kk * NX + j];
            double v = -(2. * cx + ru + rd) * xc
                       + cx * (x[(size_t)kk * NX + (j + NX - 1) % NX] + x[(size_t)kk * NX + (j + 1) % NX]);
            if (kk + 1 < NK) v += ru * x[(size_t)(kk + 1) * NX + j];
            if (kk > 0) v += rd * x[(size_t)(kk - 1) * NX + j];
            y[(size_t)kk * NX + j] = v;
        }
    }
}

void orc_solve_psi(orc_model* m, const double* b, double* x) {
    int NK = m->nz - 3;
    double* cf = (double*)malloc(sizeof(double) * 3 * NK);
    for (int kk = 0; kk < NK; kk++) {
        int k = kk + 2;
        cf[kk] = 1. / m->rhow[k];
        cf[NK + kk] = 1. / m->rhou[k];
        cf[2 * NK + kk] = 1. / m->rhou[k - 1];
    }
    solve_separable(m->nx - 2, NK, cf, cf + NK, cf + 2 * NK, b, x);
    free(cf);
}

/* src/PoissonSolver.cpp:124-177 (Eigen branch) with an exact solve: psi from
 * zeta (b = zetap dx^2), its ghosts, then u and w from psi. The routine's
 * w-zeroing loop runs over i < nz (line 172), which the westdown halo that
 * follows makes immaterial: w = 0 at k = 0, 1, nz-1 for every i. */
static void calpsiuw(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double* b = m->work;
    double* x = m->work + (size_t)nx * nz;
    int cnt = 0;
    for (int k = 2; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++) b[cnt++] = F2(m->zetap, i, k) * m->dx * m->dx;
    orc_solve_psi(m, b, x);
    cnt = 0;
    for (int k = 2; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++) F2(m->psi, i, k) = x[cnt++];
    for (int k = 2; k <= nz - 2; k++) {
        F2(m->psi, 0, k) = F2(m->psi, nx - 2, k);
        F2(m->psi, nx - 1, k) = F2(m->psi, 1, k);
    }
    for (int i = 0; i <= nx - 1; i++) F2(m->psi, i, 0) = F2(m->psi, i, 1) = F2(m->psi, i, nz - 1) = 0.;
    bc2d_westdown(m, m->psi);
    for (int i = 1; i <= nx - 2; i++) {
        for (int k = 1; k <= nz - 2; k++) {
            F2(m->u, i, k) = -(m->rhow[k + 1] * F2(m->psi, i, k + 1) - m->rhow[k] * F2(m->psi, i, k)) * m->rdz / m->rhou[k];
            F2(m->w, i, k) = (F2(m->psi, i + 1, k) - F2(m->psi, i, k)) * m->rdx;
        }
    }
    for (int i = 0; i < nz && i < nx; i++) F2(m->w, i, nz - 1) = F2(m->w, i, 0) = F2(m->w, i, 1) = 0.;
    bc2d_center(m, m->u);
    bc2d_westdown(m, m->w);
}

void orc_set_streamfunction(orc_model* m, int on) { m->streamfunction = on; }

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* src/PoissonSolver.cpp:580-653 (Eigen branch). The chi problem
 * chi[i-1] - 2 chi[i] + chi[i+1] = h[i] (periodic) is only used through
 * uxi = (chi[i] - chi[i-1]) / dx with its mean removed; the differences
 * d[i] = chi[i] - chi[i-1] satisfy d[i+1] - d[i] = h[i], so uxi is the prefix
 * sum of h up to an additive constant, which the mean removal cancels. */
static void cal_u(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double* h = m->work;
    double tmp = 0.;
    for (int i = 1; i <= nx - 2; i++) {
        h[i - 1] = -(0. - m->rhow[nz - 2] * F2(m->w, i, nz - 2)) / m->rhou[nz - 2] * m->dx * m->lv_hfac;
        tmp += h[i - 1];
    }
    tmp /= (nx - 2);
    for (int i = 1; i <= nx - 2; i++) h[i - 1] = h[i - 1] - tmp;
    double run = 0.;
    for (int i = 1; i <= nx - 2; i++) {
        m->uxi[i] = run * m->rdx;
        run += h[i - 1];
    }
    tmp = 0.;
    for (int i = 1; i < nx - 1; i++) tmp += m->uxi[i];
    tmp /= (nx - 2);
    for (int i = 1; i <= nx - 2; i++) m->uxi[i] -= tmp;
    m->uxi[0] = m->uxi[nx - 2];
    m->uxi[nx - 1] = m->uxi[1];
    for (int i = 1; i <= nx - 2; i++) F2(m->u, i, nz - 2) = m->uxi[i] + m->ubarTopp;
    F2(m->u, 0, nz - 2) = F2(m->u, nx - 2, nz - 2);
    F2(m->u, nx - 1, nz - 2) = F2(m->u, 1, nz - 2);
    for (int i = 1; i <= nx - 2; i++) {
        double area = 0.;
        for (int k = nz - 3; k >= 1; k--) {
            area += ((F2(m->w, i, k + 1) - F2(m->w, i - 1, k + 1)) * m->rdx - m->rhow[k + 1] * F2(m->zetap, i, k + 1)) * -m->lv_dzw[k + 1];
            F2(m->u, i, k) = area + F2(m->u, i, nz - 2);
        }
    }
    bc2d_center(m, m->u);
}

/* Domain-mean top-boundary wind tendency, AB2 (src/PoissonSolver.cpp:655-676). */
static void pubar_top(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double down = 0., kup = 0., kdown = 0.;
    double *u = m->u, *w = m->w, *K = m->RKM, *rhou = m->rhou, *rhow = m->rhow;
    for (int i = 1; i < nx - 1; i++) {
        down += 0.25 * (rhou[nz - 2] * F2(u, i, nz - 2) + rhou[nz - 3] * F2(u, i, nz - 3)) * (F2(w, i, nz - 2) + F2(w, i - 1, nz - 2));
        kup += rhow[nz - 1] * 0.25 * (F2(K, i, nz - 1) + F2(K, i, nz - 2) + F2(K, i - 1, nz - 1) + F2(K, i - 1, nz - 2))
               * (m->lv_rdz_up * (F2(u, i, nz - 1) - F2(u, i, nz - 2)));
        kdown += rhow[nz - 2] * 0.25 * (F2(K, i, nz - 2) + F2(K, i, nz - 3) + F2(K, i - 1, nz - 2) + F2(K, i - 1, nz - 3))
                 * (m->rdx * (F2(w, i, nz - 2) - F2(w, i - 1, nz - 2)) + m->lv_rdz_dn * (F2(u, i, nz - 2) - F2(u, i, nz - 3)));
    }
    down /= ((double)(nx - 2.));
    kup /= ((double)(nx - 2.));
    kdown /= ((double)(nx - 2.));
    double a = (-down) * m->lv_rdz_c / rhou[nz - 2];
    double b = (kup - kdown) * m->lv_rdz_c / rhou[nz - 2];
    int sn = (m->step + 1) % 2, so = m->step % 2;
    m->dubarTop_advect[sn] = -a + b;
    if (m->step == 0) m->dubarTop_advect[0] = m->dubarTop_advect[1];
    m->ubarTopp = m->ubarTop + 1.5 * m->dt * m->dubarTop_advect[sn] - 0.5 * m->dt * m->dubarTop_advect[so];
}

/* ----------------------------------------------------------- turbulence */

/* src/Turbulent.cpp:68-90: in-place Gauss-Seidel sweep, k outer, i inner. */
static void mparam(orc_model* m, double* v) {
    int nx = m->nx, nz = m->nz;
    double *K = m->RKM, *rhou = m->rhou, *rhow = m->rhow;
    for (int k = 1; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++)
            F2(v, i, k) += m->rdx2 * m->dt *
                (0.5 * (F2(K, i, k) + F2(K, i, k - 1)) * (F2(v, i + 1, k) - F2(v, i, k)) -
                 0.5 * (F2(K, i - 1, k) + F2(K, i - 1, k - 1)) * (F2(v, i, k) - F2(v, i - 1, k)))
                + m->lv_rdz2M[k] * m->dt / rhow[k] *
                (rhou[k] * 0.5 * (F2(K, i, k) + F2(K, i - 1, k)) * (F2(v, i, k + 1) - F2(v, i, k)) -
                 (m->lv_rdM[k] * rhou[k - 1]) * 0.5 * (F2(K, i, k - 1) + F2(K, i - 1, k - 1)) * (F2(v, i, k) - F2(v, i, k - 1)));
}

/* src/Turbulent.cpp:92-114 */
static void hparam(orc_model* m, double* v) {
    int nx = m->nx, nz = m->nz;
    double *K = m->RKH, *rhou = m->rhou, *rhow = m->rhow;
    for (int k = 1; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++)
            F2(v, i, k) += m->rdx2 * m->dt *
                (0.5 * (F2(K, i + 1, k) + F2(K, i, k)) * (F2(v, i + 1, k) - F2(v, i, k)) -
                 0.5 * (F2(K, i, k) + F2(K, i - 1, k)) * (F2(v, i, k) - F2(v, i - 1, k)))
                + m->lv_rdz2S[k] * m->dt / rhou[k] *
                (rhow[k + 1] * 0.5 * (F2(K, i, k + 1) + F2(K, i, k)) * (F2(v, i, k + 1) - F2(v, i, k)) -
                 (m->lv_rdS[k] * rhow[k]) * 0.5 * (F2(K, i, k) + F2(K, i, k - 1)) * (F2(v, i, k) - F2(v, i, k - 1)));
}

/* Eddy viscosity/diffusivity from deformation and Richardson number, then the
 * diffusion sweeps (src/Turbulent.cpp:5-62). */
static void rkm_rkh(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    double *u = m->u, *w = m->w, *thp = m->thp;
    ORC_PAR
    for (int k = 1; k <= nz - 2; k++)
        for (int i = 1; i <= nx - 2; i++) {
            double Rzeta = 0.5 * ((F2(w, i + 1, k + 1) + F2(w, i + 1, k)) - (F2(w, i - 1, k + 1) + F2(w, i - 1, k))) * m->r2dx +
                           0.5 * ((F2(u, i + 1, k + 1) + F2(u, i, k + 1)) - (F2(u, i + 1, k - 1) + F2(u, i, k - 1))) * m->lv_r2dzcc[k];
            double Rotat = pow((F2(u, i + 1, k) - F2(u, i, k)) * m->rdx + (F2(w, i, k + 1) - F2(w, i, k)) * m->lv_rdzc[k], 2);
            double Ri = (m->GRAVITY / F2(thp, i, k) * (F2(thp, i, k + 1) - F2(thp, i, k - 1)) * m->lv_r2dzcc[k]) / (pow(Rzeta, 2) + 2. * Rotat);
            double km, kh;
            if (Ri < 0) {
                km = m->lambda2[k] * sqrt(pow(Rzeta, 2) + 2. * Rotat) * sqrt(1. - 16. * Ri);
                kh = m->lambda2[k] * sqrt(pow(Rzeta, 2) + 2. * Rotat) * 1.4 * sqrt(1. - 40. * Ri);
            } else if (0 < Ri && Ri < 0.25) {
                km = m->lambda2[k] * sqrt(pow(Rzeta, 2) + 2. * Rotat) * pow(1. - 4. * Ri, 4);
                kh = m->lambda2[k] * sqrt(pow(Rzeta, 2) + 2. * Rotat) * 1.4 * (1. - 1.2 * Ri) * pow(1. - 4. * Ri, 4);
            } else {
                km = 0.;
                kh = 0.;
            }
            km = maxd(km, 10.);
            kh = maxd(kh, 10.);
            km = mind(km, m->lv_kmax[k]);
            kh = mind(kh, m->lv_kmax[k]);
            F2(m->RKM, i, k) = km;
            F2(m->RKH, i, k) = kh;
        }
    bc2d_center(m, m->RKM);
    bc2d_center(m, m->RKH);
#ifdef _OPENMP
    /* five independent in-place sweeps: one field a thread */
#pragma omp parallel for schedule(static, 1)
    for (int f = 0; f < 5; f++) {
        if (f == 0) mparam(m, m->zetap);
        else hparam(m, f == 1 ? m->thp : f == 2 ? m->qvp : f == 3 ? m->qcp : m->qrp);
    }
#else
    mparam(m, m->zetap);
    hparam(m, m->thp);
    hparam(m, m->qvp);
    hparam(m, m->qcp);
    hparam(m, m->qrp);
#endif
}

/* ---------------------------------------------------------------- nudge */

static void nudge_theta(orc_model* m) {  /* src/NumericalProcess.cpp:60-71 */
    int nz = m->nz, ks = m->lv_ks;
    for (int k = ks; k < nz - 1; k++) {
        double CGR = m->CRAD * (m->z[k] - m->z[(nz - 1) - ks]) / (m->z[nz - 1] - m->z[(nz - 1) - ks]);
        for (int i = 1; i < m->nx - 1; i++) F2(m->thp, i, k) -= m->dt * CGR * (F2(m->thp, i, k) - m->thb_init[k]);
    }
}

static void nudge_zeta(orc_model* m) {  /* src/NumericalProcess.cpp:73-85 */
    int nz = m->nz, ks = m->lv_ks;
    for (int k = ks; k < nz - 1; k++) {
        double CGR = (1. / 360.) * (m->z_zeta[k] - m->z_zeta[(nz - 1) - ks]) / (m->z_zeta[nz - 1] - m->z_zeta[(nz - 1) - ks]);
        for (int i = 1; i < m->nx - 1; i++) F2(m->zetap, i, k) -= m->dt * CGR * (F2(m->zetap, i, k));
    }
}

static void nudge_qv(orc_model* m) {  /* src/NumericalProcess.cpp:87-96 */
    if (m->moisture_nudge_time == 0) return;
    for (int i = 0; i <= m->nx - 1; i++)
        for (int k = 0; k <= m->nz - 1; k++)
            F2(m->qvp, i, k) = F2(m->qvp, i, k) + m->dt * (m->qvb0[k] - F2(m->qv, i, k)) / m->moisture_nudge_time;
}

/* ---------------------------------------------------------- time level */

/* src/Iteration.cpp:42-86 */
static void update_mean(orc_model* m) {
    int nx = m->nx, nz = m->nz;
    for (int k = 0; k < nz; k++) { m->thbm[k] = m->thb[k]; m->thvbm[k] = m->thvb[k]; }
    ORC_PAR
    for (int k = 1; k < nz - 1; k++) {
        double tb = 0., qb = 0.;
        for (int i = 1; i < nx - 1; i++) { tb += F2(m->thp, i, k); qb += F2(m->qvp, i, k); }
        m->thb[k] = tb / (double)(nx - 2.);
        m->qvb[k] = qb / (double)(nx - 2.);
        m->thvb[k] = m->thb[k] * (1 + 0.608 * m->qvb[k]);
    }
    bc1d_center(m->thb, nz);
    bc1d_center(m->thvb, nz);
    bc1d_center(m->qvb, nz);
    for (int k = 1; k < nz - 1; k++) m->thb_zeta[k] = 0.5 * (m->thb[k - 1] + m->thb[k]);
    m->thb_zeta[0] = m->thb_zeta[1];
    m->thb_zeta[nz - 1] = m->thb_zeta[nz - 2];
}

/* src/Iteration.cpp:153-204 */
static void next_time_step(orc_model* m) {
    update_mean(m);
    size_t n = (size_t)m->nx * m->nz * sizeof(double);
    memcpy(m->zetam, m->zeta, n); memcpy(m->zeta, m->zetap, n);
    memcpy(m->thm, m->th, n); memcpy(m->th, m->thp, n);
    memcpy(m->qvm, m->qv, n); memcpy(m->qv, m->qvp, n);
    memcpy(m->qcm, m->qc, n); memcpy(m->qc, m->qcp, n);
    memcpy(m->qrm, m->qr, n); memcpy(m->qr, m->qrp, n);
    m->ubarTopm = m->ubarTop;
    m->ubarTop = m->ubarTopp;
}

/* The step body of src/Iteration.cpp:246-434 (AB2, WATER, Kessler). */
static void one_step(orc_model* m) {
    levels(m);
    m->step++;
    advect_zeta(m); buoyancy(m); bc2d_westdown(m, m->zetap);                 /* pzeta_pt */
    advect_scalar(m, m->th, m->thp, m->dth_advect); bc2d_center(m, m->thp);  /* pth_pt */
    advect_scalar(m, m->qv, m->qvp, m->dqv_advect);                          /* pqv_pt */
    negative_value_process(m, m->qvp); bc2d_center(m, m->qvp);
    advect_scalar(m, m->qc, m->qcp, m->dqc_advect);                          /* pqc_pt */
    negative_value_process(m, m->qcp); bc2d_center(m, m->qcp);
    advect_scalar(m, m->qr, m->qrp, m->dqr_advect); advect_qr_vt(m);         /* pqr_pt */
    negative_value_process(m, m->qrp); precip_diag(m); bc2d_center(m, m->qrp);
    m->status_for_adding_forcing = (m->step * m->dt <= m->addforcingtime);
    add_forcing(m);
    bc_all(m);
    if (m->streamfunction) calpsiuw(m);   /* src/Iteration.cpp:289-295 */
    else { pubar_top(m); cal_w(m); cal_u(m); }
    bc_all(m);
    autoconversion(m); accretion(m); evaporation(m); condensation(m);
    negative_value_process(m, m->qvp);
    negative_value_process(m, m->qcp);
    negative_value_process(m, m->qrp);
    bc_all(m);
    update_mean(m);
    rkm_rkh(m);
    nudge_theta(m);
    if (m->CASE != 2) nudge_zeta(m);
    nudge_qv(m);
    next_time_step(m);
}

int orc_call(orc_model* m, const char* n) {
    levels(m);
    if (!strcmp(n, "pzeta_pt")) { advect_zeta(m); buoyancy(m); bc2d_westdown(m, m->zetap); }
    else if (!strcmp(n, "pth_pt")) { advect_scalar(m, m->th, m->thp, m->dth_advect); bc2d_center(m, m->thp); }
    else if (!strcmp(n, "pqv_pt")) { advect_scalar(m, m->qv, m->qvp, m->dqv_advect); negative_value_process(m, m->qvp); bc2d_center(m, m->qvp); }
    else if (!strcmp(n, "pqc_pt")) { advect_scalar(m, m->qc, m->qcp, m->dqc_advect); negative_value_process(m, m->qcp); bc2d_center(m, m->qcp); }
    else if (!strcmp(n, "pqr_pt")) { advect_scalar(m, m->qr, m->qrp, m->dqr_advect); advect_qr_vt(m); negative_value_process(m, m->qrp); precip_diag(m); bc2d_center(m, m->qrp); }
    else if (!strcmp(n, "Advection_zeta")) advect_zeta(m);
    else if (!strcmp(n, "Bouyancy")) buoyancy(m);
    else if (!strcmp(n, "Advection_thermo_th")) advect_scalar(m, m->th, m->thp, m->dth_advect);
    else if (!strcmp(n, "Advection_qrVT")) advect_qr_vt(m);
    else if (!strcmp(n, "AddForcing")) add_forcing(m);
    else if (!strcmp(n, "BoundaryProcess2D_all")) bc_all(m);
    else if (!strcmp(n, "pubarTop_pt")) pubar_top(m);
    else if (!strcmp(n, "cal_w")) cal_w(m);
    else if (!strcmp(n, "cal_u")) cal_u(m);
    else if (!strcmp(n, "calpsiuw")) calpsiuw(m);
    else if (!strcmp(n, "autoconversion")) autoconversion(m);
    else if (!strcmp(n, "accretion")) accretion(m);
    else if (!strcmp(n, "evaporation")) evaporation(m);
    else if (!strcmp(n, "condensation")) condensation(m);
    else if (!strcmp(n, "NVP_qvp")) negative_value_process(m, m->qvp);
    else if (!strcmp(n, "NVP_qcp")) negative_value_process(m, m->qcp);
    else if (!strcmp(n, "NVP_qrp")) negative_value_process(m, m->qrp);
    else if (!strcmp(n, "updateMean")) update_mean(m);
    else if (!strcmp(n, "RKM_RKH")) rkm_rkh(m);
    else if (!strcmp(n, "Nudge_theta")) nudge_theta(m);
    else if (!strcmp(n, "Nudge_zeta")) nudge_zeta(m);
    else if (!strcmp(n, "Nudge_qv")) nudge_qv(m);
    else if (!strcmp(n, "nextTimeStep")) next_time_step(m);
    else if (!strcmp(n, "one_step")) one_step(m);
    else return -1;
    return 0;
}
