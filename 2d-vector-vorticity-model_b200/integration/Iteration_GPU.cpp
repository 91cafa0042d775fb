// The GPU_STEP translation unit: vvm::Iteration::TimeMarching on the B200
// step (libvvmgpu.so, include/vvm_gpu.h).
//
// This is the binding a maintainer of the reference adds. With GPU_STEP
// defined in src/Config.hpp, this file provides TimeMarching in place of the
// one in src/Iteration.cpp (src/Iteration.cpp:208-438), and the model links
// -lvvmgpu; every other member of Iteration (pzeta_pt, updateMean,
// nextTimeStep, ...) stays as it is, so the two builds can run side by side.
// It is the whole-step version of the reference's own device boundary, the
// GPU_POISSON unit (src/PoissonSolver_GPU_mpi.cpp, hooks at
// src/main.cpp:85-87,141-145): the `vvm` object keeps owning every host
// array; the fields live on the device for the whole run and come back to
// those arrays for output and at the end.
//
// Precision and solver are compile-time choices (defaults: the reference's
// FP64 arithmetic, multigrid-PCG to ||b - A W|| / ||b|| <= 1e-10).
// Failures print the library's message and exit, as the reference does on
// fatal device errors.
#include <cstdio>
#include <cstdlib>

#include "Declare.hpp"
#include "vvm_gpu.h"

#ifndef VVM_GPU_STEP_PRECISION
#define VVM_GPU_STEP_PRECISION VVM_PREC_FP64
#endif
#ifndef VVM_GPU_STEP_SOLVER
#define VVM_GPU_STEP_SOLVER VVM_SOLVER_MGPCG
#endif
#ifndef VVM_GPU_STEP_DEVICE
#define VVM_GPU_STEP_DEVICE 0
#endif

namespace {

// Host view of the model: the contiguous blocks behind every double** field
// (allocate2DContinuousArray, src/Declare.hpp:400-407) and the 1D profiles.
vvm_gpu_host_state view(vvm& m) {
    vvm_gpu_host_state s = {};
    s.zeta = m.zetacont;  s.zetap = m.zetapcont;  s.th = m.thcont;  s.thp = m.thpcont;
    s.qv = m.qvcont;      s.qvp = m.qvpcont;      s.qc = m.qccont;  s.qcp = m.qcpcont;
    s.qr = m.qrcont;      s.qrp = m.qrpcont;      s.u = m.ucont;    s.w = m.wcont;
    s.RKM = m.RKMcont;    s.RKH = m.RKHcont;
    s.dzeta_advect = m.dzeta_advectcont;  s.dth_buoyancy = m.dth_buoyancycont;
    s.dth_advect = m.dth_advectcont;      s.dqv_advect = m.dqv_advectcont;
    s.dqc_advect = m.dqc_advectcont;      s.dqr_advect = m.dqr_advectcont;
    s.dqr_VT = m.dqr_VTcont;
    s.rhou = m.rhou; s.rhow = m.rhow; s.thb = m.thb; s.thvb = m.thvb; s.qvb = m.qvb;
    s.pib = m.pib; s.pb = m.pb; s.thb_init = m.thb_init; s.qvb0 = m.qvb0;
    s.z = m.z; s.z_zeta = m.z_zeta; s.lambda2 = m.lambda2;
#if defined(TROPICALFORCING)
    s.Q1LS = m.Q1LS; s.Q2LS = m.Q2LS;
#endif
    s.init_th_forcing = m.init_th_forcingcont;
#if defined(KESSLER_MICROPHY)
    s.precip = m.precip;
#endif
    s.ubarTop = m.ubarTop; s.ubarTopp = m.ubarTopp;
    s.dubarTop_advect[0] = m.dubarTop_advect[0]; s.dubarTop_advect[1] = m.dubarTop_advect[1];
    s.step = m.step;
    return s;
}

// The scalars a download returns by value (the arrays are filled in place).
void take_scalars(vvm& m, const vvm_gpu_host_state& s) {
    m.ubarTop = s.ubarTop;
    m.ubarTopp = s.ubarTopp;
    m.dubarTop_advect[0] = s.dubarTop_advect[0];
    m.dubarTop_advect[1] = s.dubarTop_advect[1];
}

[[noreturn]] void die(const char* what, vvm_gpu_ctx* ctx) {
    char buf[512];
    vvm_gpu_last_error(ctx, buf, sizeof buf);
    std::fprintf(stderr, "GPU_STEP: %s failed: %s\n", what, buf);
    std::exit(1);
}

void download(vvm& model, vvm_gpu_ctx* ctx, vvm_gpu_host_state& s) {
    if (vvm_gpu_download_state(ctx, &s) != VVM_GPU_OK) die("vvm_gpu_download_state", ctx);
    take_scalars(model, s);
}

}  // namespace

// src/Iteration.cpp:208-438: step from 0 to TIMEEND / dt; the whole step body
// (advection, forcing, the Poisson solves, microphysics, turbulence,
// nudging, the time-level rotation) runs on the device, one vvm_gpu_step a
// step, which increments the step counter as the loop here does.
void vvm::Iteration::TimeMarching(vvm& model) {
    model.step = 0;
    const int nmax = (int)(model.TIMEEND / model.dt);
    vvm_gpu_desc d;
    vvm_gpu_desc_default(&d, model.nx - 2, model.nz - 2, model.dx, model.dz, model.dt);
    d.case_id = model.CASE;
    d.moisture_nudge_time = model.moisture_nudge_time;
    d.addforcingtime = model.addforcingtime;
    d.precision = VVM_GPU_STEP_PRECISION;
    d.solver = VVM_GPU_STEP_SOLVER;
    vvm_gpu_ctx* ctx = nullptr;
    if (vvm_gpu_create(&d, VVM_GPU_STEP_DEVICE, &ctx) != VVM_GPU_OK) die("vvm_gpu_create", nullptr);
    vvm_gpu_host_state s = view(model);
    if (vvm_gpu_upload_state(ctx, &s) != VVM_GPU_OK) die("vvm_gpu_upload_state", ctx);
    while (model.step < nmax) {
#if defined(OUTPUTNC) || defined(OUTPUTTXT)
        if (model.step % model.OUTPUTSTEP == 0) {   // src/Iteration.cpp:229-243
            download(model, ctx, s);
#if defined(OUTPUTNC)
            vvm::Output::output_nc(model.step, model);
#endif
#if defined(OUTPUTTXT)
            vvm::Output::outputalltxt(model.step, model);
#endif
        }
#endif
        if (vvm_gpu_step(ctx, 1) != VVM_GPU_OK) die("vvm_gpu_step", ctx);
        model.step++;
    }
    download(model, ctx, s);
    vvm_gpu_destroy(ctx);
}
