// C-ABI harness around the reference VVM step, compiled together with the
// reference's own translation units (see oracle/build_ref.sh).
//
// Test infrastructure only: the library built from this file is the CPU
// checker for the GPU path and the timed CPU baseline; no product code links
// against it.
//
// This file is not compiled on its own. build_ref.sh feeds g++ a stream made
// of oracle/ref_config.hpp, the reference's src/Declare.hpp (minus its
// Config.hpp include) and then this file, so `class vvm`, `Config_VVM` and the
// Eigen sparse types are already declared when this text is reached.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

namespace {

// Silences the per-step `std::cout << model.step` of
// Iteration::TimeMarching (src/Iteration.cpp:229) while a call runs.
// Also silences C stdio on fd 1 (the vvm destructor's printf "Free vvm",
// src/Declare.hpp:99, and cal_w's solver warnings, src/PoissonSolver.cpp:464),
// so a caller's stdout carries only its own output.
struct CoutMute {
    std::ostringstream sink;  // declared first: constructed before `saved` uses it
    std::streambuf* saved;
    int fd_saved;
    CoutMute() : saved(std::cout.rdbuf(sink.rdbuf())) {
        std::fflush(stdout);
        fd_saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        if (dn >= 0) {
            dup2(dn, 1);
            close(dn);
        }
    }
    ~CoutMute() {
        std::fflush(stdout);
        if (fd_saved >= 0) {
            dup2(fd_saved, 1);
            close(fd_saved);
        }
        std::cout.rdbuf(saved);
    }
};

// One time step exactly as vvm::Iteration::TimeMarching runs it for the
// AB2 + WATER + KESSLER_MICROPHY build (src/Iteration.cpp:246-434), without
// the output and timer bookkeeping. TimeMarching itself always restarts at
// step 0 (src/Iteration.cpp:212); this replica lets a caller take snapshots
// between steps. tests/ checks it bit-for-bit against TimeMarching.
void one_step(vvm& model) {
    model.step++;
    vvm::Iteration::pzeta_pt(model);
    vvm::Iteration::pth_pt(model);
    vvm::Iteration::pqv_pt(model);
    vvm::Iteration::pqc_pt(model);
    vvm::Iteration::pqr_pt(model);
    if (model.step * model.dt <= model.addforcingtime) model.status_for_adding_forcing = true;
    else model.status_for_adding_forcing = false;
    if (model.status_for_adding_forcing == true) {
        vvm::Init::RandomPerturbation(model, model.step + 0, -0.001, 0.001, 1.);
    }
    model.AddForcing(model);
    vvm::BoundaryProcess2D_all(model);

#if defined(STREAMFUNCTION)
    vvm::PoissonSolver::calpsiuw(model);
#else
    vvm::PoissonSolver::pubarTop_pt(model);
    vvm::PoissonSolver::cal_w(model);
    vvm::PoissonSolver::cal_u(model);
#endif
    vvm::BoundaryProcess2D_all(model);

    vvm::MicroPhysics::autoconversion(model);
    vvm::MicroPhysics::accretion(model);
    vvm::MicroPhysics::evaporation(model);
    vvm::MicroPhysics::condensation(model);
    vvm::MicroPhysics::NegativeValueProcess(model.qvp, model.nx, model.nz);
    vvm::MicroPhysics::NegativeValueProcess(model.qcp, model.nx, model.nz);
    vvm::MicroPhysics::NegativeValueProcess(model.qrp, model.nx, model.nz);
    vvm::BoundaryProcess2D_all(model);

    vvm::Iteration::updateMean(model);
    vvm::Turbulence::RKM_RKH(model);
    vvm::NumericalProcess::Nudge_theta(model);
    if (model.CASE != 2) vvm::NumericalProcess::Nudge_zeta(model);
    vvm::NumericalProcess::Nudge_qv(model);

    vvm::Iteration::nextTimeStep(model);
}

}  // namespace

extern "C" {

// Builds a model the way src/main.cpp:68-74 does, with the physical constants
// hard-coded there, for an interior grid of NX x NZ cells (the model adds one
// ghost cell on each side: nx = NX + 2, nz = NZ + 2, src/Declare.hpp:33,82-83).
// addforcingtime is a parameter so parity runs can switch the random forcing
// off (main.cpp passes 10 s).
void* ref_create(int NX, int NZ, double dx, double dz, double dt, int CASE,
                 double moisture_nudge_time, double tolerance, double addforcingtime) {
    Config_VVM config(dt, dx, dz, (int)(NX * dx + 0.5), (int)(NZ * dz + 0.5), 1e9, 10000, "",
                      1 << 30, 10., 10., 0.01, tolerance, 9.80665, 1003.5, 716.5, 287., 2.5E6,
                      1E5, 96500., addforcingtime, CASE, moisture_nudge_time,
                      2025, 3, 21, 12., 0., 0., 0., 0.);
    CoutMute mute;
    return new vvm(config);
}

void ref_destroy(void* h) {
    CoutMute mute;
    delete static_cast<vvm*>(h);
}

void ref_dims(void* h, int* nx, int* nz) {
    vvm& m = *static_cast<vvm*>(h);
    *nx = m.nx;
    *nz = m.nz;
}

// Contiguous [nx][nz] block behind a 2D field (k is the fast index).
double* ref_field(void* h, const char* name) {
    vvm& m = *static_cast<vvm*>(h);
    struct { const char* n; double* p; } tab[] = {
        {"zeta", m.zetacont}, {"zetam", m.zetamcont}, {"zetap", m.zetapcont},
        {"th", m.thcont}, {"thm", m.thmcont}, {"thp", m.thpcont},
        {"u", m.ucont}, {"w", m.wcont},
        {"qv", m.qvcont}, {"qvm", m.qvmcont}, {"qvp", m.qvpcont},
        {"qc", m.qccont}, {"qcm", m.qcmcont}, {"qcp", m.qcpcont},
        {"qr", m.qrcont}, {"qrm", m.qrmcont}, {"qrp", m.qrpcont},
        {"RKM", m.RKMcont}, {"RKH", m.RKHcont}, {"U_w", m.U_wcont}, {"W_u", m.W_ucont},
        {"init_th_forcing", m.init_th_forcingcont},
        {"evaporation", m.evaporationcont}, {"accretion", m.accretioncont},
        {"autoconversion", m.autoconversioncont}, {"condensation", m.condensationcont},
#if defined(STREAMFUNCTION)
        {"psi", m.psi[0]},
#endif
    };
    for (auto& e : tab) if (std::strcmp(e.n, name) == 0) return e.p;
    return nullptr;
}

// Contiguous [nx][nz][2] block behind an AB2 tendency history.
double* ref_hist(void* h, const char* name) {
    vvm& m = *static_cast<vvm*>(h);
    struct { const char* n; double* p; } tab[] = {
        {"dth_advect", m.dth_advectcont}, {"dth_buoyancy", m.dth_buoyancycont},
        {"dzeta_advect", m.dzeta_advectcont}, {"dqv_advect", m.dqv_advectcont},
        {"dqc_advect", m.dqc_advectcont}, {"dqr_advect", m.dqr_advectcont},
        {"dqr_VT", m.dqr_VTcont},
    };
    for (auto& e : tab) if (std::strcmp(e.n, name) == 0) return e.p;
    return nullptr;
}

// 1D profiles ([nz], [nz+1] for *_lev, [nx] for xi/uxi/precip).
double* ref_prof(void* h, const char* name) {
    vvm& m = *static_cast<vvm*>(h);
    struct { const char* n; double* p; } tab[] = {
        {"thb", m.thb}, {"thbm", m.thbm}, {"thb_zeta", m.thb_zeta}, {"thb_init", m.thb_init},
        {"rhou", m.rhou}, {"rhow", m.rhow}, {"pib", m.pib}, {"pib_lev", m.pib_lev},
        {"qvb", m.qvb}, {"qvb0", m.qvb0}, {"qvsb", m.qvsb}, {"pb", m.pb}, {"pb_lev", m.pb_lev},
        {"xi", m.xi}, {"uxi", m.uxi}, {"thvb", m.thvb}, {"thvbm", m.thvbm}, {"z", m.z},
        {"z_zeta", m.z_zeta}, {"lambda2", m.lambda2}, {"precip", m.precip},
#if defined(TROPICALFORCING)
        {"Q1LS", m.Q1LS}, {"Q2LS", m.Q2LS},
#endif
    };
    for (auto& e : tab) if (std::strcmp(e.n, name) == 0) return e.p;
    return nullptr;
}

double* ref_scalar(void* h, const char* name) {
    vvm& m = *static_cast<vvm*>(h);
    if (!std::strcmp(name, "ubarTopp")) return &m.ubarTopp;
    if (!std::strcmp(name, "ubarTop")) return &m.ubarTop;
    if (!std::strcmp(name, "ubarTopm")) return &m.ubarTopm;
    if (!std::strcmp(name, "dubarTop_advect")) return m.dubarTop_advect;
    if (!std::strcmp(name, "CRAD")) return &m.CRAD;
    return nullptr;
}

int* ref_step_ptr(void* h) { return &static_cast<vvm*>(h)->step; }

void ref_init_poisson(void* h) {
    CoutMute mute;
    vvm::PoissonSolver::InitPoissonMatrix(*static_cast<vvm*>(h));
}

// Runs one reference routine by name; returns 0, or -1 for an unknown name.
int ref_call(void* h, const char* name) {
    vvm& m = *static_cast<vvm*>(h);
    CoutMute mute;
    std::string n(name);
    if (n == "pzeta_pt") vvm::Iteration::pzeta_pt(m);
    else if (n == "pth_pt") vvm::Iteration::pth_pt(m);
    else if (n == "pqv_pt") vvm::Iteration::pqv_pt(m);
    else if (n == "pqc_pt") vvm::Iteration::pqc_pt(m);
    else if (n == "pqr_pt") vvm::Iteration::pqr_pt(m);
    else if (n == "Advection_zeta") vvm::Advection_zeta(m);
    else if (n == "Bouyancy") vvm::Bouyancy(m);
    else if (n == "Advection_thermo_th") vvm::Advection_thermo(m.thm, m.th, m.thp, m.dth_advect, m);
    else if (n == "Advection_qrVT") vvm::Advection_qrVT(m);
    else if (n == "AddForcing") m.AddForcing(m);
    else if (n == "BoundaryProcess2D_all") vvm::BoundaryProcess2D_all(m);
#if defined(STREAMFUNCTION)
    else if (n == "calpsiuw") vvm::PoissonSolver::calpsiuw(m);
#else
    else if (n == "pubarTop_pt") vvm::PoissonSolver::pubarTop_pt(m);
    else if (n == "cal_w") vvm::PoissonSolver::cal_w(m);
    else if (n == "cal_u") vvm::PoissonSolver::cal_u(m);
#endif
    else if (n == "autoconversion") vvm::MicroPhysics::autoconversion(m);
    else if (n == "accretion") vvm::MicroPhysics::accretion(m);
    else if (n == "evaporation") vvm::MicroPhysics::evaporation(m);
    else if (n == "condensation") vvm::MicroPhysics::condensation(m);
    else if (n == "NVP_qvp") vvm::MicroPhysics::NegativeValueProcess(m.qvp, m.nx, m.nz);
    else if (n == "NVP_qcp") vvm::MicroPhysics::NegativeValueProcess(m.qcp, m.nx, m.nz);
    else if (n == "NVP_qrp") vvm::MicroPhysics::NegativeValueProcess(m.qrp, m.nx, m.nz);
    else if (n == "updateMean") vvm::Iteration::updateMean(m);
    else if (n == "RKM_RKH") vvm::Turbulence::RKM_RKH(m);
    else if (n == "Nudge_theta") vvm::NumericalProcess::Nudge_theta(m);
    else if (n == "Nudge_zeta") vvm::NumericalProcess::Nudge_zeta(m);
    else if (n == "Nudge_qv") vvm::NumericalProcess::Nudge_qv(m);
    else if (n == "nextTimeStep") vvm::Iteration::nextTimeStep(m);
    else if (n == "one_step") one_step(m);
    else return -1;
    return 0;
}

// The sounding file this build's Init1d reads ("" without LOADFILE).
const char* ref_init_path() {
#if defined(LOADFILE)
    return LOADINITPATH;
#else
    return "";
#endif
}

// vvm::Init::Init1d then Init2d, as src/main.cpp:81-82 runs them.
void ref_init(void* h) {
    vvm& m = *static_cast<vvm*>(h);
    CoutMute mute;
    vvm::Init::Init1d(m);
    vvm::Init::Init2d(m);
}

// vvm::Init::RandomPerturbation(model, t, min_range, max_range,
// standard_deviation) (src/Init.cpp:488-515) into model.init_th_forcing.
void ref_random_perturbation(void* h, int t, double min_range, double max_range, double standard_deviation) {
    vvm::Init::RandomPerturbation(*static_cast<vvm*>(h), t, min_range, max_range, standard_deviation);
}

// Runs vvm::Iteration::TimeMarching for nsteps from step 0
// (src/Iteration.cpp:208-438); TIMEEND = nsteps * dt.
void ref_time_marching(void* h, int nsteps) {
    vvm& m = *static_cast<vvm*>(h);
    m.TIMEEND = nsteps * m.dt;
    CoutMute mute;
    vvm::Iteration::TimeMarching(m);
}

// y = A x with the assembled w-equation matrix (src/PoissonSolver.cpp:760-796).
void ref_apply_A(void* h, const double* x, double* y) {
    vvm& m = *static_cast<vvm*>(h);
    int n = (m.nx - 2) * (m.nz - 3);
    Eigen::Map<const Eigen::VectorXd> xv(x, n);
    Eigen::Map<Eigen::VectorXd> yv(y, n);
    yv = m.A * xv;
}

// x = A^{-1} b with the solver configuration of cal_w
// (src/PoissonSolver.cpp:453-462): BiCGSTAB + IncompleteLUT, zero initial
// guess, tolerance model.tolerance, at most 10000 iterations.
int ref_solve_A(void* h, const double* b, double* x, int* iters, double* err) {
    vvm& m = *static_cast<vvm*>(h);
    CoutMute mute;
    int n = (m.nx - 2) * (m.nz - 3);
    Eigen::Map<const Eigen::VectorXd> bv(b, n);
    Eigen::BiCGSTAB<Eigen::SparseMatrix<double>, Eigen::IncompleteLUT<double> > solver;
    solver.setTolerance(m.tolerance);
    solver.setMaxIterations(10000);
    Eigen::SparseMatrix<double> A = m.A;
    solver.compute(A);
    Eigen::VectorXd xv = solver.solve(bv);
    for (int i = 0; i < n; i++) x[i] = xv[i];
    if (iters) *iters = (int)solver.iterations();
    if (err) *err = solver.error();
    return solver.info() == Eigen::Success ? 0 : 1;
}

}  // extern "C"
