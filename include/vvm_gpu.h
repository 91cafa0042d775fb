/*
 * vvm_gpu.h -- C ABI of the B200 VVM time step (libvvmgpu.so).
 *
 * The reference model (Aaron-Hsieh-0129/2D-Vector-Vorticity-Model) has no
 * plugin layer: its step is a sequence of static member functions of
 * `class vvm` called from vvm::Iteration::TimeMarching
 * (src/Iteration.cpp:262-434), each `static void F(vvm &model)`. Its only
 * device boundary is the GPU_POISSON translation unit, which swaps in
 * another definition of the same members behind InitAMGX / CleanupAMGX hooks
 * (src/PoissonSolver_GPU_mpi.cpp, src/main.cpp:85-87,141-145). This header is
 * the same kind of swap at the granularity of the whole step: one entry per
 * reference routine (so a GPU_STEP build of TimeMarching replaces each body
 * one for one), plus a fused multi-step entry and a standalone Poisson solve.
 *
 * Conventions
 *  - Every entry returns an int status: 0 = OK, see VVM_GPU_E* below; the
 *    message of the last failure is available from vvm_gpu_last_error().
 *  - Host arrays use the reference model's layout (src/Declare.hpp:400-427):
 *    2D fields are [nx][nz] doubles with k (height) the fast index, ghost
 *    cells included (nx = NX + 2, nz = NZ + 2); AB2 histories are
 *    [nx][nz][2]; profiles are [nz]. On the device every field is stored
 *    x-contiguous ([k][i], rows padded to a multiple of 32 cells) and stays
 *    resident in HBM across calls; upload/download transpose.
 *  - One context owns its device memory and stream; calls on one context must
 *    come from one host thread at a time.
 *  - The routine entries advance no step counter: TimeMarching increments
 *    model.step before the physics (src/Iteration.cpp:246), so a caller does
 *    the same with vvm_gpu_set_step(). vvm_gpu_step() does it itself.
 */
#ifndef VVM_GPU_H
#define VVM_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VVM_GPU_OK 0
#define VVM_GPU_EINVAL 1     /* bad argument or descriptor */
#define VVM_GPU_ECUDA 2      /* CUDA runtime error (message has details) */
#define VVM_GPU_ENOCONV 3    /* Poisson solve did not reach its tolerance */
#define VVM_GPU_ESTATE 4     /* call out of order (e.g. step before upload) */

/* Arithmetic of the step. */
#define VVM_PREC_FP64 0   /* every field and solve in FP64 (the plain GPU step) */
#define VVM_PREC_MIXED 1  /* FP32 fields, stencils, microphysics and inner CG;
                             FP64 Poisson residual, refinement and reductions */

/* Preconditioner of the Poisson CG (cal_w). */
#define VVM_SOLVER_MGPCG 0    /* geometric multigrid: x-semicoarsening, z-line relaxation */
#define VVM_SOLVER_LEARNED 1  /* learned BF16 conv preconditioner in flexible CG,
                                 multigrid-PCG as fallback (vvm_gpu_learned_*) */
#define VVM_SOLVER_SPECTRAL 2 /* exact Fourier-mode solve (row FFTs in x, one
                                 tridiagonal z solve per mode) applied directly in
                                 FP64, its residual checked, FP64 CG preconditioned
                                 by it only if the check fails (the iterations
                                 vvm_gpu_last_solve reports); NX a power of two;
                                 serves VVM_PREC_MIXED as well */

/* Model description; mirrors Config_VVM (src/Declare.hpp:27-70) and the
 * constants main.cpp passes (src/main.cpp:68-72). */
typedef struct vvm_gpu_desc {
    int NX, NZ;                  /* interior cells (VVM_XRANGE/dx, VVM_ZRANGE/dz) */
    double dx, dz, dt;           /* grid spacings [m], time step [s] */
    double gravity, cp, cv, rd, lv, p0, psurf;   /* 9.80665 1003.5 716.5 287 2.5e6 1e5 96500 */
    double poisson_tol;          /* relative residual ||b - A W||/||b|| of cal_w */
    int poisson_maxit;           /* CG iteration cap (0 = default 200) */
    int case_id;                 /* VVM_CASE; zeta nudging is skipped for case 2 */
    double moisture_nudge_time;  /* VVM_MOISTURE_NUDGE_TIME; 0 disables Nudge_qv */
    double addforcingtime;       /* random th forcing while step*dt <= this */
    int precision;               /* VVM_PREC_* */
    int solver;                  /* VVM_SOLVER_* */
    int warm_start;              /* 1: start cal_w from the previous W (the
                                    reference starts from zero) */
    int flags;                   /* VVM_FLAG_* below, 0 = the reference's behaviour */
} vvm_gpu_desc;

/* desc.flags: keep the uploaded init_th_forcing at every forced step instead
 * of regenerating it each step the way TimeMarching does
 * (src/Iteration.cpp:276-283; see vvm_gpu_random_perturbation). */
#define VVM_FLAG_FIXED_FORCING 1
/* desc.flags: the streamfunction formulation (the reference's STREAMFUNCTION
 * switch, src/Config.hpp:8, which it ships off and marks as debugging):
 * vvm_gpu_step calls vvm_gpu_calpsiuw where TimeMarching would call
 * pubarTop_pt, cal_w and cal_u (src/Iteration.cpp:289-295). Its steps run
 * the host loop (no CUDA graph); batches refuse it. */
#define VVM_FLAG_STREAMFUNCTION 2

/* Fills a descriptor with the reference's constants for an NX x NZ grid. */
void vvm_gpu_desc_default(vvm_gpu_desc* d, int NX, int NZ, double dx, double dz, double dt);

typedef struct vvm_gpu_ctx vvm_gpu_ctx;

/* Host view of the model state, reference layout. Pointers may be NULL on
 * download to skip a field; on upload every prognostic pointer is required
 * (the *p fields, histories and diagnostics may be NULL = zero). */
typedef struct vvm_gpu_host_state {
    /* [nx][nz] */
    double *zeta, *zetap, *th, *thp, *qv, *qvp, *qc, *qcp, *qr, *qrp, *u, *w, *RKM, *RKH;
    /* [nx][nz][2] AB2 tendency histories */
    double *dzeta_advect, *dth_buoyancy, *dth_advect, *dqv_advect, *dqc_advect, *dqr_advect,
        *dqr_VT;
    /* [nz] profiles */
    double *rhou, *rhow, *thb, *thvb, *qvb, *pib, *pb, *thb_init, *qvb0, *z, *z_zeta, *lambda2;
    double *Q1LS, *Q2LS;          /* [nz] large-scale forcing (NULL = none) */
    double *init_th_forcing;      /* [nx][nz] random th forcing field (NULL = zero) */
    double *precip;               /* [nx] surface rain diagnostic */
    /* scalars */
    double ubarTop, ubarTopp;
    double dubarTop_advect[2];
    int step;
} vvm_gpu_host_state;

/* -- lifetime --------------------------------------------------------------
 * Replaces `vvm model(config)` + PoissonSolver::InitPoissonMatrix
 * (src/main.cpp:74,88; src/Declare.hpp:78-96; src/PoissonSolver.cpp:681-813). */
int vvm_gpu_create(const vvm_gpu_desc* desc, int device, vvm_gpu_ctx** out);
/* Replaces the vvm destructor (src/Declare.hpp:98-249) / CleanupAMGX. */
int vvm_gpu_destroy(vvm_gpu_ctx* ctx);
/* Runs the context's kernels on `stream` (a cudaStream_t) from now on;
 * NULL restores the context's own stream. */
int vvm_gpu_set_stream(vvm_gpu_ctx* ctx, void* stream);
int vvm_gpu_synchronize(vvm_gpu_ctx* ctx);
/* Message of the last failure on this context (or of vvm_gpu_create when
 * ctx is NULL). */
int vvm_gpu_last_error(vvm_gpu_ctx* ctx, char* buf, size_t len);

/* -- state transfer (host [i][k] <-> device [k][i]) -----------------------
 * Replaces Init::Init1d/Init2d as the source of the state (src/Init.cpp:14-266).
 * After a whole step (vvm_gpu_step, or vvm_gpu_next_step) the future arrays
 * zetap, thp, qvp, qcp, qrp come back equal to the present ones, as the
 * reference's nextTimeStep leaves them (src/Iteration.cpp:153-204); between
 * routine calls inside a step they come back as the routines left them. */
int vvm_gpu_upload_state(vvm_gpu_ctx* ctx, const vvm_gpu_host_state* st);
int vvm_gpu_download_state(vvm_gpu_ctx* ctx, vvm_gpu_host_state* st);
/* Prognostic fields only (zeta, th, qv, qc, qr, u, w): the per-step traffic
 * of an output call. The copies run on the context's own copy stream, each
 * field's copy beside the previous field's layout kernel. The upload returns
 * once the work is queued (work on the context's stream that follows sees the
 * fields; the host buffers must stay unchanged until then, as for any
 * asynchronous copy); the download returns with the host buffers filled. */
int vvm_gpu_upload_prognostic(vvm_gpu_ctx* ctx, const vvm_gpu_host_state* st);
int vvm_gpu_download_prognostic(vvm_gpu_ctx* ctx, vvm_gpu_host_state* st);
int vvm_gpu_set_step(vvm_gpu_ctx* ctx, int step);
int vvm_gpu_get_step(vvm_gpu_ctx* ctx, int* step);

/* -- one entry per reference routine (src/Iteration.cpp:262-434) ---------- */
int vvm_gpu_pzeta(vvm_gpu_ctx* ctx);        /* Iteration::pzeta_pt, Iteration.cpp:29-34 */
int vvm_gpu_pth(vvm_gpu_ctx* ctx);          /* Iteration::pth_pt, Iteration.cpp:36-40 */
int vvm_gpu_pqv(vvm_gpu_ctx* ctx);          /* Iteration::pqv_pt, Iteration.cpp:90-98 */
int vvm_gpu_pqc(vvm_gpu_ctx* ctx);          /* Iteration::pqc_pt, Iteration.cpp:100-107 */
int vvm_gpu_pqr(vvm_gpu_ctx* ctx);          /* Iteration::pqr_pt, Iteration.cpp:109-124 */
int vvm_gpu_add_forcing(vvm_gpu_ctx* ctx);  /* vvm::AddForcing, AddForcing.cpp:6-28 */
/* Init::RandomPerturbation(model, t, min_range, max_range, standard_deviation)
 * (src/Init.cpp:488-515): the random theta forcing field of step t, made on
 * the host with the reference's own generator (std::mt19937 seeded with t,
 * std::normal_distribution<> redrawn until inside [min_range, max_range], in
 * the cells with z = (k - 0.5) dz < 200 m, k outer and i inner), so the same
 * numbers as the reference, and written to the device's init_th_forcing.
 * TimeMarching calls it before AddForcing while step*dt <= addforcingtime
 * with (step, -0.001, 0.001, 1.); vvm_gpu_step does the same unless
 * VVM_FLAG_FIXED_FORCING is set. EINVAL when min_range > max_range or
 * standard_deviation <= 0 (the reference's redraw loop would not end). */
int vvm_gpu_random_perturbation(vvm_gpu_ctx* ctx, int t, double min_range, double max_range,
                                double standard_deviation);
/* The same field for an NX x NZ grid of level spacing dz, on the host only
 * (no context, no device): out is [NX+2][NZ+2] in the reference layout, its
 * ghost cells filled as BoundaryProcess2D_center fills them
 * (src/Boundary.cpp:9-19). Init2d adds the t = 0 field of the declaration's
 * default range (-0.25, 0.25, 1., src/Declare.hpp:870) to th
 * (src/Init.cpp:169-175 and :193-196). */
int vvm_gpu_random_perturbation_host(int NX, int NZ, double dz, int t, double min_range,
                                     double max_range, double standard_deviation, double* out);
int vvm_gpu_halo_all(vvm_gpu_ctx* ctx);     /* BoundaryProcess2D_all, Boundary.cpp:32-52 */
int vvm_gpu_pubartop(vvm_gpu_ctx* ctx);     /* PoissonSolver::pubarTop_pt, PoissonSolver.cpp:655-676 */
int vvm_gpu_cal_w(vvm_gpu_ctx* ctx);        /* PoissonSolver::cal_w, PoissonSolver.cpp:439-479 */
int vvm_gpu_cal_u(vvm_gpu_ctx* ctx);        /* PoissonSolver::cal_u, PoissonSolver.cpp:580-653 */
/* autoconversion, accretion, evaporation, condensation, then
 * NegativeValueProcess on qvp, qcp, qrp (Iteration.cpp:303-311,
 * MicroPhysics.cpp:7-138); halos are left to vvm_gpu_halo_all as in the
 * reference. */
int vvm_gpu_kessler(vvm_gpu_ctx* ctx);
int vvm_gpu_update_mean(vvm_gpu_ctx* ctx);  /* Iteration::updateMean, Iteration.cpp:42-86 */
int vvm_gpu_turbulence(vvm_gpu_ctx* ctx);   /* Turbulence::RKM_RKH, Turbulent.cpp:5-114 */
/* Nudge_theta, Nudge_zeta (case != 2), Nudge_qv (NumericalProcess.cpp:60-96). */
int vvm_gpu_nudge(vvm_gpu_ctx* ctx);
int vvm_gpu_next_step(vvm_gpu_ctx* ctx);    /* Iteration::nextTimeStep, Iteration.cpp:153-204 */
/* PoissonSolver::calpsiuw, PoissonSolver.cpp:124-177 (STREAMFUNCTION): solves
 * A_psi psi = zetap dx^2 with the matrix of InitPoissonMatrix's
 * STREAMFUNCTION branch (PoissonSolver.cpp:726-756) to
 * ||b - A_psi psi|| / ||b|| <= desc.poisson_tol, from zero, then sets psi's
 * ghosts, u = -d(rhow psi)/dz / rhou and w = d(psi)/dx with the routine's
 * halos. The reference defines the diagonal shift POISSONPARAM nowhere (a
 * compile error upstream); this entry takes it as 0, which makes A_psi the
 * negative of the symmetric w-equation operator. Uniform levels only. */
int vvm_gpu_calpsiuw(vvm_gpu_ctx* ctx);
/* The psi field of the last vvm_gpu_calpsiuw, [nx][nz] with ghosts
 * (model.psi, src/Declare.hpp:584-586); VVM_GPU_ESTATE before the first. */
int vvm_gpu_download_psi(vvm_gpu_ctx* ctx, double* psi);

/* -- fused path -------------------------------------------------------------
 * nsteps complete steps of TimeMarching's body (step++ first), with fused
 * kernels and the time levels rotated by pointer swap. */
int vvm_gpu_step(vvm_gpu_ctx* ctx, int nsteps);

/* -- standalone elliptic solve (tests, solves/s) ------------------------------
 * Solves A W = b for the cal_w matrix (src/PoissonSolver.cpp:760-796) to
 * ||b - A W||_2 / ||b||_2 <= tol. Host arrays of (NX)*(NZ-1) doubles, unknown
 * index (k-2)*NX + (i-1), k = 2..nz-2, i = 1..nx-2 -- the reference's vector
 * ordering. W is used as the initial guess when warm_start is set.
 *
 * Stretched levels (no counterpart in the reference, whose levels are
 * uniform): when the uploaded heights z (centres) and z_zeta (faces) are not
 * uniform with spacing dz, A is the same anelastic operator discretised on
 * those levels, times dx^2: ru_k = rhow_k h_k / (a_k rhou_k), rd_k = rhow_k
 * h_{k-1} / (a_k rhou_{k-1}), a_k = (z_k - z_{k-1}) / dx, h_k = dx / (2 (z_k -
 * z_zeta_k)) (centres midway between faces); b is unchanged. Such a context
 * supports the Poisson and learned-preconditioner entries only; the step and
 * routine entries return VVM_GPU_EINVAL. */
int vvm_gpu_poisson_solve(vvm_gpu_ctx* ctx, const double* b, double* W, double tol,
                          int* iters, double* relres);
/* Same on device buffers (cudaMalloc'd, same ordering); no host copies. */
int vvm_gpu_poisson_solve_device(vvm_gpu_ctx* ctx, const double* d_b, double* d_W,
                                 double tol, int* iters, double* relres);

/* Iterations and final relative residual of the last cal_w solve. */
int vvm_gpu_last_solve(vvm_gpu_ctx* ctx, int* iters, double* relres);

/* -- the learned preconditioner's tensor-core convolution ------------------------
 * One 3x3 convolution of 32 channels in and out (or, with adjoint != 0, its
 * adjoint: taps mirrored, channels transposed) on the tensor cores, from and
 * to host arrays: x, y [H][W][32] FP32 (rounded to BF16 on the device),
 * w [9 taps][32 in][32 out] FP32 (BF16 on the device), periodic in the W
 * direction and zero outside the H direction, FP32 accumulation, BF16 output.
 * A diagnostic of the building block; the network runs it on device buffers.
 * Failures: vvm_gpu_last_error(NULL, ...). */
int vvm_gpu_conv3x3_c32(const float* x, const float* w, float* y, int H, int W, int adjoint, int device);

/* -- learned preconditioner (VVM_SOLVER_LEARNED) -------------------------------
 * No counterpart in the reference. The preconditioner is a two-level cycle
 * whose coarse correction is learned: the exact z-line solve L of the
 * residual r (the multigrid's finest line operator), za = L r; the network
 * on what it leaves, r1 = r - S za, giving d = ||r1|| net(r1 / ||r1||); the
 * Galerkin step za += gam d, gam = (d, r1) / (d, S d), which minimises the
 * S-norm error along d, so that a poor network can slow nothing down; and a
 * second line solve, z = za + L (r - S za). The network is linear, 4 levels
 * of 3x3 convolutions (lift 1 -> 32 channels, three levels down by 2x2
 * average pooling and three up by nearest upsampling with skips, projection
 * 32 -> 1; the 32 -> 32 convolutions on the tensor cores, BF16 weights and
 * activations, FP32 accumulation). Its grid is the cal_w grid padded to H0 = round_up(NZ-1, 8)
 * rows by W0 = NX columns (NX a multiple of 8); arrays of it are [H0][W0].
 * The solve is flexible CG from W = 0 to the same FP64 residual as the other
 * solvers, each new direction S-orthogonalised against the previous seven
 * (the preconditioner varies between applications, so one is not enough); after `cap` iterations the multigrid PCG takes over from the
 * current iterate. Weights: nparams FP32 values (vvm_gpu_learned_shape), the
 * lift [9][32], six convolutions [9 taps][32 in][32 out] (down at levels 1,
 * 2, 3, up at levels 2, 1, 0) and the projection [9][32]; seeded initial
 * values until set or trained.
 *   _weights: copies them out (get) and/or in (set).
 *   _eval: z = net(x); with t, the loss L = 1 - (z, S t)^2 / ((z, S z)(t, S t))
 *     (the S-norm error of t left by the best multiple of z, relative to
 *     ||t||_S^2; S the cal_w operator in symmetric form on the rows < NZ-1)
 *     and dL/dweights.
 *   _train: collects npairs pairs from the model's own next steps solved by
 *     the plain solver (the state is put back afterwards) and as many from
 *     white-noise right-hand sides: input r1 / ||r1||, r1 = rhs - S L rhs,
 *     target (W - L rhs) / ||r1|| = S^{-1} r1 / ||r1||; then runs
 *     `steps` Adam steps (learning rate lr) on random mini-batches of `batch`
 *     pairs; returns the mean loss of the first and the last ten steps.
 *   _config: mode 0 = the cycle with the network, 1 = the same cycle without
 *     it (two line solves: the method without the network), 2 = identity;
 *     cap = iterations before the multigrid fallback (default 200).
 *   _last: flexible-CG iterations of the last solve, and whether it fell back. */
int vvm_gpu_learned_shape(vvm_gpu_ctx* ctx, int* H0, int* W0, int* nparams);
int vvm_gpu_learned_weights(vvm_gpu_ctx* ctx, float* get, const float* set, int n);
int vvm_gpu_learned_eval(vvm_gpu_ctx* ctx, const float* x, const float* t, float* z, float* grad, double* loss);
int vvm_gpu_learned_train(vvm_gpu_ctx* ctx, int npairs, int steps, int batch, double lr, int seed,
                          double* loss_first, double* loss_last);
/* As _train, with the caller's right-hand sides: b holds npairs vectors of
 * NX*(NZ-1) values in vvm_gpu_poisson_solve's ordering; each is solved by the
 * plain multigrid PCG to make its pair, and as many white-noise right-hand
 * sides are added (the rough residuals flexible CG meets). The source of
 * model-like pairs on stretched levels, where the step does not run. */
int vvm_gpu_learned_train_rhs(vvm_gpu_ctx* ctx, const double* b, int npairs, int steps, int batch, double lr,
                              int seed, double* loss_first, double* loss_last);
int vvm_gpu_learned_config(vvm_gpu_ctx* ctx, int mode, int cap);
/* Times `reps` network forward passes on a white-noise input, and `reps`
 * passes of its six tensor-core convolutions alone, each between one pair of
 * events on the context's stream: milliseconds per pass. Changes no model
 * state (only the preconditioner's work arrays). */
int vvm_gpu_learned_time(vvm_gpu_ctx* ctx, int reps, double* ms_forward, double* ms_convs);
int vvm_gpu_learned_last(vvm_gpu_ctx* ctx, int* fcg_iters, int* fell_back);

/* -- launch-shape knobs --------------------------------------------------------
 * gs_tile_rows selects the Gauss-Seidel schedule: 4, 8, 16 or 32 = tiles of
 * that many rows (128 columns and one warp each; the passes run to the same
 * fixed point whatever the height, so results are identical across heights);
 * 1 = one thread-block cluster a field (a single pass, the schedule for many
 * cases stepping at once; it agrees with the tiles to round-off, its carries
 * associate differently). fft_threads sets the threads of a row-FFT block of
 * the spectral solve (no result changes). 0 selects the automatic value
 * (tiles of 16 rows in FP64, 8 in the mixed step; 512 threads or half the
 * row). Setting them drops the context's captured graphs. get
 * returns the values in use. */
int vvm_gpu_set_tuning(vvm_gpu_ctx* ctx, int gs_tile_rows, int fft_threads);
int vvm_gpu_get_tuning(vvm_gpu_ctx* ctx, int* gs_tile_rows, int* fft_threads);

/* -- batches of independent cases ------------------------------------------------
 * The reference runs one case per process. A batch holds many cases of any
 * sizes (one context each, created from descs[i] on `device`) that advance
 * together: from the third step on, one CUDA graph per step runs every
 * case's step, launched on the batch's own stream. Cases with the same grid,
 * precision and tuning whose step uses the exact Fourier-mode solve and the
 * tiled Gauss-Seidel passes step as grouped launches: one launch a kernel
 * for all cases of the group (each case reads its own arguments and loop
 * flags), each group a parallel branch; other cases run as branches of
 * their own. Either way each case's results are those it computes alone.
 * vvm_gpu_batch_case returns case i's context, owned by the batch, for
 * upload, download, queries and the routine entries; every case must be at
 * the same step when vvm_gpu_batch_step runs (VVM_GPU_ESTATE otherwise).
 * vvm_gpu_batch_autotune times one step of each group of cases with the same
 * grid, precision and solver for each value of the launch-shape knobs above
 * and for the cases a grouped launch takes (`reps` graph launches per
 * candidate), keeps the fastest, and restores
 * every case's state exactly; *ngroups receives the number of groups.
 * vvm_gpu_batch_synchronize waits for the batch and reports any case's
 * device error. Failures of batch calls: vvm_gpu_batch_last_error. */
typedef struct vvm_gpu_batch vvm_gpu_batch;
int vvm_gpu_batch_create(const vvm_gpu_desc* descs, int ncases, int device, vvm_gpu_batch** out);
int vvm_gpu_batch_destroy(vvm_gpu_batch* b);
int vvm_gpu_batch_case(vvm_gpu_batch* b, int i, vvm_gpu_ctx** ctx);
int vvm_gpu_batch_step(vvm_gpu_batch* b, int nsteps);
int vvm_gpu_batch_synchronize(vvm_gpu_batch* b);
int vvm_gpu_batch_autotune(vvm_gpu_batch* b, int reps, int* ngroups);
/* The stream the batch graphs run on (cudaStream_t), for events around them. */
int vvm_gpu_batch_stream(vvm_gpu_batch* b, void** stream);
/* The most cases one grouped launch takes (default 32; a shape with more
 * cases is split into sub-groups of even size, parallel branches of the
 * graph); 0 or 1: no grouped launches, every case its own branch; < 0 leaves
 * the setting. Grids of more than 65536 cells step case by case unless
 * vvm_gpu_batch_autotune found grouped launches faster for them. Setting it
 * clears the autotuner's per-group choice and drops the batch's graphs. *groups (may be null) receives the number of grouped
 * launch groups in the last captured step graph. No counterpart in the
 * reference, which runs one case per process (src/main.cpp:29-147). */
int vvm_gpu_batch_grouping(vvm_gpu_batch* b, int max_cases, int* groups);
int vvm_gpu_batch_last_error(vvm_gpu_batch* b, char* buf, size_t len);

/* -- elliptic solve that allocates nothing ------------------------------------
 * No counterpart in the reference.
 *
 * Solves the same system as vvm_gpu_poisson_solve_device (same unknown
 * ordering, same stopping test ||b - A W||_2 / ||b||_2 <= tol) without a
 * context, and without allocating device memory. It is for callers that
 * cannot allocate during the solve, for example a host model that reserves
 * the device memory for its own pool at start-up and forbids allocation in
 * its time loop, or a GPU_POISSON-style replacement of cal_w that has b and W
 * on the device but keeps no context of this library.
 *
 * rhou, rhow: host profiles of NZ+2 doubles (the model's [nz] arrays).
 * d_b, d_W: device buffers of NX*(NZ-1) doubles on the current device; the
 * incoming W is ignored (the solve starts from W = 0). Runs FP64 CG with exact
 * z-line solves as preconditioner, at most maxit iterations, on `stream`
 * (NULL: the legacy default stream), and returns after the solve completed.
 *
 * Working memory is a fixed file-scope device array of
 * VVM_NOALLOC_SCRATCH_BYTES per device, so NX*(NZ-1) may not exceed
 * VVM_NOALLOC_MAX_UNKNOWNS and NZ-1 may not exceed VVM_NOALLOC_MAX_ROWS;
 * larger problems return VVM_GPU_EINVAL (message from
 * vvm_gpu_last_error(NULL, ...), like every failure of this entry).
 * None of that memory has to start at zero: each call writes every word
 * before reading it. The first call on each device does a one-time set-up
 * (it looks up the array's device address, which may load the library's
 * device code): make it, with that device current, before any stream capture
 * begins (a captured first call returns VVM_GPU_ESTATE). Each later call made
 * outside capture looks the address up again, so a cudaDeviceReset between
 * calls is harmless if the next call is not captured; a captured call uses
 * the address of the last uncaptured one. Calls that overlap on one device
 * (two host threads, or two streams without ordering between them) share the
 * one array and race: serialise them. */
#define VVM_NOALLOC_MAX_UNKNOWNS 131072
#define VVM_NOALLOC_MAX_ROWS 1024
#define VVM_NOALLOC_SCRATCH_BYTES 4251712
int vvm_gpu_poisson_solve_noalloc(int NX, int NZ, const double* rhou, const double* rhow,
                                  const double* d_b, double* d_W, double tol, int maxit,
                                  void* stream, int* iters, double* relres);

/* -- timers -------------------------------------------------------------------
 * The reference keeps per-phase wall timers of each step (t_advection,
 * t_poisson, t_microphysics, t_diffusion, t_all; src/Iteration.cpp:286-435).
 * Here, with profiling enabled, every kernel launch is bracketed by CUDA
 * events on the context's stream and accumulated per kernel class
 * (VVM_K_*); phases are the sums of their classes. The launch counter runs
 * always. Enabling resets both. */
#define VVM_K_PZETA 0       /* vorticity advection + buoyancy */
#define VVM_K_PADV 1        /* scalar advection + sedimentation + NVP sums */
#define VVM_K_APPLY 2       /* NVP rescale, forcing, halos */
#define VVM_K_PUBAR 3       /* pubarTop */
#define VVM_K_POISSON_RHS 4 /* cal_w right-hand side, w from W */
#define VVM_K_CG 5          /* CG vector kernels and reductions */
#define VVM_K_MG_SWEEP 6    /* multigrid z-line sweeps */
#define VVM_K_MG_RESTRICT 7 /* multigrid restriction */
#define VVM_K_MG_COARSE 8   /* multigrid coarse-level block */
#define VVM_K_CAL_U 9       /* cal_u top row and column integral */
#define VVM_K_KESSLER 10    /* Kessler + NVP sums */
#define VVM_K_RKM 11        /* eddy coefficients */
#define VVM_K_GS 12         /* Gauss-Seidel diffusion (+ nudging) */
#define VVM_K_MEAN 13       /* updateMean, nudging passes, transfers */
#define VVM_K_LEARNED 14    /* learned preconditioner: network (not its convolutions), training */
#define VVM_K_CONV 15       /* learned preconditioner: tensor-core 3x3 convolutions */
#define VVM_K_COUNT 16
int vvm_gpu_profile(vvm_gpu_ctx* ctx, int enable);
/* Accumulated device milliseconds and launches of one kernel class. */
int vvm_gpu_profile_read(vvm_gpu_ctx* ctx, int kernel_class, double* ms, long long* launches);
/* Kernel launches of this context since creation or the last profile(1). */
int vvm_gpu_launch_count(vvm_gpu_ctx* ctx, long long* launches);

#ifdef __cplusplus
}
#endif
#endif
