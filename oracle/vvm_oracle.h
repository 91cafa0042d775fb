/* CPU restatement of the reference VVM time step (AB2 + WATER + Kessler).
 *
 * Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it as the checker. The product path never links it.
 *
 * Layout and names follow the reference model object (src/Declare.hpp):
 * 2D fields are [nx][nz] doubles with k the fast index and one ghost cell on
 * each side; AB2 histories are [nx][nz][2]; profiles are [nz].
 *
 * Every stencil routine keeps the reference's floating-point expression
 * order, so on the reference's grids it reproduces the reference bit for
 * bit. The two elliptic solves are exact instead of iterative:
 *   cal_w : the w-equation matrix is separable (coefficients depend on k
 *           only, periodic in x), so it is solved by a real discrete Fourier
 *           transform in x and one tridiagonal (Thomas) solve in z per mode;
 *   cal_u : the periodic 1D Poisson problem for chi only enters through
 *           d(chi)/dx with its mean removed, which is a prefix sum of h.
 * The reference reaches the same solutions to its solver tolerances
 * (BiCGSTAB at 1e-22 requested, CG at 1e-12), i.e. to round-off.
 */
#ifndef VVM_ORACLE_H
#define VVM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;

orc_model* orc_create(int NX, int NZ, double dx, double dz, double dt, int CASE,
                      double moisture_nudge_time, double addforcingtime);
void orc_destroy(orc_model* m);
void orc_dims(orc_model* m, int* nx, int* nz);
double* orc_field(orc_model* m, const char* name);
double* orc_hist(orc_model* m, const char* name);
double* orc_prof(orc_model* m, const char* name);
double* orc_scalar(orc_model* m, const char* name);
int* orc_step_ptr(orc_model* m);
/* Runs one routine by the reference's name (see the dispatch table in
 * vvm_oracle.c); returns 0, or -1 for an unknown name. "one_step" runs the
 * whole TimeMarching step body (src/Iteration.cpp:246-434). */
int orc_call(orc_model* m, const char* name);
/* Solves A x = b exactly for the cal_w matrix (src/PoissonSolver.cpp:760-796);
 * unknown index (k-2)*(nx-2) + (i-1). */
void orc_solve_A(orc_model* m, const double* b, double* x);
void orc_apply_A(orc_model* m, const double* x, double* y);
/* The cal_w system on the model's (possibly stretched) levels: the matrix of
 * oracle/stretched_poisson.py, the reference's on uniform levels. */
void orc_solve_W(orc_model* m, const double* b, double* x);
/* The streamfunction formulation (STREAMFUNCTION, src/PoissonSolver.cpp:14-177,
 * matrix 726-756 with POISSONPARAM = 0): y = A_psi x, x = A_psi^{-1} b exactly,
 * and the switch that makes "one_step" call calpsiuw in place of
 * pubarTop_pt + cal_w + cal_u (src/Iteration.cpp:289-295). */
void orc_apply_psi(orc_model* m, const double* x, double* y);
void orc_solve_psi(orc_model* m, const double* b, double* x);
void orc_set_streamfunction(orc_model* m, int on);
/* Threads the library runs its loops on: 1 for the serial checker, the
 * OpenMP team size for the threaded CPU baseline (libvvmoracle_mt.so). */
int orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
