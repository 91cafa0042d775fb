// Compile-time switches for building the reference VVM step as a CPU oracle.
//
// Test infrastructure only: nothing in the product links against the library
// this produces. It stands in for the reference's own src/Config.hpp
// (src/Config.hpp:1-32), which enables P3, RRTMGP, tropical forcing and file
// loading; the oracle wants the warm-rain configuration instead:
//   AB2                Adams-Bashforth 2 time stepping (src/Config.hpp:6)
//   WATER              qv, qc, qr prognostics (src/Config.hpp:14)
//   KESSLER_MICROPHY   Kessler warm rain (src/Config.hpp:15)
// Everything else (output, P3, radiation, PETSc, GPU_POISSON) stays off.
#define AB2
#define WATER
#define KESSLER_MICROPHY
