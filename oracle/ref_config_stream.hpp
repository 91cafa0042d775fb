// Compile-time switches for building the reference's streamfunction
// formulation as a CPU oracle (oracle/build_ref.sh with REF_VARIANT=stream).
//
// Test infrastructure only. The reference ships this formulation switched off
// and unfinished (src/Config.hpp:8, "Don't turn this on. Debugging"): with
// STREAMFUNCTION on, its sources do not compile as they stand, for two
// reasons that this header and the build script supply without touching the
// sources:
//   * src/Declare.hpp:143,305 allocate and free `psicont`, the contiguous
//     block behind `psi`, but the class never declares it; here it names a
//     per-object slot (a table keyed by the model's address), which the
//     constructor and the destructor, the only places that name it, reach
//     through `this`;
//   * src/PoissonSolver.cpp:732 adds POISSONPARAM to the diagonal of the psi
//     matrix, a macro defined nowhere; build_ref.sh passes
//     -DPOISSONPARAM=0.0, which makes the matrix the negative of the
//     symmetric w-equation operator (the value the GPU entry takes too).
#define AB2
#define WATER
#define KESSLER_MICROPHY
#define STREAMFUNCTION
#include <map>
inline double*& vvm_psicont_slot(const void* model) {
    static std::map<const void*, double*> slots;
    return slots[model];
}
#define psicont (vvm_psicont_slot(this))
