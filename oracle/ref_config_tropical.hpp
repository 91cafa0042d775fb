// Compile-time switches of the second reference build (test infrastructure
// only): the warm-rain configuration of ref_config.hpp plus the sounding file
// and large-scale forcing that the reference's own src/Config.hpp turns on
// (src/Config.hpp:18-22):
//   TROPICALFORCING  Q1LS/Q2LS forcing, th = thb + RandomPerturbation(0) in Init2d
//   LOADFILE         Init1d reads the 1D base state from LOADINITPATH
// The path comes from the build (-DREF_INIT_PATH=...).
#define AB2
#define WATER
#define KESSLER_MICROPHY
#define TROPICALFORCING
#define LOADFILE
#define LOADINITPATH REF_INIT_PATH
