// Pre-included after testcases/sedov/parameter.h for the harness build
// ref_sph_bal: the same Sedov configuration with the Balsara viscosity switch
// (parameter.h's BALSARA_SWITCH) turned on.  Test infrastructure only.
#undef BALSARA_SWITCH
#define BALSARA_SWITCH 1
