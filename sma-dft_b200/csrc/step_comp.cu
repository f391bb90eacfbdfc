// step_comp.cu -- the compressible loop body (compressible/compressible.cpp:1265-2720).
#include "comp.cuh"
#include "steps.h"

namespace smadft {

// each precision builds as its own object (SMADFT_INST_FLOAT / SMADFT_INST_DOUBLE); a plain
// compile without either instantiates both
#if !defined(SMADFT_INST_DOUBLE)
template int comp_pre_loop<float>(Ctx &);
template int comp_step<float>(Ctx &, long long, bool);
template int reduce_comp_mass_energy<float>(Ctx &, const float *, double *);
#endif
#if !defined(SMADFT_INST_FLOAT)
template int comp_pre_loop<double>(Ctx &);
template int comp_step<double>(Ctx &, long long, bool);
template int reduce_comp_mass_energy<double>(Ctx &, const double *, double *);
#endif

}  // namespace smadft
