// step_quasi.cu -- the quasi-incompressible loop body (quasi/quasi.cpp:1099-2190).
#include "quasi.cuh"
#include "steps.h"

namespace smadft {

// each precision builds as its own object (SMADFT_INST_FLOAT / SMADFT_INST_DOUBLE); a plain
// compile without either instantiates both
#if !defined(SMADFT_INST_DOUBLE)
template int quasi_step<float>(Ctx &, long long, bool);
template int reduce_mass_energy<float>(Ctx &, double *);
#endif
#if !defined(SMADFT_INST_FLOAT)
template int quasi_step<double>(Ctx &, long long, bool);
template int reduce_mass_energy<double>(Ctx &, double *);
#endif

}  // namespace smadft
