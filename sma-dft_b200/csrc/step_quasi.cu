// step_quasi.cu -- the quasi-incompressible loop body (quasi/quasi.cpp:1099-2190).
#include "quasi.cuh"
#include "steps.h"

namespace smadft {

template int quasi_step<float>(Ctx &, long long, bool);
template int quasi_step<double>(Ctx &, long long, bool);
template int reduce_mass_energy<float>(Ctx &, double *);
template int reduce_mass_energy<double>(Ctx &, double *);

}  // namespace smadft
