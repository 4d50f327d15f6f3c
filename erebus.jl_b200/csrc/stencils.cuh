// stencils.cuh -- host wrappers of the node-parallel phases (stencils.cu).
#pragma once
#include "solver.cuh"

namespace erebus {
int gravity_post(erebus_state *s);
int bulk_viscosity(erebus_state *s);
int hydro_post(erebus_state *s, const double *S);
int finalize_plastic(erebus_state *s, int rollback);
int heating(erebus_state *s);
int adiabatic(erebus_state *s);
int thermal_post(erebus_state *s, const double *S);
int velocities_rotation(erebus_state *s);
}  // namespace erebus
