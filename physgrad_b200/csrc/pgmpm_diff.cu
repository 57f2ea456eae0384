// pgmpm_diff.cu -- differentiation entry points (filled in below).
#include "../../include/pgmpm.h"
extern "C" {
int pgmpm_forward_checkpointed(pgmpm_solver, int32_t, int32_t, void*) { return PGMPM_ERR_UNSUPPORTED; }
int pgmpm_backward(pgmpm_solver, const float*, const float*, const float*, const float*, float*, float*, float*,
                   float*, float*, int32_t, void*) { return PGMPM_ERR_UNSUPPORTED; }
void launch_mpm_timestep_forward(float*, float*, const float*, int, int, float, const float*, void*) {}
}
