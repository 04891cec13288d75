// Solver instantiations: float, neumann boundary, N = 256.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, neumann, float, true, 256)
