// Solver instantiations: float, neumann boundary, N = 512.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, neumann, float, true, 512)
