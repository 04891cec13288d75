// Solver instantiations: float, neumann boundary, N = 128.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, neumann, float, true, 128)
