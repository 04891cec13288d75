// Solver instantiations: float, neumann boundary, N = 16, 32, 64.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, neumann, float, true, 16)
SHB_INST_UNIT(f32, neumann, float, true, 32)
SHB_INST_UNIT(f32, neumann, float, true, 64)
