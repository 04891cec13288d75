// Solver instantiations: float, periodic boundary, N = 16, 32, 64.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, periodic, float, false, 16)
SHB_INST_UNIT(f32, periodic, float, false, 32)
SHB_INST_UNIT(f32, periodic, float, false, 64)
