// Solver instantiations: float, periodic boundary, N = 128.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, periodic, float, false, 128)
