// Solver instantiations: float, periodic boundary, N = 256.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, periodic, float, false, 256)
