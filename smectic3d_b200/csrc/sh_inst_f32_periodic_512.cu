// Solver instantiations: float, periodic boundary, N = 512.
#include "sh_inst.cuh"
SHB_INST_UNIT(f32, periodic, float, false, 512)
