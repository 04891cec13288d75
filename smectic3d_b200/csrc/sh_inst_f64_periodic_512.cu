// Solver instantiations: double, periodic boundary, N = 512.
#include "sh_inst.cuh"
SHB_INST_UNIT(f64, periodic, double, false, 512)
