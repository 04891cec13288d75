// Instantiation of the solver for every supported grid size.  Included by one
// translation unit per (precision, boundary) so that they compile in parallel.
#pragma once
#include "sh_solver.cuh"

namespace shb {

// cluster size of the plane pass: NC = N / (2 CL) column lines per CTA
template <int N> constexpr int cluster_for() {
  return N <= 64 ? 1 : (N == 128 ? 2 : (N == 256 ? 4 : 16));
}

template <typename T, bool DCT>
SolverBase* make_solver(int n) {
  switch (n) {
    case 16: return new Solver<T, 16, cluster_for<16>(), DCT>();
    case 32: return new Solver<T, 32, cluster_for<32>(), DCT>();
    case 64: return new Solver<T, 64, cluster_for<64>(), DCT>();
    case 128: return new Solver<T, 128, cluster_for<128>(), DCT>();
    case 256: return new Solver<T, 256, cluster_for<256>(), DCT>();
#ifdef SHB_WITH_512
    case 512: return new Solver<T, 512, cluster_for<512>(), DCT>();
#endif
    default: return nullptr;
  }
}

}  // namespace shb
