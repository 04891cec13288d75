// Instantiation of the solver for every supported grid size.  Included by one
// translation unit per (precision, boundary) so that they compile in parallel.
#pragma once
#include "sh_solver.cuh"

namespace shb {

// Cluster size CL of the plane pass (NC = N / (2 CL) column lines per CTA).
// ``variant`` selects a CL explicitly (0 = default); a CL whose working set
// does not fit one CTA's shared memory is not built.
template <typename T, int N, int CL, bool DCT, int TKV = 0>
SolverBase* make_if_fits() {
  if constexpr (PlaneCfg<T, N, CL, DCT>::fits) {
    return new Solver<T, N, CL, DCT, TKV>();
  } else {
    return nullptr;
  }
}

// Pencil tiles of 8, 16 or 32 lines per CTA (``tile``, 0 = the default), with
// the plane cluster size ``CL``: built for the batched replicas' 64^3 and for
// 128^3 without clusters
template <typename T, int N, int CL, bool DCT>
SolverBase* make_tiled(int tile) {
  constexpr int def = PencilCfg<T, N, DCT>::TK;
  if (tile == 0 || tile == def) return make_if_fits<T, N, CL, DCT>();
  if constexpr (def != 8) {
    if (tile == 8) return make_if_fits<T, N, CL, DCT, 8>();
  }
  if constexpr (def != 16) {
    if (tile == 16) return make_if_fits<T, N, CL, DCT, 16>();
  }
  if constexpr (def != 32) {
    if (tile == 32) return make_if_fits<T, N, CL, DCT, 32>();
  }
  return nullptr;
}

// Solver of one grid size N with cluster size ``cl`` (0 = the default) and
// pencil tile ``tile`` (0 = the default; other tiles at 64^3, and at 128^3 with
// cluster size 1).
template <typename T, int N, bool DCT>
SolverBase* make_sized(int cl, int tile) {
  const bool other_tile = tile != 0 && tile != PencilCfg<T, N, DCT>::TK;
  if (other_tile && !(N == 64 || (N == 128 && cl <= 1))) return nullptr;
  if constexpr (N <= 32) {
    return cl == 0 || cl == 1 ? make_if_fits<T, N, 1, DCT>() : nullptr;
  } else if constexpr (N == 64) {
    if (cl == 0 || cl == 1) return make_tiled<T, 64, 1, DCT>(tile);
    if (cl == 2) return make_tiled<T, 64, 2, DCT>(tile);
    return nullptr;
  } else if constexpr (N == 128) {
    if (cl == 0 || cl == 1) return make_tiled<T, 128, 1, DCT>(tile);
    if (cl == 2) return make_if_fits<T, 128, 2, DCT>();
    if (cl == 4) return make_if_fits<T, 128, 4, DCT>();
    return nullptr;
  } else if constexpr (N == 256) {
    // default: 8 for FP32 (three CTAs per SM), 16 for FP64 (half the shared
    // memory of 8, two CTAs per SM)
    if (cl == 4) return make_if_fits<T, 256, 4, DCT>();
    if (cl == 8 || (cl == 0 && sizeof(T) == 4)) return make_if_fits<T, 256, 8, DCT>();
    if (cl == 16 || (cl == 0 && sizeof(T) == 8)) return make_if_fits<T, 256, 16, DCT>();
    return nullptr;
  } else {
    if (cl == 0 || cl == 16) return make_if_fits<T, 512, 16, DCT>();
    return nullptr;
  }
}

}  // namespace shb

// One translation unit per (precision, boundary, size group) so that nvcc
// compiles them in parallel: SHB_INST_UNIT(f32, neumann, float, true, 256)
// defines shb::make_solver_f32_neumann_n256.
#define SHB_INST_UNIT(P, B, T, DCT, N) \
  namespace shb {                       \
  SolverBase* make_solver_##P##_##B##_n##N(int cl, int tile) { return make_sized<T, N, DCT>(cl, tile); } \
  }
