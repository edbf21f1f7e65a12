// 16-byte shared-memory moves for the tiled stage kernels: four floats or two
// doubles in one access. The kernels store a plane's per-cell values as
// groups of U = 16 / sizeof(real) values, each group cell by cell
// ([value / U][cell][value % U]), so one group moves in one access and a
// warp's accesses to one group are contiguous (no bank conflicts).
#pragma once
#include <cuda_runtime.h>

namespace clv {

template <class real> struct Smem16 {
  static constexpr int U = 16 / (int)sizeof(real);          // values in 16 bytes
  static constexpr int pad(int n) { return (n + U - 1) / U * U; }  // n rounded up to whole groups
};

template <class real> __device__ __forceinline__ void ld16(const real* p, real* o) {
  if constexpr (sizeof(real) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
  } else {
    const double2 t = *reinterpret_cast<const double2*>(p);
    o[0] = t.x; o[1] = t.y;
  }
}
template <class real> __device__ __forceinline__ void st16(real* p, const real* v) {
  if constexpr (sizeof(real) == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

// the NG groups of slot c of an array of n slots (base = &X[0][0][0]) into or
// from v[NG * U]; groups whose values go unused are dropped by the compiler
template <class real, int NG> __device__ __forceinline__ void grp_load(const real* base, int n, int c, real* v) {
  constexpr int U = Smem16<real>::U;
#pragma unroll
  for (int g = 0; g < NG; g++) ld16<real>(base + ((size_t)g * n + c) * U, v + U * g);
}
template <class real, int NG> __device__ __forceinline__ void grp_store(real* base, int n, int c, const real* v) {
  constexpr int U = Smem16<real>::U;
#pragma unroll
  for (int g = 0; g < NG; g++) st16<real>(base + ((size_t)g * n + c) * U, v + U * g);
}

}  // namespace clv
