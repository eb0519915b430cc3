// Device helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace dgpu {

// Bilinear blend of one coarse cell, float32 with the reference's fused
// multiply-adds (src/subtract.cpp:196-204 as compiled with FMA contraction).
__device__ __forceinline__ float cell_blend(float a00, float a01, float a10, float a11, float fy,
                                            float wx) {
  const float base = __fmaf_rn(a10 - a00, fy, a00);
  const float top = a01 - a00;
  const float slope = __fmaf_rn((a11 - a10) - top, fy, top);
  return __fmaf_rn(slope, wx, base);
}

// a_f(x, y) (f == nc is the background), CoarseFields::point
// (src/subtract.cpp:187-205).
__device__ __forceinline__ float field_point(const DevFields& F, int f, int x, int y) {
  if (F.exact) return F.full[(static_cast<size_t>(f) * F.h + y) * F.w + x];
  const int jx = F.cellx[x], jy = F.celly[y];
  const float* c0 = F.latf + (static_cast<size_t>(f) * F.ncy + jy) * F.ncx;
  const float* c1 = c0 + F.ncx;
  return cell_blend(c0[jx], c0[jx + 1], c1[jx], c1[jx + 1], F.wy[y], F.wx[x]);
}

__device__ __forceinline__ void set_status(unsigned* st, unsigned bit) {
  if (st) atomicOr(st, bit);
}

// Monotone uint32 key of a float (total order matching operator< on finite
// values, -0 before +0).
__device__ __forceinline__ uint32_t float_key(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace dgpu
