// Morton codes on the device, bit-exact with computeMortonCodes
// (src/physics/mortonTree.js:43-62): cubic bbox over finite particles, 10-bit
// quantisation per axis in IEEE double, ToInt32 (`| 0`), clamp to 1023, and the
// part1by2 interleave x | y<<1 | z<<2.
#pragma once
#include "common.cuh"

namespace gs {

// Double-precision frame of the quantisation, derived once per build.
struct __align__(16) MortonFrame {
  double mn[3];
  double s;     // 1024 / size
  double size;  // rootSize
};

// mortonTree.js:29-36
__host__ __device__ inline uint32_t part1by2(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x30000ff;
  v = (v | (v << 8)) & 0x300f00f;
  v = (v | (v << 4)) & 0x30c30c3;
  v = (v | (v << 2)) & 0x9249249;
  return v;
}

// ECMA-262 ToInt32 of a double (the `x | 0` of mortonTree.js:56-58): truncate,
// wrap modulo 2^32, NaN/Inf -> 0. All steps are exact in IEEE double.
__device__ inline int32_t js_toint32(double d) {
  if (!isfinite(d)) return 0;
  if (d > -2147483648.0 && d < 2147483648.0) return (int32_t)d;  // truncation
  double t = trunc(d);
  double m = fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}

// Math.max(a, b, c) with NaN propagation.
__device__ inline double js_max3(double a, double b, double c) {
  if (isnan(a) || isnan(b) || isnan(c)) return __longlong_as_double(0x7ff8000000000000ll);
  double m = a;
  if (b > m) m = b;
  if (c > m) m = c;
  return m;
}

// The double frame from the float bbox, exactly as mortonTree.js:53-54:
// size = max(extent) * 1.0001 + 1e-9 (no contraction), s = 1024 / size.
__device__ inline MortonFrame frame_from_bbox(const float mn[3], const float mx[3]) {
  MortonFrame f;
  double e[3];
  for (int k = 0; k < 3; k++) {
    f.mn[k] = (double)mn[k];
    e[k] = __dsub_rn((double)mx[k], (double)mn[k]);
  }
  f.size = __dadd_rn(__dmul_rn(js_max3(e[0], e[1], e[2]), 1.0001), 1e-9);
  f.s = __ddiv_rn(1024.0, f.size);
  return f;
}

__device__ inline uint32_t morton_code(const MortonFrame& f, float x, float y, float z) {
  int32_t q[3];
  const float v[3] = {x, y, z};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    int32_t t = js_toint32(__dmul_rn(__dsub_rn((double)v[k], f.mn[k]), f.s));
    q[k] = t > 1023 ? 1023 : t;
  }
  return part1by2((uint32_t)q[0]) | (part1by2((uint32_t)q[1]) << 1) |
         (part1by2((uint32_t)q[2]) << 2);
}

}  // namespace gs
