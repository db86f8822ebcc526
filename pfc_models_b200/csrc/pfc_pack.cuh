// Two-lane complex arithmetic on the packed FP32 pipe of sm_100a.
//
// A `pc` value holds one complex number of each of two independent transforms: the
// real parts of lanes 0 and 1 in one 64-bit register pair and the imaginary parts in
// another. Every operation is issued as packed f32x2 instructions (add/sub/mul/fma .f32x2),
// so each instruction advances both transforms: the butterflies, twiddle products and
// pointwise terms of two rows (or two columns) cost the issue slots of one. Both lanes
// run the same code on the same indices, so their rounding is identical.
#pragma once
#include <cuda_runtime.h>

namespace pfc {

__device__ __forceinline__ unsigned long long f2u(float2 a) { return *reinterpret_cast<unsigned long long*>(&a); }
__device__ __forceinline__ float2 u2f(unsigned long long a) { return *reinterpret_cast<float2*>(&a); }

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
  return u2f(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }

struct pc {
  float2 r, i;
};

__device__ __forceinline__ pc mkpc(float2 r, float2 i) { pc v; v.r = r; v.i = i; return v; }
// from one complex value per lane
__device__ __forceinline__ pc mkpc2(float2 lane0, float2 lane1) {
  return mkpc(make_float2(lane0.x, lane1.x), make_float2(lane0.y, lane1.y));
}
__device__ __forceinline__ float2 lane0(pc v) { return make_float2(v.r.x, v.i.x); }
__device__ __forceinline__ float2 lane1(pc v) { return make_float2(v.r.y, v.i.y); }

__device__ __forceinline__ pc operator+(pc a, pc b) { return mkpc(add2(a.r, b.r), add2(a.i, b.i)); }
__device__ __forceinline__ pc operator-(pc a, pc b) { return mkpc(sub2(a.r, b.r), sub2(a.i, b.i)); }
// a + rot(b) and a - rot(b), rot = multiply by -i (forward) or +i (inverse)
template <bool INV> __device__ __forceinline__ pc addrot(pc a, pc b) {
  return INV ? mkpc(sub2(a.r, b.i), add2(a.i, b.r)) : mkpc(add2(a.r, b.i), sub2(a.i, b.r));
}
template <bool INV> __device__ __forceinline__ pc subrot(pc a, pc b) {
  return INV ? mkpc(add2(a.r, b.i), sub2(a.i, b.r)) : mkpc(sub2(a.r, b.i), add2(a.i, b.r));
}
// a * (c + i s), the same compile-time (c, s) for both lanes
__device__ __forceinline__ pc pmulc(pc a, float c, float s) {
  return mkpc(fma2(a.i, bc2(-s), mul2(a.r, bc2(c))), fma2(a.i, bc2(c), mul2(a.r, bc2(s))));
}
__device__ __forceinline__ pc pscale(pc a, float s) { return mkpc(mul2(a.r, bc2(s)), mul2(a.i, bc2(s))); }

// ---------------------------------------------------------------- small DFTs on two lanes
// The radix-2 decimation-in-time structure and constants of the scalar dft2..dft16 of
// pfc_fft.cuh (forward e^{-2 pi i jk/R}, inverse unnormalised).
template <bool INV> __device__ __forceinline__ void pdft2(pc& a, pc& b) {
  const pc t = a - b;
  a = a + b;
  b = t;
}

template <bool INV> __device__ __forceinline__ void pdft4(pc* v) {
  const pc t0 = v[0] + v[2], t1 = v[0] - v[2];
  const pc t2 = v[1] + v[3], d = v[1] - v[3];
  v[0] = t0 + t2;
  v[2] = t0 - t2;
  v[1] = addrot<INV>(t1, d);
  v[3] = subrot<INV>(t1, d);
}

// multiply by exp(-+ 2 pi i k / 8), k = 1, 3
template <bool INV, int K> __device__ __forceinline__ pc pw8(pc a) {
  const float c = 0.70710678118654752440f;
  if (K == 1) {
    return INV ? mkpc(mul2(sub2(a.r, a.i), bc2(c)), mul2(add2(a.r, a.i), bc2(c)))
               : mkpc(mul2(add2(a.r, a.i), bc2(c)), mul2(sub2(a.i, a.r), bc2(c)));
  }
  // K == 3
  return INV ? mkpc(mul2(add2(a.r, a.i), bc2(-c)), mul2(sub2(a.r, a.i), bc2(c)))
             : mkpc(mul2(sub2(a.i, a.r), bc2(c)), mul2(add2(a.r, a.i), bc2(-c)));
}

template <bool INV> __device__ __forceinline__ void pdft8(pc* v) {
  pc e[4] = {v[0], v[2], v[4], v[6]};
  pc o[4] = {v[1], v[3], v[5], v[7]};
  pdft4<INV>(e);
  pdft4<INV>(o);
  o[1] = pw8<INV, 1>(o[1]);
  o[3] = pw8<INV, 3>(o[3]);
  v[0] = e[0] + o[0];
  v[4] = e[0] - o[0];
  v[1] = e[1] + o[1];
  v[5] = e[1] - o[1];
  v[2] = addrot<INV>(e[2], o[2]);   // o[2] * exp(-+ i pi/2)
  v[6] = subrot<INV>(e[2], o[2]);
  v[3] = e[3] + o[3];
  v[7] = e[3] - o[3];
}

template <bool INV> __device__ __forceinline__ void pdft16(pc* v) {
  pc e[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
  pdft8<INV>(e);
  pdft8<INV>(o);
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
  const float c2 = 0.70710678118654752440f;
  const float cs[8] = {1.f, c1, c2, s1, 0.f, -s1, -c2, -c1};
  const float sn[8] = {0.f, s1, c2, c1, 1.f, c1, c2, s1};
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    if (k == 4) continue;
    o[k] = pmulc(o[k], cs[k], INV ? sn[k] : -sn[k]);
  }
  v[0] = e[0] + o[0];
  v[8] = e[0] - o[0];
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    if (k == 4) {
      v[4] = addrot<INV>(e[4], o[4]);
      v[12] = subrot<INV>(e[4], o[4]);
    } else {
      v[k] = e[k] + o[k];
      v[k + 8] = e[k] - o[k];
    }
  }
}

template <int R, bool INV> __device__ __forceinline__ void pdft(pc* v) {
  if constexpr (R == 2) pdft2<INV>(v[0], v[1]);
  else if constexpr (R == 4) pdft4<INV>(v);
  else if constexpr (R == 8) pdft8<INV>(v);
  else pdft16<INV>(v);
}

}  // namespace pfc
