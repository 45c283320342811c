// Two FP32 values processed as one packed pair with the sm_100 paired-FP32 instructions
// (fma/add/mul .rn.f32x2): each component is rounded exactly as the scalar operation would round
// it, so a pair of cells computed this way gives the results of two scalar evaluations.  Subtraction
// is a - b = fma(b, -1, a) (exact negation, one rounding).
#pragma once

#include <cuda_runtime.h>

namespace mpdg
{
  using ::fma; // the scalar overloads stay visible beside the packed ones below

  struct F2
  {
    float2 v;
  };

  __device__ __forceinline__ F2
  f2(float a, float b)
  {
    return F2{make_float2(a, b)};
  }
  __device__ __forceinline__ F2
  f2(float s)
  {
    return F2{make_float2(s, s)};
  }
  __device__ __forceinline__ F2
  operator+(F2 a, F2 b)
  {
    return F2{__fadd2_rn(a.v, b.v)};
  }
  __device__ __forceinline__ F2
  operator-(F2 a, F2 b)
  {
    return F2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)};
  }
  __device__ __forceinline__ F2
  operator*(F2 a, F2 b)
  {
    return F2{__fmul2_rn(a.v, b.v)};
  }
  __device__ __forceinline__ F2
  operator*(float s, F2 b)
  {
    return F2{__fmul2_rn(make_float2(s, s), b.v)};
  }
  __device__ __forceinline__ F2 &
  operator+=(F2 &a, F2 b)
  {
    a = a + b;
    return a;
  }
  __device__ __forceinline__ F2 &
  operator*=(F2 &a, F2 b)
  {
    a = a * b;
    return a;
  }
  __device__ __forceinline__ F2
  fma(F2 a, F2 b, F2 c)
  {
    return F2{__ffma2_rn(a.v, b.v, c.v)};
  }
  __device__ __forceinline__ F2
  fma(float s, F2 b, F2 c)
  {
    return F2{__ffma2_rn(make_float2(s, s), b.v, c.v)};
  }
} // namespace mpdg
