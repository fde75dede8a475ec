// Packed float pairs for the FP32 shell quartets of mixed precision.
//
// The FP32 J/K kernels are bound by instruction issue, not by the FP32
// pipe: one scalar FFMA per issue slot fills only half of what the FP32
// units of an sm_100 SM can do.  Blackwell's packed instructions (FFMA2,
// FADD2, FMUL2 -- the __ffma2_rn family) carry two FP32 operations per
// issue slot, so a lane that evaluates two primitive quartets at once in
// F2 values runs the generated Obara-Saika recursions at twice the FP32
// work per instruction.  The generated class code (eri_classes.cuh) is
// written in pf_fma / * / + on its template type, so F2 instantiates it as
// is.
#pragma once
#include <cuda_runtime.h>

namespace pyfacc {

struct F2 {
  float2 v;
  __device__ __forceinline__ F2() {}
  __device__ __forceinline__ explicit F2(float a) : v(make_float2(a, a)) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};

__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2 r;
  r.v = __fmul2_rn(a.v, b.v);
  return r;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2 r;
  r.v = __fadd2_rn(a.v, b.v);
  return r;
}
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) {
  a.v = __fadd2_rn(a.v, b.v);
  return a;
}
__device__ __forceinline__ F2 pf_fma(F2 a, F2 b, F2 c) {
  F2 r;
  r.v = __ffma2_rn(a.v, b.v, c.v);
  return r;
}

}  // namespace pyfacc
