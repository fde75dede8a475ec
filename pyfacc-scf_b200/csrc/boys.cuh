// Boys function F_m(T) = int_0^1 t^(2m) exp(-T t^2) dt on the device.
//
// Accurate mode (default): F_L (L = the highest order a class needs) from an
// 8-term Taylor expansion about the nearest point T_k of a 0.1-spaced grid
// (|dT| <= 0.05, remainder < 1e-16 relative), read as 8 coefficients
// F_{L+j}(T_k) / j! per grid point (so the Horner step is one FMA), for
// T < 36; for T >= 36 from F_0 = sqrt(pi/T)/2 (erfc(6) ~ 2e-17) and the
// upward recursion F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T) (stable for
// T > m).  The lower orders follow from the stable downward recursion
// F_m = (2T F_{m+1} + e^{-T}) / (2m+1), with e^{-T} = e^{-T_k} e^{T_k - T}
// from e^{-T_k} tabulated on the same 0.1 grid up to T = 100 and the
// degree-8 Taylor polynomial of e^x on |x| <= 0.05 (remainder < 6e-18
// relative); beyond T = 100, e^{-T} < 4e-44 and is dropped (a relative
// change below 1e-29 of F_6).  The grid values are computed once on the host
// in long double from the positive series (ensure_boys_tables, kernels.cu).
// FP32 mode (mixed precision) uses the same per-order scaled grid in float
// with 5 Taylor terms, and expf.
//
// Reference mode: boys.f90:9-43 of PyFAcc-SCF -- Taylor 1/(2m+1) - x/(2m+3)
// for x <= 1e-6, else the 1001-point trapezoid rule on [0,1].  It is used for
// the nuclear-attraction matrix only, so that V reproduces the reference.
#pragma once
#include <cuda_runtime.h>

#include "f2.cuh"

#define PF_BOYS_NGRID 361
#define PF_BOYS_STEP 0.1
#define PF_BOYS_INV_STEP 10.0
#define PF_BOYS_TMAX 36.0
#define PF_BOYS_MMAX 9       // highest order needed: (dd|dd) gradient = 9
#define PF_BOYS_NT 8         // Taylor terms, FP64
#define PF_BOYS_NTF 5        // Taylor terms, FP32
#define PF_BOYS_EMAX 100.0   // e^{-T} table end
#define PF_BOYS_NEXP 1001    // e^{-T_k}, T_k = 0.1 k <= PF_BOYS_EMAX
#define PF_BOYS_NCOL (PF_BOYS_MMAX + PF_BOYS_NT)

namespace pyfacc {

// Grid tables, one copy per translation unit that includes this header
// (kernels.cu and kernels_d.cu; each fills its copy per device with
// cudaMemcpyToSymbol, see ensure_boys_tables):
// g_boys_tl[L][k][j] = F_{L+j}(T_k) / j!, g_boys_exp[k] = e^{-T_k},
// g_boys_tlf[L][k][j] = F_{L+j}(T_k) / j! in float (j < 5 used).
static __device__ __align__(16) double g_boys_tl[(PF_BOYS_MMAX + 1) * PF_BOYS_NGRID * PF_BOYS_NT];
static __device__ double g_boys_exp[PF_BOYS_NEXP];
static __device__ __align__(16) float g_boys_tlf[(PF_BOYS_MMAX + 1) * PF_BOYS_NGRID * PF_BOYS_NT];

// Branch-free: every lane evaluates the Taylor value (from row 0 when T is
// beyond the grid) and the asymptotic value and selects, so a warp whose
// quartets straddle T = 36 does not execute both paths one after the other.
template <int L>
__device__ __forceinline__ void boys_fp64(double T, double* __restrict__ F) {
  const bool tab = T < PF_BOYS_TMAX;
  // nearest grid point by adding and subtracting 1.5 * 2^52 (round to
  // nearest in the FMA pipe, no conversion instructions): kd = round(10 T),
  // the integer sits in the low word of the biased value
  const double biased = fmin(T, PF_BOYS_EMAX) * PF_BOYS_INV_STEP + 6755399441055744.0;
  const int ke = __double2loint(biased);
  const double kd = biased - 6755399441055744.0;
  const int k = tab ? ke : 0;
  const double x = kd * PF_BOYS_STEP - T;  // F_L(T) = sum_j F_{L+j}(T_k) x^j / j! (T < 36)
  const double2* row = reinterpret_cast<const double2*>(g_boys_tl + ((size_t)L * PF_BOYS_NGRID + k) * PF_BOYS_NT);
  const double2 c01 = __ldg(row), c23 = __ldg(row + 1), c45 = __ldg(row + 2), c67 = __ldg(row + 3);
  double f = fma(c67.y, x, c67.x);
  f = fma(f, x, c45.y);
  f = fma(f, x, c45.x);
  f = fma(f, x, c23.y);
  f = fma(f, x, c23.x);
  f = fma(f, x, c01.y);
  f = fma(f, x, c01.x);
  const double rt = rsqrt(fmax(T, PF_BOYS_TMAX));
  double fa = 0.88622692545275801365 * rt;  // sqrt(pi/T)/2
  if (L == 0) {
    F[0] = tab ? f : fa;
    return;
  }
  // e^x on |x| <= 0.05, Taylor coefficients 1/j!, j = 8 .. 0
  double ex = 1.0 / 40320.0;
  ex = fma(ex, x, 1.0 / 5040.0);
  ex = fma(ex, x, 1.0 / 720.0);
  ex = fma(ex, x, 1.0 / 120.0);
  ex = fma(ex, x, 1.0 / 24.0);
  ex = fma(ex, x, 1.0 / 6.0);
  ex = fma(ex, x, 0.5);
  ex = fma(ex, x, 1.0);
  ex = fma(ex, x, 1.0);
  const double e = (T < PF_BOYS_EMAX) ? __ldg(g_boys_exp + ke) * ex : 0.0;
  const double o2t = 0.5 * rt * rt;
#pragma unroll
  for (int m = 0; m < L; ++m) fa = ((2 * m + 1) * fa - e) * o2t;
  F[L] = tab ? f : fa;
  const double t2 = 2.0 * T;
#pragma unroll
  for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
}

template <int L>
__device__ __forceinline__ void boys_fp32(float T, float* __restrict__ F) {
  const bool tab = T < (float)PF_BOYS_TMAX;
  // nearest grid point by adding and subtracting 1.5 * 2^23 (see boys_fp64)
  const float biased = fminf(T, (float)PF_BOYS_TMAX) * (float)PF_BOYS_INV_STEP + 12582912.0f;
  const int k = tab ? (__float_as_int(biased) & 0x7fffff) - 0x400000 : 0;
  const float x = (biased - 12582912.0f) * (float)PF_BOYS_STEP - T;
  const float4* row = reinterpret_cast<const float4*>(g_boys_tlf + ((size_t)L * PF_BOYS_NGRID + k) * PF_BOYS_NT);
  const float4 c0 = __ldg(row), c1 = __ldg(row + 1);
  float f = fmaf(c1.x, x, c0.w);  // 5 terms: F_{L+j}(T_k) / j!, j = 4 .. 0
  f = fmaf(f, x, c0.z);
  f = fmaf(f, x, c0.y);
  f = fmaf(f, x, c0.x);
  const float rt = rsqrtf(fmaxf(T, (float)PF_BOYS_TMAX));
  float fa = 0.88622692545275801365f * rt;
  if (L == 0) {
    F[0] = tab ? f : fa;
    return;
  }
  const float e = expf(-T);
  const float o2t = 0.5f * rt * rt;
#pragma unroll
  for (int m = 0; m < L; ++m) fa = ((2 * m + 1) * fa - e) * o2t;
  F[L] = tab ? f : fa;
  const float t2 = 2.0f * T;
#pragma unroll
  for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0f / (2 * m + 1));
}

// Two arguments at once in packed float pairs (F2, f2.cuh): the grid rows
// are gathered per argument, the Taylor sum and the recursions run on both
// in FFMA2/FMUL2; the per-argument selections (Taylor or asymptotic, grid
// index) stay scalar.  The same arithmetic as boys_fp32, argument by
// argument.
template <int L>
__device__ __forceinline__ void boys_fp32x2(F2 T, F2* __restrict__ F) {
  const float Tx = T.v.x, Ty = T.v.y;
  const bool tabx = Tx < (float)PF_BOYS_TMAX, taby = Ty < (float)PF_BOYS_TMAX;
  const F2 biased = pf_fma(F2(fminf(Tx, (float)PF_BOYS_TMAX), fminf(Ty, (float)PF_BOYS_TMAX)),
                           F2((float)PF_BOYS_INV_STEP), F2(12582912.0f));
  const int kx = tabx ? (__float_as_int(biased.v.x) & 0x7fffff) - 0x400000 : 0;
  const int ky = taby ? (__float_as_int(biased.v.y) & 0x7fffff) - 0x400000 : 0;
  const F2 kd = biased + F2(-12582912.0f);
  const F2 x = pf_fma(kd, F2((float)PF_BOYS_STEP), T * F2(-1.0f));
  const float4* rx = reinterpret_cast<const float4*>(g_boys_tlf + ((size_t)L * PF_BOYS_NGRID + kx) * PF_BOYS_NT);
  const float4* ry = reinterpret_cast<const float4*>(g_boys_tlf + ((size_t)L * PF_BOYS_NGRID + ky) * PF_BOYS_NT);
  const float4 x0 = __ldg(rx), x1 = __ldg(rx + 1), y0 = __ldg(ry), y1 = __ldg(ry + 1);
  F2 f = pf_fma(F2(x1.x, y1.x), x, F2(x0.w, y0.w));
  f = pf_fma(f, x, F2(x0.z, y0.z));
  f = pf_fma(f, x, F2(x0.y, y0.y));
  f = pf_fma(f, x, F2(x0.x, y0.x));
  const F2 rt(rsqrtf(fmaxf(Tx, (float)PF_BOYS_TMAX)), rsqrtf(fmaxf(Ty, (float)PF_BOYS_TMAX)));
  F2 fa = F2(0.88622692545275801365f) * rt;
  if (L == 0) {
    F[0] = F2(tabx ? f.v.x : fa.v.x, taby ? f.v.y : fa.v.y);
    return;
  }
  const F2 e(expf(-Tx), expf(-Ty));
  const F2 ne = e * F2(-1.0f);
  const F2 o2t = F2(0.5f) * rt * rt;
#pragma unroll
  for (int m = 0; m < L; ++m) fa = pf_fma(F2((float)(2 * m + 1)), fa, ne) * o2t;
  F[L] = F2(tabx ? f.v.x : fa.v.x, taby ? f.v.y : fa.v.y);
  const F2 t2 = T + T;
#pragma unroll
  for (int m = L - 1; m >= 0; --m) F[m] = pf_fma(t2, F[m + 1], e) * F2(1.0f / (2 * m + 1));
}

template <int L, typename R> struct Boys;
template <int L> struct Boys<L, double> {
  __device__ static __forceinline__ void eval(double T, double* F) { boys_fp64<L>(T, F); }
};
template <int L> struct Boys<L, float> {
  __device__ static __forceinline__ void eval(float T, float* F) { boys_fp32<L>(T, F); }
};

// boys.f90:9-43, literally: small-x Taylor, else 1001-point trapezoid.
__device__ __forceinline__ double boys_trapezoid(int nu, double x) {
  if (x <= 1.0e-6) return 1.0 / (2.0 * nu + 1.0) - x / (2.0 * nu + 3.0);
  const int N = 1000;
  const double dt = 1.0 / N;
  double sum = 0.0;
  for (int i = 0; i <= N; ++i) {
    const double t = i * dt;
    const double e = exp(-x * t * t);
    double tp = 1.0;
    for (int k = 0; k < 2 * nu; ++k) tp *= t;
    sum += (i == 0 || i == N) ? 0.5 * tp * e : tp * e;
  }
  return sum * dt;
}

// F_0..F_lmax with a runtime order bound (one-electron kernels).
__device__ __forceinline__ void boys_runtime(int mode, int lmax, double T, double* F) {
  if (mode == 1) {
    for (int m = 0; m <= lmax; ++m) F[m] = boys_trapezoid(m, T);
    return;
  }
  switch (lmax) {
    case 0: boys_fp64<0>(T, F); break;
    case 1: boys_fp64<1>(T, F); break;
    case 2: boys_fp64<2>(T, F); break;
    case 3: boys_fp64<3>(T, F); break;
    case 4: boys_fp64<4>(T, F); break;
    case 5: boys_fp64<5>(T, F); break;
    case 6: boys_fp64<6>(T, F); break;
    case 7: boys_fp64<7>(T, F); break;
    case 8: boys_fp64<8>(T, F); break;
    default: boys_fp64<9>(T, F); break;
  }
}

}  // namespace pyfacc
