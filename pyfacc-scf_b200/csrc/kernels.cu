// Device code of the B200 Hartree-Fock engine (sm_100a).
//
//  * Boys tables (boys.cuh)
//  * shell-pair construction, Schwarz factors, sorted gather
//  * J/K digestion: one warp per task = one bra shell pair x 32 ket pairs,
//    one contracted shell quartet per lane, OS/HGP class code from
//    eri_classes.cuh, J_ab reduced across the warp with shuffles, the other
//    J/K blocks added with FP64 atomics; the ERI tensor is never stored
//  * nuclear-gradient two-electron kernel with the same task layout
//  * one-electron S/T/V and their derivatives (the reference's formulas,
//    overlap.f90 / kinetic.f90 / nuclear.f90, evaluated per shell pair)
//  * dense helpers for the SCF step and an FP64 peak probe
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <atomic>
#include <mutex>
#include <vector>

#include "boys.cuh"
#include "engine.h"
#include "eri_classes.cuh"

namespace pyfacc {

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ===========================================================================
// Boys tables: F_m(T_k), T_k = 0.1 k, from the positive series in long double
// ===========================================================================
static long double boys_series_ld(int m, long double x) {
  if (x <= 0.0L) return 1.0L / (2 * m + 1);
  long double term = 1.0L / (2 * m + 1), sum = term;
  for (int k = 1; k < 2000; ++k) {
    term *= 2.0L * x / (2 * m + 2 * k + 1);
    sum += term;
    if (term < sum * 1e-22L) break;
  }
  return expl(-x) * sum;
}

void ensure_boys_tables(int device) {
  static std::mutex mu;
  static std::vector<double> tl, ex;
  static std::vector<float> tabf;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (tl.empty()) {
    std::vector<long double> F((size_t)PF_BOYS_NGRID * PF_BOYS_NCOL);
    for (int k = 0; k < PF_BOYS_NGRID; ++k)
      for (int m = 0; m < PF_BOYS_NCOL; ++m) F[(size_t)k * PF_BOYS_NCOL + m] = boys_series_ld(m, (long double)k * 0.1L);
    tl.resize((size_t)(PF_BOYS_MMAX + 1) * PF_BOYS_NGRID * PF_BOYS_NT);
    for (int L = 0; L <= PF_BOYS_MMAX; ++L)
      for (int k = 0; k < PF_BOYS_NGRID; ++k) {
        long double fact = 1.0L;
        for (int j = 0; j < PF_BOYS_NT; ++j) {
          if (j > 0) fact *= j;
          tl[((size_t)L * PF_BOYS_NGRID + k) * PF_BOYS_NT + j] = (double)(F[(size_t)k * PF_BOYS_NCOL + L + j] / fact);
        }
      }
    ex.resize(PF_BOYS_NEXP);
    for (int k = 0; k < PF_BOYS_NEXP; ++k) ex[k] = (double)expl(-(long double)k * 0.1L);
    tabf.resize(tl.size());
    for (size_t i = 0; i < tl.size(); ++i) tabf[i] = (float)tl[i];
  }
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (!done[device]) {
    PF_CUDA(cudaMemcpyToSymbol(g_boys_tl, tl.data(), tl.size() * sizeof(double)));
    PF_CUDA(cudaMemcpyToSymbol(g_boys_exp, ex.data(), ex.size() * sizeof(double)));
    PF_CUDA(cudaMemcpyToSymbol(g_boys_tlf, tabf.data(), tabf.size() * sizeof(float)));
    upload_boys_tables_d(tl.data(), tl.size(), ex.data(), ex.size());
    done[device] = 1;
  }
}

__global__ void boys_test_kernel(int mode, int fp32, int mmax, int n, const double* __restrict__ x,
                                 double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double F[PF_BOYS_MMAX + 1];
  if (fp32) {
    float Ff[PF_BOYS_MMAX + 1];
    float T = (float)x[i];
    switch (mmax) {
      case 0: boys_fp32<0>(T, Ff); break;
      case 1: boys_fp32<1>(T, Ff); break;
      case 2: boys_fp32<2>(T, Ff); break;
      case 3: boys_fp32<3>(T, Ff); break;
      case 4: boys_fp32<4>(T, Ff); break;
      case 5: boys_fp32<5>(T, Ff); break;
      default: boys_fp32<6>(T, Ff); break;
    }
    for (int m = 0; m <= mmax; ++m) F[m] = Ff[m];
  } else {
    boys_runtime(mode, mmax, x[i], F);
  }
  for (int m = 0; m <= mmax; ++m) out[(size_t)i * (mmax + 1) + m] = F[m];
}

void launch_boys_test(int mode, int fp32, int mmax, int n, const double* x, double* out, cudaStream_t s) {
  if (n <= 0) return;
  boys_test_kernel<<<(n + 127) / 128, 128, 0, s>>>(mode, fp32, mmax, n, x, out);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ===========================================================================
// Shell pairs
// ===========================================================================
__device__ __forceinline__ double prim_norm(int l, double a) {
  // gaussian.f90:80-98: (2a/pi)^(3/4) (4a)^(l/2) / sqrt((2l-1)!!) for the
  // x^l component (the (2a_x-1)!! product is 1 for s and p); the other d
  // components differ by comp_ratio
  double n = pow(2.0 * a * 0.31830988618379067154, 0.75);
  if (l == 0) return n;
  if (l == 1) return n * 2.0 * sqrt(a);
  return n * 4.0 * a * 0.57735026918962576451;  // 4a / sqrt(3)
}

// norm of Cartesian component k of an l shell / norm of its x^l component:
// sqrt(3) for d_xy, d_xz, d_yz, else 1
__device__ __forceinline__ double comp_ratio(int l, int k) {
  return (l == 2 && (k == 1 || k == 2 || k == 4)) ? 1.7320508075688772935 : 1.0;
}

// pl0 = {shell a, shell b, prim_start, first shell of the molecule},
// pl1 = {mat_off, ld, molecule, dmax_off}; info1 holds molecule-local shell
// indices (the density-maximum blocks of a molecule start at dmax_off).
// Every primitive pair is written (the Schwarz factors use them all);
// kept[i] counts those with |K| >= cut, the ones the gather keeps.
__global__ void build_pairs_kernel(int npair, const double4* __restrict__ cen, const int4* __restrict__ desc,
                                   const int* __restrict__ nprim, const double* __restrict__ ex,
                                   const double* __restrict__ co, const int4* __restrict__ pl0,
                                   const int4* __restrict__ pl1, int4* __restrict__ info0,
                                   int4* __restrict__ info1, int4* __restrict__ info2,
                                   double4* __restrict__ geom, double4* __restrict__ prim, double cut,
                                   int* __restrict__ kept) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npair) return;
  const int4 p0 = pl0[i];
  const int a = p0.x, b = p0.y, ps = p0.z;
  const int4 da = desc[a], db = desc[b];
  const int na = nprim[a], nb = nprim[b];
  const double4 A = cen[a], B = cen[b];
  const double ABx = A.x - B.x, ABy = A.y - B.y, ABz = A.z - B.z;
  const double ab2 = ABx * ABx + ABy * ABy + ABz * ABz;
  info0[i] = make_int4(da.z, db.z, ps, na * nb);
  info1[i] = make_int4(a - p0.w, b - p0.w, da.y, db.y);
  info2[i] = pl1[i];
  geom[i] = make_double4(ABx, ABy, ABz, 0.0);
  const double c0 = 5.9149671727956128778;  // sqrt(2) * pi^(5/4)
  int nk = 0;
  for (int ka = 0; ka < na; ++ka) {
    const double al = ex[da.w + ka], ca = co[da.w + ka] * prim_norm(da.x, ex[da.w + ka]);
    for (int kb = 0; kb < nb; ++kb) {
      const double be = ex[db.w + kb], cb = co[db.w + kb] * prim_norm(db.x, ex[db.w + kb]);
      const double p = al + be, op = 1.0 / p;
      const double K = ca * cb * exp(-al * be * op * ab2) * c0 * op;
      const double Px = (al * A.x + be * B.x) * op, Py = (al * A.y + be * B.y) * op, Pz = (al * A.z + be * B.z) * op;
      double4* r = prim + 3 * (size_t)(ps + ka * nb + kb);
      r[0] = make_double4(p, 0.5 * op, K, al);
      r[1] = make_double4(Px, Py, Pz, 0.0);
      r[2] = make_double4(Px - A.x, Py - A.y, Pz - A.z, 0.0);
      nk += fabs(K) >= cut;
    }
  }
  if (kept) kept[i] = nk;
}

void launch_build_pairs(const ShellDev& sh, int npair, const int4* pl0, const int4* pl1, int4* info0,
                        int4* info1, int4* info2, double4* geom, double4* prim, double cut, int* kept,
                        cudaStream_t s) {
  if (npair <= 0) return;
  build_pairs_kernel<<<(npair + 127) / 128, 128, 0, s>>>(npair, sh.cen, sh.desc, sh.nprim, sh.ex, sh.co, pl0, pl1,
                                                         info0, info1, info2, geom, prim, cut, kept);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ---------------------------------------------------------------------------
// One primitive quartet: prefactors, Boys, VRR (shared by J/K, Schwarz,
// gradient and tensor kernels).
// ---------------------------------------------------------------------------
template <typename R>
struct PrimGeo {
  R I[PF_BOYS_MMAX + 1];
  R WP[3], WQ[3];
  R o2p, nrp, o2q, nrq, o2pq;  // nrp = -rho/p, nrq = -rho/q
};

template <typename R> struct Rec;  // primitive-pair record vector of a precision
template <> struct Rec<double> { using T = double4; };
template <> struct Rec<float> { using T = float4; };

// bra record b0..b2 and ket record k0..k2 (3 vectors each)
template <typename R, int LM, typename V>
__device__ __forceinline__ void prim_setup(const V& b0, const V& b1, const V& k0, const V& k1, PrimGeo<R>& g) {
  const R p = (R)b0.x, q = (R)k0.x;
  const R PQx = (R)(b1.x - k1.x), PQy = (R)(b1.y - k1.y), PQz = (R)(b1.z - k1.z);
  const R zeta = p + q;
  R rs, oz;
  if constexpr (sizeof(R) == 8) {
    rs = rsqrt((double)zeta);
  } else {
    rs = rsqrtf((float)zeta);
  }
  oz = rs * rs;
  const R rho = p * q * oz;
  const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
  const R pref = (R)b0.z * (R)k0.z * rs;
  R F[LM + 1];
  Boys<LM, R>::eval(T, F);
#pragma unroll
  for (int m = 0; m <= LM; ++m) g.I[m] = pref * F[m];
  const R qz = q * oz, pz = p * oz;
  g.WP[0] = -qz * PQx; g.WP[1] = -qz * PQy; g.WP[2] = -qz * PQz;
  g.WQ[0] = pz * PQx;  g.WQ[1] = pz * PQy;  g.WQ[2] = pz * PQz;
  g.o2p = (R)b0.y;
  g.o2q = (R)k0.y;
  g.nrp = -qz;  // -rho / p
  g.nrq = -pz;  // -rho / q
  g.o2pq = (R)0.5 * oz;
}

template <int L> struct NC { static constexpr int v = (L + 1) * (L + 2) / 2; };

// Contracted (ab|cd) for one bra pair and one ket pair (records of the
// kernel's precision: double4 for FP64 quartets, float4 for FP32 ones).
// Primitive pairs are stored in order of decreasing |K|, so with kcut > 0
// both loops stop at the first primitive quartet with |K_ab K_cd| < kcut.
// With kq_step > 1 only the ket primitives kq0, kq0 + kq_step, ... are
// summed (a share of the quartet; the shares add up to the integral).
// brec: the bra pair's first primitive record (in global memory, or the
// copy a warp staged in shared memory); prim: all records (the kets').
template <typename R, int LA, int LB, int LC, int LD>
__device__ __forceinline__ int contracted_quartet(const typename Rec<R>::T* __restrict__ prim,
                                                  const typename Rec<R>::T* brec, int4 bi0, int4 ki0,
                                                  const double4& bgeo, const double4& kgeo,
                                                  R out[EriClass<R, LA, LB, LC, LD>::NOUT], double kcut = 0.0,
                                                  int kq0 = 0, int kq_step = 1) {
  using C = EriClass<R, LA, LB, LC, LD>;
  using V = typename Rec<R>::T;
  R acc[C::NACC];
#pragma unroll
  for (int i = 0; i < C::NACC; ++i) acc[i] = (R)0;
  // the cut is compared in the records' precision (no FP64 work in the FP32
  // loop); a cut beyond the float range becomes +inf, which skips everything
  const R cut = (R)kcut;
  const R kab_max = fabs((R)brec[0].z);
  int nprim = 0;
  for (int kq = kq0; kq < ki0.w; kq += kq_step) {
    const V* kr = prim + 3 * (size_t)(ki0.z + kq);
    const V k0 = kr[0], k1 = kr[1], k2 = kr[2];
    const R kcd = fabs((R)k0.z);
    if (kab_max * kcd < cut) break;
    const R QC[3] = {(R)k2.x, (R)k2.y, (R)k2.z};
#pragma unroll 1
    for (int kp = 0; kp < bi0.w; ++kp) {
      const V* br = brec + 3 * kp;
      const V b0 = br[0], b1 = br[1], b2 = br[2];
      if (fabs((R)b0.z) * kcd < cut) break;
      const R PA[3] = {(R)b2.x, (R)b2.y, (R)b2.z};
      PrimGeo<R> g;
      prim_setup<R, C::L>(b0, b1, k0, k1, g);
      C::vrr(g.I, PA, g.WP, QC, g.WQ, g.o2p, g.nrp, g.o2q, g.nrq, g.o2pq, acc);
      ++nprim;
    }
  }
  const R AB[3] = {(R)bgeo.x, (R)bgeo.y, (R)bgeo.z};
  const R CD[3] = {(R)kgeo.x, (R)kgeo.y, (R)kgeo.z};
  C::hrr(acc, AB, CD, out);
  return nprim;
}

// The FP32 contracted quartet with two bra primitives per step in packed
// float pairs (FFMA2, f2.cuh): the same primitive quartets, cuts and sums as
// contracted_quartet<float>, but each Obara-Saika step of the generated
// recursion does the work of both primitives in one instruction.  An odd
// bra primitive count, or a second primitive below the cut, fills the upper
// half with the lower primitive at zero weight.
template <int L>
__device__ __forceinline__ void prim_setup_f2(const float4& blo0, const float4& blo1, const float4& bhi0,
                                              const float4& bhi1, float khi_weight, const float4& k0,
                                              const float4& k1, PrimGeo<F2>& g) {
  const F2 p(blo0.x, bhi0.x), q(k0.x);
  const F2 PQx = F2(blo1.x, bhi1.x) + F2(-k1.x), PQy = F2(blo1.y, bhi1.y) + F2(-k1.y),
           PQz = F2(blo1.z, bhi1.z) + F2(-k1.z);
  const F2 zeta = p + q;
  const F2 rs(rsqrtf(zeta.v.x), rsqrtf(zeta.v.y));
  const F2 oz = rs * rs;
  const F2 rho = p * q * oz;
  const F2 T = rho * pf_fma(PQx, PQx, pf_fma(PQy, PQy, PQz * PQz));
  const F2 pref = F2(blo0.z, bhi0.z * khi_weight) * F2(k0.z) * rs;
  F2 F[L + 1];
  boys_fp32x2<L>(T, F);
#pragma unroll
  for (int m = 0; m <= L; ++m) g.I[m] = pref * F[m];
  const F2 qz = q * oz, pz = p * oz;
  const F2 nqz = qz * F2(-1.0f);
  g.WP[0] = nqz * PQx; g.WP[1] = nqz * PQy; g.WP[2] = nqz * PQz;
  g.WQ[0] = pz * PQx;  g.WQ[1] = pz * PQy;  g.WQ[2] = pz * PQz;
  g.o2p = F2(blo0.y, bhi0.y);
  g.o2q = F2(k0.y);
  g.nrp = nqz;               // -rho / p
  g.nrq = pz * F2(-1.0f);    // -rho / q
  g.o2pq = F2(0.5f) * oz;
}

template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ int contracted_quartet_f2(const float4* __restrict__ prim, const float4* brec, int4 bi0,
                                                     int4 ki0, const double4& bgeo, const double4& kgeo,
                                                     float out[EriClass<float, LA, LB, LC, LD>::NOUT],
                                                     double kcut = 0.0, int kq0 = 0, int kq_step = 1) {
  using C2 = EriClass<F2, LA, LB, LC, LD>;
  using C1 = EriClass<float, LA, LB, LC, LD>;
  F2 acc[C2::NACC];
#pragma unroll
  for (int i = 0; i < C2::NACC; ++i) acc[i] = F2(0.0f);
  const float cut = (float)kcut;
  const float kab_max = fabsf(brec[0].z);
  int nprim = 0;
  for (int kq = kq0; kq < ki0.w; kq += kq_step) {
    const float4* kr = prim + 3 * (size_t)(ki0.z + kq);
    const float4 k0 = kr[0], k1 = kr[1], k2 = kr[2];
    const float kcd = fabsf(k0.z);
    if (kab_max * kcd < cut) break;
    const F2 QC[3] = {F2(k2.x), F2(k2.y), F2(k2.z)};
#pragma unroll 1
    for (int kp = 0; kp < bi0.w; kp += 2) {
      const float4* br = brec + 3 * kp;
      const float4 b0 = br[0], b1 = br[1], b2 = br[2];
      if (fabsf(b0.z) * kcd < cut) break;
      // the second primitive, or the first again at zero weight
      bool two = kp + 1 < bi0.w;
      float4 c0 = b0, c1 = b1, c2 = b2;
      if (two) {
        c0 = br[3];
        two = fabsf(c0.z) * kcd >= cut;
        if (two) {
          c1 = br[4];
          c2 = br[5];
        } else {
          c0 = b0;
        }
      }
      const F2 PA[3] = {F2(b2.x, c2.x), F2(b2.y, c2.y), F2(b2.z, c2.z)};
      PrimGeo<F2> g;
      prim_setup_f2<C2::L>(b0, b1, c0, c1, two ? 1.0f : 0.0f, k0, k1, g);
      C2::vrr(g.I, PA, g.WP, QC, g.WQ, g.o2p, g.nrp, g.o2q, g.nrq, g.o2pq, acc);
      nprim += two ? 2 : 1;
      if (!two) break;
    }
  }
  float accs[C1::NACC];
#pragma unroll
  for (int i = 0; i < C1::NACC; ++i) accs[i] = acc[i].v.x + acc[i].v.y;
  const float AB[3] = {(float)bgeo.x, (float)bgeo.y, (float)bgeo.z};
  const float CD[3] = {(float)kgeo.x, (float)kgeo.y, (float)kgeo.z};
  C1::hrr(accs, AB, CD, out);
  return nprim;
}

// Schwarz factor of every pair of one class: Q = sqrt(max |(ab|ab)|).
template <int LA, int LB>
__global__ void schwarz_kernel(int begin, int end, const int4* __restrict__ info0, const double4* __restrict__ geom,
                               const double4* __restrict__ prim, double* __restrict__ q) {
  int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= end) return;
  using C = EriClass<double, LA, LB, LA, LB>;
  double out[C::NOUT];
  const int4 i0 = info0[i];
  const double4 g = geom[i];
  contracted_quartet<double, LA, LB, LA, LB>(prim, prim + 3 * (size_t)i0.z, i0, i0, g, g, out);
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v;
  double mx = 0.0;
#pragma unroll
  for (int a = 0; a < NA; ++a)
#pragma unroll
    for (int b = 0; b < NB; ++b) mx = fmax(mx, fabs(out[((a * NB + b) * NA + a) * NB + b]));
  q[i] = sqrt(mx);
}

void launch_schwarz(const PairData& pd, int off[NCLASS + 1], double* q, cudaStream_t s, cudaStream_t side,
                    cudaEvent_t fork, cudaEvent_t join) {
  const bool two = side && fork && join;
  if (two) {
    PF_CUDA(cudaEventRecord(fork, s));
    PF_CUDA(cudaStreamWaitEvent(side, fork, 0));
  }
  for (int c = NCLASS - 1; c >= 0; --c) {  // the longest class first
    int n = off[c + 1] - off[c];
    if (n <= 0) continue;
    dim3 grid((n + 63) / 64), block(64);
    cudaStream_t st = (two && c == NCLASS - 1) ? side : s;
    if (c == 0) schwarz_kernel<0, 0><<<grid, block, 0, st>>>(off[c], off[c + 1], pd.info0, pd.geom, pd.prim, q);
    if (c == 1) schwarz_kernel<1, 0><<<grid, block, 0, st>>>(off[c], off[c + 1], pd.info0, pd.geom, pd.prim, q);
    if (c == 2) schwarz_kernel<1, 1><<<grid, block, 0, st>>>(off[c], off[c + 1], pd.info0, pd.geom, pd.prim, q);
    PF_CUDA(cudaGetLastError());
    count_launch();
  }
  if (two) {
    PF_CUDA(cudaEventRecord(join, side));
    PF_CUDA(cudaStreamWaitEvent(s, join, 0));
  }
}

// Sorted copy of the pair records; primitive pairs with |K| < cut are left
// out (their count was taken by build_pairs_kernel).
__global__ void gather_pairs_kernel(int npair, const int* __restrict__ perm, const int* __restrict__ new_ps,
                                    const int4* __restrict__ i0, const int4* __restrict__ i1,
                                    const int4* __restrict__ i2, const double4* __restrict__ g,
                                    const double4* __restrict__ pr, const double* __restrict__ q, double cut,
                                    int4* __restrict__ o0, int4* __restrict__ o1, int4* __restrict__ o2,
                                    double4* __restrict__ og, double4* __restrict__ opr,
                                    float4* __restrict__ oprf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npair) return;
  const int j = perm[i];
  int4 a = i0[j];
  const int old_ps = a.z, old_np = a.w;
  a.z = new_ps[i];
  // kept primitive pairs in order of decreasing |K| (so that a loop over
  // them can stop at a cut); pairs with more than 64 primitive pairs keep
  // the input order
  int order[64];
  int nk = 0;
  for (int k = 0; k < old_np; ++k)
    if (fabs(pr[3 * (size_t)(old_ps + k)].z) >= cut) {
      if (old_np <= 64) order[nk] = k;
      ++nk;
    }
  if (old_np <= 64) {
    for (int x = 1; x < nk; ++x) {
      const int v = order[x];
      const double kv = fabs(pr[3 * (size_t)(old_ps + v)].z);
      int y = x - 1;
      while (y >= 0 && fabs(pr[3 * (size_t)(old_ps + order[y])].z) < kv) {
        order[y + 1] = order[y];
        --y;
      }
      order[y + 1] = v;
    }
  }
  const int nkept = nk;
  nk = 0;
  for (int kk = 0; kk < (old_np <= 64 ? nkept : old_np); ++kk) {
    const int k = (old_np <= 64) ? order[kk] : kk;
    const double4* src = pr + 3 * (size_t)(old_ps + k);
    const double4 r0 = src[0];
    if (fabs(r0.z) < cut) continue;
    double4* dst = opr + 3 * (size_t)(a.z + nk);
    const double4 r1 = src[1], r2 = src[2];
    dst[0] = r0;
    dst[1] = r1;
    dst[2] = r2;
    if (oprf) {
      float4* df = oprf + 3 * (size_t)(a.z + nk);
      df[0] = make_float4((float)r0.x, (float)r0.y, (float)r0.z, (float)r0.w);
      df[1] = make_float4((float)r1.x, (float)r1.y, (float)r1.z, 0.0f);
      df[2] = make_float4((float)r2.x, (float)r2.y, (float)r2.z, 0.0f);
    }
    ++nk;
  }
  a.w = nk;
  o0[i] = a;
  o1[i] = i1[j];
  o2[i] = i2[j];
  double4 gg = g[j];
  gg.w = q[j];
  og[i] = gg;
}

void launch_gather_pairs(int npair, const int* perm, const int* new_pstart, const int4* i0, const int4* i1,
                         const int4* i2, const double4* g, const double4* pr, const double* q, double cut,
                         int4* o0, int4* o1, int4* o2, double4* og, double4* opr, float4* oprf, cudaStream_t s) {
  if (npair <= 0) return;
  gather_pairs_kernel<<<(npair + 127) / 128, 128, 0, s>>>(npair, perm, new_pstart, i0, i1, i2, g, pr, q, cut, o0,
                                                          o1, o2, og, opr, oprf);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ===========================================================================
// J/K digestion
// ===========================================================================
__device__ __forceinline__ int find_bra(const int* __restrict__ task_off, int nbra, int t) {
  int lo = 0, hi = nbra;  // task_off[lo] <= t < task_off[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(task_off + mid) <= t) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float dmax_bound(const float* __restrict__ dm, int ld, int a, int b, int c, int d) {
  float m = 2.0f * fmaxf(__ldg(dm + a * ld + b), __ldg(dm + c * ld + d));
  m = fmaxf(m, __ldg(dm + a * ld + c));
  m = fmaxf(m, __ldg(dm + a * ld + d));
  m = fmaxf(m, __ldg(dm + b * ld + c));
  m = fmaxf(m, __ldg(dm + b * ld + d));
  return m;
}

struct JkKernelArgs {
  JkArgs a;
  const int* ntasks_dev;
  const int4* info0;
  const int4* info1;
  const int4* info2;
  const double4* geom;
  const double4* prim;
  const float4* primf;
  const int* task_off;
  const int* ket_lo;
  const int* ket_hi;
  int nbra, ntasks, bra_base, ket_base, same_class, qclass, prec, task_begin;
  int lwidth;  // log2 of the task width: one warp runs 32 >> lwidth tasks of (1 bra) x (1 << lwidth kets)
  int psplit;  // warps per task (each takes every psplit-th ket primitive)
  int stage;   // primitive records staged per bra in shared memory (0: read from global memory)
};

// Warps per task for a list of the given length: lists with too few warps
// to fill the GPU (the (pp|pp) class: one quartet per lane and up to 81
// primitive quartets each) spread each task's ket primitives over up to 8
// warps; the grid is then even, so that 4-warp blocks keep groups whole.
static int primitive_split(long long warps, int num_sms) {
  int ps = 1;
  while (ps < 8 && warps * ps < (long long)num_sms * 32) ps *= 2;
  return ps;
}

// Whether any lane of this lane's aligned group of w lanes is active.
__device__ __forceinline__ bool active_any(unsigned mask, int lane, int w) {
  const unsigned gm = (w == 32) ? 0xffffffffu : (((1u << w) - 1u) << (lane & ~(w - 1)));
  return (mask & gm) != 0u;
}

// Sum over the aligned group of w lanes (w a power of two <= 32).
__device__ __forceinline__ double group_sum(double v, int w) {
  for (int o = w >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename R> __device__ __forceinline__ const typename Rec<R>::T* records(const JkKernelArgs& a);
template <> __device__ __forceinline__ const double4* records<double>(const JkKernelArgs& a) { return a.prim; }
template <> __device__ __forceinline__ const float4* records<float>(const JkKernelArgs& a) { return a.primf; }

template <typename R, int LA, int LB, int LC, int LD, int NK>
__global__ void __launch_bounds__(128) jk_kernel(const JkKernelArgs args) {
  using C = EriClass<R, LA, LB, LC, LD>;
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v, NCc = NC<LC>::v, ND = NC<LD>::v;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const JkArgs& A = args.a;
  const int ntasks = args.ntasks_dev ? *args.ntasks_dev : args.ntasks;
  const int lw = args.lwidth, W = 1 << lw, sub = lane & (W - 1), tpw = 32 >> lw;
  // (pp|pp) only: a task is shared by psplit consecutive warps, each summing
  // every psplit-th ket primitive and digesting its share (J and K are
  // linear in the integrals); the other classes compile with a unit stride
  constexpr bool kSplit = C::L == 4;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ps = kSplit ? args.psplit : 1, slice = kSplit ? gw % ps : 0;
  for (int tb = (gw / ps) * tpw; tb < ntasks; tb += (nw / ps) * tpw) {
    const int tl = tb + (lane >> lw);
    const bool valid = tl < ntasks;
    const int t = args.task_begin + (valid ? tl : ntasks - 1);
    const int ib = find_bra(args.task_off, args.nbra, t);
    const int ket = __ldg(args.ket_lo + ib) + (t - __ldg(args.task_off + ib)) * W + sub;
    const int bp = args.bra_base + ib;
    const int kp = args.ket_base + ket;
    bool active = valid && ket < __ldg(args.ket_hi + ib);
    const int4 bi0 = args.info0[bp], bi1 = args.info1[bp], bi2 = args.info2[bp];
    const double4 bg = args.geom[bp];
    int4 ki0 = bi0, ki1 = bi1;
    double4 kg = bg;
    double kcut = 0.0;
    if (active) {
      ki0 = args.info0[kp];
      ki1 = args.info1[kp];
      kg = args.geom[kp];
      if (A.dmax) {
        const float dm = dmax_bound(A.dmax + bi2.w, A.ns_ld, bi1.x, bi1.y, ki1.x, ki1.y);
        active = (float)(bg.w * kg.w) * dm >= (float)A.thresh;
        if (A.prim_thresh > 0.0) kcut = A.prim_thresh / fmax((double)dm, 1e-300);
      }
    }
    const unsigned amask = __ballot_sync(0xffffffffu, active);
    if (amask == 0u) continue;
    // the bra's primitive records, read by every primitive of every lane of
    // the group: staged once per task into this warp's shared-memory area
    // (one coalesced copy by the group's lanes) when the launch gave one
    using V = typename Rec<R>::T;
    const V* brec = records<R>(args) + 3 * (size_t)bi0.z;
    // FP32 kernels only: the FP64 ones read their bra records from L1
    // (staging measured 2% slower there, and its mere branch 2.5%)
    if (sizeof(R) == 4 && args.stage > 0) {
      extern __shared__ __align__(16) unsigned char jk_stage_smem[];
      V* st = reinterpret_cast<V*>(jk_stage_smem) +
              ((size_t)(threadIdx.x >> 5) * tpw + (lane >> lw)) * 3 * (size_t)args.stage;
      __syncwarp();
      for (int i = sub; i < 3 * bi0.w; i += W) st[i] = brec[i];
      __syncwarp();
      brec = st;
    }
    R out[C::NOUT];
    int nprim = 0;
    if (active) {
      // FP32 quartets: two primitives per step in packed pairs, except
      // (pp|pp), whose 81 packed accumulators would not fit the registers
      if constexpr (sizeof(R) == 4 && C::L < 4)
        nprim = contracted_quartet_f2<LA, LB, LC, LD>(args.primf, brec, bi0, ki0, bg, kg, out, kcut, slice, ps);
      else
        nprim = contracted_quartet<R, LA, LB, LC, LD>(records<R>(args), brec, bi0, ki0, bg, kg, out, kcut, slice, ps);
    } else {
#pragma unroll
      for (int i = 0; i < C::NOUT; ++i) out[i] = (R)0;
    }
    if (A.stats) {  // contracted and evaluated primitive quartets
      unsigned long long tot = (unsigned long long)nprim;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if (lane == 0) {
        if (slice == 0) atomicAdd(A.stats + args.prec * NQCLASS + args.qclass, (unsigned long long)__popc(amask));
        atomicAdd(A.stats + (2 + args.prec) * NQCLASS + args.qclass, tot);
      }
    }
    // degeneracy factor of the canonical quartet
    double fac = active ? 1.0 : 0.0;
    if (bi1.x == bi1.y) fac *= 0.5;
    if (ki1.x == ki1.y) fac *= 0.5;
    if (args.same_class && bp == kp) fac *= 0.5;
    const size_t mo = (size_t)bi2.x;
    const int ld = bi2.y;
    const int ma = bi0.x, mb = bi0.y, mc = ki0.x, md = ki0.y;
    // ---- Coulomb
    double Dab[NA * NB], Dcd[NCc * ND];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) Dab[a * NB + b] = __ldg(A.Dj + mo + (size_t)(ma + a) * ld + mb + b);
#pragma unroll
    for (int c = 0; c < NCc; ++c)
#pragma unroll
      for (int d = 0; d < ND; ++d)
        Dcd[c * ND + d] = active ? __ldg(A.Dj + mo + (size_t)(mc + c) * ld + md + d) : 0.0;
    double jab[NA * NB], jcd[NCc * ND];
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) jab[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NCc * ND; ++i) jcd[i] = 0.0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NCc; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const double v = fac * (double)out[((a * NB + b) * NCc + c) * ND + d];
            jab[a * NB + b] += v * Dcd[c * ND + d];
            jcd[c * ND + d] += v * Dab[a * NB + b];
          }
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) {
      const double s = group_sum(jab[i], W);
      if (sub == 0 && s != 0.0) atomicAdd(A.J + mo + (size_t)(ma + i / NB) * ld + mb + i % NB, 2.0 * s);
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < NCc; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) atomicAdd(A.J + mo + (size_t)(mc + c) * ld + md + d, 2.0 * jcd[c * ND + d]);
    }
    // ---- exchange, one or two densities
    if (active) {
#pragma unroll
      for (int k = 0; k < NK; ++k) {
        const double* Dk = (k == 0) ? A.Dk0 : A.Dk1;
        double* Kk = (k == 0) ? A.K0 : A.K1;
        double kac[NA * NCc], kad[NA * ND], kbc[NB * NCc], kbd[NB * ND];
#pragma unroll
        for (int i = 0; i < NA * NCc; ++i) kac[i] = 0.0;
#pragma unroll
        for (int i = 0; i < NA * ND; ++i) kad[i] = 0.0;
#pragma unroll
        for (int i = 0; i < NB * NCc; ++i) kbc[i] = 0.0;
#pragma unroll
        for (int i = 0; i < NB * ND; ++i) kbd[i] = 0.0;
        double Dbd[NB * ND], Dbc[NB * NCc], Dad[NA * ND], Dac[NA * NCc];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
#pragma unroll
          for (int d = 0; d < ND; ++d) Dbd[b * ND + d] = __ldg(Dk + mo + (size_t)(mb + b) * ld + md + d);
#pragma unroll
          for (int c = 0; c < NCc; ++c) Dbc[b * NCc + c] = __ldg(Dk + mo + (size_t)(mb + b) * ld + mc + c);
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) {
#pragma unroll
          for (int d = 0; d < ND; ++d) Dad[a * ND + d] = __ldg(Dk + mo + (size_t)(ma + a) * ld + md + d);
#pragma unroll
          for (int c = 0; c < NCc; ++c) Dac[a * NCc + c] = __ldg(Dk + mo + (size_t)(ma + a) * ld + mc + c);
        }
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int c = 0; c < NCc; ++c)
#pragma unroll
              for (int d = 0; d < ND; ++d) {
                const double v = fac * (double)out[((a * NB + b) * NCc + c) * ND + d];
                kac[a * NCc + c] += v * Dbd[b * ND + d];
                kad[a * ND + d] += v * Dbc[b * NCc + c];
                kbc[b * NCc + c] += v * Dad[a * ND + d];
                kbd[b * ND + d] += v * Dac[a * NCc + c];
              }
#pragma unroll
        for (int a = 0; a < NA; ++a) {
#pragma unroll
          for (int c = 0; c < NCc; ++c) atomicAdd(Kk + mo + (size_t)(ma + a) * ld + mc + c, kac[a * NCc + c]);
#pragma unroll
          for (int d = 0; d < ND; ++d) atomicAdd(Kk + mo + (size_t)(ma + a) * ld + md + d, kad[a * ND + d]);
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
#pragma unroll
          for (int c = 0; c < NCc; ++c) atomicAdd(Kk + mo + (size_t)(mb + b) * ld + mc + c, kbc[b * NCc + c]);
#pragma unroll
          for (int d = 0; d < ND; ++d) atomicAdd(Kk + mo + (size_t)(mb + b) * ld + md + d, kbd[b * ND + d]);
        }
      }
    }
  }
}

static int qclass_of(int bc, int kc) {
  // (ss|ss)=0 (ps|ss)=1 (ps|ps)=2 (pp|ss)=3 (pp|ps)=4 (pp|pp)=5
  static const int tab[3][3] = {{0, -1, -1}, {1, 2, -1}, {3, 4, 5}};
  return tab[bc][kc];
}

template <typename R, int LA, int LB, int LC, int LD>
static void jk_dispatch_nk(int nk, dim3 grid, dim3 block, size_t smem, cudaStream_t s, const JkKernelArgs& k) {
  if (nk == 1) jk_kernel<R, LA, LB, LC, LD, 1><<<grid, block, smem, s>>>(k);
  else jk_kernel<R, LA, LB, LC, LD, 2><<<grid, block, smem, s>>>(k);
}

template <typename R>
static void jk_dispatch(int qc, int nk, dim3 grid, dim3 block, size_t smem, cudaStream_t s, const JkKernelArgs& k) {
  switch (qc) {
    case 0: jk_dispatch_nk<R, 0, 0, 0, 0>(nk, grid, block, smem, s, k); break;
    case 1: jk_dispatch_nk<R, 1, 0, 0, 0>(nk, grid, block, smem, s, k); break;
    case 2: jk_dispatch_nk<R, 1, 0, 1, 0>(nk, grid, block, smem, s, k); break;
    case 3: jk_dispatch_nk<R, 1, 1, 0, 0>(nk, grid, block, smem, s, k); break;
    case 4: jk_dispatch_nk<R, 1, 1, 1, 0>(nk, grid, block, smem, s, k); break;
    default: jk_dispatch_nk<R, 1, 1, 1, 1>(nk, grid, block, smem, s, k); break;
  }
}

// Shared memory per 128-thread block for the staged bra records, above
// which a launch reads them from global memory instead (STO-6G pairs of 36
// primitive pairs with 8-wide tasks would take 55 KB and cost resident
// blocks).  Only the FP32 quartets stage: at C40H82 an all-FP32 build gains
// 3.5% (2.44 -> 2.35 ms), an FP64 build loses 2% (4.03 -> 4.11 ms), the
// FP64 kernels' bra records being L1 hits already.
constexpr size_t JK_STAGE_MAX_BYTES = 16 * 1024;

static int width_log2(int w) {
  if (w != 8 && w != 16 && w != 32) throw Error(PYFACC_ERR_INVALID, "task width must be 8, 16 or 32");
  return w == 8 ? 3 : (w == 16 ? 4 : 5);
}

// Blocks of four warps for a grid-stride loop over the tasks: at most 32
// per SM, of which 5-8 are resident at a time (registers); the rest queue
// and take the tail, so warps whose tasks cost more do not hold back the
// end (C40H82: FP64 step -2.2%, mixed -0.6% against 16 per SM; 8 per SM
// +3-4%, 128 per SM no better than 32)
static int grid_for(int ntasks, int num_sms) {
  long long warps_needed = ntasks;
  long long blocks = (warps_needed + 3) / 4;
  long long cap = (long long)num_sms * 32;
  return (int)std::max(1LL, std::min(blocks, cap));
}

void launch_jk(const PairData& pd, const TaskList& tl, int bc, int kc, bool fp32, int nk, const JkArgs& a,
               int num_sms, cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  JkKernelArgs k;
  k.a = a;
  k.ntasks_dev = tl.ntasks_dev;
  k.info0 = pd.info0; k.info1 = pd.info1; k.info2 = pd.info2;
  k.geom = pd.geom; k.prim = pd.prim; k.primf = pd.primf;
  if (fp32 && !pd.primf) throw Error(PYFACC_ERR_INVALID, "FP32 quartets need float primitive records");
  k.task_off = tl.task_off; k.ket_lo = tl.ket_lo; k.ket_hi = tl.ket_hi;
  k.nbra = tl.nbra; k.ntasks = tl.ntasks; k.task_begin = tl.task_begin;
  k.bra_base = pd.class_off[bc] + tl.bra_offset; k.ket_base = pd.class_off[kc];
  k.same_class = (bc == kc);
  k.qclass = qclass_of(bc, kc);
  k.prec = fp32 ? 1 : 0;
  k.lwidth = width_log2(tl.width);
  const long long warps = (tl.ntasks + (32 / tl.width) - 1) / (32 / tl.width);
  k.psplit = k.qclass == NQCLASS - 1 ? primitive_split(warps, num_sms) : 1;
  int nblk = grid_for((int)std::min<long long>(warps * k.psplit, 1LL << 30), num_sms);
  nblk = (nblk + 1) / 2 * 2;
  dim3 grid(nblk), block(128);
  const size_t rec = fp32 ? sizeof(float4) : sizeof(double4);
  const int tpw = 32 / tl.width;
  const size_t smem = (size_t)4 * tpw * 3 * rec * pd.class_maxprim[bc];
  k.stage = (fp32 && pd.class_maxprim[bc] > 0 && smem <= JK_STAGE_MAX_BYTES) ? pd.class_maxprim[bc] : 0;
  const size_t dyn = k.stage ? smem : 0;
  if (fp32) jk_dispatch<float>(k.qclass, nk, grid, block, dyn, s, k);
  else jk_dispatch<double>(k.qclass, nk, grid, block, dyn, s, k);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ---------------------------------------------------------------------------
// Task lists of one Fock build, built on the device (no host round trip).
// One block per list: per bra a ket prefix by binary search over the ket
// class's Q (descending), then a block-wide exclusive scan of the task counts.
// ---------------------------------------------------------------------------
__global__ void dmax_global_kernel(long long n, const float* __restrict__ dm, double* __restrict__ out) {
  __shared__ float sh[32];
  float m = 0.0f;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, dm[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = fmaxf(m, sh[k]);
    m = fmaxf(m, sh[0]);
    out[0] = (double)m;
  }
}

struct DynListArgs {
  int nbra, bra_base, ket_base, nket, same, part;  // part 0: FP64, 1: FP32
  int* task_off;
  int* ket_lo;
  int* ket_hi;
  int* ntasks;
};
struct DynAllArgs {
  DynListArgs l[2 * NQCLASS];
  const double4* geom;
  const double* dmax_global;
  double thresh, fp32_thresh;
  int width;
};

__device__ __forceinline__ int ket_prefix(const double4* __restrict__ geom, int ket_base, int nket, double qb, double t) {
  int lo = 0, hi = nket;  // count of j with qb * Q_j >= t, Q descending
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (qb * geom[ket_base + mid].w >= t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(1024) dyn_tasks_kernel(const DynAllArgs A) {
  const DynListArgs& L = A.l[blockIdx.x];
  __shared__ int wsum[32];
  __shared__ int carry;
  const double dm = fmax(A.dmax_global[0], 1e-300);
  const double t = A.thresh / dm, t64 = A.fp32_thresh / dm;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < L.nbra; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int cnt = 0;
    if (i < L.nbra) {
      const double qb = A.geom[L.bra_base + i].w;
      int m = ket_prefix(A.geom, L.ket_base, L.nket, qb, t);
      if (L.same) m = min(m, i + 1);
      const int m64 = min(ket_prefix(A.geom, L.ket_base, L.nket, qb, t64), m);
      const int lo = L.part == 0 ? 0 : m64, hi = L.part == 0 ? m64 : m;
      L.ket_lo[i] = lo;
      L.ket_hi[i] = hi;
      cnt = (hi - lo + A.width - 1) / A.width;
    }
    // block exclusive scan of cnt
    int v = cnt;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    if (w == 0) {
      int x = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      wsum[lane] = x;  // inclusive over warps
    }
    __syncthreads();
    const int excl = carry + (w > 0 ? wsum[w - 1] : 0) + v - cnt;
    if (i < L.nbra) L.task_off[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + cnt;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    L.task_off[L.nbra] = carry;
    L.ntasks[0] = carry;
  }
}

void launch_dyn_tasks(const PairData& pd, const float* dmax, int ns, double thresh, double fp32_thresh,
                      DynTaskSet& dt, cudaStream_t s) {
  dmax_global_kernel<<<1, 1024, 0, s>>>((long long)ns * ns, dmax, dt.dmax_global);
  PF_CUDA(cudaGetLastError());
  count_launch();
  DynAllArgs A;
  A.geom = pd.geom;
  A.dmax_global = dt.dmax_global;
  A.thresh = thresh;
  A.fp32_thresh = fp32_thresh;
  A.width = dt.lists[0].width;
  int k = 0;
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int qc = qclass_of(bc, kc);
      for (int part = 0; part < 2; ++part, ++k) {
        TaskList& tl = dt.lists[2 * qc + part];
        DynListArgs& L = A.l[2 * qc + part];
        L.nbra = tl.nbra;
        L.bra_base = pd.class_off[bc];
        L.ket_base = pd.class_off[kc];
        L.nket = pd.class_off[kc + 1] - pd.class_off[kc];
        L.same = bc == kc;
        L.part = part;
        L.task_off = tl.task_off;
        L.ket_lo = tl.ket_lo;
        L.ket_hi = tl.ket_hi;
        L.ntasks = dt.ntasks_dev + 2 * qc + part;
      }
    }
  dyn_tasks_kernel<<<2 * NQCLASS, 1024, 0, s>>>(A);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ===========================================================================
// Nuclear gradient, two-electron part
// ===========================================================================
struct GradKernelArgs {
  GradArgs a;
  const int4* info0;
  const int4* info1;
  const int4* info2;
  const double4* geom;
  const double4* prim;
  const float4* primf;
  const int* task_off;
  const int* ket_lo;
  const int* ket_hi;
  const int* ntasks_dev;  // device count of a list built on the GPU (else ntasks)
  int nbra, ntasks, bra_base, ket_base, same_class, qclass, task_begin;
  int lwidth;
  int smem_atoms;  // atoms summed in shared memory (0: global atomics)
  int psplit;      // warps per task: warp k of a group takes ket primitives k, k + psplit, ...
  int stage;       // FP32: bra primitive records staged per task in shared memory (0: global)
  int stage_off;   // byte offset of the staging area in the dynamic shared memory
};

template <typename R> __device__ __forceinline__ const typename Rec<R>::T* grecords(const GradKernelArgs& a);
template <> __device__ __forceinline__ const double4* grecords<double>(const GradKernelArgs& a) { return a.prim; }
template <> __device__ __forceinline__ const float4* grecords<float>(const GradKernelArgs& a) { return a.primf; }

template <typename R, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) grad2e_kernel(const GradKernelArgs args) {
  using C = EriClass<R, LA, LB, LC, LD>;
  using V = typename Rec<R>::T;
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v, NCc = NC<LC>::v, ND = NC<LD>::v;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const GradArgs& A = args.a;
  const int lw = args.lwidth, W = 1 << lw, sub = lane & (W - 1), tpw = 32 >> lw;
  // per-atom sums of the block in shared memory (one global add per atom
  // and block at the end) when the gradient is small enough
  extern __shared__ double gsh[];
  constexpr bool kGamSmem = C::L >= 4;
  const int nsm = args.smem_atoms * 3;
  for (int i = threadIdx.x; i < nsm; i += blockDim.x) gsh[i] = 0.0;
  if (nsm) __syncthreads();
  double* G = nsm ? gsh : A.grad;
  const int ntasks = args.ntasks_dev ? *args.ntasks_dev : args.ntasks;
  // a task is shared by psplit consecutive warps (the gradient is a sum over
  // primitive quartets, so each warp adds its share with the same atomics)
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ps = args.psplit, slice = gw % ps;
  for (int tb = (gw / ps) * tpw; tb < ntasks; tb += (nw / ps) * tpw) {
    const int tl = tb + (lane >> lw);
    const bool valid = tl < ntasks;
    const int t = args.task_begin + (valid ? tl : ntasks - 1);
    const int ib = find_bra(args.task_off, args.nbra, t);
    const int ket = __ldg(args.ket_lo + ib) + (t - __ldg(args.task_off + ib)) * W + sub;
    const int bp = args.bra_base + ib;
    const int kp = args.ket_base + ket;
    bool active = valid && ket < __ldg(args.ket_hi + ib);
    const int4 bi0 = args.info0[bp], bi1 = args.info1[bp], bi2 = args.info2[bp];
    const double4 bg = args.geom[bp];
    int4 ki0 = bi0, ki1 = bi1;
    double4 kg = bg;
    double kcut = 0.0;
    if (active) {
      ki0 = args.info0[kp];
      ki1 = args.info1[kp];
      kg = args.geom[kp];
      if (A.dmax) {
        const float dm = dmax_bound(A.dmax + bi2.w, A.ns_ld, bi1.x, bi1.y, ki1.x, ki1.y);
        active = (float)(bg.w * kg.w) * dm >= (float)A.thresh;
        if (A.prim_thresh > 0.0) kcut = A.prim_thresh / fmax((double)dm, 1e-300);
      }
    }
    const unsigned amask = __ballot_sync(0xffffffffu, active);
    if (amask == 0u) continue;
    // the bra's primitive records; FP32 kernels stage them once per task in
    // this warp's shared-memory area, as jk_kernel does
    const V* brec = grecords<R>(args) + 3 * (size_t)bi0.z;
    if (sizeof(R) == 4 && args.stage > 0) {
      V* st = reinterpret_cast<V*>(reinterpret_cast<unsigned char*>(gsh) + args.stage_off) +
              ((size_t)(threadIdx.x >> 5) * tpw + (lane >> lw)) * 3 * (size_t)args.stage;
      __syncwarp();
      for (int i = sub; i < 3 * bi0.w; i += W) st[i] = brec[i];
      __syncwarp();
      brec = st;
    }
    int nprim = 0;
    double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (active) {
      const size_t mo = (size_t)bi2.x;
      const int ld = bi2.y;
      const int ma = bi0.x, mb = bi0.y, mc = ki0.x, md = ki0.y;
      // the density products Gamma_abcd of the quartet
      auto fill_gam = [&](R* gam) {
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int c = 0; c < NCc; ++c)
#pragma unroll
              for (int d = 0; d < ND; ++d) {
                const size_t mu = ma + a, nu = mb + b, la = mc + c, si = md + d;
                const double* Pt = A.Pt + mo;
                double v = __ldg(Pt + mu * ld + nu) * __ldg(Pt + la * ld + si);
                if (A.uhf) {
                  const double* Pa = A.Pa + mo;
                  const double* Pb = A.Pb + mo;
                  v -= 0.5 * (__ldg(Pa + mu * ld + la) * __ldg(Pa + nu * ld + si) +
                              __ldg(Pa + mu * ld + si) * __ldg(Pa + nu * ld + la));
                  v -= 0.5 * (__ldg(Pb + mu * ld + la) * __ldg(Pb + nu * ld + si) +
                              __ldg(Pb + mu * ld + si) * __ldg(Pb + nu * ld + la));
                } else {
                  v -= 0.25 * (__ldg(Pt + mu * ld + la) * __ldg(Pt + nu * ld + si) +
                               __ldg(Pt + mu * ld + si) * __ldg(Pt + nu * ld + la));
                }
                gam[((a * NB + b) * NCc + c) * ND + d] = (R)v;
              }
      };
      const R AB[3] = {(R)bg.x, (R)bg.y, (R)bg.z};
      const R CD[3] = {(R)kg.x, (R)kg.y, (R)kg.z};
      R gr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const V* prim = grecords<R>(args);
      const R cut = (R)kcut;
      const R kab_max = fabs((R)brec[0].z);
      if constexpr (C::GCON) {
        // exponent-weighted sums over the primitive quartets, then one HRR
        // and one contraction with Gamma per contracted quartet
        R acc[C::NGACC];
#pragma unroll
        for (int i = 0; i < C::NGACC; ++i) acc[i] = (R)0;
#pragma unroll 1
        for (int kq = slice; kq < ki0.w; kq += ps) {
          const V* kr = prim + 3 * (size_t)(ki0.z + kq);
          const V k0 = kr[0], k1 = kr[1], k2 = kr[2];
          const R kcd = fabs((R)k0.z);
          if (kab_max * kcd < cut) break;
          const R QC[3] = {(R)k2.x, (R)k2.y, (R)k2.z};
          const R tc = (R)(2 * k0.w);
#pragma unroll 1
          for (int kpp = 0; kpp < bi0.w; ++kpp) {
            const V* br = brec + 3 * kpp;
            const V b0 = br[0], b1 = br[1], b2 = br[2];
            if (fabs((R)b0.z) * kcd < cut) break;
            ++nprim;
            const R PA[3] = {(R)b2.x, (R)b2.y, (R)b2.z};
            PrimGeo<R> pg;
            prim_setup<R, C::L + 1>(b0, b1, k0, k1, pg);
            C::gacc(pg.I, PA, pg.WP, QC, pg.WQ, pg.o2p, pg.nrp, pg.o2q, pg.nrq, pg.o2pq, (R)(2 * b0.w),
                    (R)(2 * (b0.x - b0.w)), tc, acc);
          }
        }
        if (nprim > 0) {
          R gam[C::NOUT];
          fill_gam(gam);
          C::gfin(acc, AB, CD, gam, gr);
        }
      } else {
        // the (pp|pp) derivative routines are compiled out of line and read
        // the density products through a pointer: for that class they live
        // in shared memory (after the per-atom sums) rather than in local
        // memory, which spilled to DRAM
        R gam_reg[kGamSmem ? 1 : C::NOUT];
        R* gam = kGamSmem ? reinterpret_cast<R*>(gsh + nsm) + (size_t)threadIdx.x * C::NOUT : gam_reg;
        fill_gam(gam);
#pragma unroll 1
        for (int kq = slice; kq < ki0.w; kq += ps) {
          const V* kr = prim + 3 * (size_t)(ki0.z + kq);
          const V k0 = kr[0], k1 = kr[1], k2 = kr[2];
          const R kcd = fabs((R)k0.z);
          if (kab_max * kcd < cut) break;
          const R QC[3] = {(R)k2.x, (R)k2.y, (R)k2.z};
#pragma unroll 1
          for (int kpp = 0; kpp < bi0.w; ++kpp) {
            const V* br = brec + 3 * kpp;
            const V b0 = br[0], b1 = br[1], b2 = br[2];
            if (fabs((R)b0.z) * kcd < cut) break;
            ++nprim;
            const R PA[3] = {(R)b2.x, (R)b2.y, (R)b2.z};
            PrimGeo<R> pg;
            prim_setup<R, C::L + 1>(b0, b1, k0, k1, pg);
            C::gradA(pg.I, PA, pg.WP, QC, pg.WQ, pg.o2p, pg.nrp, pg.o2q, pg.nrq, pg.o2pq, AB, CD, (R)(2 * b0.w), gam,
                     gr);
            C::gradB(pg.I, PA, pg.WP, QC, pg.WQ, pg.o2p, pg.nrp, pg.o2q, pg.nrq, pg.o2pq, AB, CD,
                     (R)(2 * (b0.x - b0.w)), gam, gr + 3);
            C::gradC(pg.I, PA, pg.WP, QC, pg.WQ, pg.o2p, pg.nrp, pg.o2q, pg.nrq, pg.o2pq, AB, CD, (R)(2 * k0.w), gam,
                     gr + 6);
          }
        }
      }
      double fac = 4.0;
      if (bi1.x == bi1.y) fac *= 0.5;
      if (ki1.x == ki1.y) fac *= 0.5;
      if (args.same_class && bp == kp) fac *= 0.5;
#pragma unroll
      for (int i = 0; i < 9; ++i) g[i] = fac * (double)gr[i];
    }
    if (A.stats) {  // contracted and evaluated primitive quartets
      unsigned long long tot = (unsigned long long)nprim;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if (lane == 0) {
        if (slice == 0) atomicAdd(A.stats + args.qclass, (unsigned long long)__popc(amask));
        atomicAdd(A.stats + NQCLASS + args.qclass, tot);
      }
    }
    // centre A and B are the bra's, uniform across a task's lanes
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double sa = group_sum(g[x], W);
      const double sb = group_sum(g[3 + x], W);
      if (sub == 0 && active_any(amask, lane, W)) {
        atomicAdd(G + 3 * bi1.z + x, sa);
        atomicAdd(G + 3 * bi1.w + x, sb);
      }
    }
    if (active) {
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(G + 3 * ki1.z + x, g[6 + x]);
        atomicAdd(G + 3 * ki1.w + x, -(g[x] + g[3 + x] + g[6 + x]));
      }
    }
  }
  if (nsm) {
    __syncthreads();
    for (int i = threadIdx.x; i < nsm; i += blockDim.x)
      if (gsh[i] != 0.0) atomicAdd(A.grad + i, gsh[i]);
  }
}

template <typename R, int LA, int LB, int LC, int LD>
static void grad2e_launch(dim3 grid, dim3 block, size_t smem, cudaStream_t s, const GradKernelArgs& k) {
  if (smem > 48 * 1024)
    PF_CUDA(cudaFuncSetAttribute(grad2e_kernel<R, LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  grad2e_kernel<R, LA, LB, LC, LD><<<grid, block, smem, s>>>(k);
}

template <typename R>
static void grad2e_dispatch(int qc, dim3 grid, dim3 block, size_t smem, cudaStream_t s, const GradKernelArgs& k) {
  switch (qc) {
    case 0: grad2e_launch<R, 0, 0, 0, 0>(grid, block, smem, s, k); break;
    case 1: grad2e_launch<R, 1, 0, 0, 0>(grid, block, smem, s, k); break;
    case 2: grad2e_launch<R, 1, 0, 1, 0>(grid, block, smem, s, k); break;
    case 3: grad2e_launch<R, 1, 1, 0, 0>(grid, block, smem, s, k); break;
    case 4: grad2e_launch<R, 1, 1, 1, 0>(grid, block, smem, s, k); break;
    default: grad2e_launch<R, 1, 1, 1, 1>(grid, block, smem, s, k); break;
  }
}

void launch_grad2e(const PairData& pd, const TaskList& tl, int bc, int kc, bool fp32, const GradArgs& a,
                   int num_sms, cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  GradKernelArgs k;
  k.a = a;
  k.info0 = pd.info0; k.info1 = pd.info1; k.info2 = pd.info2;
  k.geom = pd.geom; k.prim = pd.prim; k.primf = pd.primf;
  if (fp32 && !pd.primf) throw Error(PYFACC_ERR_INVALID, "FP32 quartets need float primitive records");
  k.task_off = tl.task_off; k.ket_lo = tl.ket_lo; k.ket_hi = tl.ket_hi;
  k.ntasks_dev = tl.ntasks_dev;
  k.nbra = tl.nbra; k.ntasks = tl.ntasks; k.task_begin = tl.task_begin;
  k.bra_base = pd.class_off[bc] + tl.bra_offset; k.ket_base = pd.class_off[kc];
  k.same_class = (bc == kc);
  k.qclass = qclass_of(bc, kc);
  k.lwidth = width_log2(tl.width);
  // up to 256 atoms (6 KB of per-block sums; above that the end-of-block
  // flush costs more than the contention it saves)
  k.smem_atoms = (a.natoms_total > 0 && a.natoms_total <= 256) ? a.natoms_total : 0;
  // the (pp|pp) kernels keep each thread's density products in shared memory
  const size_t gam_bytes = k.qclass == NQCLASS - 1 ? 128 * 81 * (fp32 ? sizeof(float) : sizeof(double)) : 0;
  const int tpw = 32 / tl.width;
  const size_t base = 3 * (size_t)k.smem_atoms * sizeof(double) + gam_bytes;
  const size_t stage_bytes = (size_t)4 * tpw * 3 * sizeof(float4) * pd.class_maxprim[bc];
  k.stage_off = (int)((base + 15) / 16 * 16);
  k.stage = (fp32 && pd.class_maxprim[bc] > 0 && stage_bytes <= JK_STAGE_MAX_BYTES) ? pd.class_maxprim[bc] : 0;
  const size_t smem = k.stage ? (size_t)k.stage_off + stage_bytes : base;
  const long long warps = (tl.ntasks + tpw - 1) / tpw;
  k.psplit = primitive_split(warps, num_sms);
  int nblk = grid_for((int)std::min<long long>(warps * k.psplit, 1LL << 30), num_sms);
  nblk = (nblk + 1) / 2 * 2;
  dim3 grid(nblk), block(128);
  if (fp32) grad2e_dispatch<float>(k.qclass, grid, block, smem, s, k);
  else grad2e_dispatch<double>(k.qclass, grid, block, smem, s, k);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ===========================================================================
// Full ERI tensor (small systems, tests): every canonical quartet writes its
// eight images.
// ===========================================================================
template <int LA, int LB, int LC, int LD>
__global__ void eri_tensor_kernel(const JkKernelArgs args, int n, double* __restrict__ eri) {
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v, NCc = NC<LC>::v, ND = NC<LD>::v;
  using C = EriClass<double, LA, LB, LC, LD>;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int lw = args.lwidth, tpw = 32 >> lw;
  for (int tb = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * tpw; tb < args.ntasks; tb += nw * tpw) {
    const int t = tb + (lane >> lw);
    if (t >= args.ntasks) continue;
    const int ib = find_bra(args.task_off, args.nbra, t);
    const int ket = args.ket_lo[ib] + (t - args.task_off[ib]) * (1 << lw) + (lane & ((1 << lw) - 1));
    if (ket >= args.ket_hi[ib]) continue;
    const int bp = args.bra_base + ib, kp = args.ket_base + ket;
    const int4 bi0 = args.info0[bp], ki0 = args.info0[kp];
    double out[C::NOUT];
    contracted_quartet<double, LA, LB, LC, LD>(args.prim, args.prim + 3 * (size_t)bi0.z, bi0, ki0, args.geom[bp],
                                               args.geom[kp], out);
    for (int a = 0; a < NA; ++a)
      for (int b = 0; b < NB; ++b)
        for (int c = 0; c < NCc; ++c)
          for (int d = 0; d < ND; ++d) {
            const size_t i = bi0.x + a, j = bi0.y + b, k = ki0.x + c, l = ki0.y + d;
            const double v = out[((a * NB + b) * NCc + c) * ND + d];
            const size_t N = n;
            eri[((i * N + j) * N + k) * N + l] = v;
            eri[((j * N + i) * N + k) * N + l] = v;
            eri[((i * N + j) * N + l) * N + k] = v;
            eri[((j * N + i) * N + l) * N + k] = v;
            eri[((k * N + l) * N + i) * N + j] = v;
            eri[((l * N + k) * N + i) * N + j] = v;
            eri[((k * N + l) * N + j) * N + i] = v;
            eri[((l * N + k) * N + j) * N + i] = v;
          }
  }
}

void launch_eri_tensor(const PairData& pd, const TaskList& tl, int bc, int kc, int nbf, double* eri,
                       cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  JkKernelArgs k{};
  k.psplit = 1;
  k.info0 = pd.info0; k.info1 = pd.info1; k.info2 = pd.info2;
  k.geom = pd.geom; k.prim = pd.prim;
  k.task_off = tl.task_off; k.ket_lo = tl.ket_lo; k.ket_hi = tl.ket_hi;
  k.nbra = tl.nbra; k.ntasks = tl.ntasks;
  k.bra_base = pd.class_off[bc]; k.ket_base = pd.class_off[kc];
  k.lwidth = width_log2(tl.width);
  dim3 grid((tl.ntasks + 3) / 4), block(128);
  switch (qclass_of(bc, kc)) {
    case 0: eri_tensor_kernel<0, 0, 0, 0><<<grid, block, 0, s>>>(k, nbf, eri); break;
    case 1: eri_tensor_kernel<1, 0, 0, 0><<<grid, block, 0, s>>>(k, nbf, eri); break;
    case 2: eri_tensor_kernel<1, 0, 1, 0><<<grid, block, 0, s>>>(k, nbf, eri); break;
    case 3: eri_tensor_kernel<1, 1, 0, 0><<<grid, block, 0, s>>>(k, nbf, eri); break;
    case 4: eri_tensor_kernel<1, 1, 1, 0><<<grid, block, 0, s>>>(k, nbf, eri); break;
    default: eri_tensor_kernel<1, 1, 1, 1><<<grid, block, 0, s>>>(k, nbf, eri); break;
  }
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ===========================================================================
// One-electron integrals and their gradient.
// Overlap by the 1-D Obara-Saika recursion of overlap.f90:121-145, kinetic
// energy by the directional formula of kinetic.f90:20-54 on the same 1-D
// overlaps, nuclear attraction by the OS recursion of the generated
// NucClass (the Cook/THO sum of nuclear.f90:66-136 in recursive form).
// One warp per shell pair of one class (l_a >= l_b); the lanes share the
// (primitive pair, nucleus) work; primitive pairs whose prefactor is below
// 1e-17 are skipped.
// ===========================================================================
template <int NI, int NJ>
__device__ __forceinline__ void ovl1d(double s00, double PA, double PB, double o2p, double (&S)[NI][NJ]) {
#pragma unroll
  for (int i = 0; i < NI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      double v;
      if (i == 0 && j == 0) v = s00;
      else if (i > 0) {
        v = PA * S[i - 1][j];
        if (i > 1) v += (i - 1) * o2p * S[i - 2][j];
        if (j > 0) v += j * o2p * S[i - 1][j - 1];
      } else {
        v = PB * S[i][j - 1];
        if (j > 1) v += (j - 1) * o2p * S[i][j - 2];
      }
      S[i][j] = v;
    }
}

__device__ __forceinline__ void cart_comp(int l, int k, int* c) {
  // x descending, then y (cartesian.f90:7-23), l <= 2
  if (l == 0) { c[0] = c[1] = c[2] = 0; return; }
  if (l == 1) { c[0] = (k == 0); c[1] = (k == 1); c[2] = (k == 2); return; }
  // xx, xy, xz, yy, yz, zz
  const int tab[6][3] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};
  c[0] = tab[k][0]; c[1] = tab[k][1]; c[2] = tab[k][2];
}

// S_ab and T_ab of unnormalised Cartesian components a, b from 1-D tables
// (the Gaussian prefactor is carried by the tables).
template <int NI, int NJ>
__device__ __forceinline__ double ovl3(const double (&S)[3][NI][NJ], const int* a, const int* b) {
  if (a[0] < 0 || a[1] < 0 || a[2] < 0 || b[0] < 0 || b[1] < 0 || b[2] < 0) return 0.0;
  return S[0][a[0]][b[0]] * S[1][a[1]][b[1]] * S[2][a[2]][b[2]];
}
template <int NI, int NJ>
__device__ __forceinline__ double kin3(const double (&S)[3][NI][NJ], const int* a, const int* b, double al,
                                       double be) {
  if (a[0] < 0 || a[1] < 0 || a[2] < 0 || b[0] < 0 || b[1] < 0 || b[2] < 0) return 0.0;
  double t = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int x = a[d], y = b[d];
    double k = 4.0 * al * be * S[d][x + 1][y + 1];
    if (y > 0) k -= 2.0 * al * y * S[d][x + 1][y - 1];
    if (x > 0) k -= 2.0 * be * x * S[d][x - 1][y + 1];
    if (x > 0 && y > 0) k += x * y * S[d][x - 1][y - 1];
    t += 0.5 * k * S[(d + 1) % 3][a[(d + 1) % 3]][b[(d + 1) % 3]] * S[(d + 2) % 3][a[(d + 2) % 3]][b[(d + 2) % 3]];
  }
  return t;
}

struct Prim1e {
  double al, be, p, o2p, w;  // w = c_a c_b N_a N_b exp(-al be/p |AB|^2)
  double P[3], PA[3], PB[3];
};
// primitive pairs of a shell pair kept in shared memory by grad1e_kernel
// (STO-6G: 36); shell pairs with more set them up per nucleus
constexpr int GRAD1E_MAXPP = 36;

// normalize = false: the coefficients multiply unnormalised primitives
__device__ __forceinline__ void prim1e_setup(double al, double ca, int la, double be, double cb, int lb,
                                             const double4& A, const double4& B, Prim1e& g, bool normalize = true) {
  g.al = al; g.be = be; g.p = al + be; g.o2p = 0.5 / g.p;
  const double A3[3] = {A.x, A.y, A.z}, B3[3] = {B.x, B.y, B.z};
  double ab2 = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    g.P[x] = (al * A3[x] + be * B3[x]) / g.p;
    g.PA[x] = g.P[x] - A3[x];
    g.PB[x] = g.P[x] - B3[x];
    ab2 += (A3[x] - B3[x]) * (A3[x] - B3[x]);
  }
  g.w = ca * cb * (normalize ? prim_norm(la, al) * prim_norm(lb, be) : 1.0) * exp(-al * be / g.p * ab2);
}

// 1-D overlap tables of one primitive pair: (pi/p)^{3/2} w carried by z.
template <int NI, int NJ>
__device__ __forceinline__ void st_tables(const Prim1e& g, double (&S)[3][NI][NJ]) {
  const double pre = g.w * pow(3.14159265358979323846 / g.p, 1.5);
  ovl1d<NI, NJ>(1.0, g.PA[0], g.PB[0], g.o2p, S[0]);
  ovl1d<NI, NJ>(1.0, g.PA[1], g.PB[1], g.o2p, S[1]);
  ovl1d<NI, NJ>(pre, g.PA[2], g.PB[2], g.o2p, S[2]);
}

template <int LA, int LB>
__global__ void __launch_bounds__(128) one_electron_kernel(int npair, const int2* __restrict__ pairs,
                                                           const double4* __restrict__ cen,
                                                           const int4* __restrict__ desc, const int* __restrict__ nprim,
                                                           const double* __restrict__ ex,
                                                           const double* __restrict__ co,
                                                           const int4* __restrict__ mol, OneEArgs args) {
  using NCl = NucClass<double, LA, LB>;
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v;
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= npair) return;
  const int2 pr = pairs[w];
  // the molecule of the pair: its nuclei and its matrix block
  const int4 mi = mol ? mol[pr.x] : make_int4(0, args.natoms, 0, args.nbf);
  const double4* atoms = args.atoms + mi.x;
  const int natoms = mi.y;
  const int4 da = desc[pr.x], db = desc[pr.y];
  const int na = nprim[pr.x], nb = nprim[pr.y];
  const double4 A = cen[pr.x], B = cen[pr.y];
  const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
  double s[NA * NB], t[NA * NB], v[NA * NB];
#pragma unroll
  for (int i = 0; i < NA * NB; ++i) s[i] = t[i] = v[i] = 0.0;
  // lpp lanes share one primitive pair (its Gaussian product is set up once)
  // and split the nuclei between them
  const int npp = na * nb;
  const int lpp = npp >= 32 ? 1 : 32 / npp;
  const int sub = lane % lpp;
  for (int pp = lane / lpp; pp < npp; pp += 32 / lpp) {
    const int ka = pp / nb, kb = pp % nb;
    Prim1e g;
    prim1e_setup(ex[da.w + ka], co[da.w + ka], LA, ex[db.w + kb], co[db.w + kb], LB, A, B, g);
    if (fabs(g.w) * 6.2831853071795864769 / g.p < 1e-17) continue;
    if (sub == 0) {
      double S[3][LA + 2][LB + 2];
      st_tables<LA + 2, LB + 2>(g, S);
#pragma unroll
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
          int ca[3], cb[3];
          cart_comp(LA, ia, ca);
          cart_comp(LB, ib, cb);
          s[ia * NB + ib] += ovl3(S, ca, cb);
          t[ia * NB + ib] += kin3(S, ca, cb, g.al, g.be);
        }
    }
    const double wp = g.w * 6.2831853071795864769 / g.p;
    for (int c = sub; c < natoms; c += lpp) {
      const double4 Cn = atoms[c];
      const double PC[3] = {g.P[0] - Cn.x, g.P[1] - Cn.y, g.P[2] - Cn.z};
      double F[PF_BOYS_MMAX + 1];
      boys_runtime(args.boys_mode, LA + LB, g.p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
      const double pref = -Cn.w * wp;
      double I[LA + LB + 1];
#pragma unroll
      for (int m = 0; m <= LA + LB; ++m) I[m] = pref * F[m];
      NCl::vint(I, g.PA, PC, g.o2p, AB, v);
    }
  }
#pragma unroll
  for (int i = 0; i < NA * NB; ++i) {
    s[i] = warp_sum(s[i]);
    t[i] = warp_sum(t[i]);
    v[i] = warp_sum(v[i]);
  }
  if (lane == 0) {
    const size_t n = mi.w, mo = mi.z;
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        const size_t mu = da.z + ia, nu = db.z + ib;
        const int k = ia * NB + ib;
        const double r = comp_ratio(LA, ia) * comp_ratio(LB, ib);
        if (args.S) { args.S[mo + mu * n + nu] = r * s[k]; args.S[mo + nu * n + mu] = r * s[k]; }
        if (args.T) { args.T[mo + mu * n + nu] = r * t[k]; args.T[mo + nu * n + mu] = r * t[k]; }
        if (args.V) { args.V[mo + mu * n + nu] = r * v[k]; args.V[mo + nu * n + mu] = r * v[k]; }
      }
  }
}

template <int LA, int LB>
static void one_electron_launch(int n, const int2* pairs, const ShellDev& sh, const OneEArgs& a, cudaStream_t s) {
  one_electron_kernel<LA, LB><<<(n + 3) / 4, 128, 0, s>>>(n, pairs, sh.cen, sh.desc, sh.nprim, sh.ex, sh.co, sh.mol, a);
}

// pairs[c] for the pair classes c = ss, ps, pp, ds, dp, dd (l_a >= l_b);
// molecules without d shells have the last three empty
void launch_one_electron(const ShellDev& sh, const int* npair, const int2* const* pairs, const OneEArgs& a,
                         cudaStream_t s) {
  for (int c = 0; c < NPAIRCLASS; ++c) {
    if (npair[c] <= 0) continue;
    switch (c) {
      case 0: one_electron_launch<0, 0>(npair[c], pairs[c], sh, a, s); break;
      case 1: one_electron_launch<1, 0>(npair[c], pairs[c], sh, a, s); break;
      case 2: one_electron_launch<1, 1>(npair[c], pairs[c], sh, a, s); break;
      case 3: one_electron_launch<2, 0>(npair[c], pairs[c], sh, a, s); break;
      case 4: one_electron_launch<2, 1>(npair[c], pairs[c], sh, a, s); break;
      default: one_electron_launch<2, 2>(npair[c], pairs[c], sh, a, s); break;
    }
    PF_CUDA(cudaGetLastError());
    count_launch();
  }
}

// ---------------------------------------------------------------------------
// One-body integrals of a single shell pair with caller-given contraction
// coefficients, for the libint_*_c entry points (the reference's unused
// Libint one-body wrapper, src/cpp/libint_wrapper.cpp:16-327): the
// coefficients multiply unnormalised Cartesian primitives x^i y^j z^k
// exp(-a r^2) as given, and the potential is that of a unit positive
// charge at C, int phi_a phi_b / |r - C| (Libint's elecpot sign).  One warp;
// its lanes take the primitive pairs.  la >= lb; a transposed request
// writes out[ib * NA + ia].
// ---------------------------------------------------------------------------
struct Libint1eArgs {
  int kind;  // 0 overlap, 1 kinetic, 2 potential
  int na, nb, transpose;
  double A[3], B[3], C[3];
  double ea[LIBINT1E_MAX_PRIM], ca[LIBINT1E_MAX_PRIM], eb[LIBINT1E_MAX_PRIM], cb[LIBINT1E_MAX_PRIM];
};

static __device__ double g_libint1e_out[36];  // up to 6 x 6 components (d|d)

template <int LA, int LB>
__global__ void __launch_bounds__(32) libint_1e_kernel(const Libint1eArgs a) {
  using NCl = NucClass<double, LA, LB>;
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v;
  const int lane = threadIdx.x & 31;
  const double4 A = make_double4(a.A[0], a.A[1], a.A[2], 0.0), B = make_double4(a.B[0], a.B[1], a.B[2], 0.0);
  const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
  double acc[NA * NB];
#pragma unroll
  for (int i = 0; i < NA * NB; ++i) acc[i] = 0.0;
  for (int pp = lane; pp < a.na * a.nb; pp += 32) {
    const int ka = pp / a.nb, kb = pp % a.nb;
    Prim1e g;
    prim1e_setup(a.ea[ka], a.ca[ka], LA, a.eb[kb], a.cb[kb], LB, A, B, g, false);
    if (a.kind < 2) {
      double S[3][LA + 2][LB + 2];
      st_tables<LA + 2, LB + 2>(g, S);
#pragma unroll
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
          int c1[3], c2[3];
          cart_comp(LA, ia, c1);
          cart_comp(LB, ib, c2);
          acc[ia * NB + ib] += a.kind == 0 ? ovl3(S, c1, c2) : kin3(S, c1, c2, g.al, g.be);
        }
    } else {
      const double PC[3] = {g.P[0] - a.C[0], g.P[1] - a.C[1], g.P[2] - a.C[2]};
      double F[PF_BOYS_MMAX + 1];
      boys_runtime(0, LA + LB, g.p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
      const double pref = g.w * 6.2831853071795864769 / g.p;
      double I[LA + LB + 1];
#pragma unroll
      for (int m = 0; m <= LA + LB; ++m) I[m] = pref * F[m];
      NCl::vint(I, g.PA, PC, g.o2p, AB, acc);
    }
  }
#pragma unroll
  for (int i = 0; i < NA * NB; ++i) acc[i] = warp_sum(acc[i]);
  if (lane == 0)
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib)
        g_libint1e_out[a.transpose ? ib * NA + ia : ia * NB + ib] = acc[ia * NB + ib];
}

void libint_one_body(int kind, int la, int na, const double* A, const double* ea, const double* ca, int lb, int nb,
                     const double* B, const double* eb, const double* cb, const double* C, double* out) {
  if (kind < 0 || kind > 2) throw Error(PYFACC_ERR_INVALID, "unknown one-body integral kind");
  if (la < 0 || lb < 0 || la > 2 || lb > 2)
    throw Error(PYFACC_ERR_UNSUPPORTED_L, "one-body shell pairs up to d (l <= 2)");
  if (na <= 0 || nb <= 0 || na > LIBINT1E_MAX_PRIM || nb > LIBINT1E_MAX_PRIM)
    throw Error(PYFACC_ERR_INVALID, "contraction depth must be 1.." + std::to_string(LIBINT1E_MAX_PRIM));
  if (!A || !B || !ea || !ca || !eb || !cb || !out || (kind == 2 && !C))
    throw Error(PYFACC_ERR_INVALID, "null argument");
  int device = 0;
  PF_CUDA(cudaGetDevice(&device));
  ensure_boys_tables(device);
  // the kernel's class has l_a >= l_b; a (lower | higher) request is the
  // transposed (higher | lower) one
  const bool swap = la < lb;
  Libint1eArgs a{};
  a.kind = kind;
  a.transpose = swap ? 1 : 0;
  a.na = swap ? nb : na;
  a.nb = swap ? na : nb;
  for (int x = 0; x < 3; ++x) {
    a.A[x] = swap ? B[x] : A[x];
    a.B[x] = swap ? A[x] : B[x];
    a.C[x] = kind == 2 ? C[x] : 0.0;
  }
  for (int k = 0; k < a.na; ++k) {
    a.ea[k] = swap ? eb[k] : ea[k];
    a.ca[k] = swap ? cb[k] : ca[k];
  }
  for (int k = 0; k < a.nb; ++k) {
    a.eb[k] = swap ? ea[k] : eb[k];
    a.cb[k] = swap ? ca[k] : cb[k];
  }
  const int L1 = swap ? lb : la, L2 = swap ? la : lb;
  // calls share the 36-double result array on the device: one at a time
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  switch (L1 * 3 + L2) {
    case 0: libint_1e_kernel<0, 0><<<1, 32>>>(a); break;
    case 3: libint_1e_kernel<1, 0><<<1, 32>>>(a); break;
    case 4: libint_1e_kernel<1, 1><<<1, 32>>>(a); break;
    case 6: libint_1e_kernel<2, 0><<<1, 32>>>(a); break;
    case 7: libint_1e_kernel<2, 1><<<1, 32>>>(a); break;
    default: libint_1e_kernel<2, 2><<<1, 32>>>(a); break;
  }
  PF_CUDA(cudaGetLastError());
  count_launch();
  const int n = ((la + 1) * (la + 2) / 2) * ((lb + 1) * (lb + 2) / 2);
  PF_CUDA(cudaMemcpyFromSymbol(out, g_libint1e_out, n * sizeof(double)));
}

// Gradient of the one-electron energy: sum P (dT + dV) - sum W dS over the
// pairs of one class; d/dB = -d/dA for the two-centre S and T, and
// d/dC V^C = -(d/dA + d/dB) V^C for every nucleus C.  Each lane owns a set
// of nuclei; the nuclear (C) terms go to a shared-memory gradient that the
// block adds to the global one at the end.
template <int LA, int LB>
__global__ void __launch_bounds__(128) grad1e_kernel(int npair, const int2* __restrict__ pairs,
                                                     const double4* __restrict__ cen, const int4* __restrict__ desc,
                                                     const int* __restrict__ nprim, const double* __restrict__ ex,
                                                     const double* __restrict__ co,
                                                     const int4* __restrict__ mol, int use_smem,
                                                     OneEGradArgs args) {
  using NCl = NucClass<double, LA, LB>;
  constexpr int NA = NC<LA>::v, NB = NC<LB>::v;
  extern __shared__ double gsh[];  // 3 * natoms_total when use_smem
  if (use_smem) {
    for (int i = threadIdx.x; i < 3 * args.natoms_total; i += blockDim.x) gsh[i] = 0.0;
    __syncthreads();
  }
  double* gacc = use_smem ? gsh : args.grad;  // per-atom accumulator (shared or global)
  __shared__ Prim1e g1e_pp[4][GRAD1E_MAXPP];  // per warp: the current shell pair's primitive pairs
  const int lane = threadIdx.x & 31;
  const int nwarp_total = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < npair; w += nwarp_total) {
    const int2 pr = pairs[w];
    const int4 mi = mol ? mol[pr.x] : make_int4(0, args.natoms, 0, args.nbf);
    const size_t n = mi.w, mo = mi.z;
    const int4 da = desc[pr.x], db = desc[pr.y];
    const int na = nprim[pr.x], nb = nprim[pr.y];
    const double4 A = cen[pr.x], B = cen[pr.y];
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const double wgt = (pr.x == pr.y) ? 1.0 : 2.0;
    double Pd[NA * NB], Wd[NA * NB];
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        const size_t k = mo + (size_t)(da.z + ia) * n + db.z + ib;
        const double r = comp_ratio(LA, ia) * comp_ratio(LB, ib);
        Pd[ia * NB + ib] = wgt * r * args.P[k];
        Wd[ia * NB + ib] = wgt * r * args.W[k];
      }
    double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
    const int npp = na * nb;
    // the primitive pairs' Gaussian products are set up once (kinetic and
    // overlap loop) and kept in this warp's shared memory for the nuclear
    // attraction loop, where every lane needs all of them
    const bool cached = npp <= GRAD1E_MAXPP;
    Prim1e* gpp = g1e_pp[threadIdx.x >> 5];
    __syncwarp();
    // kinetic and overlap: lanes over primitive pairs
    for (int pp = lane; pp < npp; pp += 32) {
      const int ka = pp / nb, kb = pp % nb;
      Prim1e g;
      prim1e_setup(ex[da.w + ka], co[da.w + ka], LA, ex[db.w + kb], co[db.w + kb], LB, A, B, g);
      if (cached) gpp[pp] = g;
      if (fabs(g.w) * 6.2831853071795864769 / g.p < 1e-17) continue;
      double S[3][LA + 3][LB + 2];
      st_tables<LA + 3, LB + 2>(g, S);
#pragma unroll
      for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
          int ca[3], cb[3];
          cart_comp(LA, ia, ca);
          cart_comp(LB, ib, cb);
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            int up[3] = {ca[0], ca[1], ca[2]}, dn[3] = {ca[0], ca[1], ca[2]};
            up[x] += 1;
            dn[x] -= 1;
            double ds = 2.0 * g.al * ovl3(S, up, cb);
            double dt = 2.0 * g.al * kin3(S, up, cb, g.al, g.be);
            if (ca[x] > 0) {
              ds -= ca[x] * ovl3(S, dn, cb);
              dt -= ca[x] * kin3(S, dn, cb, g.al, g.be);
            }
            const double d = Pd[ia * NB + ib] * dt - Wd[ia * NB + ib] * ds;
            gA[x] += d;
            gB[x] -= d;
          }
        }
    }
    __syncwarp();
    // nuclear attraction: lanes over nuclei, all primitive pairs each
    for (int c = lane; c < mi.y; c += 32) {
      const double4 Cn = args.atoms[mi.x + c];
      double gv[6] = {0, 0, 0, 0, 0, 0};
      for (int pp = 0; pp < npp; ++pp) {
        const int ka = pp / nb, kb = pp % nb;
        Prim1e g;
        if (cached) g = gpp[pp];
        else prim1e_setup(ex[da.w + ka], co[da.w + ka], LA, ex[db.w + kb], co[db.w + kb], LB, A, B, g);
        if (fabs(g.w) * 6.2831853071795864769 / g.p < 1e-17) continue;
        const double PC[3] = {g.P[0] - Cn.x, g.P[1] - Cn.y, g.P[2] - Cn.z};
        double F[PF_BOYS_MMAX + 1];
        boys_runtime(args.boys_mode, LA + LB + 1, g.p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
        const double pref = -Cn.w * g.w * 6.2831853071795864769 / g.p;
        double I[LA + LB + 2];
#pragma unroll
        for (int m = 0; m <= LA + LB + 1; ++m) I[m] = pref * F[m];
        const double tw[2] = {2.0 * g.al, 2.0 * g.be};
        NCl::vgrad(I, g.PA, PC, g.o2p, AB, tw, Pd, gv);
      }
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        gA[x] += gv[x];
        gB[x] += gv[3 + x];
        atomicAdd(gacc + 3 * (mi.x + c) + x, -(gv[x] + gv[3 + x]));
      }
    }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double sa = warp_sum(gA[x]), sb = warp_sum(gB[x]);
      if (lane == 0) {
        atomicAdd(gacc + 3 * da.y + x, sa);
        atomicAdd(gacc + 3 * db.y + x, sb);
      }
    }
  }
  if (!use_smem) return;
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * args.natoms_total; i += blockDim.x)
    if (gsh[i] != 0.0) atomicAdd(args.grad + i, gsh[i]);
}

template <int LA, int LB>
static void grad1e_launch(int blocks, size_t smem, int use_smem, int n, const int2* pairs, const ShellDev& sh,
                          const OneEGradArgs& a, cudaStream_t s) {
  PF_CUDA(cudaFuncSetAttribute(grad1e_kernel<LA, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  grad1e_kernel<LA, LB><<<blocks, 128, smem, s>>>(n, pairs, sh.cen, sh.desc, sh.nprim, sh.ex, sh.co, sh.mol, use_smem,
                                                  a);
}

void launch_grad1e(const ShellDev& sh, const int* npair, const int2* const* pairs, const OneEGradArgs& a,
                   int num_sms, cudaStream_t s) {
  // per-atom partial sums in shared memory while they fit (one molecule),
  // straight global atomics for the many atoms of a batch
  const size_t need = 3 * (size_t)a.natoms_total * sizeof(double);
  const int use_smem = need <= 96 * 1024;
  const size_t smem = use_smem ? need : 0;
  for (int c = 0; c < NPAIRCLASS; ++c) {
    if (npair[c] <= 0) continue;
    // one warp per pair; with global atomics up to 16 blocks per SM (a batch's
    // many pairs), with per-block sums 4 (each block flushes 3 natoms sums)
    const int blocks = std::max(1, std::min((npair[c] + 3) / 4, (use_smem ? 4 : 16) * num_sms));
    switch (c) {
      case 0: grad1e_launch<0, 0>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
      case 1: grad1e_launch<1, 0>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
      case 2: grad1e_launch<1, 1>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
      case 3: grad1e_launch<2, 0>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
      case 4: grad1e_launch<2, 1>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
      default: grad1e_launch<2, 2>(blocks, smem, use_smem, npair[c], pairs[c], sh, a, s); break;
    }
    PF_CUDA(cudaGetLastError());
    count_launch();
  }
}

// ===========================================================================
// Dense helpers
// ===========================================================================
__global__ void symmetrize_add_kernel(int n, double* A) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || j > i) return;
  const double s = A[(size_t)i * n + j] + A[(size_t)j * n + i];
  A[(size_t)i * n + j] = s;
  A[(size_t)j * n + i] = s;
}
// A = diag(f d) (n x n)
__global__ void set_diag_kernel(long long n2, int n, const double* __restrict__ d, double f, double* __restrict__ A) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2; k += (long long)gridDim.x * blockDim.x)
    A[k] = (k % (n + 1) == 0) ? f * d[k / (n + 1)] : 0.0;
}
void launch_set_diag(int n, const double* d, double f, double* A, cudaStream_t s) {
  const long long n2 = (long long)n * n;
  const int g = (int)std::min<long long>((n2 + 255) / 256, 2048);
  set_diag_kernel<<<std::max(g, 1), 256, 0, s>>>(n2, n, d, f, A);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// out = min_i L_ii^2 (one block; NaN pivots propagate as NaN)
__global__ void min_diag_sq_kernel(int n, const double* __restrict__ L, double* __restrict__ out) {
  __shared__ double part[32];
  double m = 1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = L[(size_t)i * n + i] * L[(size_t)i * n + i];
    m = (v < m || v != v) ? v : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(0xffffffffu, m, o);
    m = (y < m || y != y) ? y : m;
  }
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = (part[w] < m || part[w] != part[w]) ? part[w] : m;
    *out = m;
  }
}
void launch_min_diag_sq(int n, const double* L, double* out, cudaStream_t s) {
  min_diag_sq_kernel<<<1, 256, 0, s>>>(n, L, out);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

__global__ void identity_kernel(long long n2, int n, double* A) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2; k += (long long)gridDim.x * blockDim.x)
    A[k] = (k % (n + 1) == 0) ? 1.0 : 0.0;
}
void launch_identity(int n, double* A, cudaStream_t s) {
  const long long n2 = (long long)n * n;
  const int g = (int)std::min<long long>((n2 + 255) / 256, 2048);
  identity_kernel<<<std::max(g, 1), 256, 0, s>>>(n2, n, A);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_symmetrize_add(int n, double* A, cudaStream_t s) {
  dim3 b(32, 8), g((n + 31) / 32, (n + 7) / 8);
  symmetrize_add_kernel<<<g, b, 0, s>>>(n, A);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// E = B - B^T (the commutator F'P' - P'F' from B = F'P' with F', P' symmetric)
__global__ void antisym_kernel(int n, const double* __restrict__ B, double* __restrict__ E) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || j >= n) return;
  E[(size_t)i * n + j] = B[(size_t)i * n + j] - B[(size_t)j * n + i];
}
void launch_antisym(int n, const double* B, double* E, cudaStream_t s) {
  dim3 b(32, 8), g((n + 31) / 32, (n + 7) / 8);
  antisym_kernel<<<g, b, 0, s>>>(n, B, E);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

__global__ void axpby_kernel(long long n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}
void launch_axpby(long long n, double a, const double* x, double b, double* y, cudaStream_t s) {
  int g = (int)std::min<long long>((n + 255) / 256, 4096);
  axpby_kernel<<<std::max(g, 1), 256, 0, s>>>(n, a, x, b, y);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// F = H + (Jh + Jh^T) - kf (Kh + Kh^T) from the unsymmetrised halves
__global__ void fock_half_kernel(int n, const double* __restrict__ H, const double* __restrict__ J, double kf,
                                 const double* __restrict__ K, double* __restrict__ F) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || j >= n) return;
  const size_t ij = (size_t)i * n + j, ji = (size_t)j * n + i;
  F[ij] = H[ij] + (J[ij] + J[ji]) - kf * (K[ij] + K[ji]);
}
void launch_fock_half(int n, const double* H, const double* J, double kf, const double* K, double* F,
                      cudaStream_t s) {
  dim3 b(32, 8), g((n + 31) / 32, (n + 7) / 8);
  fock_half_kernel<<<g, b, 0, s>>>(n, H, J, kf, K, F);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// out = x - y, then y = x
__global__ void diff_kernel(long long n, const double* __restrict__ x, double* __restrict__ y,
                            double* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i];
    out[i] = v - y[i];
    y[i] = v;
  }
}
void launch_diff_update(long long n, const double* x, double* y, double* out, cudaStream_t s) {
  int g = (int)std::min<long long>((n + 255) / 256, 4096);
  diff_kernel<<<std::max(g, 1), 256, 0, s>>>(n, x, y, out);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

__global__ void fock_kernel(long long n, const double* __restrict__ H, const double* __restrict__ J, double kf,
                            const double* __restrict__ K, double* __restrict__ F) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    F[i] = H[i] + J[i] - kf * K[i];
}
void launch_fock(long long n, const double* H, const double* J, double kf, const double* K, double* F,
                 cudaStream_t s) {
  int g = (int)std::min<long long>((n + 255) / 256, 4096);
  fock_kernel<<<std::max(g, 1), 256, 0, s>>>(n, H, J, kf, K, F);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}

// out[j] = <x, ys[j]>: RED_BLOCKS blocks per j write partial sums into
// part[j * RED_BLOCKS + b]; sum_parts_kernel adds them in a fixed order, so
// the result does not depend on scheduling.
__global__ void dot_many_kernel(long long n, const double* __restrict__ x, const double* const* ys,
                                double* __restrict__ part) {
  __shared__ double sh[32];
  const double* y = ys[blockIdx.y];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += x[i] * y[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// out[j] = sum_b part[j * nb + b] (or the max for the rows flagged in
// max_rows), one warp per row, lanes in a fixed order
__global__ void sum_parts_kernel(const double* __restrict__ part, int rows, int nb, unsigned max_rows,
                                 double* __restrict__ out, int split = 1 << 30, double* __restrict__ out2 = nullptr) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int j = w; j < rows; j += blockDim.x >> 5) {
    const bool mx = (max_rows >> j) & 1u;
    double v = 0.0;
    for (int b = l; b < nb; b += 32) v = mx ? fmax(v, part[j * nb + b]) : v + part[j * nb + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_xor_sync(0xffffffffu, v, o);
      v = mx ? fmax(v, u) : v + u;
    }
    if (l == 0) {
      if (j < split) out[j] = v;
      else out2[j - split] = v;
    }
  }
}

struct LinCombArgs {
  const double* src[8];
  double c[8];
  int m, accumulate;
};

__global__ void lincomb_kernel(long long n, const LinCombArgs a, double* __restrict__ out) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = a.accumulate ? out[i] : 0.0;
    for (int k = 0; k < a.m; ++k) v += a.c[k] * __ldg(a.src[k] + i);
    out[i] = v;
  }
}

void launch_lincomb(long long n, int m, const double* const* src, const double* c, double* out, cudaStream_t s) {
  if (n <= 0 || m <= 0) return;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  for (int k0 = 0; k0 < m; k0 += 8) {  // eight terms per pass
    LinCombArgs a{};
    a.m = std::min(8, m - k0);
    a.accumulate = k0 > 0;
    for (int k = 0; k < a.m; ++k) {
      a.src[k] = src[k0 + k];
      a.c[k] = c[k0 + k];
    }
    lincomb_kernel<<<blocks, 256, 0, s>>>(n, a, out);
    PF_CUDA(cudaGetLastError());
    count_launch();
  }
}

void launch_dot_many(long long n, const double* x, int m, const double* const* ys, double* out, double* part,
                     cudaStream_t s) {
  if (m <= 0) return;
  dot_many_kernel<<<dim3(RED_BLOCKS, m), 256, 0, s>>>(n, x, ys, part);
  PF_CUDA(cudaGetLastError());
  sum_parts_kernel<<<1, 256, 0, s>>>(part, m, RED_BLOCKS, 0u, out);
  PF_CUDA(cudaGetLastError());
  count_launches(2);
}

// out[0] = sum Pt H + sum Pa Fa + sum Pb Fb (x 1/2 applied by the caller),
// out[1] = max |Ea|,|Eb|, out[2] = ||dP||_F^2: RED_BLOCKS blocks write
// partials part[{0,1,2} * RED_BLOCKS + b], sum_parts_kernel combines them.
__global__ void scf_reduce_kernel(long long n, int uhf, const double* __restrict__ H, const double* __restrict__ Pa,
                                  const double* __restrict__ Pb, const double* __restrict__ Fa,
                                  const double* __restrict__ Fb, const double* __restrict__ Ea,
                                  const double* __restrict__ Eb, const double* __restrict__ Pa_old,
                                  const double* __restrict__ Pb_old, double* __restrict__ part, long long nd,
                                  const double* __restrict__ x, const double* const* ys) {
  __shared__ double sh[32];
  if (blockIdx.y > 0) {  // the DIIS overlaps <x, ys[y-1]>: partials into row 2 + y
    const double* y = ys[blockIdx.y - 1];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += (long long)gridDim.x * blockDim.x)
      acc += x[i] * y[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[(2 + blockIdx.y) * gridDim.x + blockIdx.x] = acc;
    return;
  }
  double e = 0.0, dp = 0.0;
  double emx = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (uhf) {
      e += (Pa[i] + Pb[i]) * H[i] + Pa[i] * Fa[i] + Pb[i] * Fb[i];
      emx = fmax(emx, fmax(fabs(Ea[i]), fabs(Eb[i])));
      if (Pa_old) {
        const double d1 = Pa[i] - Pa_old[i], d2 = Pb[i] - Pb_old[i];
        dp += d1 * d1 + d2 * d2;
      }
    } else {
      e += Pa[i] * (H[i] + Fa[i]);
      emx = fmax(emx, fabs(Ea[i]));
      if (Pa_old) {
        const double d1 = Pa[i] - Pa_old[i];
        dp += d1 * d1;
      }
    }
  }
  e = block_sum(e, sh);
  dp = block_sum(dp, sh);
  // max reduction
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) emx = fmax(emx, __shfl_xor_sync(0xffffffffu, emx, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = emx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmax(m, sh[k]);
    part[blockIdx.x] = e;
    part[gridDim.x + blockIdx.x] = m;
    part[2 * gridDim.x + blockIdx.x] = dp;
  }
}
void launch_scf_reduce(long long n, int uhf, const double* H, const double* Pa, const double* Pb, const double* Fa,
                       const double* Fb, const double* Ea, const double* Eb, const double* Pa_old,
                       const double* Pb_old, double* out, double* part, cudaStream_t s, long long nd,
                       const double* x, int m, const double* const* ys, double* out_dots) {
  scf_reduce_kernel<<<dim3(RED_BLOCKS, 1 + std::max(m, 0)), 256, 0, s>>>(n, uhf, H, Pa, Pb, Fa, Fb, Ea, Eb, Pa_old,
                                                                         Pb_old, part, nd, x, ys);
  PF_CUDA(cudaGetLastError());
  sum_parts_kernel<<<1, 256, 0, s>>>(part, 3 + std::max(m, 0), RED_BLOCKS, 2u, out, 3, out_dots);
  PF_CUDA(cudaGetLastError());
  count_launches(2);
}


// dmax[a][b] = max |A|, |B| over the (a, b) shell block.
__global__ void dmax_kernel(int ns, const int* __restrict__ bf_off, const int* __restrict__ nfun, int nbf,
                            const double* __restrict__ A, const double* __restrict__ B,
                            const double* __restrict__ Cc, float* __restrict__ dm) {
  const int a = blockIdx.y * blockDim.y + threadIdx.y, b = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= ns || b >= ns) return;
  double m = 0.0;
  for (int i = 0; i < nfun[a]; ++i)
    for (int j = 0; j < nfun[b]; ++j) {
      const size_t k = (size_t)(bf_off[a] + i) * nbf + bf_off[b] + j;
      m = fmax(m, fabs(A[k]));
      if (B) m = fmax(m, fabs(B[k]));
      if (Cc) m = fmax(m, fabs(Cc[k]));
    }
  dm[(size_t)a * ns + b] = (float)m;
}
void launch_dmax(int ns, const int* bf_off, const int* nfun, int nbf, const double* A, const double* B,
                 const double* C, float* dmax, cudaStream_t s) {
  dim3 b(16, 16), g((ns + 15) / 16, (ns + 15) / 16);
  dmax_kernel<<<g, b, 0, s>>>(ns, bf_off, nfun, nbf, A, B, C, dmax);
  PF_CUDA(cudaGetLastError());
  count_launch();
}


// ---------------------------------------------------------------------------
// Trace-correcting density-matrix purification (TC2, Niklasson 2002) of the
// orthogonalised Fock matrix: X_0 = (l_max I - F')/(l_max - l_min) with
// Gershgorin bounds, then X <- X^2 or X <- 2X - X^2, whichever moves Tr X
// towards the occupation N.  X converges to the projector onto the N lowest
// eigenvectors of F'.  The choice and the convergence test run on the device
// (one block), so a purification needs no host round trip per step.
// state: [0] l_min, [1] l_max, [2] Tr X, [3] Tr X^2, [4] converged flag,
//        [5] steps taken, [6] remaining final steps.
// ---------------------------------------------------------------------------
__global__ void gersh_kernel(int n, const double* __restrict__ F, double* __restrict__ state) {
  __shared__ double smin[32], smax[32];
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) r += fabs(F[(size_t)j * n + i]);
    const double d = F[(size_t)i * n + i];
    lo = fmin(lo, d - r);
    hi = fmax(hi, d + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { smin[w] = lo; smax[w] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { lo = fmin(lo, smin[k]); hi = fmax(hi, smax[k]); }
    lo = fmin(lo, smin[0]);
    hi = fmax(hi, smax[0]);
    state[0] = lo;
    state[1] = hi;
    state[4] = 0.0;
    state[5] = 0.0;
    state[6] = 0.0;
  }
}

__global__ void tc2_init_kernel(long long n2, int n, const double* __restrict__ F, const double* __restrict__ state,
                                double* __restrict__ X) {
  const double lo = state[0], hi = state[1];
  const double sc = 1.0 / (hi - lo);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n), j = (int)(k / n);
    X[k] = ((i == j ? hi : 0.0) - F[k]) * sc;
  }
}

// One TC2 step, out of place: Xout = a Xin + b X2 with X2 = Xin Xin.
// Every block reduces the two traces from the diagonals itself (the same
// reduction order in every block, so all blocks take the same decision) and
// updates its grid-stride share; block 0 writes the next state into the
// other state buffer (sin and sout alternate), so no block reads a value
// written during the same launch.  Once Tr X - Tr X^2 < 1e-9 two more steps
// run (quadratic convergence takes the rest to round-off); afterwards X is
// copied unchanged.
__global__ void tc2_step_kernel(int n, double nocc, const double* __restrict__ Xin, const double* __restrict__ X2,
                                double* __restrict__ Xout, const double* __restrict__ sin, double* __restrict__ sout) {
  __shared__ double s1[32], s2[32];
  __shared__ double coef[2];
  __shared__ int done;
  double t1 = 0.0, t2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    t1 += Xin[(size_t)i * n + i];
    t2 += X2[(size_t)i * n + i];
  }
  t1 = warp_sum(t1);
  t2 = warp_sum(t2);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { s1[w] = t1; s2[w] = t2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    t1 = 0.0; t2 = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { t1 += s1[k]; t2 += s2[k]; }
    const bool was_done = sin[4] != 0.0;
    double countdown = sin[6];
    bool now_done = was_done;
    if (!was_done) {
      if (countdown > 0.0) {
        countdown -= 1.0;
        if (countdown <= 0.0) now_done = true;
      } else if (t1 - t2 < 1e-9 && fabs(t1 - nocc) < 1e-6) {
        countdown = 2.0;
      }
    }
    done = was_done;
    // X <- X^2 takes the trace to t2, X <- 2X - X^2 to 2 t1 - t2
    if (fabs(t2 - nocc) < fabs(2.0 * t1 - t2 - nocc)) { coef[0] = 0.0; coef[1] = 1.0; }
    else { coef[0] = 2.0; coef[1] = -1.0; }
    if (blockIdx.x == 0) {
      sout[0] = sin[0];
      sout[1] = sin[1];
      sout[2] = t1;
      sout[3] = t2;
      sout[4] = now_done ? 1.0 : 0.0;
      sout[5] = sin[5] + (was_done ? 0.0 : 1.0);
      sout[6] = countdown;
    }
  }
  __syncthreads();
  const long long n2 = (long long)n * n;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (done) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2; k += stride) Xout[k] = Xin[k];
    return;
  }
  const double a = coef[0], b = coef[1];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2; k += stride)
    Xout[k] = a * Xin[k] + b * X2[k];
}

void launch_gersh(int n, const double* F, double* state, cudaStream_t s) {
  gersh_kernel<<<1, 1024, 0, s>>>(n, F, state);
  PF_CUDA(cudaGetLastError());
  count_launch();
}
void launch_tc2_init(int n, const double* F, const double* state, double* X, cudaStream_t s) {
  const long long n2 = (long long)n * n;
  const int g = (int)std::min<long long>((n2 + 255) / 256, 2048);
  tc2_init_kernel<<<std::max(g, 1), 256, 0, s>>>(n2, n, F, state, X);
  PF_CUDA(cudaGetLastError());
  count_launch();
}
void launch_tc2_step(int n, double nocc, const double* Xin, const double* X2, double* Xout, const double* sin,
                     double* sout, cudaStream_t s) {
  const long long n2 = (long long)n * n;
  const int blocks = (int)std::max<long long>(1, std::min<long long>((n2 + 511) / 512, 296));
  tc2_step_kernel<<<blocks, 512, 0, s>>>(n, nocc, Xin, X2, Xout, sin, sout);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_zero(void* p, size_t bytes, cudaStream_t s) { PF_CUDA(cudaMemsetAsync(p, 0, bytes, s)); }

// ===========================================================================
// FP64 / FP32 FMA throughput probe: independent FMA chains per thread.
// ===========================================================================
template <typename R>
__global__ void fma_probe_kernel(R* out, int iters, R a, R b) {
  R x0 = threadIdx.x * (R)1e-3, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
    x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  R s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (R)-12345.678) out[0] = s;  // keep the chains alive
}

double probe_fp64(int device, double* fp32) {
  PF_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  PF_CUDA(cudaGetDeviceProperties(&prop, device));
  double* d = nullptr;
  PF_CUDA(cudaMalloc(&d, 64));
  cudaEvent_t e0, e1;
  PF_CUDA(cudaEventCreate(&e0));
  PF_CUDA(cudaEventCreate(&e1));
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  double best64 = 0.0, best32 = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    PF_CUDA(cudaEventRecord(e0));
    fma_probe_kernel<double><<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    PF_CUDA(cudaEventRecord(e1));
    PF_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    if (rep > 0) best64 = std::max(best64, flops / (ms * 1e-3) / 1e9);
    PF_CUDA(cudaEventRecord(e0));
    fma_probe_kernel<float><<<blocks, threads>>>(reinterpret_cast<float*>(d), iters * 2, 0.999999f, 1e-7f);
    PF_CUDA(cudaEventRecord(e1));
    PF_CUDA(cudaEventSynchronize(e1));
    PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best32 = std::max(best32, 2.0 * flops / (ms * 1e-3) / 1e9);
  }
  PF_CUDA(cudaEventDestroy(e0));
  PF_CUDA(cudaEventDestroy(e1));
  PF_CUDA(cudaFree(d));
  if (fp32) *fp32 = best32;
  return best64;
}

}  // namespace pyfacc

namespace pyfacc {

// ---------------------------------------------------------------------------
// Algorithmic flop counts (from the generated class routines)
// ---------------------------------------------------------------------------
const ClassFlops& class_flops(int qc) {
  using C0 = EriClass<double, 0, 0, 0, 0>;
  using C1 = EriClass<double, 1, 0, 0, 0>;
  using C2 = EriClass<double, 1, 0, 1, 0>;
  using C3 = EriClass<double, 1, 1, 0, 0>;
  using C4 = EriClass<double, 1, 1, 1, 0>;
  using C5 = EriClass<double, 1, 1, 1, 1>;
  static const ClassFlops tab[NQCLASS] = {
      {C0::L, C0::NOUT, C0::VRR_FLOPS, C0::HRR_FLOPS, C0::GCON ? C0::GACC_FLOPS : C0::GRAD_FLOPS, C0::GFIN_FLOPS},
      {C1::L, C1::NOUT, C1::VRR_FLOPS, C1::HRR_FLOPS, C1::GCON ? C1::GACC_FLOPS : C1::GRAD_FLOPS, C1::GFIN_FLOPS},
      {C2::L, C2::NOUT, C2::VRR_FLOPS, C2::HRR_FLOPS, C2::GCON ? C2::GACC_FLOPS : C2::GRAD_FLOPS, C2::GFIN_FLOPS},
      {C3::L, C3::NOUT, C3::VRR_FLOPS, C3::HRR_FLOPS, C3::GCON ? C3::GACC_FLOPS : C3::GRAD_FLOPS, C3::GFIN_FLOPS},
      {C4::L, C4::NOUT, C4::VRR_FLOPS, C4::HRR_FLOPS, C4::GCON ? C4::GACC_FLOPS : C4::GRAD_FLOPS, C4::GFIN_FLOPS},
      {C5::L, C5::NOUT, C5::VRR_FLOPS, C5::HRR_FLOPS, C5::GCON ? C5::GACC_FLOPS : C5::GRAD_FLOPS, C5::GFIN_FLOPS},
  };
  return tab[qc];
}

// Per primitive quartet outside the VRR: P-Q (3), T (6), prefactor (2),
// zeta/rho/W terms (12), Boys (Taylor 2*8 + downward recursion 4L), I_m (L+1).
double prim_overhead_flops(int qc, bool) {
  const int L = class_flops(qc).L;
  return 3 + 6 + 2 + 12 + 16 + 4 * L + (L + 1);
}

// Digestion per contracted quartet: J (4 flops per integral) and K (8 per
// integral and exchange density).
double digest_flops(int qc, int nk) { return (double)class_flops(qc).nout * (4.0 + 8.0 * nk); }

}  // namespace pyfacc
