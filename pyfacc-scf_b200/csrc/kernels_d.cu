// Shell quartets with a d shell: Schwarz factors, J/K digestion and the
// two-electron nuclear gradient, one warp per contracted quartet.
//
// The recursions of these classes (up to 961 contracted accumulators and
// 2330 intermediates per primitive quartet for (dd|dd)) do not fit a lane's
// registers, so gen_programs.py flattens them into operation lists with
// dependency levels (eri_programs.cuh).  A warp keeps the tables of its
// quartet in shared memory; per primitive quartet every lane computes the
// prefactors, the lanes share the Boys values I_m, then execute the VRR
// operations of one level at a time (32 at once, __syncwarp between
// levels) and add the [e0|f0] needed to the contracted accumulators.  After
// the primitive loop the HRR operations run the same way on the
// accumulators, and the lanes digest the (ab|cd) into J and K (FP64
// atomics, the layout of the s/p kernels: J = Jh + Jh^T afterwards).
//
// The gradient sums the primitive [e0|f0] four times (plain and weighted by
// 2 alpha, 2 beta, 2 gamma) and builds the shifted classes (a+-1 b|, (a b+-1|,
// |c+-1 d) from those sums, contracted with the two-particle density on the
// fly; centre D follows from translational invariance.
//
// Primitives carry the x^l normalisation of their shell (gaussian.f90:80-98
// for l <= 1); the d components xy, xz, yz get the factor sqrt(3) that the
// x^2 normalisation leaves out, as in the oracle.  All arithmetic is FP64
// (mixed precision leaves the d quartets in FP64).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "boys.cuh"
#include "engine.h"
#include "eri_programs.cuh"

namespace pyfacc {

void upload_boys_tables_d(const double* tl, size_t ntl, const double* ex, size_t nex) {
  PF_CUDA(cudaMemcpyToSymbol(g_boys_tl, tl, ntl * sizeof(double)));
  PF_CUDA(cudaMemcpyToSymbol(g_boys_exp, ex, nex * sizeof(double)));
}

namespace {

// Component factor of Cartesian component k of a shell with angular
// momentum l: 1 for s and p, and for d (xx, xy, xz, yy, yz, zz) sqrt(3) on
// the mixed ones.
__device__ __forceinline__ double comp_ratio_d(int l, int k) {
  return (l == 2 && (k == 1 || k == 2 || k == 4)) ? 1.7320508075688772935 : 1.0;
}

__device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }

__device__ __forceinline__ void boys_any(int L, double T, double* F) {
  switch (L) {
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

__device__ __forceinline__ double pick3(double x, double y, double z, int a) { return a == 0 ? x : (a == 1 ? y : z); }

struct PrimQ {  // one primitive quartet, the same on every lane
  double PA[3], WP[3], QC[3], WQ[3];
  double o2p, rp, o2q, rq, o2pq;
  double ta, tb, tc;  // 2 alpha, 2 beta, 2 gamma
};

// Prefactors of primitive pair records b (bra) and k (ket); T[0..L] = I_m.
__device__ __forceinline__ void prim_quartet(const double4* __restrict__ br, const double4* __restrict__ kr, int L,
                                             PrimQ& g, double* T, int lane) {
  const double4 b0 = br[0], b1 = br[1], b2 = br[2];
  const double4 k0 = kr[0], k1 = kr[1], k2 = kr[2];
  const double p = b0.x, q = k0.x;
  const double PQx = b1.x - k1.x, PQy = b1.y - k1.y, PQz = b1.z - k1.z;
  const double rs = rsqrt(p + q), oz = rs * rs;
  const double rho = p * q * oz;
  const double Tv = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
  const double pref = b0.z * k0.z * rs;
  double F[PF_BOYS_MMAX + 1];
  boys_any(L, Tv, F);
  if (lane <= L) {
    double v = F[0];
#pragma unroll
    for (int m = 1; m <= PF_BOYS_MMAX; ++m)
      if (m == lane) v = F[m];
    T[lane] = pref * v;
  }
  const double qz = q * oz, pz = p * oz;
  g.PA[0] = b2.x; g.PA[1] = b2.y; g.PA[2] = b2.z;
  g.QC[0] = k2.x; g.QC[1] = k2.y; g.QC[2] = k2.z;
  g.WP[0] = -qz * PQx; g.WP[1] = -qz * PQy; g.WP[2] = -qz * PQz;
  g.WQ[0] = pz * PQx;  g.WQ[1] = pz * PQy;  g.WQ[2] = pz * PQz;
  g.o2p = b0.y;
  g.o2q = k0.y;
  g.rp = qz;
  g.rq = pz;
  g.o2pq = 0.5 * oz;
  g.ta = 2.0 * b0.w;
  g.tb = 2.0 * (b0.x - b0.w);
  g.tc = 2.0 * k0.w;
}

// The VRR operations of one primitive quartet on the table T (one warp).
__device__ __forceinline__ void run_vrr(const DOps& o, const PrimQ& g, double* T, int lane) {
  int start = 0;
  for (int lv = 0; lv < o.nlev; ++lv) {
    const int end = __ldg(g_dlev + o.lev + lv);
    for (int i = start + lane; i < end; i += 32) {
      const uint4 op = __ldg(g_dvrr + o.begin + i);
      const int dst = op.x & 0xffff, s1 = op.x >> 16, s2 = op.y & 0xffff, s3 = op.y >> 16, s4 = op.z & 0xffff,
                s5 = op.z >> 16;
      const int ax = op.w & 3, ket = (op.w >> 2) & 1, c3 = (op.w >> 4) & 15, c5 = (op.w >> 8) & 15;
      double v;
      if (!ket) {
        v = pick3(g.PA[0], g.PA[1], g.PA[2], ax) * T[s1] + pick3(g.WP[0], g.WP[1], g.WP[2], ax) * T[s2];
        if (c3) v += c3 * g.o2p * (T[s3] - g.rp * T[s4]);
      } else {
        v = pick3(g.QC[0], g.QC[1], g.QC[2], ax) * T[s1] + pick3(g.WQ[0], g.WQ[1], g.WQ[2], ax) * T[s2];
        if (c3) v += c3 * g.o2q * (T[s3] - g.rq * T[s4]);
        if (c5) v += c5 * g.o2pq * T[s5];
      }
      T[dst] = v;
    }
    start = end;
    __syncwarp();
  }
}

// The HRR operations on the table H (one warp); AB = A - B, CD = C - D.
__device__ __forceinline__ void run_hrr(const DOps& o, const double4& AB, const double4& CD, double* H, int lane) {
  int start = 0;
  for (int lv = 0; lv < o.nlev; ++lv) {
    const int end = __ldg(g_dlev + o.lev + lv);
    for (int i = start + lane; i < end; i += 32) {
      const uint4 op = __ldg(g_dhrr + o.begin + i);
      const int dst = op.x & 0xffff, sa = op.x >> 16, sb = op.y;
      const int ax = op.z & 3, ket = (op.z >> 2) & 1;
      const double X = ket ? pick3(CD.x, CD.y, CD.z, ax) : pick3(AB.x, AB.y, AB.z, ax);
      H[dst] = H[sa] + X * H[sb];
    }
    start = end;
    __syncwarp();
  }
}

// Contracted (ab|cd) of bra pair bp and ket pair kp into WORK (outputs at
// the program's output slots); ACC and WORK are this warp's tables.
// Primitive quartets with |K_ab K_cd| < kcut are skipped (records sorted by
// |K| per pair, as in the s/p kernels).
__device__ void contracted_d(const DProg& P, const double4* __restrict__ prim, int4 bi0, int4 ki0,
                             const double4& bg, const double4& kg, double kcut, double* ACC, double* WORK,
                             int lane) {
  for (int k = lane; k < P.nacc; k += 32) ACC[k] = 0.0;
  __syncwarp();
  const double kab_max = fabs(prim[3 * (size_t)bi0.z].z);
  for (int kq = 0; kq < ki0.w; ++kq) {
    const double4* kr = prim + 3 * (size_t)(ki0.z + kq);
    const double kcd = fabs(kr[0].z);
    if (kab_max * kcd < kcut) break;
    for (int kp = 0; kp < bi0.w; ++kp) {
      const double4* br = prim + 3 * (size_t)(bi0.z + kp);
      if (fabs(br[0].z) * kcd < kcut) break;
      PrimQ g;
      prim_quartet(br, kr, P.L, g, WORK, lane);
      __syncwarp();
      run_vrr(P.vrr, g, WORK, lane);
      for (int k = lane; k < P.nacc; k += 32) ACC[k] += WORK[__ldg(g_dmap + P.acc + k)];
      __syncwarp();
    }
  }
  for (int k = lane; k < P.nacc; k += 32) WORK[k] = ACC[k];
  __syncwarp();
  run_hrr(P.hrr, bg, kg, WORK, lane);
}

__device__ __forceinline__ int find_bra_d(const int* __restrict__ task_off, int nbra, int t) {
  int lo = 0, hi = nbra;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(task_off + mid) <= t) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ float dmax_bound_d(const float* __restrict__ dm, int ld, int a, int b, int c, int d) {
  float m = 2.0f * fmaxf(__ldg(dm + a * ld + b), __ldg(dm + c * ld + d));
  m = fmaxf(m, __ldg(dm + a * ld + c));
  m = fmaxf(m, __ldg(dm + a * ld + d));
  m = fmaxf(m, __ldg(dm + b * ld + c));
  m = fmaxf(m, __ldg(dm + b * ld + d));
  return m;
}

struct DListArgs {
  const int4* info0;
  const int4* info1;
  const int4* info2;
  const double4* geom;
  const double4* prim;
  const int* task_off;
  const int* ket_lo;
  const int* ket_hi;
  int nbra, ntasks, bra_base, ket_base, same_class, task_begin, width, prog, wpb;
  int words;  // doubles of shared memory per warp
};

// ---------------------------------------------------------------------------
// Schwarz factors of the d pairs: Q = sqrt(max |(ab|ab)|), one warp per pair.
// ---------------------------------------------------------------------------
__global__ void schwarz_d_kernel(int begin, int end, const int4* __restrict__ info0,
                                 const double4* __restrict__ geom, const double4* __restrict__ prim, int prog,
                                 int words, double* __restrict__ q) {
  extern __shared__ double dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double* ACC = dsm + (size_t)wib * words;
  const DProg P = g_dprog[prog];
  double* WORK = ACC + P.nacc;
  for (int i = begin + blockIdx.x * wpb + wib; i < end; i += gridDim.x * wpb) {
    const int4 i0 = info0[i];
    const double4 g = geom[i];
    contracted_d(P, prim, i0, i0, g, g, 0.0, ACC, WORK, lane);
    const int na = ncart(P.la), nb = ncart(P.lb);
    double mx = 0.0;
    for (int ab = lane; ab < na * nb; ab += 32) {
      const int a = ab / nb, b = ab % nb;
      const double r = comp_ratio_d(P.la, a) * comp_ratio_d(P.lb, b);
      const int o = ab * na * nb + ab;
      mx = fmax(mx, fabs(WORK[__ldg(g_dmap + P.out + o)]) * r * r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) q[i] = sqrt(mx);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// J/K digestion of a d-class task list: a warp takes a task (one bra, up to
// `width` kets) and runs its quartets one after the other.
// ---------------------------------------------------------------------------
template <int NK>
__global__ void jk_d_kernel(const DListArgs L, const JkArgs A) {
  extern __shared__ double dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* ACC = dsm + (size_t)wib * L.words;
  const DProg P = g_dprog[L.prog];
  double* WORK = ACC + P.nacc;
  const int na = ncart(P.la), nb = ncart(P.lb), nc = ncart(P.lc), nd = ncart(P.ld);
  for (int t = blockIdx.x * L.wpb + wib; t < L.ntasks; t += gridDim.x * L.wpb) {
    const int tg = L.task_begin + t;
    const int ib = find_bra_d(L.task_off, L.nbra, tg);
    const int k0 = __ldg(L.ket_lo + ib) + (tg - __ldg(L.task_off + ib)) * L.width;
    const int k1 = min(k0 + L.width, __ldg(L.ket_hi + ib));
    const int bp = L.bra_base + ib;
    const int4 bi0 = L.info0[bp], bi1 = L.info1[bp], bi2 = L.info2[bp];
    const double4 bg = L.geom[bp];
    for (int ket = k0; ket < k1; ++ket) {
      const int kp = L.ket_base + ket;
      const int4 ki0 = L.info0[kp], ki1 = L.info1[kp];
      const double4 kg = L.geom[kp];
      double kcut = 0.0;
      if (A.dmax) {
        const float dm = dmax_bound_d(A.dmax + bi2.w, A.ns_ld, bi1.x, bi1.y, ki1.x, ki1.y);
        if ((float)(bg.w * kg.w) * dm < (float)A.thresh) continue;  // uniform across the warp
        if (A.prim_thresh > 0.0) kcut = A.prim_thresh / fmax((double)dm, 1e-300);
      }
      contracted_d(P, L.prim, bi0, ki0, bg, kg, kcut, ACC, WORK, lane);
      double fac = 1.0;
      if (bi1.x == bi1.y) fac *= 0.5;
      if (ki1.x == ki1.y) fac *= 0.5;
      if (L.same_class && bp == kp) fac *= 0.5;
      const size_t mo = (size_t)bi2.x;
      const int ld = bi2.y;
      for (int o = lane; o < P.nout; o += 32) {
        const int d = o % nd, c = (o / nd) % nc, b = (o / (nd * nc)) % nb, a = o / (nd * nc * nb);
        const double v = fac * WORK[__ldg(g_dmap + P.out + o)] * comp_ratio_d(P.la, a) * comp_ratio_d(P.lb, b) *
                         comp_ratio_d(P.lc, c) * comp_ratio_d(P.ld, d);
        const size_t mu = bi0.x + a, nu = bi0.y + b, la = ki0.x + c, si = ki0.y + d;
        atomicAdd(A.J + mo + mu * ld + nu, 2.0 * v * __ldg(A.Dj + mo + la * ld + si));
        atomicAdd(A.J + mo + la * ld + si, 2.0 * v * __ldg(A.Dj + mo + mu * ld + nu));
#pragma unroll
        for (int k = 0; k < NK; ++k) {
          const double* Dk = k == 0 ? A.Dk0 : A.Dk1;
          double* Kk = k == 0 ? A.K0 : A.K1;
          atomicAdd(Kk + mo + mu * ld + la, v * __ldg(Dk + mo + nu * ld + si));
          atomicAdd(Kk + mo + mu * ld + si, v * __ldg(Dk + mo + nu * ld + la));
          atomicAdd(Kk + mo + nu * ld + la, v * __ldg(Dk + mo + mu * ld + si));
          atomicAdd(Kk + mo + nu * ld + si, v * __ldg(Dk + mo + mu * ld + la));
        }
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Two-electron gradient of a d-class task list (same task walk).
// ---------------------------------------------------------------------------
__global__ void grad2e_d_kernel(const DListArgs L, const GradArgs A) {
  extern __shared__ double dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const DGradProg G = g_dgrad[L.prog];
  double* GAM = dsm + (size_t)wib * L.words;
  double* ACC = GAM + G.nout;
  double* WORK = ACC + G.nacc_all;
  const int la = G.la, lb = G.lb, lc = G.lc, ldd = G.ld;
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ldd);
  for (int t = blockIdx.x * L.wpb + wib; t < L.ntasks; t += gridDim.x * L.wpb) {
    const int tg = L.task_begin + t;
    const int ib = find_bra_d(L.task_off, L.nbra, tg);
    const int k0 = __ldg(L.ket_lo + ib) + (tg - __ldg(L.task_off + ib)) * L.width;
    const int k1 = min(k0 + L.width, __ldg(L.ket_hi + ib));
    const int bp = L.bra_base + ib;
    const int4 bi0 = L.info0[bp], bi1 = L.info1[bp], bi2 = L.info2[bp];
    const double4 bg = L.geom[bp];
    for (int ket = k0; ket < k1; ++ket) {
      const int kp = L.ket_base + ket;
      const int4 ki0 = L.info0[kp], ki1 = L.info1[kp];
      const double4 kg = L.geom[kp];
      double kcut = 0.0;
      if (A.dmax) {
        const float dm = dmax_bound_d(A.dmax + bi2.w, A.ns_ld, bi1.x, bi1.y, ki1.x, ki1.y);
        if ((float)(bg.w * kg.w) * dm < (float)A.thresh) continue;
        if (A.prim_thresh > 0.0) kcut = A.prim_thresh / fmax((double)dm, 1e-300);
      }
      double fac = 4.0;
      if (bi1.x == bi1.y) fac *= 0.5;
      if (ki1.x == ki1.y) fac *= 0.5;
      if (L.same_class && bp == kp) fac *= 0.5;
      // two-particle density of the quartet with the component factors
      const size_t mo = (size_t)bi2.x;
      const int ldm = bi2.y;
      for (int o = lane; o < G.nout; o += 32) {
        const int d = o % nd, c = (o / nd) % nc, b = (o / (nd * nc)) % nb, a = o / (nd * nc * nb);
        const size_t mu = bi0.x + a, nu = bi0.y + b, lam = ki0.x + c, si = ki0.y + d;
        const double* Pt = A.Pt + mo;
        double v = __ldg(Pt + mu * ldm + nu) * __ldg(Pt + lam * ldm + si);
        if (A.uhf) {
          const double* Pa = A.Pa + mo;
          const double* Pb = A.Pb + mo;
          v -= 0.5 * (__ldg(Pa + mu * ldm + lam) * __ldg(Pa + nu * ldm + si) +
                      __ldg(Pa + mu * ldm + si) * __ldg(Pa + nu * ldm + lam));
          v -= 0.5 * (__ldg(Pb + mu * ldm + lam) * __ldg(Pb + nu * ldm + si) +
                      __ldg(Pb + mu * ldm + si) * __ldg(Pb + nu * ldm + lam));
        } else {
          v -= 0.25 * (__ldg(Pt + mu * ldm + lam) * __ldg(Pt + nu * ldm + si) +
                       __ldg(Pt + mu * ldm + si) * __ldg(Pt + nu * ldm + lam));
        }
        GAM[o] = fac * v * comp_ratio_d(la, a) * comp_ratio_d(lb, b) * comp_ratio_d(lc, c) * comp_ratio_d(ldd, d);
      }
      for (int k = lane; k < G.nacc_all; k += 32) ACC[k] = 0.0;
      __syncwarp();
      // primitive quartets: VRR to L + 1, four weighted sums
      const double kab_max = fabs(L.prim[3 * (size_t)bi0.z].z);
      for (int kq = 0; kq < ki0.w; ++kq) {
        const double4* kr = L.prim + 3 * (size_t)(ki0.z + kq);
        const double kcd = fabs(kr[0].z);
        if (kab_max * kcd < kcut) break;
        for (int kpp = 0; kpp < bi0.w; ++kpp) {
          const double4* br = L.prim + 3 * (size_t)(bi0.z + kpp);
          if (fabs(br[0].z) * kcd < kcut) break;
          PrimQ g;
          prim_quartet(br, kr, G.L, g, WORK, lane);
          __syncwarp();
          run_vrr(G.vrr, g, WORK, lane);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            const double w = s == 0 ? 1.0 : (s == 1 ? g.ta : (s == 2 ? g.tb : g.tc));
            for (int k = lane; k < G.set_n[s]; k += 32) ACC[G.set_base[s] + k] += w * WORK[__ldg(g_dmap + G.set_map[s] + k)];
          }
          __syncwarp();
        }
      }
      // shifted classes, contracted with the density as they come
      double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0}, gC[3] = {0, 0, 0};
      for (int part = 0; part < 6; ++part) {
        const DGradPart& Q = G.part[part];
        if (!Q.present) continue;
        const int n0 = G.set_n[Q.set];
        for (int k = lane; k < n0; k += 32) WORK[k] = ACC[G.set_base[Q.set] + k];
        __syncwarp();
        run_hrr(Q.hrr, bg, kg, WORK, lane);
        const double sign = (part & 1) ? -1.0 : 1.0;
        for (int idx = lane; idx < 3 * G.nout; idx += 32) {
          const int slot = __ldg(g_dmap + Q.cmap + idx);
          if (slot == 0xffff) continue;
          const double v = sign * __ldg(g_dmap + Q.cfac + idx) * GAM[idx / 3] * WORK[slot];
          const int x = idx % 3;
          if (part < 2) gA[x] += v;
          else if (part < 4) gB[x] += v;
          else gC[x] += v;
        }
        __syncwarp();
      }
#pragma unroll
      for (int x = 0; x < 3; ++x) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          gA[x] += __shfl_xor_sync(0xffffffffu, gA[x], o);
          gB[x] += __shfl_xor_sync(0xffffffffu, gB[x], o);
          gC[x] += __shfl_xor_sync(0xffffffffu, gC[x], o);
        }
      }
      if (lane == 0) {
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          atomicAdd(A.grad + 3 * bi1.z + x, gA[x]);
          atomicAdd(A.grad + 3 * bi1.w + x, gB[x]);
          atomicAdd(A.grad + 3 * ki1.z + x, gC[x]);
          atomicAdd(A.grad + 3 * ki1.w + x, -(gA[x] + gB[x] + gC[x]));
        }
      }
      __syncwarp();
    }
  }
}

// Full ERI tensor (small systems, tests): every quartet of the list writes
// its eight images.
__global__ void eri_tensor_d_kernel(const DListArgs L, int n, double* __restrict__ eri) {
  extern __shared__ double dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* ACC = dsm + (size_t)wib * L.words;
  const DProg P = g_dprog[L.prog];
  double* WORK = ACC + P.nacc;
  const int na = ncart(P.la), nb = ncart(P.lb), nc = ncart(P.lc), nd = ncart(P.ld);
  for (int t = blockIdx.x * L.wpb + wib; t < L.ntasks; t += gridDim.x * L.wpb) {
    const int ib = find_bra_d(L.task_off, L.nbra, t);
    const int k0 = __ldg(L.ket_lo + ib) + (t - __ldg(L.task_off + ib)) * L.width;
    const int k1 = min(k0 + L.width, __ldg(L.ket_hi + ib));
    const int bp = L.bra_base + ib;
    const int4 bi0 = L.info0[bp];
    const double4 bg = L.geom[bp];
    for (int ket = k0; ket < k1; ++ket) {
      const int kp = L.ket_base + ket;
      const int4 ki0 = L.info0[kp];
      contracted_d(P, L.prim, bi0, ki0, bg, L.geom[kp], 0.0, ACC, WORK, lane);
      for (int o = lane; o < P.nout; o += 32) {
        const int d = o % nd, c = (o / nd) % nc, b = (o / (nd * nc)) % nb, a = o / (nd * nc * nb);
        const double v = WORK[__ldg(g_dmap + P.out + o)] * comp_ratio_d(P.la, a) * comp_ratio_d(P.lb, b) *
                         comp_ratio_d(P.lc, c) * comp_ratio_d(P.ld, d);
        const size_t i = bi0.x + a, j = bi0.y + b, k = ki0.x + c, l = ki0.y + d, N = n;
        eri[((i * N + j) * N + k) * N + l] = v;
        eri[((j * N + i) * N + k) * N + l] = v;
        eri[((i * N + j) * N + l) * N + k] = v;
        eri[((j * N + i) * N + l) * N + k] = v;
        eri[((k * N + l) * N + i) * N + j] = v;
        eri[((l * N + k) * N + i) * N + j] = v;
        eri[((k * N + l) * N + j) * N + i] = v;
        eri[((l * N + k) * N + j) * N + i] = v;
      }
      __syncwarp();
    }
  }
}

// Warps per block and shared memory per warp for a table of `words`
// doubles: as many warps as fit 200 KB, at most 4.
void block_shape(int words, int* wpb, size_t* smem) {
  const size_t per = (size_t)words * sizeof(double);
  int w = (int)std::max<size_t>(1, std::min<size_t>(4, (200u * 1024u) / std::max<size_t>(per, 1)));
  *wpb = w;
  *smem = per * w;
}

template <typename K>
void set_smem(K kernel, size_t smem) {
  if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

DListArgs list_args(const PairData& pd, const TaskList& tl, int bc, int kc) {
  DListArgs L{};
  L.info0 = pd.info0; L.info1 = pd.info1; L.info2 = pd.info2;
  L.geom = pd.geom; L.prim = pd.prim;
  L.task_off = tl.task_off; L.ket_lo = tl.ket_lo; L.ket_hi = tl.ket_hi;
  L.nbra = tl.nbra; L.ntasks = tl.ntasks; L.task_begin = tl.task_begin;
  L.bra_base = pd.class_off[bc] + tl.bra_offset;
  L.ket_base = pd.class_off[kc];
  L.same_class = bc == kc;
  L.width = tl.width;
  L.prog = dclass_index(bc, kc);
  return L;
}

int grid_d(long long items, int wpb, int num_sms) {
  const long long blocks = (items + wpb - 1) / wpb;
  return (int)std::max(1LL, std::min(blocks, (long long)num_sms * 8));
}

}  // namespace

void launch_schwarz_d(const PairData& pd, const int* off, double* q, int num_sms, cudaStream_t s) {
  for (int c = NCLASS; c < NPAIRCLASS; ++c) {
    const int n = off[c + 1] - off[c];
    if (n <= 0) continue;
    const int prog = dclass_index(c, c);
    const int words = PF_DPROG_SIZES[prog][1] + std::max(PF_DPROG_SIZES[prog][0], PF_DPROG_SIZES[prog][2]);
    int wpb;
    size_t smem;
    block_shape(words, &wpb, &smem);
    set_smem(schwarz_d_kernel, smem);
    schwarz_d_kernel<<<grid_d(n, wpb, num_sms), 32 * wpb, smem, s>>>(off[c], off[c + 1], pd.info0, pd.geom, pd.prim,
                                                                      prog, words, q);
    PF_CUDA(cudaGetLastError());
    count_launch();
  }
}

void launch_jk_d(const PairData& pd, const TaskList& tl, int bc, int kc, int nk, const JkArgs& a, int num_sms,
                 cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  DListArgs L = list_args(pd, tl, bc, kc);
  L.words = PF_DPROG_SIZES[L.prog][1] + std::max(PF_DPROG_SIZES[L.prog][0], PF_DPROG_SIZES[L.prog][2]);
  size_t smem;
  block_shape(L.words, &L.wpb, &smem);
  const int grid = grid_d(tl.ntasks, L.wpb, num_sms);
  if (nk == 1) {
    set_smem(jk_d_kernel<1>, smem);
    jk_d_kernel<1><<<grid, 32 * L.wpb, smem, s>>>(L, a);
  } else {
    set_smem(jk_d_kernel<2>, smem);
    jk_d_kernel<2><<<grid, 32 * L.wpb, smem, s>>>(L, a);
  }
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_eri_tensor_d(const PairData& pd, const TaskList& tl, int bc, int kc, int nbf, double* eri,
                         cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  DListArgs L = list_args(pd, tl, bc, kc);
  L.words = PF_DPROG_SIZES[L.prog][1] + std::max(PF_DPROG_SIZES[L.prog][0], PF_DPROG_SIZES[L.prog][2]);
  size_t smem;
  block_shape(L.words, &L.wpb, &smem);
  set_smem(eri_tensor_d_kernel, smem);
  eri_tensor_d_kernel<<<grid_d(tl.ntasks, L.wpb, 148), 32 * L.wpb, smem, s>>>(L, nbf, eri);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_grad2e_d(const PairData& pd, const TaskList& tl, int bc, int kc, const GradArgs& a, int num_sms,
                     cudaStream_t s) {
  if (tl.ntasks <= 0) return;
  DListArgs L = list_args(pd, tl, bc, kc);
  const int* z = PF_DGRAD_SIZES[L.prog];
  L.words = z[3] + z[1] + std::max(z[0], z[2]);
  size_t smem;
  block_shape(L.words, &L.wpb, &smem);
  set_smem(grad2e_d_kernel, smem);
  grad2e_d_kernel<<<grid_d(tl.ntasks, L.wpb, num_sms), 32 * L.wpb, smem, s>>>(L, a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

}  // namespace pyfacc
