// Trace-correcting purification (TC2, Niklasson 2002) of an orthogonalised
// Fock matrix in ONE cooperative launch: every block stays resident, the
// blocks meet at a grid barrier twice per step, and no step returns to the
// host.  A step squares the symmetric iterate X over the tiles of its upper
// triangle (row panels of X staged in shared memory by cp.async; X2[i][j] =
// sum_k X[i][k] X[j][k]), every block then sums the per-block partial traces
// in the same order, takes the same step choice (X <- X^2 or 2X - X^2,
// whichever moves Tr X towards N) and updates the elements of its own tiles.
// The stopping rule is that of the single-launch-per-step kernels: once
// Tr X - Tr X^2 < 1e-9 at the right trace, two more steps.
//
// The grid barrier is a counter plus a generation word in global memory; a
// block that waits longer than its spin limit (seconds) raises an error flag
// in the state and every block returns, so the caller falls back to the
// eigensolver path.  The cooperative launch guarantees that all blocks are
// resident, so the limit is never reached in normal operation.
#include <cuda_runtime.h>

#include <algorithm>

#include "engine.h"

namespace pyfacc {

namespace {

constexpr int kThreads = 256;
constexpr int kPad = 2;  // panel row stride = tile + 2 doubles (16-byte aligned pairs)

struct Tc2Args {
  int n, nocc, ts, ntile, nup, kc;
  const double* Fp;
  double* X;
  double* X2;
  double* part;        // [0, 2G): Gershgorin lo/hi; then [2][2][G] traces by step parity
  unsigned* bar;       // [0] arrivals, [1] generation
  double* state;       // [0] lo [1] hi [4] converged [5] steps [7] error
};

__device__ __forceinline__ double blk_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += red[k];
    red[32] = r;
  }
  __syncthreads();
  const double r = red[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;\n" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void red_add_release(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier with a bounded wait; false when this or another block gave
// up.  Thread 0 of every block arrives with an acquire-release add on the
// counter (the block's writes, ordered before it by the block barrier, are
// released with it); the last arrival resets the counter and releases the
// generation word, which the others poll with acquire loads.
__device__ bool grid_barrier(unsigned* bar, volatile double* state, int* ok_s) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire(bar + 1);
    int ok = 1;
    if (atom_add_acq_rel(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      red_add_release(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (ld_acquire(bar + 1) == g) {
        if (++spins > (1LL << 26)) {
          ok = 0;
          break;
        }
        if (spins > 256) __nanosleep(32);
      }
    }
    if (!ok) state[7] = 1.0;
    *ok_s = ok && state[7] == 0.0;
  }
  __syncthreads();
  return *ok_s != 0;
}

// Sum of v[0..m) and of w[0..m) (m <= 4 * blockDim.x) by the whole block in
// a fixed order, read from L2 (the partial sums of the other blocks).
__device__ __forceinline__ void blk_sum2(const double* v, const double* w, int m, double* red, double* s1,
                                         double* s2) {
  double a = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    a += __ldcg(v + i);
    c += __ldcg(w + i);
  }
  *s1 = blk_sum(a, red);
  *s2 = blk_sum(c, red);
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? 8 : 0;  // 0: zero-fill without reading
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz));
}

__device__ __forceinline__ void tile_of(int t, int ntile, int* ti, int* tj) {
  int i = 0;
  while (t >= ntile - i) {
    t -= ntile - i;
    ++i;
  }
  *ti = i;
  *tj = i + t;
}

// X2 tile (ti, tj) = X[rows i0..] . X[rows j0..]^T, RT x RT outputs per
// thread (tile ts = 16 RT).  Panels are staged k-major with stride ts + kPad.
template <int RT>
__device__ void square_tile(const Tc2Args& a, int ti, int tj, double* As, double* Bs, double (&acc)[RT][RT]) {
  constexpr int TS = 16 * RT;
  const int n = a.n, i0 = ti * TS, j0 = tj * TS;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  const bool diag = ti == tj;
  double* Bp = diag ? As : Bs;
#pragma unroll
  for (int u = 0; u < RT; ++u)
#pragma unroll
    for (int v = 0; v < RT; ++v) acc[u][v] = 0.0;
  for (int k0 = 0; k0 < n; k0 += a.kc) {
    const int kn = min(a.kc, n - k0);
    for (int idx = threadIdx.x; idx < TS * kn; idx += blockDim.x) {
      const int r = idx / kn, k = idx - (idx / kn) * kn;
      const int gi = i0 + r, gk = k0 + k;
      cp_async8(As + k * (TS + kPad) + r, a.X + (gi < n ? (size_t)gi * n + gk : 0), gi < n);
      if (!diag) {
        const int gj = j0 + r;
        cp_async8(Bs + k * (TS + kPad) + r, a.X + (gj < n ? (size_t)gj * n + gk : 0), gj < n);
      }
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    for (int kk = 0; kk < kn; ++kk) {
      const double* ar = As + kk * (TS + kPad) + ty * RT;
      const double* br = Bp + kk * (TS + kPad) + tx * RT;
      double av[RT], bv[RT];
#pragma unroll
      for (int u = 0; u < RT; ++u) av[u] = ar[u];
#pragma unroll
      for (int v = 0; v < RT; ++v) bv[v] = br[v];
#pragma unroll
      for (int u = 0; u < RT; ++u)
#pragma unroll
        for (int v = 0; v < RT; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
    }
    __syncthreads();
  }
}

template <int RT>
__global__ void __launch_bounds__(kThreads) tc2_coop_kernel(const Tc2Args a) {
  constexpr int TS = 16 * RT;
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[33];
  __shared__ double bcast[2];
  __shared__ int ok_s;
  double* As = sm;
  double* Bs = sm + (size_t)a.kc * (TS + kPad);
  const int G = gridDim.x, b = blockIdx.x, n = a.n;
  const size_t n2 = (size_t)n * n;
  volatile double* state = a.state;
  double* part_g = a.part;
  double* part_t = a.part + 2 * G;  // [parity][0: tr X, 1: tr X2][G]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const double nocc = a.nocc;
  // ---- Gershgorin bounds of the symmetrised F' (rows over warps)
  {
    __shared__ double mn[32], mx[32];
    double l2 = 1e300, h2 = -1e300;
    for (int i = b * nw + warp; i < n; i += G * nw) {
      double r = 0.0;
      for (int j = lane; j < n; j += 32)
        if (j != i) r += fabs(0.5 * (a.Fp[(size_t)i * n + j] + a.Fp[(size_t)j * n + i]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
      const double d = a.Fp[(size_t)i * n + i];
      l2 = fmin(l2, d - r);
      h2 = fmax(h2, d + r);
    }
    if (lane == 0) {
      mn[warp] = l2;
      mx[warp] = h2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double l3 = 1e300, h3 = -1e300;
      for (int k = 0; k < nw; ++k) {
        l3 = fmin(l3, mn[k]);
        h3 = fmax(h3, mx[k]);
      }
      part_g[b] = l3;
      part_g[G + b] = h3;
    }
  }
  if (!grid_barrier(a.bar, state, &ok_s)) return;
  {
    __shared__ double mn[32], mx[32];
    double l2 = 1e300, h2 = -1e300;
    for (int k = threadIdx.x; k < G; k += blockDim.x) {
      l2 = fmin(l2, __ldcg(part_g + k));
      h2 = fmax(h2, __ldcg(part_g + G + k));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      l2 = fmin(l2, __shfl_xor_sync(0xffffffffu, l2, o));
      h2 = fmax(h2, __shfl_xor_sync(0xffffffffu, h2, o));
    }
    if (lane == 0) {
      mn[warp] = l2;
      mx[warp] = h2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double l3 = 1e300, h3 = -1e300;
      for (int k = 0; k < nw; ++k) {
        l3 = fmin(l3, mn[k]);
        h3 = fmax(h3, mx[k]);
      }
      bcast[0] = l3;
      bcast[1] = h3;
      if (b == 0) {
        state[0] = l3;
        state[1] = h3;
      }
    }
    __syncthreads();
  }
  const double lo = bcast[0], hi = bcast[1];
  const double sc = 1.0 / fmax(hi - lo, 1e-300);
  // ---- X0 = (hi I - F') / (hi - lo), exactly symmetric
  double t1 = 0.0;
  for (size_t idx = (size_t)b * blockDim.x + threadIdx.x; idx < n2; idx += (size_t)G * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx - (idx / n) * n);
    const double f = 0.5 * (a.Fp[idx] + a.Fp[(size_t)j * n + i]);
    const double x = ((i == j ? hi : 0.0) - f) * sc;
    a.X[idx] = x;
    if (i == j) t1 += x;
  }
  t1 = blk_sum(t1, red);
  if (threadIdx.x == 0) part_t[0 * 2 * G + 0 * G + b] = t1;
  if (!grid_barrier(a.bar, state, &ok_s)) return;
  int countdown = 0;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  for (int k = 0; k < 200; ++k) {
    const int p = k & 1;
    // ---- X2 = X X over the upper tiles (mirrored into the lower ones)
    double t2 = 0.0;
    for (int t = b; t < a.nup; t += G) {
      int ti, tj;
      tile_of(t, a.ntile, &ti, &tj);
      double acc[RT][RT];
      square_tile<RT>(a, ti, tj, As, Bs, acc);
#pragma unroll
      for (int u = 0; u < RT; ++u)
#pragma unroll
        for (int v = 0; v < RT; ++v) {
          const int i = ti * TS + ty * RT + u, j = tj * TS + tx * RT + v;
          if (i < n && j < n) {
            a.X2[(size_t)i * n + j] = acc[u][v];
            if (ti != tj) a.X2[(size_t)j * n + i] = acc[u][v];
            if (i == j) t2 += acc[u][v];
          }
        }
    }
    t2 = blk_sum(t2, red);
    if (threadIdx.x == 0) part_t[p * 2 * G + G + b] = t2;
    if (!grid_barrier(a.bar, state, &ok_s)) return;
    // ---- the same traces, step choice and stopping decision in every block
    double tr1, tr2;
    blk_sum2(part_t + p * 2 * G, part_t + p * 2 * G + G, G, red, &tr1, &tr2);
    bool finish = false;
    if (countdown > 0) {
      if (--countdown == 0) finish = true;
    } else if (tr1 - tr2 < 1e-9 && fabs(tr1 - nocc) < 1e-6) {
      countdown = 2;
    }
    double ca = 2.0, cb = -1.0;  // X <- X^2 takes the trace to tr2, 2X - X^2 to 2 tr1 - tr2
    if (fabs(tr2 - nocc) < fabs(2.0 * tr1 - tr2 - nocc)) {
      ca = 0.0;
      cb = 1.0;
    }
    // ---- update the elements of this block's tiles; partial Tr X of the new X
    double tn = 0.0;
    for (int t = b; t < a.nup; t += G) {
      int ti, tj;
      tile_of(t, a.ntile, &ti, &tj);
#pragma unroll
      for (int u = 0; u < RT; ++u)
#pragma unroll
        for (int v = 0; v < RT; ++v) {
          const int i = ti * TS + ty * RT + u, j = tj * TS + tx * RT + v;
          if (i < n && j < n) {
            const size_t q = (size_t)i * n + j;
            const double x = ca * a.X[q] + cb * a.X2[q];
            a.X[q] = x;
            if (ti != tj) a.X[(size_t)j * n + i] = x;
            if (i == j) tn += x;
          }
        }
    }
    tn = blk_sum(tn, red);
    if (threadIdx.x == 0) part_t[(1 - p) * 2 * G + b] = tn;
    if (!grid_barrier(a.bar, state, &ok_s)) return;
    if (finish) {
      if (b == 0 && threadIdx.x == 0) {
        state[4] = 1.0;
        state[5] = k + 1;
      }
      return;
    }
  }
  if (b == 0 && threadIdx.x == 0) {
    state[4] = 0.0;
    state[5] = 200;
  }
}

template <int RT>
static int coop_grid(size_t smem, int nup, int num_sms) {
  int per_sm = 0;
  PF_CUDA(cudaFuncSetAttribute(tc2_coop_kernel<RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc2_coop_kernel<RT>, kThreads, smem));
  return std::max(1, std::min(nup, std::min(per_sm, 4) * num_sms));
}

}  // namespace

// at most 4 blocks per SM take part: 6 partial sums per block
size_t tc2_coop_scratch_doubles(int num_sms) { return 24 * (size_t)num_sms + 64; }

// state (host-visible after the launch): [4] converged, [5] steps, [7] error.
void launch_tc2_coop(int n, int nocc, const double* Fp, double* X, double* X2, double* part, unsigned* bar,
                     double* state, int num_sms, cudaStream_t s) {
  const int RT = n <= 256 ? 1 : 2;
  const int TS = 16 * RT;
  Tc2Args a;
  a.n = n;
  a.nocc = nocc;
  a.ts = TS;
  a.ntile = (n + TS - 1) / TS;
  a.nup = a.ntile * (a.ntile + 1) / 2;
  a.kc = std::min(384, (n + 31) / 32 * 32);
  a.Fp = Fp;
  a.X = X;
  a.X2 = X2;
  a.part = part;
  a.bar = bar;
  a.state = state;
  const size_t smem = 2 * (size_t)a.kc * (TS + kPad) * sizeof(double);
  PF_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
  PF_CUDA(cudaMemsetAsync(state, 0, 8 * sizeof(double), s));
  void* args[] = {&a};
  if (RT == 1) {
    const int grid = coop_grid<1>(smem, a.nup, num_sms);
    PF_CUDA(cudaLaunchCooperativeKernel((void*)tc2_coop_kernel<1>, grid, kThreads, args, smem, s));
  } else {
    const int grid = coop_grid<2>(smem, a.nup, num_sms);
    PF_CUDA(cudaLaunchCooperativeKernel((void*)tc2_coop_kernel<2>, grid, kThreads, args, smem, s));
  }
  count_launch();
}

}  // namespace pyfacc
