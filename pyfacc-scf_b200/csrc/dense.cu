// Dense FP64 work of the single-molecule SCF step on the FP64 tensor cores.
//
//  * dgemm_kernel: C = alpha op(A) op(B) + beta Y for row-major matrices,
//    one block of eight warps (symmetric outputs) or four (full ones) per
//    16 x 16 output tile (2 x 2 tiles of mma.sync m8n8k4 f64), the k range
//    split between the warps and
//    the partial tiles added through shared memory; operands read from
//    L2/L1 (the matrices of one molecule are a few MB at most and stay
//    resident), 16 loads per lane in flight; optionally only the
//    upper-triangle tiles of a symmetric
//    result, mirrored on the store, and optionally op(A) = A - A^T (the
//    commutator F P S - S P F of the DIIS error).
//  * TC2 purification (Niklasson 2002) of F' = X^T F X as one CUDA graph per
//    occupation number: Gershgorin bounds, X_0, then a conditional WHILE node
//    whose body is four fused steps X <- X^2 or 2X - X^2 (product, update,
//    traces of the new iterate) chained by programmatic-dependent-launch
//    edges, so a whole purification is one graph launch and the host reads
//    the outcome once.  This replaces the rscf.f90:140-
//    156 / la.f90:28-57 diagonalisation (dsyev of X^T F X, then D = 2 C C^T)
//    by the equivalent projector onto the nocc lowest eigenvectors.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "engine.h"

namespace pyfacc {

namespace {

struct GemmArgs {
  int m, n, k;
  const double* A;
  int lda;
  const double* B;
  int ldb;
  double* C;
  int ldc;
  double alpha;
  const double* Y;  // may be null (beta ignored)
  int ldy;
  double beta;
};

__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Tile (ti, tj) of the t-th warp: all nt x nt tiles, or with SYM only
// ti <= tj in row-major order of the upper triangle.
template <bool SYM>
__device__ __forceinline__ bool tile_of(int t, int ntm, int ntn, int& ti, int& tj) {
  if (!SYM) {
    if (t >= ntm * ntn) return false;
    ti = t / ntn;
    tj = t - ti * ntn;
    return true;
  }
  const int nt = ntn;
  if (t >= nt * (nt + 1) / 2) return false;
  int i = 0, start = 0;
  while (start + (nt - i) <= t) {
    start += nt - i;
    ++i;
  }
  ti = i;
  tj = i + (t - start);
  return true;
}

// Accumulate the 16 x 16 tile at (i0, j0) of op(A) op(B) over k in
// [kb, ke): acc[r][c][0..1] for the 8 x 8 sub-tile (r, c).  Elements outside
// the matrices read as zero.
template <bool TA, bool TB, bool ASYMA>
__device__ __forceinline__ void tile_product(const GemmArgs& g, int i0, int j0, int kb, int ke,
                                             double (&acc)[2][2][2]) {
  const int lane = threadIdx.x & 31, gr = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
  const int ra[2] = {i0 + gr, i0 + 8 + gr};
  const int cb[2] = {j0 + gr, j0 + 8 + gr};
  const bool rok[2] = {ra[0] < g.m, ra[1] < g.m};
  const bool cok[2] = {cb[0] < g.n, cb[1] < g.n};
  auto opA = [&](int i, int k) -> double {
    double v = TA ? __ldg(g.A + (size_t)k * g.lda + i) : __ldg(g.A + (size_t)i * g.lda + k);
    if (ASYMA) v -= __ldg(g.A + (size_t)k * g.lda + i);
    return v;
  };
  auto opB = [&](int k, int j) -> double {
    return TB ? __ldg(g.B + (size_t)j * g.ldb + k) : __ldg(g.B + (size_t)k * g.ldb + j);
  };
  // the operands of the 16-wide k chunk at k0 (zero beyond ke)
  auto load = [&](int k0, double (&a)[4][2], double (&b)[4][2]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int kk = k0 + 4 * u + tq;
      const bool kok = kk < ke;
#pragma unroll
      for (int r = 0; r < 2; ++r) a[u][r] = (kok && rok[r]) ? opA(ra[r], kk) : 0.0;
#pragma unroll
      for (int c = 0; c < 2; ++c) b[u][c] = (kok && cok[c]) ? opB(kk, cb[c]) : 0.0;
    }
  };
  if (kb >= ke) return;
  // register double buffering: the next chunk's loads are in flight while
  // the current chunk's products run, so a warp waits for one load latency
  // instead of one per chunk
  double a[4][2], b[4][2];
  load(kb, a, b);
  for (int k0 = kb; k0 < ke; k0 += 16) {
    double an[4][2], bn[4][2];
    const bool more = k0 + 16 < ke;
    if (more) load(k0 + 16, an, bn);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) mma_f64(acc[r][c][0], acc[r][c][1], a[u][r], b[u][c]);
    if (more) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          a[u][r] = an[u][r];
          b[u][r] = bn[u][r];
        }
    }
  }
}

// One 16 x 16 tile per block of SPLITK warps: warp w sums its share of k
// (the matrices here are at most a few hundred wide, so a warp alone would
// spend the kernel waiting on one L2 round trip per 16 k; split eight ways
// the waits overlap, and at n = 282 each warp has at most three k chunks),
// then warp 0 adds the other warps' partial tiles from shared memory.
// Returns true on warp 0, whose acc holds the tile.
constexpr int SPLITK = 8;
// Full (not symmetric) products have twice the tiles of a symmetric one
// (324 against 171 at n = 282): with eight warps a block, two blocks per SM
// (registers) hold 296 of them and the rest form a second wave; with four
// warps all fit at once.
constexpr int SPLITK_FULL = 4;
template <bool TA, bool TB, bool ASYMA, int WARPS = SPLITK>
__device__ __forceinline__ bool block_tile(const GemmArgs& g, int i0, int j0, double (&acc)[2][2][2]) {
  __shared__ double part[WARPS - 1][8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunk = (g.k + 15) >> 4, per = (nchunk + WARPS - 1) / WARPS;
  const int kb = min(warp * per * 16, g.k), ke = min((warp + 1) * per * 16, g.k);
  tile_product<TA, TB, ASYMA>(g, i0, j0, kb, ke, acc);
  if (warp > 0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) part[warp - 1][q][lane] = acc[q >> 2][(q >> 1) & 1][q & 1];
  }
  __syncthreads();
  if (warp > 0) return false;
#pragma unroll
  for (int w = 0; w < WARPS - 1; ++w)
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q >> 2][(q >> 1) & 1][q & 1] += part[w][q][lane];
  return true;
}

template <bool TA, bool TB, bool SYM, bool ASYMA, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) dgemm_kernel(const GemmArgs g) {
  const int ntm = (g.m + 15) >> 4, ntn = (g.n + 15) >> 4;
  int ti, tj;
  if (!tile_of<SYM>(blockIdx.x, ntm, ntn, ti, tj)) return;
  const int i0 = ti << 4, j0 = tj << 4;
  double acc[2][2][2];
  if (!block_tile<TA, TB, ASYMA, WARPS>(g, i0, j0, acc)) return;
  const int lane = threadIdx.x & 31, gr = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = i0 + 8 * r + gr, col = j0 + 8 * c + 2 * tq + h;
        if (row >= g.m || col >= g.n) continue;
        if (SYM && ti == tj && row > col) continue;  // the mirror of (col, row) covers it
        double v = g.alpha * acc[r][c][h];
        if (g.Y) v += g.beta * g.Y[(size_t)row * g.ldy + col];
        g.C[(size_t)row * g.ldc + col] = v;
        if (SYM && row != col) g.C[(size_t)col * g.ldc + row] = v;
      }
}

template <bool TA, bool TB, bool SYM, bool ASYMA>
void gemm_launch(const GemmArgs& g, cudaStream_t s) {
  const int ntm = (g.m + 15) / 16, ntn = (g.n + 15) / 16;
  const long long tiles = SYM ? (long long)ntn * (ntn + 1) / 2 : (long long)ntm * ntn;
  constexpr int W = SYM ? SPLITK : SPLITK_FULL;
  dgemm_kernel<TA, TB, SYM, ASYMA, W><<<(int)tiles, 32 * W, 0, s>>>(g);
}

// ---------------------------------------------------------------------------
// TC2 purification graph.  State (doubles): [0] l_min, [1] l_max,
// [2..7] traces {Tr X, Tr X^2} of three consecutive iterates (step k reads
// slot k % 3, accumulates its result's traces into slot (k+1) % 3 and clears
// slot (k+2) % 3), [8..15] and [16..23] the control words of the two
// parities {countdown, done, steps, k, failed}: a step of parity p reads
// control p and writes control 1 - p, so no thread reads a word written in
// the same launch.
// ---------------------------------------------------------------------------
constexpr int ST_ACC = 2, ST_CTL = 8;

__global__ void tc2g_bounds_kernel(int n, const double* __restrict__ F, double* __restrict__ st) {
  __shared__ double smin[32], smax[32];
  double lo = 1e300, hi = -1e300;
  // one warp per row (coalesced reads of the row), lanes split the columns
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = threadIdx.x >> 5; i < n; i += nw) {
    const double* row = F + (size_t)i * n;
    double r = 0.0;
    for (int j = lane; j < n; j += 32)
      if (j != i) r += fabs(row[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    const double d = row[i];
    lo = fmin(lo, d - r);
    hi = fmax(hi, d + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    smin[w] = lo;
    smax[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      lo = fmin(lo, smin[k]);
      hi = fmax(hi, smax[k]);
    }
    lo = fmin(lo, smin[0]);
    hi = fmax(hi, smax[0]);
    st[0] = lo;
    st[1] = hi;
  }
  if (threadIdx.x < 22) st[ST_ACC + threadIdx.x] = 0.0;  // traces and both control words
}

// X_0 = (l_max I - F) / (l_max - l_min) and its traces into slot 0.
__global__ void tc2g_init_kernel(int n, const double* __restrict__ F, double* __restrict__ st,
                                 double* __restrict__ X) {
  const double lo = st[0], hi = st[1];
  const double sc = 1.0 / (hi - lo);
  const long long n2 = (long long)n * n;
  double t1 = 0.0, t2 = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n2; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n), j = (int)(q - (q / n) * n);
    const double v = ((i == j ? hi : 0.0) - F[q]) * sc;
    X[q] = v;
    if (i == j) t1 += v;
    t2 += v * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    t1 += __shfl_xor_sync(0xffffffffu, t1, o);
    t2 += __shfl_xor_sync(0xffffffffu, t2, o);
  }
  // one pair of atomics per block, not per warp (all blocks add to the
  // same two words)
  __shared__ double s1[32], s2[32];
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s1[w] = t1;
    s2[w] = t2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nw; ++k) {
      t1 += s1[k];
      t2 += s2[k];
    }
    atomicAdd(st + ST_ACC + 0, t1);
    atomicAdd(st + ST_ACC + 1, t2);
  }
}

struct Tc2StepArgs {
  int n;
  double nocc;
  const double* Xin;
  double* Xout;
  double* st;
  int parity;
  int kmax;
  cudaGraphConditionalHandle cond;
  int set_cond;  // the body's last step decides whether the WHILE loop goes on
};

// One TC2 step, fused: Xout = a Xin + b Xin^2 over the upper-triangle tiles
// (mirrored), with (a, b) = (0, 1) if Tr X^2 is closer to nocc than
// 2 Tr X - Tr X^2, else (2, -1) -- the choice every warp makes from the
// traces of Xin that the previous step accumulated.  Once Tr X - Tr X^2 <
// 1e-9 at the right trace, two more steps run, then the iterate is copied.
__global__ void __launch_bounds__(32 * SPLITK) tc2g_step_kernel(const Tc2StepArgs s) {
  const int n = s.n;
  const int nt = (n + 15) >> 4;
  int ti = 0, tj = 0;
  tile_of<true>(blockIdx.x, nt, nt, ti, tj);  // the grid is the upper-triangle tile count
  const int i0 = ti << 4, j0 = tj << 4;
  const int lane = threadIdx.x & 31, gr = lane >> 2, tq = lane & 3;
  // Programmatic dependent launch: within a WHILE body the next step's grid
  // is launched while this one runs (its blocks wait here), so a step does
  // not pay the whole launch latency.  Nothing of X, the traces or the
  // control words is read before the previous step has completed.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // Every load that does not depend on the control words is issued first,
  // so that one L2 round trip covers them all: this lane's entries of X for
  // the update (warp 0), the control words, all three trace slots, and the
  // product's operands (evaluated even after convergence, when the update
  // discards it, rather than waiting for the done flag).
  double xin[2][2][2];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = i0 + 8 * r + gr, col = j0 + 8 * c + 2 * tq + h;
        xin[r][c][h] = (threadIdx.x < 32 && row < n && col < n) ? s.Xin[(size_t)row * n + col] : 0.0;
      }
  const double* cin = s.st + ST_CTL + 8 * s.parity;
  double* cout = s.st + ST_CTL + 8 * (1 - s.parity);
  const double countdown0 = cin[0];
  const bool was_done = cin[1] != 0.0;
  const double steps = cin[2];
  const int k = (int)cin[3];
  const double failed0 = cin[4];
  double tr[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) tr[q] = s.st[ST_ACC + q];
  double acc[2][2][2];
  const GemmArgs g{n, n, n, s.Xin, n, s.Xin, n, nullptr, n, 1.0, nullptr, n, 0.0};
  const bool warp0 = block_tile<false, false, false>(g, i0, j0, acc);
  const int k3 = k % 3;
  const double t1 = tr[2 * k3], t2 = tr[2 * k3 + 1];
  double a = 0.0, b = 1.0;
  if (!(fabs(t2 - s.nocc) < fabs(2.0 * t1 - t2 - s.nocc))) {
    a = 2.0;
    b = -1.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double countdown = countdown0;
    bool now_done = was_done;
    if (!was_done) {
      if (countdown > 0.0) {
        countdown -= 1.0;
        if (countdown <= 0.0) now_done = true;
      } else if (t1 - t2 < 1e-9 && fabs(t1 - s.nocc) < 1e-6) {
        countdown = 2.0;
      }
    }
    const double steps_out = steps + (was_done ? 0.0 : 1.0);
    const bool failed = failed0 != 0.0 || (!now_done && steps_out >= (double)s.kmax);
    cout[0] = countdown;
    cout[1] = now_done ? 1.0 : 0.0;
    cout[2] = steps_out;
    cout[3] = (double)(k + 1);
    cout[4] = failed ? 1.0 : 0.0;
    s.st[ST_ACC + 2 * ((k + 2) % 3)] = 0.0;
    s.st[ST_ACC + 2 * ((k + 2) % 3) + 1] = 0.0;
    if (s.set_cond) cudaGraphSetConditional(s.cond, (now_done || failed) ? 0u : 1u);
  }
  if (!warp0) return;
  if (was_done) {  // converged: the iterate is copied unchanged
    a = 1.0;
    b = 0.0;
  }
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = i0 + 8 * r + gr, col = j0 + 8 * c + 2 * tq + h;
        if (row >= n || col >= n) continue;
        if (ti == tj && row > col) continue;
        const double v = a * xin[r][c][h] + b * acc[r][c][h];
        s.Xout[(size_t)row * n + col] = v;
        if (row != col) {
          s.Xout[(size_t)col * n + row] = v;
          s2 += 2.0 * v * v;
        } else {
          s1 += v;
          s2 += v * v;
        }
      }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    double* nx = s.st + ST_ACC + 2 * ((k + 1) % 3);
    if (s1 != 0.0) atomicAdd(nx, s1);
    if (s2 != 0.0) atomicAdd(nx + 1, s2);
  }
}

}  // namespace

void launch_dgemm(int m, int n, int k, bool ta, const double* A, int lda, bool tb, const double* B, int ldb,
                  double* C, int ldc, double alpha, const double* Y, int ldy, double beta, bool sym, bool asym_a,
                  cudaStream_t s) {
  if (m <= 0 || n <= 0) return;
  if (sym && m != n) throw Error(PYFACC_ERR_INVALID, "symmetric product needs m == n");
  if (asym_a && ta) throw Error(PYFACC_ERR_INVALID, "A - A^T with a transposed A");
  const GemmArgs g{m, n, k, A, lda, B, ldb, C, ldc, alpha, Y, ldy, beta};
  const int code = (ta ? 8 : 0) | (tb ? 4 : 0) | (sym ? 2 : 0) | (asym_a ? 1 : 0);
  switch (code) {
    case 0: gemm_launch<false, false, false, false>(g, s); break;
    case 1: gemm_launch<false, false, false, true>(g, s); break;
    case 2: gemm_launch<false, false, true, false>(g, s); break;
    case 3: gemm_launch<false, false, true, true>(g, s); break;
    case 4: gemm_launch<false, true, false, false>(g, s); break;
    case 5: gemm_launch<false, true, false, true>(g, s); break;
    case 6: gemm_launch<false, true, true, false>(g, s); break;
    case 7: gemm_launch<false, true, true, true>(g, s); break;
    case 8: gemm_launch<true, false, false, false>(g, s); break;
    case 10: gemm_launch<true, false, true, false>(g, s); break;
    case 12: gemm_launch<true, true, false, false>(g, s); break;
    case 14: gemm_launch<true, true, true, false>(g, s); break;
    default: throw Error(PYFACC_ERR_INVALID, "unsupported product form");
  }
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// The purification graph of one occupation number (see above): bounds,
// X_0, WHILE { TC2_BODY_STEPS steps of alternating parity: 0 (Xa -> Xb),
// 1 (Xb -> Xa), ... }.  The
// result is in Xa; st[ST_CTL + 1] (done), [+2] (steps), [+4] (failed) of
// parity 0 tell the outcome.
static cudaGraphExec_t build_tc2_graph_impl(int n, int nocc, const double* Fp, double* Xa, double* Xb, double* st,
                                            int kmax, bool programmatic) {
  cudaGraph_t graph = nullptr;
  PF_CUDA(cudaGraphCreate(&graph, 0));
  cudaGraphExec_t exec = nullptr;
  try {
    // bounds (one block) -> X_0
    cudaGraphNode_t nb = nullptr, ni = nullptr, nw = nullptr;
    {
      int nn = n;
      const double* f = Fp;
      double* sp = st;
      void* args[] = {&nn, &f, &sp};
      cudaKernelNodeParams p{};
      p.func = reinterpret_cast<void*>(tc2g_bounds_kernel);
      p.gridDim = dim3(1);
      p.blockDim = dim3(1024);
      p.kernelParams = args;
      PF_CUDA(cudaGraphAddKernelNode(&nb, graph, nullptr, 0, &p));
    }
    {
      int nn = n;
      const double* f = Fp;
      double* sp = st;
      double* x = Xa;
      void* args[] = {&nn, &f, &sp, &x};
      cudaKernelNodeParams p{};
      p.func = reinterpret_cast<void*>(tc2g_init_kernel);
      const long long n2 = (long long)n * n;
      p.gridDim = dim3((unsigned)std::max<long long>(1, std::min<long long>((n2 + 255) / 256, 1024)));
      p.blockDim = dim3(256);
      p.kernelParams = args;
      PF_CUDA(cudaGraphAddKernelNode(&ni, graph, &nb, 1, &p));
    }
    cudaGraphConditionalHandle h;
    PF_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    PF_CUDA(cudaGraphAddNode(&nw, graph, &ni, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const int nt = (n + 15) / 16;
    const int blocks = nt * (nt + 1) / 2;
    // TC2_BODY_STEPS steps per WHILE iteration, chained by programmatic
    // edges (the next step's launch overlaps the current one; the kernel
    // waits for its predecessor's completion before reading anything), or
    // by plain edges where the runtime does not take programmatic ones
    cudaGraphNode_t prev = nullptr;
    for (int q = 0; q < TC2_BODY_STEPS; ++q) {
      const int par = q & 1;
      Tc2StepArgs a;
      a.n = n;
      a.nocc = (double)nocc;
      a.Xin = par == 0 ? Xa : Xb;
      a.Xout = par == 0 ? Xb : Xa;
      a.st = st;
      a.parity = par;
      a.kmax = kmax;
      a.cond = h;
      a.set_cond = q == TC2_BODY_STEPS - 1;
      void* args[] = {&a};
      cudaKernelNodeParams p{};
      p.func = reinterpret_cast<void*>(tc2g_step_kernel);
      p.gridDim = dim3(blocks);
      p.blockDim = dim3(32 * SPLITK);
      p.kernelParams = args;
      cudaGraphNode_t node = nullptr;
      PF_CUDA(cudaGraphAddKernelNode(&node, body, nullptr, 0, &p));
      if (prev) {
        cudaGraphEdgeData ed{};
        ed.from_port = cudaGraphKernelNodePortProgrammatic;
        ed.type = cudaGraphDependencyTypeProgrammatic;
        if (!programmatic || cudaGraphAddDependencies_v2(body, &prev, &node, &ed, 1) != cudaSuccess) {
          (void)cudaGetLastError();
          PF_CUDA(cudaGraphAddDependencies(body, &prev, &node, 1));
        }
      }
      prev = node;
    }
    const cudaError_t rc = cudaGraphInstantiate(&exec, graph, 0);
    if (rc != cudaSuccess) throw Error(PYFACC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(rc));
  } catch (...) {
    cudaGraphDestroy(graph);
    throw;
  }
  cudaGraphDestroy(graph);
  return exec;
}

cudaGraphExec_t build_tc2_graph(int n, int nocc, const double* Fp, double* Xa, double* Xb, double* st, int kmax) {
  try {
    return build_tc2_graph_impl(n, nocc, Fp, Xa, Xb, st, kmax, true);
  } catch (const Error&) {  // a runtime that does not instantiate programmatic edges in a WHILE body
    (void)cudaGetLastError();
    return build_tc2_graph_impl(n, nocc, Fp, Xa, Xb, st, kmax, false);
  }
}

}  // namespace pyfacc
