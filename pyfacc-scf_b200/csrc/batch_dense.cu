// Dense per-molecule work of the batched engine.  One thread block per
// molecule; every n x n product is computed by the block itself on the FP64
// tensor cores (mma.sync m8n8k4) from L1/L2-resident operands (the
// matrices of a molecule of up to 160 basis functions are at most 200 KB),
// the TC2 iterate stays in shared memory, reductions go through shared
// memory, and nothing returns to the host between the Fock build and the
// next build density.
//
// The SCF step follows the single-molecule engine (rscf.f90:118-156 with
// DIIS and purification): F = H + J - K/2, E = 1/2 sum P (H + F), the DIIS
// error X (F P S - S P F) X, Pulay extrapolation over up to 8 stored
// matrices, F' = X F X, TC2 purification of F' to the projector on the nocc
// lowest orbitals, P = 2 X P' X.  X = S^{-1/2} (Loewdin orthogonalisation,
// from a coupled Newton-Schulz iteration, so no eigensolver is needed).
#include <cuda_runtime.h>

#include <cmath>

#include "batch.h"

namespace pyfacc {

namespace {

__device__ __forceinline__ double red_op(double a, double b, bool mx) { return mx ? fmax(a, b) : a + b; }

// Block-wide sum (mx = false) or maximum; every thread receives the result.
__device__ double blk_reduce(double v, bool mx) {
  __shared__ double red[33];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = red_op(v, __shfl_xor_sync(0xffffffffu, v, o), mx);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = red_op(r, red[k], mx);
    red[32] = r;
  }
  __syncthreads();
  const double r = red[32];
  __syncthreads();
  return r;
}

// C = alpha A B (+ beta C) for n x n row-major matrices with leading
// dimension n, on the FP64 tensor cores: each warp owns 8 x 8 output tiles
// and runs mma.sync.m8n8k4 (f64) over k in steps of 4; elements beyond n
// are read as zero and not written.  A, B, C may be global or shared; C
// must not alias A or B.  Ends with a block barrier.
//
// Fragments of m8n8k4 (f64, row.col): lane l holds A[l/4][l%4],
// B[l%4][l/4] and C[l/4][2(l%4)], C[l/4][2(l%4)+1].
__device__ void bgemm(int n, const double* A, const double* B, double* C, double alpha, double beta) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nt = (n + 7) >> 3;
  for (int tile = warp; tile < nt * nt; tile += nwarp) {
    const int i0 = (tile / nt) << 3, j0 = (tile % nt) << 3;
    const int ra = i0 + g;          // row of A this lane reads
    const int cb = j0 + g;          // column of B this lane reads
    // two accumulator chains (even and odd k-steps) so that consecutive
    // MMAs do not wait on each other
    double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
    for (int k0 = 0; k0 < n; k0 += 8) {
      const int ka = k0 + t, kb = k0 + 4 + t;
      const double a = (ra < n && ka < n) ? A[(size_t)ra * n + ka] : 0.0;
      const double b = (ka < n && cb < n) ? B[(size_t)ka * n + cb] : 0.0;
      const double a2 = (ra < n && kb < n) ? A[(size_t)ra * n + kb] : 0.0;
      const double b2 = (kb < n && cb < n) ? B[(size_t)kb * n + cb] : 0.0;
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                   : "+d"(d0), "+d"(d1)
                   : "d"(a), "d"(b));
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                   : "+d"(e0), "+d"(e1)
                   : "d"(a2), "d"(b2));
    }
    d0 += e0;
    d1 += e1;
    const int r = i0 + g, c = j0 + 2 * t;
    if (r < n) {
      if (c < n) {
        const size_t q = (size_t)r * n + c;
        C[q] = (beta == 0.0) ? alpha * d0 : alpha * d0 + beta * C[q];
      }
      if (c + 1 < n) {
        const size_t q = (size_t)r * n + c + 1;
        C[q] = (beta == 0.0) ? alpha * d1 : alpha * d1 + beta * C[q];
      }
    }
  }
  __syncthreads();
}

// TC2 purification (Niklasson 2002) of the orthogonalised Fock matrix Fp:
// Xs <- projector onto the nocc lowest eigenvectors.  X2 is n x n work
// space.  The step choice and the stopping rule are those of the
// single-molecule kernels (Tr X - Tr X^2 < 1e-9 at the right trace, then two
// more steps).  Returns the steps taken, or -1 without convergence.
__device__ int tc2(int n, int nocc, const double* Fp, double* Xs, double* X2) {
  const int n2 = n * n;
  if (nocc <= 0 || nocc >= n) {
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
      const int i = idx / n, j = idx - (idx / n) * n;
      Xs[idx] = (nocc > 0 && i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    return 0;
  }
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) r += fabs(Fp[(size_t)i * n + j]);
    const double d = Fp[(size_t)i * n + i];
    lo = fmin(lo, d - r);
    hi = fmax(hi, d + r);
  }
  lo = -blk_reduce(-lo, true);
  hi = blk_reduce(hi, true);
  const double sc = 1.0 / fmax(hi - lo, 1e-300);
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    Xs[idx] = ((i == j ? hi : 0.0) - Fp[idx]) * sc;
  }
  __syncthreads();
  int countdown = 0;
  for (int k = 0; k < 200; ++k) {
    bgemm(n, Xs, Xs, X2, 1.0, 0.0);
    double t1 = 0.0, t2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      t1 += Xs[(size_t)i * n + i];
      t2 += X2[(size_t)i * n + i];
    }
    t1 = blk_reduce(t1, false);
    t2 = blk_reduce(t2, false);
    bool finish = false;
    if (countdown > 0) {
      if (--countdown == 0) finish = true;
    } else if (t1 - t2 < 1e-9 && fabs(t1 - nocc) < 1e-6) {
      countdown = 2;
    }
    // X <- X^2 takes the trace to t2, X <- 2X - X^2 to 2 t1 - t2
    double a = 2.0, b = -1.0;
    if (fabs(t2 - nocc) < fabs(2.0 * t1 - t2 - nocc)) { a = 0.0; b = 1.0; }
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) Xs[idx] = a * Xs[idx] + b * X2[idx];
    __syncthreads();
    if (finish) return k + 1;
  }
  return -1;
}

// Pulay DIIS solve: B c = 0 with sum c = 1 over the slots in use (m <= 8),
// Gaussian elimination with partial pivoting on the bordered system.
__device__ bool diis_solve(int m, const double* B, double* c) {
  double A[(BATCH_DIIS_MAX + 1) * (BATCH_DIIS_MAX + 1)], b[BATCH_DIIS_MAX + 1];
  const int q = m + 1;
  double scl = 0.0;
  for (int i = 0; i < m; ++i) scl = fmax(scl, fabs(B[i * m + i]));
  scl = scl > 0.0 ? 1.0 / scl : 1.0;
  for (int i = 0; i < q; ++i) {
    for (int j = 0; j < q; ++j) A[i * q + j] = (i < m && j < m) ? B[i * m + j] * scl : ((i == m && j == m) ? 0.0 : -1.0);
    b[i] = (i == m) ? -1.0 : 0.0;
  }
  for (int col = 0; col < q; ++col) {
    int piv = col;
    for (int r = col + 1; r < q; ++r)
      if (fabs(A[r * q + col]) > fabs(A[piv * q + col])) piv = r;
    if (fabs(A[piv * q + col]) < 1e-300) return false;
    if (piv != col) {
      for (int k = 0; k < q; ++k) {
        const double t = A[col * q + k];
        A[col * q + k] = A[piv * q + k];
        A[piv * q + k] = t;
      }
      const double t = b[col];
      b[col] = b[piv];
      b[piv] = t;
    }
    for (int r = col + 1; r < q; ++r) {
      const double f = A[r * q + col] / A[col * q + col];
      for (int k = col; k < q; ++k) A[r * q + k] -= f * A[col * q + k];
      b[r] -= f * b[col];
    }
  }
  for (int r = q - 1; r >= 0; --r) {
    double s = b[r];
    for (int k = r + 1; k < q; ++k) s -= A[r * q + k] * c[k];
    c[r] = s / A[r * q + r];
  }
  for (int i = 0; i < m; ++i)
    if (!isfinite(c[i])) return false;
  return true;
}

struct MolPtrs {
  int n, n2;
  const double *S, *H, *X;
  double *F, *J, *K, *Jd, *Kd, *P, *Db, *T1, *T2, *T3;
};

__device__ __forceinline__ MolPtrs mol_ptrs(const BatchDenseArgs& a, const BatchMolDev& d) {
  MolPtrs p;
  p.n = d.nbf;
  p.n2 = d.nbf * d.nbf;
  const size_t o = (size_t)d.mat_off;
  p.S = a.S + o; p.H = a.H + o; p.X = a.X + o;
  p.F = a.F + o; p.J = a.J + o; p.K = a.K + o; p.Jd = a.Jd + o; p.Kd = a.Kd + o;
  p.P = a.P + o; p.Db = a.Db + o; p.T1 = a.T1 + o; p.T2 = a.T2 + o; p.T3 = a.T3 + o;
  return p;
}

// P = 2 X P' X of the TC2 projector of F' = X Fsrc X; T1 and T3 are
// overwritten, the result goes to out.  Returns the TC2 steps or -1.
__device__ int density_from_fock(const MolPtrs& p, int nocc, const double* Fsrc, double* Xs, double* out) {
  bgemm(p.n, p.X, Fsrc, p.T3, 1.0, 0.0);
  bgemm(p.n, p.T3, p.X, p.T1, 1.0, 0.0);
  const int steps = tc2(p.n, nocc, p.T1, Xs, p.T3);
  if (steps < 0) return -1;
  bgemm(p.n, p.X, Xs, p.T1, 1.0, 0.0);
  bgemm(p.n, p.T1, p.X, out, 2.0, 0.0);
  return steps;
}

}  // namespace

// ---------------------------------------------------------------------------
// X = S^{-1/2}: coupled Newton-Schulz iteration Y0 = S/c, Z0 = I,
// T = (3I - Z Y)/2, Y <- Y T, Z <- T Z, which converges to Y = (S/c)^{1/2},
// Z = (S/c)^{-1/2} when the spectrum of S/c lies in (0, 1] (c = the largest
// absolute row sum of S, a bound on its largest eigenvalue).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(BATCH_THREADS) batch_lowdin_kernel(const BatchDenseArgs a, double* Xout) {
  const int m = blockIdx.x;
  const BatchMolDev d = a.mol[m];
  const MolPtrs p = mol_ptrs(a, d);
  const int n = p.n, n2 = p.n2;
  double c = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j) r += fabs(p.S[(size_t)i * n + j]);
    c = fmax(c, r);
  }
  c = blk_reduce(c, true);
  double* Y = p.T1;
  double* Z = p.T2;
  double* Tm = p.T3;
  double* fr = p.F;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    Y[idx] = p.S[idx] / c;
    Z[idx] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  bool ok = false;
  for (int it = 0; it < 100; ++it) {
    bgemm(n, Z, Y, Tm, 1.0, 0.0);
    double dev = 0.0;
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
      const int i = idx / n, j = idx - (idx / n) * n;
      const double v = Tm[idx], e = (i == j) ? 1.0 : 0.0;
      dev = fmax(dev, fabs(v - e));
      Tm[idx] = 1.5 * e - 0.5 * v;
    }
    dev = blk_reduce(dev, true);
    bgemm(n, Y, Tm, fr, 1.0, 0.0);
    { double* t = Y; Y = fr; fr = t; }
    bgemm(n, Tm, Z, fr, 1.0, 0.0);
    { double* t = Z; Z = fr; fr = t; }
    if (dev < 1e-13) {
      ok = true;
      break;
    }
  }
  const double rs = 1.0 / sqrt(c);
  double* Xm = Xout + (size_t)d.mat_off;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    Xm[idx] = 0.5 * (Z[idx] + Z[(size_t)j * n + i]) * rs;
  }
  if (threadIdx.x == 0 && !ok) a.st[m].failed = 1;
}

__global__ void batch_guess_kernel(const BatchDenseArgs a, const double* __restrict__ occ) {
  const int m = blockIdx.x;
  const BatchMolDev d = a.mol[m];
  double* P = a.P + (size_t)d.mat_off;
  const int n = d.nbf;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    P[idx] = (i == j) ? occ[d.occ_off + i] : 0.0;
  }
}

// Start of the SCF: per-molecule state, zero J/K accumulators, the starting
// density (core guess: purification of F = H; otherwise P already holds the
// atomic-occupation guess) and Db = P for the first (full) build.
__global__ void __launch_bounds__(BATCH_THREADS) batch_init_kernel(const BatchDenseArgs a, int core_guess) {
  extern __shared__ double xs_sh[];
  const int m = blockIdx.x;
  const BatchMolDev d = a.mol[m];
  BatchMolState& st = a.st[m];
  const MolPtrs p = mol_ptrs(a, d);
  const int failed = st.failed;
  __syncthreads();
  if (threadIdx.x == 0) {
    st.E = st.E_prev = st.err = st.dD = st.E_final = 0.0;
    for (int k = 0; k < BATCH_DIIS_MAX * BATCH_DIIS_MAX; ++k) st.B[k] = 0.0;
    for (int k = 0; k < BATCH_DIIS_MAX; ++k) st.age[k] = -1;
    st.iter = st.head = st.converged = st.tc2_steps = 0;
    st.done = failed;
  }
  for (int idx = threadIdx.x; idx < p.n2; idx += blockDim.x) {
    p.J[idx] = 0.0;
    p.K[idx] = 0.0;
    p.Jd[idx] = 0.0;
    p.Kd[idx] = 0.0;
  }
  __syncthreads();
  if (!failed && core_guess) {
    double* Xs = (p.n <= a.smem_nmax) ? xs_sh : p.T2;
    const int steps = density_from_fock(p, d.nocc, p.H, Xs, p.P);
    if (steps < 0 && threadIdx.x == 0) {
      st.failed = 1;
      st.done = 1;
    }
    __syncthreads();
  }
  const bool skip = failed || st.done;
  for (int idx = threadIdx.x; idx < p.n2; idx += blockDim.x) p.Db[idx] = skip ? 0.0 : p.P[idx];
}

// One SCF step after the J/K build of Db (partial J, K in Jd, Kd).
__global__ void __launch_bounds__(BATCH_THREADS) batch_step_kernel(const BatchDenseArgs a) {
  extern __shared__ double xs_sh[];
  __shared__ double bro[BATCH_DIIS_MAX], coef[BATCH_DIIS_MAX];
  __shared__ int nuse;
  const int m = blockIdx.x;
  BatchMolState& st = a.st[m];
  if (st.done || st.failed) return;
  const BatchMolDev d = a.mol[m];
  const MolPtrs p = mol_ptrs(a, d);
  const int n = p.n, n2 = p.n2;
  const int it = st.iter + 1;
  const double E_prev = st.E_prev, dD_prev = st.dD;
  const bool built_full = a.built_full != 0;
  // ---- J, K (J = Jh + Jh^T of the build), F and the energy of P
  double e = 0.0;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    const size_t t = (size_t)j * n + i;
    const double jn = (built_full ? 0.0 : p.J[idx]) + p.Jd[idx] + p.Jd[t];
    const double kn = (built_full ? 0.0 : p.K[idx]) + p.Kd[idx] + p.Kd[t];
    p.J[idx] = jn;
    p.K[idx] = kn;
    const double f = p.H[idx] + jn - 0.5 * kn;
    p.F[idx] = f;
    e += p.P[idx] * (p.H[idx] + f);
  }
  const double E = 0.5 * blk_reduce(e, false);
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    p.Jd[idx] = 0.0;
    p.Kd[idx] = 0.0;
  }
  // ---- DIIS error X (F P S - S P F) X  (S P F = (F P S)^T)
  bgemm(n, p.F, p.P, p.T1, 1.0, 0.0);
  bgemm(n, p.T1, p.S, p.T2, 1.0, 0.0);
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    p.T1[idx] = p.T2[idx] - p.T2[(size_t)j * n + i];
  }
  __syncthreads();
  bgemm(n, p.X, p.T1, p.T3, 1.0, 0.0);
  bgemm(n, p.T3, p.X, p.T1, 1.0, 0.0);
  double em = 0.0;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) em = fmax(em, fabs(p.T1[idx]));
  em = blk_reduce(em, true);
  const double dE = fabs(E - E_prev);
  if (threadIdx.x == 0 && a.max_err) atomicMax(a.max_err, (unsigned long long)__double_as_longlong(em));
  bool conv = !a.coarse && dE < a.e_tol && em < a.eps_diis;
  if (a.eps_density > 0) conv = conv && it > 1 && dD_prev < a.eps_density;
  if (threadIdx.x == 0) {
    st.E = E;
    st.err = em;
    st.iter = it;
    st.E_final = E;
  }
  if (conv || it >= a.max_iter) {
    if (threadIdx.x == 0) {
      st.done = 1;
      st.converged = conv ? 1 : 0;
    }
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) p.Db[idx] = 0.0;
    return;
  }
  // ---- DIIS: store F and the error, overlaps, extrapolate
  const double* Fuse = p.F;
  if (a.ndiis > 0) {
    double* dF = a.diis + d.diis_off;
    double* dEr = dF + (size_t)a.ndiis * n2;
    const int slot = st.head;
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
      dF[(size_t)slot * n2 + idx] = p.F[idx];
      dEr[(size_t)slot * n2 + idx] = p.T1[idx];
    }
    __syncthreads();
    for (int k = 0; k < a.ndiis; ++k) {
      if (k != slot && st.age[k] < 0) continue;
      double v = 0.0;
      for (int idx = threadIdx.x; idx < n2; idx += blockDim.x)
        v += dEr[(size_t)slot * n2 + idx] * dEr[(size_t)k * n2 + idx];
      v = blk_reduce(v, false);
      if (threadIdx.x == 0) bro[k] = v;
    }
    __syncthreads();  // every thread has read the slot ages before thread 0 changes them
    if (threadIdx.x == 0) {
      const int D = BATCH_DIIS_MAX;
      st.age[slot] = it;
      for (int k = 0; k < a.ndiis; ++k)
        if (st.age[k] >= 0) {
          st.B[slot * D + k] = bro[k];
          st.B[k * D + slot] = bro[k];
        }
      st.head = (slot + 1) % a.ndiis;
      for (int k = 0; k < BATCH_DIIS_MAX; ++k) coef[k] = 0.0;
      nuse = 0;
      int use[BATCH_DIIS_MAX], nu = 0;
      for (int k = 0; k < a.ndiis; ++k)
        if (st.age[k] >= 0) use[nu++] = k;
      // drop the oldest vectors until the system is solvable
      while (nu >= 2) {
        double Bs[BATCH_DIIS_MAX * BATCH_DIIS_MAX], c[BATCH_DIIS_MAX + 1];
        for (int i = 0; i < nu; ++i)
          for (int j = 0; j < nu; ++j) Bs[i * nu + j] = st.B[use[i] * D + use[j]];
        if (diis_solve(nu, Bs, c)) {
          for (int i = 0; i < nu; ++i) coef[use[i]] = c[i];
          nuse = nu;
          break;
        }
        int oldest = 0;
        for (int i = 1; i < nu; ++i)
          if (st.age[use[i]] < st.age[use[oldest]]) oldest = i;
        st.age[use[oldest]] = -1;
        for (int i = oldest; i + 1 < nu; ++i) use[i] = use[i + 1];
        --nu;
      }
    }
    __syncthreads();
    if (nuse >= 2) {
      for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
        double v = 0.0;
        for (int k = 0; k < a.ndiis; ++k)
          if (coef[k] != 0.0) v += coef[k] * dF[(size_t)k * n2 + idx];
        p.T2[idx] = v;
      }
      __syncthreads();
      Fuse = p.T2;
    }
  }
  // ---- new density: Fuse (F or T2) is read before T2 is reused
  double* Xs = (n <= a.smem_nmax) ? xs_sh : p.T2;
  double* Pn = (p.T2 == Xs) ? p.F : p.T2;
  const int steps = density_from_fock(p, d.nocc, Fuse, Xs, Pn);
  if (steps < 0) {
    if (threadIdx.x == 0) {
      st.failed = 1;
      st.done = 1;
    }
    for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) p.Db[idx] = 0.0;
    return;
  }
  // ---- next build density: P_new - P for an incremental build, else P_new
  // (a full rebuild of an incremental run sets Db = P before its build)
  const bool next_full = !a.incremental;
  double dd = 0.0;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const double pn = Pn[idx], diff = pn - p.P[idx];
    dd += diff * diff;
    p.Db[idx] = next_full ? pn : diff;
    p.P[idx] = pn;
  }
  dd = blk_reduce(dd, false);
  if (threadIdx.x == 0) {
    st.dD = sqrt(dd);
    st.E_prev = E;
    st.tc2_steps += steps;
    atomicAdd(a.active, 1);
  }
}

// F and E of the converged density after a full build of Db = P (the FP64
// polish of mixed precision); J, K, F are replaced, E -> st.E_final.
__global__ void __launch_bounds__(BATCH_THREADS) batch_polish_kernel(const BatchDenseArgs a) {
  const int m = blockIdx.x;
  BatchMolState& st = a.st[m];
  if (st.failed || !st.done) return;
  const BatchMolDev d = a.mol[m];
  const MolPtrs p = mol_ptrs(a, d);
  const int n = p.n, n2 = p.n2;
  double e = 0.0;
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    const int i = idx / n, j = idx - (idx / n) * n;
    const size_t t = (size_t)j * n + i;
    const double jn = p.Jd[idx] + p.Jd[t], kn = p.Kd[idx] + p.Kd[t];
    p.J[idx] = jn;
    p.K[idx] = kn;
    const double f = p.H[idx] + jn - 0.5 * kn;
    p.F[idx] = f;
    e += p.P[idx] * (p.H[idx] + f);
  }
  e = blk_reduce(e, false);
  for (int idx = threadIdx.x; idx < n2; idx += blockDim.x) {
    p.Jd[idx] = 0.0;
    p.Kd[idx] = 0.0;
  }
  if (threadIdx.x == 0) st.E_final = 0.5 * e;
}

// Db = P for the molecules that finished (FP64 polish build), 0 otherwise.
__global__ void batch_polish_density_kernel(const BatchDenseArgs a) {
  const int m = blockIdx.x;
  const BatchMolState& st = a.st[m];
  const BatchMolDev d = a.mol[m];
  const MolPtrs p = mol_ptrs(a, d);
  const bool use = st.done && !st.failed;
  for (int idx = threadIdx.x; idx < p.n2; idx += blockDim.x) p.Db[idx] = use ? p.P[idx] : 0.0;
}

// W = 1/2 P F P (RHF energy-weighted density at convergence).
__global__ void __launch_bounds__(BATCH_THREADS) batch_wdens_kernel(const BatchDenseArgs a, double* out) {
  const int m = blockIdx.x;
  const BatchMolDev d = a.mol[m];
  const MolPtrs p = mol_ptrs(a, d);
  bgemm(p.n, p.F, p.P, p.T1, 1.0, 0.0);
  bgemm(p.n, p.P, p.T1, out + (size_t)d.mat_off, 0.5, 0.0);
}

__global__ void batch_dmax_kernel(int ns_max, const int4* __restrict__ mt, const int* __restrict__ bf_off,
                                  const int* __restrict__ nfun, const double* __restrict__ D, float* __restrict__ dm) {
  const int m = blockIdx.y;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ns_max * ns_max) return;
  const int4 t = mt[m];  // {first shell, ns, mat_off, nbf}
  const int a = idx / ns_max, b = idx - (idx / ns_max) * ns_max;
  float* out = dm + (size_t)m * ns_max * ns_max;
  if (a >= t.y || b >= t.y) {
    out[idx] = 0.0f;
    return;
  }
  const int sa = t.x + a, sb = t.x + b;
  double mx = 0.0;
  for (int i = 0; i < nfun[sa]; ++i)
    for (int j = 0; j < nfun[sb]; ++j)
      mx = fmax(mx, fabs(D[(size_t)t.z + (size_t)(bf_off[sa] + i) * t.w + bf_off[sb] + j]));
  out[idx] = (float)mx;
}

static size_t xs_bytes(const BatchDenseArgs& a) { return (size_t)a.smem_nmax * a.smem_nmax * sizeof(double); }

void batch_set_smem(const BatchDenseArgs& a) {
  const int sm = (int)xs_bytes(a);
  PF_CUDA(cudaFuncSetAttribute(batch_init_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  PF_CUDA(cudaFuncSetAttribute(batch_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
}

__global__ void __launch_bounds__(BATCH_THREADS) batch_full_density_kernel(const BatchDenseArgs a) {
  const int m = blockIdx.x;
  const BatchMolState& st = a.st[m];
  if (st.done || st.failed) return;
  const BatchMolDev d = a.mol[m];
  const size_t n2 = (size_t)d.nbf * d.nbf;
  const double* P = a.P + d.mat_off;
  double* Db = a.Db + d.mat_off;
  for (size_t idx = threadIdx.x; idx < n2; idx += blockDim.x) Db[idx] = P[idx];
}

void launch_batch_full_density(int nmol, const BatchDenseArgs& a, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_full_density_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_lowdin(int nmol, const BatchDenseArgs& a, double* Xout, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_lowdin_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a, Xout);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_guess(int nmol, const BatchDenseArgs& a, const double* occ, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_guess_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a, occ);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_init(int nmol, const BatchDenseArgs& a, int core_guess, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_init_kernel<<<nmol, BATCH_THREADS, xs_bytes(a), s>>>(a, core_guess);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

// ---------------------------------------------------------------------------
// Control of the whole-SCF graph (one thread each).
// ---------------------------------------------------------------------------
__global__ void batch_ctl_select_kernel(const BatchScfCtl* __restrict__ c, int* __restrict__ report,
                                        cudaGraphConditionalHandle variant) {
  report[0] = 0;  // active molecules
  report[1] = 0;
  report[2] = 0;  // largest DIIS error (bits of a double, two ints)
  report[3] = 0;
  cudaGraphSetConditional(variant, (unsigned)c->variant);
}

__global__ void batch_ctl_update_kernel(BatchScfCtl* __restrict__ c, const int* __restrict__ report,
                                        cudaGraphConditionalHandle loop) {
  c->counts[c->variant] += 1;
  const int it = ++c->it;
  const int active = report[0];
  const double err = __longlong_as_double(*reinterpret_cast<const long long*>(report + 2));
  bool go = active > 0;
  if (go && c->coarse && (err < c->coarse_err || it >= c->coarse_max_iter)) {
    c->coarse = 0;
    c->restart = 1;
  }
  if (it >= c->max_iter) go = false;
  if (go) {
    int v;
    if (c->coarse) {
      v = G_CINC;
    } else {
      const bool full = !c->incremental || c->restart || c->since_full + 1 >= c->rebuild_every;
      c->since_full = full ? 0 : c->since_full + 1;
      c->restart = 0;
      v = full ? G_FULL : G_INC;
    }
    c->variant = v;
  }
  c->stop = go ? 0 : 1;
  cudaGraphSetConditional(loop, go ? 1u : 0u);
}

void add_batch_select_node(cudaGraph_t g, cudaGraphNode_t* node, BatchScfCtl* ctl, int* report,
                           cudaGraphConditionalHandle variant) {
  const BatchScfCtl* c = ctl;
  void* args[] = {&c, &report, &variant};
  cudaKernelNodeParams p{};
  p.func = reinterpret_cast<void*>(batch_ctl_select_kernel);
  p.gridDim = dim3(1);
  p.blockDim = dim3(1);
  p.kernelParams = args;
  PF_CUDA(cudaGraphAddKernelNode(node, g, nullptr, 0, &p));
}

void add_batch_update_node(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* dep, BatchScfCtl* ctl,
                           const int* report, cudaGraphConditionalHandle loop) {
  void* args[] = {&ctl, &report, &loop};
  cudaKernelNodeParams p{};
  p.func = reinterpret_cast<void*>(batch_ctl_update_kernel);
  p.gridDim = dim3(1);
  p.blockDim = dim3(1);
  p.kernelParams = args;
  PF_CUDA(cudaGraphAddKernelNode(node, g, dep, 1, &p));
}

void launch_batch_step(int nmol, const BatchDenseArgs& a, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_step_kernel<<<nmol, BATCH_THREADS, xs_bytes(a), s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_polish(int nmol, const BatchDenseArgs& a, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_polish_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_polish_density(int nmol, const BatchDenseArgs& a, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_polish_density_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_wdens(int nmol, const BatchDenseArgs& a, double* out, cudaStream_t s) {
  if (nmol <= 0) return;
  batch_wdens_kernel<<<nmol, BATCH_THREADS, 0, s>>>(a, out);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_dmax(int nmol, int ns_max, const int4* mt, const int* bf_off, const int* nfun, const double* D,
                       float* dm, cudaStream_t s) {
  if (nmol <= 0 || ns_max <= 0) return;
  dim3 grid((ns_max * ns_max + 127) / 128, nmol), block(128);
  batch_dmax_kernel<<<grid, block, 0, s>>>(ns_max, mt, bf_off, nfun, D, dm);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

}  // namespace pyfacc
