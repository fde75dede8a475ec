// SCF step of the B200 engine: Fock builds, DIIS, diagonalisation, density,
// energy and the analytic gradient (see engine.cpp for the overview).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "engine.h"
#include "system.h"

namespace pyfacc {

#define PF_CUBLAS(x)                                                                    \
  do {                                                                                  \
    cublasStatus_t s_ = (x);                                                            \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                                    \
      throw Error(PYFACC_ERR_CUDA, std::string(#x) + ": cuBLAS status " + std::to_string((int)s_)); \
  } while (0)
#define PF_CUSOLVER(x)                                                                  \
  do {                                                                                  \
    cusolverStatus_t s_ = (x);                                                          \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                                  \
      throw Error(PYFACC_ERR_CUDA, std::string(#x) + ": cuSOLVER status " + std::to_string((int)s_)); \
  } while (0)

float System::elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  PF_CUDA(cudaEventElapsedTime(&ms, a, b));
  return ms;
}

void System::one_electron() {
  OneEArgs a;
  a.natoms = natoms;
  a.atoms = atoms_dev;
  a.boys_mode = opt.boys_mode;
  a.S = S;
  a.T = T;
  a.V = Vm;
  a.nbf = nbf;
  // pairs left out of the lists (negligible overlap) keep zeros
  launch_zero(S, (size_t)nbf * nbf * sizeof(double), stream);
  launch_zero(T, (size_t)nbf * nbf * sizeof(double), stream);
  launch_zero(Vm, (size_t)nbf * nbf * sizeof(double), stream);
  launch_one_electron(shd, n1e, pairs1e, a, stream);
  launch_axpby((long long)nbf * nbf, 1.0, T, 0.0, H, stream);
  launch_axpby((long long)nbf * nbf, 1.0, Vm, 1.0, H, stream);
  one_e_done = true;
}

// One Fock build: zero the outputs, shell-block density maxima for the
// density-weighted Schwarz test, the six class kernels (FP64 task lists, or
// the FP64 and FP32 halves of the mixed lists), then J = Jh + Jh^T.
void System::jk(const double* Dj, int nk, const double* const* Dk, double* Jo, double* const* Ko, int precision,
                bool dynamic, double thresh, double fp32_thresh, int out) {
  if (thresh <= 0) thresh = opt.schwarz_thresh;
  if (out == JK_ADD && reducer) throw Error(PYFACC_ERR_INVALID, "J/K cannot be added in place across shards");
  const size_t n2 = (size_t)nbf * nbf;
  if (out != JK_ADD) {
    launch_zero(Jo, n2 * sizeof(double), stream);
    for (int k = 0; k < nk; ++k) launch_zero(Ko[k], n2 * sizeof(double), stream);
  }
  launch_dmax(ns, bf_off_dev, nfun_dev, nbf, Dj, Dk[0], nk > 1 ? Dk[1] : nullptr, dmax, stream);
  JkArgs a;
  a.Dj = Dj;
  a.Dk0 = Dk[0];
  a.Dk1 = nk > 1 ? Dk[1] : Dk[0];
  a.J = Jo;
  a.K0 = Ko[0];
  a.K1 = nk > 1 ? Ko[1] : Ko[0];
  a.dmax = (thresh > 0) ? dmax : nullptr;
  a.ns_ld = ns;
  a.thresh = thresh;
  a.stats = stats_dev;
  a.prim_thresh = thresh * PRIM_QUARTET_REL;
  const bool mixed = precision == PYFACC_PRECISION_MIXED;
  if (opt.shard_count > 1) dynamic = false;  // shards use their static sub-lists
  const double t32 = fp32_thresh >= 0 ? fp32_thresh : opt.fp32_thresh;
  if (dynamic) launch_dyn_tasks(pd, dmax, ns, thresh, mixed ? t32 : 0.0, dyn, stream);
  // an all-FP32 build (the coarse phase: t32 beyond every Q_ab Q_cd max|D|)
  // has empty FP64 lists, whose kernels are not launched
  const bool fp64_part = !(dynamic && mixed && t32 >= 1e299);
  // the FP64 and FP32 halves of a mixed build run on different streams,
  // which swap from class to class; an FP64 build alternates its classes
  // between the two streams (every launch only adds into J and K)
  cudaStream_t s32 = ctx.side;
  PF_CUDA(cudaEventRecord(ctx.fork, stream));
  PF_CUDA(cudaStreamWaitEvent(ctx.side, ctx.fork, 0));
  int nth = 0;
  for (int bc = NCLASS - 1; bc >= 0; --bc)
    for (int kc = bc; kc >= 0; --kc, ++nth) {
      const int qc = (bc == 0) ? 0 : (bc == 1 ? 1 + kc : 3 + kc);
      cudaStream_t s64 = (nth & 1) ? s32 : stream, s32c = (nth & 1) ? stream : s32;
      if (dynamic) {
        if (fp64_part) launch_jk(pd, dyn.lists[2 * qc], bc, kc, false, nk, a, num_sms, mixed ? s64 : stream);
        if (mixed) launch_jk(pd, dyn.lists[2 * qc + 1], bc, kc, true, nk, a, num_sms, s32c);
      } else if (mixed) {
        launch_jk(pd, tasks[bc][kc][1], bc, kc, false, nk, a, num_sms, stream);
        launch_jk(pd, tasks[bc][kc][2], bc, kc, true, nk, a, num_sms, s32);
      } else {
        launch_jk(pd, tasks[bc][kc][0], bc, kc, false, nk, a, num_sms, (nth & 1) ? ctx.side : stream);
      }
    }
  // quartets with a d pair: FP64, warp-cooperative kernels (full lists,
  // Schwarz-screened; the density test is made per quartet in the kernel)
  if (has_d)
    for (int bc = NCLASS; bc < NPAIRCLASS; ++bc)
      for (int kc = 0; kc <= bc; ++kc) launch_jk_d(pd, tasks[bc][kc][0], bc, kc, nk, a, num_sms, stream);
  PF_CUDA(cudaEventRecord(ctx.join, ctx.side));
  PF_CUDA(cudaStreamWaitEvent(stream, ctx.join, 0));
  if (reducer) {  // partial J/K of this shard -> sums over all shards
    reduce(Jo, (long long)n2);
    for (int k = 0; k < nk; ++k) reduce(Ko[k], (long long)n2);
  }
  if (out == JK_FULL) {
    launch_symmetrize_add(nbf, Jo, stream);
    for (int k = 0; k < nk; ++k) launch_symmetrize_add(nbf, Ko[k], stream);
  }
  st.n_fock++;
}

void System::jk_counters(int nk, double out[6], double* per_class) {
  JkStats js;
  PF_CUDA(cudaMemcpy(&js, stats_dev, sizeof(JkStats), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 6; ++k) out[k] = 0.0;
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < NQCLASS; ++q) {
      const ClassFlops& cf = class_flops(q);
      out[p] += (double)js.prims[p][q] * (cf.vrr + prim_overhead_flops(q, p == 1)) +
                (double)js.quartets[p][q] * (cf.hrr + digest_flops(q, nk));
      out[2 + p] += (double)js.quartets[p][q];
      out[4 + p] += (double)js.prims[p][q];
      if (per_class) {
        per_class[p * NQCLASS + q] = (double)js.quartets[p][q];
        per_class[(2 + p) * NQCLASS + q] = (double)js.prims[p][q];
      }
    }
}

void System::reduce(double* data, long long count) {
  PF_CUDA(cudaStreamSynchronize(stream));
  const int rc = reducer(reducer_ctx, data, count);
  if (rc != 0) throw Error(PYFACC_ERR_CUDA, "shard reduction failed (" + std::to_string(rc) + ")");
}

void System::eri_tensor(double* eri) {
  const size_t n = nbf;
  launch_zero(eri, n * n * n * n * sizeof(double), stream);
  // unscreened canonical quartets: use a system-local zero-threshold task set
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) launch_eri_tensor(pd, tasks[bc][kc][0], bc, kc, nbf, eri, stream);
  for (int bc = NCLASS; bc < NPAIRCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) launch_eri_tensor_d(pd, tasks[bc][kc][0], bc, kc, nbf, eri, stream);
}

// X = U s^-1/2 from S (la.f90:28-57).  cuSOLVER works column-major; S is
// symmetric, and U comes back with eigenvector j in column j.
// X with X^T S X = I from the Cholesky factor S = L L^T: X = L^{-T}
// (cuSOLVER potrf + cuBLAS trsm).  Any S-orthonormalising X gives the same
// density, energy and orbital energies; la.f90:7-57 uses U s^{-1/2}, which
// costs a full eigendecomposition.  A non-positive-definite S is reported
// as PYFACC_ERR_LINDEP, as before.
void System::orthogonalizer() {
  const size_t n2 = (size_t)nbf * nbf;
  double* L = W3;
  PF_CUDA(cudaMemcpyAsync(L, S, n2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  int lwork = 0;
  PF_CUSOLVER(cusolverDnDpotrf_bufferSize(cusolver, CUBLAS_FILL_MODE_LOWER, nbf, L, nbf, &lwork));
  if ((size_t)lwork * sizeof(double) > syev_work.bytes) syev_work.ensure((size_t)lwork * sizeof(double));
  PF_CUSOLVER(cusolverDnDpotrf(cusolver, CUBLAS_FILL_MODE_LOWER, nbf, L, nbf, syev_work.as<double>(), lwork,
                               info_dev));
  // the status and the smallest pivot go to pinned memory and are checked
  // after the next synchronisation (check_overlap_factor): nothing that runs
  // before it can fault on a bad factor, it only computes with it
  launch_min_diag_sq(nbf, L, pmin_dev, stream);
  PF_CUDA(cudaMemcpyAsync(ctx.pinned + ORTHO_PINNED, pmin_dev, sizeof(double), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaMemcpyAsync(ctx.pinned + ORTHO_PINNED + 1, info_dev, sizeof(int), cudaMemcpyDeviceToHost, stream));
  launch_identity(nbf, X, stream);
  const double one = 1.0;
  PF_CUBLAS(cublasDtrsm(cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, nbf, nbf,
                        &one, L, nbf, X, nbf));
}

// The overlap factorisation's outcome (after a synchronisation that follows
// orthogonalizer()): a non-positive-definite S is PYFACC_ERR_LINDEP.
void System::check_overlap_factor() {
  int info = 0;
  std::memcpy(&info, ctx.pinned + ORTHO_PINNED + 1, sizeof(int));
  const double pmin = ctx.pinned[ORTHO_PINNED];
  if (info > 0) throw Error(PYFACC_ERR_LINDEP, "overlap matrix is not positive definite");
  if (info < 0) throw Error(PYFACC_ERR_CUDA, "overlap factorisation failed");
  // Cholesky pivots L_ii^2 bound the smallest eigenvalue of S from above;
  // coincident atoms give a pivot at round-off level without a negative
  // one.  la.f90:40-44 warns below an eigenvalue of 1e-8 and goes on into
  // 1/sqrt of it; here a pivot below 1e-10 (S_ii = 1) is reported.
  if (!(pmin >= LINDEP_PIVOT))
    throw Error(PYFACC_ERR_LINDEP, "overlap matrix is numerically singular (smallest Cholesky pivot " +
                                       std::to_string(pmin) + "; coincident atoms?)");
}

// Eigenpairs of F' = X^T F X (= R F R^T, symmetric) given directly, C = X C'.
void System::diagonalize_orth(const double* Fp, double* C, double* eps) {
  const double one = 1.0, zero = 0.0;
  PF_CUDA(cudaMemcpyAsync(W2, Fp, (size_t)nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  PF_CUSOLVER(cusolverDnDsyevd(cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nbf, W2, nbf, eps,
                               syev_work.as<double>(), syev_lwork, info_dev));
  PF_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_N, CUBLAS_OP_N, nbf, nbf, nbf, &one, X, nbf, W2, nbf, &zero, C, nbf));
}

// F' = X^T F X, eigenpairs, C = X C' (all column-major).
void System::diagonalize(const double* Fm, double* C, double* eps) {
  const double one = 1.0, zero = 0.0;
  PF_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_N, CUBLAS_OP_N, nbf, nbf, nbf, &one, Fm, nbf, X, nbf, &zero, W1, nbf));
  PF_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_T, CUBLAS_OP_N, nbf, nbf, nbf, &one, X, nbf, W1, nbf, &zero, W2, nbf));
  PF_CUSOLVER(cusolverDnDsyevd(cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nbf, W2, nbf, eps,
                               syev_work.as<double>(), syev_lwork, info_dev));
  PF_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_N, CUBLAS_OP_N, nbf, nbf, nbf, &one, X, nbf, W2, nbf, &zero, C, nbf));
}

// P = scale * C_occ C_occ^T
void System::density_from(const double* C, int nocc, double scale, double* Pm) {
  const double zero = 0.0;
  if (nocc <= 0) {
    launch_zero(Pm, (size_t)nbf * nbf * sizeof(double), stream);
    return;
  }
  PF_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, nocc, &scale, C, nbf, C, nbf, &zero, Pm, nbf));
}

// Diagonal starting density from atomic aufbau occupations of the
// minimal-basis shells: Z electrons per atom over 1s, 2s, 2p, ... (2 per s,
// 6 per p shell, in the order the basis lists them), scaled to nelec.
std::vector<double> atomic_occupations(const Basis& basis, const std::vector<int>& Z, int nelec) {
  const int natoms = (int)Z.size(), ns = (int)basis.shells.size();
  std::vector<double> occ(basis.nbf, 0.0);
  double total = 0.0;
  for (int a = 0; a < natoms; ++a) {
    std::vector<int> ss, ps, ds;
    for (int s = 0; s < ns; ++s)
      if (basis.shells[s].atom == a) (basis.shells[s].l == 0 ? ss : (basis.shells[s].l == 1 ? ps : ds)).push_back(s);
    std::vector<int> order;
    for (size_t k = 0; k < std::max(ss.size(), ps.size() + 1); ++k) {
      if (k < ss.size()) order.push_back(ss[k]);
      if (k >= 1 && k - 1 < ps.size()) order.push_back(ps[k - 1]);
    }
    // d shells (3d of Sc..Zn, core 3d/4d of heavier atoms) before the
    // outermost p shell: 4s then 3d then 4p
    if (!ds.empty() && !order.empty() && basis.shells[order.back()].l == 1)
      order.insert(order.end() - 1, ds.begin(), ds.end());
    else
      order.insert(order.end(), ds.begin(), ds.end());
    double left = Z[a];
    for (int s : order) {
      const int l = basis.shells[s].l, nf = (l + 1) * (l + 2) / 2;
      const double take = std::min(left, l == 0 ? 2.0 : (l == 1 ? 6.0 : 10.0));
      left -= take;
      for (int f = 0; f < nf; ++f) occ[basis.bf_off[s] + f] = take / nf;
      total += take;
    }
  }
  if (total > 0)
    for (double& v : occ) v *= (double)nelec / total;  // charge
  return occ;
}

std::vector<double> System::atomic_occupations() const {
  return pyfacc::atomic_occupations(basis, Z, nalpha + nbeta);
}

// The buffer X holds, read row-major, R = L^{-1} (cuBLAS wrote X = L^{-T}
// column-major), so X^T F X = R F R^T and X P' X^T = R^T P' R in the
// row-major products of dense.cu.
bool System::purify(const double* Fm, int nocc, double scale, double* Pm, double* Pp) {
  const int n = nbf;
  if (nocc > 0 && nocc < n) {  // F' = R F R^T into the graph's input
    launch_dgemm(n, n, n, false, Fm, n, true, X, n, W1, n, 1.0, nullptr, n, 0.0, false, false, stream);
    launch_dgemm(n, n, n, false, X, n, false, W1, n, Pu[0], n, 1.0, nullptr, n, 0.0, true, false, stream);
  }
  return purify_core(nocc, scale, Pm, Pp);
}

bool System::purify_orth(const double* Fp, int nocc, double scale, double* Pm, double* Pp) {
  if (nocc > 0 && nocc < nbf && Fp != Pu[0])
    PF_CUDA(cudaMemcpyAsync(Pu[0], Fp, (size_t)nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  return purify_core(nocc, scale, Pm, Pp);
}

// TC2 on F' (in Pu[0]): P = scale R^T P' R, and P' into Pp when given.
bool System::purify_core(int nocc, double scale, double* Pm, double* Pp) {
  const int n = nbf;
  const size_t bytes = (size_t)n * n * sizeof(double);
  if (nocc <= 0) {
    launch_zero(Pm, bytes, stream);
    if (Pp) launch_zero(Pp, bytes, stream);
    return true;
  }
  if (nocc >= n) {  // every orbital occupied: P = scale * X X^T = scale * S^-1, P' = I
    launch_dgemm(n, n, n, true, X, n, false, X, n, Pm, n, scale, nullptr, n, 0.0, true, false, stream);
    if (Pp) launch_identity(n, Pp, stream);
    return true;
  }
  double* Xa = Pu[1];
  // the whole TC2 iteration is one graph launch (conditional WHILE loop on
  // the device); the host reads the outcome once
  if (opt.verbose) PF_CUDA(cudaEventRecord(ctx.ev0, stream));
  PF_CUDA(cudaGraphLaunch(tc2_graph(nocc), stream));
  if (opt.verbose) PF_CUDA(cudaEventRecord(ctx.ev1, stream));
  // the outcome into pinned memory; the projector's copy and the
  // back-transform are queued before it is read, so they run while the host
  // waits (after a failed purification the eigensolver fallback overwrites
  // Pm, and the caller does not use Pp)
  double* ctl_pinned = ctx.pinned + PURIFY_PINNED;
  PF_CUDA(cudaMemcpyAsync(ctl_pinned, pstate + 8, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaEventRecord(ctx.ready, stream));
  if (Pp) PF_CUDA(cudaMemcpyAsync(Pp, Xa, bytes, cudaMemcpyDeviceToDevice, stream));
  // P = scale R^T Xp R
  launch_dgemm(n, n, n, false, Xa, n, false, X, n, W1, n, 1.0, nullptr, n, 0.0, false, false, stream);
  launch_dgemm(n, n, n, true, X, n, false, W1, n, Pm, n, scale, nullptr, n, 0.0, true, false, stream);
  PF_CUDA(cudaEventSynchronize(ctx.ready));
  double ctl[8];
  std::memcpy(ctl, ctl_pinned, sizeof(ctl));
  const int steps = (int)ctl[2];
  count_launches(2 + (steps + TC2_BODY_STEPS - 1) / TC2_BODY_STEPS * TC2_BODY_STEPS);
  purify_steps += steps;
  if (opt.verbose) purify_ms += elapsed(ctx.ev0, ctx.ev1);
  return !(ctl[1] == 0.0 || ctl[4] != 0.0);
}

// The purification graph of one occupation number (dense.cu): built once
// per system and occupation, replayed by every purify() of that occupation.
cudaGraphExec_t System::tc2_graph(int nocc) {
  for (auto& g : tc2_graphs)
    if (g.first == nocc) return g.second;
  cudaGraphExec_t exec = build_tc2_graph(nbf, nocc, Pu[0], Pu[1], Pu[3], pstate, TC2_KMAX);
  tc2_graphs.emplace_back(nocc, exec);
  return exec;
}

// New density from a Fock matrix: purification, or eigenvectors when the
// purification does not converge (no gap at the occupation number).
bool System::density_step(const double* Fm, int nocc, double scale, double* Pm, double* C, double* eps,
                          double* Pp) {
  if (purify(Fm, nocc, scale, Pm, Pp)) return Pp != nullptr;
  purify_fallbacks++;
  diagonalize(Fm, C, eps);
  density_from(C, nocc, scale, Pm);
  return false;
}

bool System::density_step_orth(const double* Fp, int nocc, double scale, double* Pm, double* C, double* eps,
                               double* Pp) {
  if (purify_orth(Fp, nocc, scale, Pm, Pp)) return Pp != nullptr;
  purify_fallbacks++;
  diagonalize_orth(Fp, C, eps);
  density_from(C, nocc, scale, Pm);
  return false;
}

// Orbitals of the final Fock matrices, for the caller's outputs.
void System::final_orbitals() {
  if (orbitals_ready) return;
  const int nsp = uhf ? 2 : 1;
  for (int s = 0; s < nsp; ++s) diagonalize(F[s], Cm[s], eps_dev + s * nbf);
  orbitals_ready = true;
}

static bool solve_small(int m, std::vector<double> A, std::vector<double> b, std::vector<double>& x) {
  // Gaussian elimination with partial pivoting on an m x m system.
  for (int c = 0; c < m; ++c) {
    int piv = c;
    for (int r = c + 1; r < m; ++r)
      if (std::fabs(A[r * m + c]) > std::fabs(A[piv * m + c])) piv = r;
    if (std::fabs(A[piv * m + c]) < 1e-300) return false;
    if (piv != c) {
      for (int k = 0; k < m; ++k) std::swap(A[c * m + k], A[piv * m + k]);
      std::swap(b[c], b[piv]);
    }
    for (int r = c + 1; r < m; ++r) {
      const double f = A[r * m + c] / A[c * m + c];
      for (int k = c; k < m; ++k) A[r * m + k] -= f * A[c * m + k];
      b[r] -= f * b[c];
    }
  }
  x.assign(m, 0.0);
  for (int r = m - 1; r >= 0; --r) {
    double s = b[r];
    for (int k = r + 1; k < m; ++k) s -= A[r * m + k] * x[k];
    x[r] = s / A[r * m + r];
  }
  for (double v : x)
    if (!std::isfinite(v)) return false;
  return true;
}

void System::run_scf() {
  const size_t n2 = (size_t)nbf * nbf;
  const int nsp = uhf ? 2 : 1;
  const int nocc[2] = {uhf ? nalpha : (nalpha + nbeta + 1) / 2, uhf ? nbeta : 0};  // rscf.f90:54-55
  const double pscale = uhf ? 1.0 : 2.0;
  const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
  const bool incremental = opt.incremental < 0 ? mixed : (opt.incremental != 0);
  // Incremental builds of mixed mode may screen harder: the reported energy
  // comes from a full FP64 build at the converged density, and an error
  // delta in F only moves that density by O(delta), the energy by O(delta^2).
  const double inc_thresh =
      (mixed && opt.incremental_thresh > 0) ? std::max(opt.incremental_thresh, opt.schwarz_thresh) : opt.schwarz_thresh;
  st = ScfState();
  PF_CUDA(cudaMemsetAsync(stats_dev, 0, sizeof(JkStats), stream));
  cudaEvent_t t0, t1, a0, a1;
  PF_CUDA(cudaEventCreate(&t0));
  PF_CUDA(cudaEventCreate(&t1));
  PF_CUDA(cudaEventCreate(&a0));
  PF_CUDA(cudaEventCreate(&a1));
  cudaEvent_t d0, d1;
  PF_CUDA(cudaEventCreate(&d0));
  PF_CUDA(cudaEventCreate(&d1));
  bool diag_pending = false;
  // one-electron matrices, the overlap factor and the starting density are
  // queued without a synchronisation; their timings and the factor's status
  // are read at the first one (the first iteration's readback)
  cudaEvent_t q1, q2;
  PF_CUDA(cudaEventCreate(&q1));
  PF_CUDA(cudaEventCreate(&q2));
  PF_CUDA(cudaEventRecord(t0, stream));
  one_electron();
  PF_CUDA(cudaEventRecord(q1, stream));
  orthogonalizer();
  PF_CUDA(cudaEventRecord(q2, stream));
  float ms_orth = 0.0f;
  bool ortho_checked = false;
  auto ortho_check = [&]() {
    if (ortho_checked) return;
    check_overlap_factor();
    st.ms_1e = elapsed(t0, q1);
    ms_orth = elapsed(q1, q2);
    ortho_checked = true;
  };
  orbitals_ready = false;
  purify_steps = purify_fallbacks = 0;
  purify_ms = 0.0;
  // DIIS on the orthonormal-basis Fock matrices F' = R F R^T: with P =
  // scale R^T P' R the error R (F P S - S P F) R^T is scale (F' P' - P' F'),
  // and the extrapolated F' goes to the purification as it is (5 dense
  // products per iteration instead of 8).  pp_ok: Pp holds P' of the
  // current density (not after the atomic guess or an eigensolver fallback).
  const bool orth_diis = opt.diis_size > 0;
  bool pp_ok[2] = {false, false};
  if (opt.guess == PYFACC_GUESS_CORE) {
    // core-Hamiltonian guess (rscf.f90:113-114, uscf.f90:140-144): it uses
    // the factor, so its status is read first
    PF_CUDA(cudaStreamSynchronize(stream));
    ortho_check();
    for (int s = 0; s < nsp; ++s) pp_ok[s] = density_step(H, nocc[s], pscale, P[s], Cm[s], eps_dev + s * nbf, Pp[s]);
  } else {
    // atomic occupations on the diagonal (occ_dev, uploaded with the system)
    const double ne = (double)(nalpha + nbeta);
    for (int s = 0; s < nsp; ++s) {
      const double f = uhf ? (s == 0 ? nalpha : nbeta) / ne : 1.0;
      launch_set_diag(nbf, occ_dev, f, P[s], stream);
    }
  }
  for (int s = 0; s < nsp; ++s) launch_zero(Pbuilt[s], n2 * sizeof(double), stream);
  launch_zero(J, n2 * sizeof(double), stream);
  for (int s = 0; s < nsp; ++s) launch_zero(K[s], n2 * sizeof(double), stream);

  const int ndiis = std::max(opt.diis_size, 0);
  for (int k = 0; k < ndiis; ++k) {
    launch_zero(diis_F[k], 2 * n2 * sizeof(double), stream);
    launch_zero(diis_E[k], 2 * n2 * sizeof(double), stream);
  }
  if (ndiis > 0) {  // the stored error vectors, for the overlaps of each new one
    std::vector<const double*> ys(ndiis);
    for (int k = 0; k < ndiis; ++k) ys[k] = diis_E[k];
    PF_CUDA(cudaMemcpyAsync(ptrs_dev, ys.data(), ndiis * sizeof(double*), cudaMemcpyHostToDevice, stream));
  }
  int nhist = 0, head = 0;
  std::vector<double> Bm;  // DIIS overlap matrix of the stored error vectors
  const int cap = std::max(ndiis, 1);
  Bm.assign(cap * cap, 0.0);
  std::vector<int> slot_age(cap, -1);
  double E_old = 0.0;
  double ms_fock = 0.0, ms_diag = 0.0;
  int since_full = 0;
  // Dynamic precision (Luehr, Ufimtsev and Martinez, JCTC 7, 949 (2011)):
  // while the DIIS error is above coarse_err every quartet runs in FP32;
  // the first build after that is a full mixed build, so the incremental
  // chain that produces the converged density starts afresh and carries no
  // error of the coarse builds.
  bool coarse = mixed && opt.coarse_err > 0 && opt.shard_count <= 1;
  bool restart = false;
  const double t32_coarse = 1e300;
  const double coarse_base = std::max(COARSE_SCREEN, opt.schwarz_thresh);
  double err_prev = -1.0;  // DIIS error of the previous iteration (none before the first)
  const double* Pspin[2] = {P[0], P[1]};
  for (int it = 1; it <= opt.max_iter; ++it) {
    st.n_iter = it;
    // ---- Fock build
    PF_CUDA(cudaEventRecord(a0, stream));
    const bool full = !incremental || it == 1 || restart || since_full + 1 >= std::max(opt.rebuild_every, 1);
    const bool coarse_build = coarse;
    // the coarse threshold follows the DIIS error: COARSE_SCREEN once the
    // error nears coarse_err, up to COARSE_SCREEN_SPAN times looser while
    // it is far above (the first build, with no error yet, at the loosest)
    const double span = (err_prev < 0 || opt.coarse_err <= 0)
                            ? COARSE_SCREEN_SPAN
                            : std::min(COARSE_SCREEN_SPAN, std::max(1.0, err_prev / opt.coarse_err));
    const double coarse_screen = coarse_base * span;
    const double t32 = coarse_build ? t32_coarse : -1.0;
    // a mixed full build (the restart after the coarse phase, periodic
    // rebuilds) screens like the incremental ones
    const double full_thresh = coarse_build ? coarse_screen : (mixed ? inc_thresh : -1.0);
    const double step_thresh = coarse_build ? std::max(coarse_screen, inc_thresh) : inc_thresh;
    restart = false;
    double* Kp[2] = {K[0], K[1]};
    // Without a shard reducer J and K hold the unsymmetrised halves Jh, Kh
    // (J = Jh + Jh^T): an incremental build adds into them in place and the
    // Fock matrix is assembled from them (launch_fock_half).  With one, they
    // are the full matrices summed over the shards.
    const bool half = !reducer;
    if (full) {
      if (uhf) {
        launch_axpby((long long)n2, 1.0, P[0], 0.0, W3, stream);
        launch_axpby((long long)n2, 1.0, P[1], 1.0, W3, stream);
        jk(W3, 2, Pspin, J, Kp, opt.precision, mixed, full_thresh, t32, half ? JK_HALF : JK_FULL);
      } else {
        jk(P[0], 1, Pspin, J, Kp, opt.precision, mixed, full_thresh, t32, half ? JK_HALF : JK_FULL);
      }
      since_full = 0;
    } else {
      // dP = P - P_built (and P_built = P); J += J[dP], K += K[dP]
      double* dP[2] = {Err[0], Err[1]};
      for (int s = 0; s < nsp; ++s) launch_diff_update((long long)n2, P[s], Pbuilt[s], dP[s], stream);
      const double* dPc[2] = {dP[0], dP[1]};
      const double* dPj = dP[0];
      if (uhf) {
        launch_axpby((long long)n2, 1.0, dP[0], 0.0, Wm, stream);
        launch_axpby((long long)n2, 1.0, dP[1], 1.0, Wm, stream);
        dPj = Wm;
      }
      if (half) {
        jk(dPj, nsp, dPc, J, Kp, opt.precision, mixed, step_thresh, t32, JK_ADD);
      } else {
        double* dK[2] = {W2, W3};
        jk(dPj, nsp, dPc, W1, dK, opt.precision, mixed, step_thresh, t32);
        launch_axpby((long long)n2, 1.0, W1, 1.0, J, stream);
        for (int s = 0; s < nsp; ++s) launch_axpby((long long)n2, 1.0, dK[s], 1.0, K[s], stream);
      }
      since_full++;
    }
    if (full)
      for (int s = 0; s < nsp; ++s)
        PF_CUDA(cudaMemcpyAsync(Pbuilt[s], P[s], n2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    for (int s = 0; s < nsp; ++s) {
      if (half) launch_fock_half(nbf, H, J, uhf ? 1.0 : 0.5, K[s], F[s], stream);
      else launch_fock((long long)n2, H, J, uhf ? 1.0 : 0.5, K[s], F[s], stream);
    }
    PF_CUDA(cudaEventRecord(a1, stream));
    // ---- DIIS error X^T (F P S - S P F) X and energy
    // R (F P S - S P F) R^T with R = L^{-1} the row-major view of X (the
    // error's sign and transpose do not matter: only max |E| and <E_i, E_j>
    // are used); FPS - SPF = A - A^T with A = F P S, or scale (F'P' - P'F')
    // = B - B^T with B = scale F' P' when P' is known
    int slot = -1;
    if (ndiis > 0) {
      slot = head;
      head = (head + 1) % ndiis;
    }
    const bool use_pp = orth_diis && pp_ok[0] && (nsp == 1 || pp_ok[1]);
    double* Eo[2] = {Err[0], Err[1]};
    for (int s = 0; s < nsp; ++s) {
      if (slot >= 0) Eo[s] = diis_E[slot] + s * n2;
      if (orth_diis) {  // F' = R F R^T, the stored DIIS vector
        double* Fo = diis_F[slot] + s * n2;
        launch_dgemm(nbf, nbf, nbf, false, F[s], nbf, true, X, nbf, W1, nbf, 1.0, nullptr, nbf, 0.0, false, false,
                     stream);
        launch_dgemm(nbf, nbf, nbf, false, X, nbf, false, W1, nbf, Fo, nbf, 1.0, nullptr, nbf, 0.0, true, false,
                     stream);
        if (use_pp) {
          launch_dgemm(nbf, nbf, nbf, false, Fo, nbf, false, Pp[s], nbf, W1, nbf, pscale, nullptr, nbf, 0.0, false,
                       false, stream);
          launch_antisym(nbf, W1, Eo[s], stream);
          continue;
        }
      }
      launch_dgemm(nbf, nbf, nbf, false, F[s], nbf, false, P[s], nbf, W1, nbf, 1.0, nullptr, nbf, 0.0, false, false,
                   stream);
      launch_dgemm(nbf, nbf, nbf, false, W1, nbf, false, S, nbf, W2, nbf, 1.0, nullptr, nbf, 0.0, false, false,
                   stream);
      launch_dgemm(nbf, nbf, nbf, false, W2, nbf, true, X, nbf, W1, nbf, 1.0, nullptr, nbf, 0.0, false, true,
                   stream);
      launch_dgemm(nbf, nbf, nbf, false, X, nbf, false, W1, nbf, Eo[s], nbf, 1.0, nullptr, nbf, 0.0, false, false,
                   stream);
    }
    // energy, errors and (DIIS: F' and the error vector are in their slot)
    // the overlaps of the new error vector with the stored ones, one launch
    launch_scf_reduce((long long)n2, uhf ? 1 : 0, H, P[0], uhf ? P[1] : nullptr, F[0], uhf ? F[1] : nullptr, Eo[0],
                      uhf ? Eo[1] : nullptr, it > 1 ? Pold[0] : nullptr, uhf ? Pold[1] : nullptr, small, red_part, stream,
                      (long long)nsp * n2, ndiis > 0 ? diis_E[slot] : nullptr, ndiis, ptrs_dev, small + 8);
    // energy, errors and DIIS overlaps into pinned memory; the copy of P
    // for the next iteration's |dP| runs while the host waits
    const int nred = 8 + std::max(ndiis, 0);
    PF_CUDA(cudaMemcpyAsync(ctx.pinned, small, nred * sizeof(double), cudaMemcpyDeviceToHost, stream));
    PF_CUDA(cudaEventRecord(ctx.ready, stream));
    for (int s = 0; s < nsp; ++s)
      PF_CUDA(cudaMemcpyAsync(Pold[s], P[s], n2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    PF_CUDA(cudaEventSynchronize(ctx.ready));
    double red[8 + 64];
    std::memcpy(red, ctx.pinned, nred * sizeof(double));
    ortho_check();
    if (diag_pending) {  // the previous iteration's density step, timed now
      ms_diag += elapsed(d0, d1);
      diag_pending = false;
    }
    const float ms_build = elapsed(a0, a1);
    ms_fock += ms_build;
    const double E = 0.5 * red[0];
    const double err = red[1];
    err_prev = err;
    const double dD = std::sqrt(red[2]);
    const double dE = std::fabs(E - E_old);
    st.last_de = dE;
    st.last_err = err;
    st.e_elec = E;
    st.energy = E + e_nuc;
    if (opt.verbose)
      std::fprintf(stderr, "pyfacc iter %3d  E = %.12f  dE = %.3e  err = %.3e  |dD| = %.3e  %s%s build %.3f ms\n", it,
                   E + e_nuc, dE, err, dD, coarse_build ? "FP32 " : "", full ? "full" : "incremental", ms_build);
    // In mixed precision the energy of incremental FP32/FP64 builds carries
    // a ~1e-10 noise floor; the density is converged on the commutator and
    // the energy is then taken from one full FP64 build (below).
    const double e_tol = mixed ? std::max(opt.eps_energy, 1e-8) : opt.eps_energy;
    bool conv = !coarse_build && dE < e_tol && err < opt.eps_diis;
    if (opt.eps_density > 0) conv = conv && it > 1 && dD < opt.eps_density;
    if (coarse && (err < opt.coarse_err || it >= COARSE_MAX_ITER)) {
      coarse = false;
      restart = true;
    }
    if (conv) {
      st.converged = true;
      break;
    }
    E_old = E;
    // ---- extrapolate
    const double* Fuse[2] = {F[0], F[1]};
    if (orth_diis) {
      Fuse[0] = diis_F[slot];
      Fuse[1] = diis_F[slot] + n2;
    }
    if (ndiis > 0) {
      slot_age[slot] = it;
      for (int k = 0; k < ndiis; ++k) {
        Bm[slot * cap + k] = red[8 + k];
        Bm[k * cap + slot] = red[8 + k];
      }
      nhist = std::min(nhist + 1, ndiis);
      if (nhist >= 2) {
        std::vector<int> use;
        for (int k = 0; k < ndiis; ++k)
          if (slot_age[k] >= 0) use.push_back(k);
        // drop the oldest vectors until the system is solvable
        while (use.size() >= 2) {
          const int m = (int)use.size();
          std::vector<double> A((m + 1) * (m + 1), 0.0), b(m + 1, 0.0), x;
          double scl = 0.0;
          for (int i = 0; i < m; ++i) scl = std::max(scl, std::fabs(Bm[use[i] * cap + use[i]]));
          scl = scl > 0 ? 1.0 / scl : 1.0;
          for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) A[i * (m + 1) + j] = Bm[use[i] * cap + use[j]] * scl;
            A[i * (m + 1) + m] = -1.0;
            A[m * (m + 1) + i] = -1.0;
          }
          b[m] = -1.0;
          if (solve_small(m + 1, A, b, x)) {
            // F'_diis = sum c_i F'_i (into W3 / Wm as the stacked spins; a
            // closed shell's straight into the purification's input)
            double* Fd = uhf ? W3 : Pu[0];
            std::vector<const double*> src(m);
            for (int i = 0; i < m; ++i) src[i] = diis_F[use[i]];
            launch_lincomb((long long)n2, m, src.data(), x.data(), Fd, stream);
            if (uhf) {
              for (int i = 0; i < m; ++i) src[i] = diis_F[use[i]] + n2;
              launch_lincomb((long long)n2, m, src.data(), x.data(), Wm, stream);
            }
            Fuse[0] = Fd;
            Fuse[1] = Wm;
            break;
          }
          int oldest = 0;
          for (int i = 1; i < (int)use.size(); ++i)
            if (slot_age[use[i]] < slot_age[use[oldest]]) oldest = i;
          slot_age[use[oldest]] = -1;
          use.erase(use.begin() + oldest);
        }
      }
    }
    // ---- diagonalise and rebuild the density (timed at the next sync, so
    // the host queues the next Fock build while this one runs)
    PF_CUDA(cudaEventRecord(d0, stream));
    for (int s = 0; s < nsp; ++s)
      pp_ok[s] = orth_diis ? density_step_orth(Fuse[s], nocc[s], pscale, P[s], Cm[s], eps_dev + s * nbf, Pp[s])
                           : density_step(Fuse[s], nocc[s], pscale, P[s], Cm[s], eps_dev + s * nbf);
    PF_CUDA(cudaEventRecord(d1, stream));
    diag_pending = true;
  }
  if (diag_pending) {
    PF_CUDA(cudaEventSynchronize(d1));
    ms_diag += elapsed(d0, d1);
    diag_pending = false;
  }
  if (mixed && st.converged && opt.polish) {
    // FP64 polish: F and E of the converged density from one full FP64 build
    PF_CUDA(cudaEventRecord(a0, stream));
    double* Kp[2] = {K[0], K[1]};
    if (uhf) {
      launch_axpby((long long)n2, 1.0, P[0], 0.0, W3, stream);
      launch_axpby((long long)n2, 1.0, P[1], 1.0, W3, stream);
      jk(W3, 2, Pspin, J, Kp, PYFACC_PRECISION_FP64);
    } else {
      jk(P[0], 1, Pspin, J, Kp, PYFACC_PRECISION_FP64);
    }
    for (int s = 0; s < nsp; ++s) launch_fock((long long)n2, H, J, uhf ? 1.0 : 0.5, K[s], F[s], stream);
    PF_CUDA(cudaEventRecord(a1, stream));
    launch_scf_reduce((long long)n2, uhf ? 1 : 0, H, P[0], uhf ? P[1] : nullptr, F[0], uhf ? F[1] : nullptr, Err[0],
                      uhf ? Err[1] : nullptr, nullptr, nullptr, small, red_part, stream);
    double red[4];
    PF_CUDA(cudaMemcpyAsync(red, small, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    PF_CUDA(cudaStreamSynchronize(stream));
    ms_fock += elapsed(a0, a1);
    st.last_de = std::fabs(0.5 * red[0] - st.e_elec);
    st.e_elec = 0.5 * red[0];
    st.energy = st.e_elec + e_nuc;
  }
  PF_CUDA(cudaEventRecord(t1, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  ortho_check();  // (no iteration ran)
  st.ms_total = elapsed(t0, t1);
  st.ms_fock = ms_fock;
  st.ms_diag = ms_diag;
  if (opt.verbose)
    std::fprintf(stderr, "pyfacc phases (ms): total %.3f  one-electron %.3f  orthogonaliser %.3f  Fock %.3f  "
                 "density %.3f  rest (DIIS, energy, guess) %.3f\n", st.ms_total, st.ms_1e, ms_orth, ms_fock, ms_diag,
                 st.ms_total - st.ms_1e - ms_orth - ms_fock - ms_diag);
  if (opt.verbose)
    std::fprintf(stderr, "pyfacc purification: %d TC2 steps in all, %.3f ms in the TC2 graphs, %d eigensolver "
                 "fallbacks\n", purify_steps, purify_ms, purify_fallbacks);
  JkStats js;
  PF_CUDA(cudaMemcpy(&js, stats_dev, sizeof(JkStats), cudaMemcpyDeviceToHost));
  st.quartets[0] = st.quartets[1] = 0;
  st.flops_fock = 0.0;
  const int nk = uhf ? 2 : 1;
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < NQCLASS; ++q) {
      st.quartets[p] += js.quartets[p][q];
      const ClassFlops& cf = class_flops(q);
      st.flops_fock += (double)js.prims[p][q] * (cf.vrr + prim_overhead_flops(q, p == 1)) +
                       (double)js.quartets[p][q] * (cf.hrr + digest_flops(q, nk));
    }
  st.done = true;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(a0);
  cudaEventDestroy(a1);
  cudaEventDestroy(d0);
  cudaEventDestroy(d1);
  cudaEventDestroy(q1);
  cudaEventDestroy(q2);
}

// Analytic gradient of the converged SCF:
//   dE/dR = sum P dH - sum W dS + 1/2 sum Gamma d(mn|ls) + dV_nn
void System::gradient(double* g_host) {
  if (!st.done) throw Error(PYFACC_ERR_NOT_READY, "gradient requested before the SCF");
  const size_t n2 = (size_t)nbf * nbf;
  cudaEvent_t a0, a1;
  PF_CUDA(cudaEventCreate(&a0));
  PF_CUDA(cudaEventCreate(&a1));
  PF_CUDA(cudaEventRecord(a0, stream));
  // Energy-weighted density without orbitals: at convergence
  // sum_occ eps_i c_i c_i^T = P_s F_s P_s (UHF), = P F P / 4 for the RHF
  // total density P = 2 C_occ C_occ^T, and W = 2 x that for RHF.
  const int nsp = uhf ? 2 : 1;
  for (int s = 0; s < nsp; ++s) {
    const double f = uhf ? 1.0 : 0.5;
    launch_dgemm(nbf, nbf, nbf, false, F[s], nbf, false, P[s], nbf, W1, nbf, 1.0, nullptr, nbf, 0.0, false, false,
                 stream);
    launch_dgemm(nbf, nbf, nbf, false, P[s], nbf, false, W1, nbf, Wm, nbf, f, s == 0 ? nullptr : Wm, nbf, 1.0, true,
                 false, stream);
  }
  // total density and spin densities of the converged SCF
  double* Pt = W2;
  double* Ps[2] = {P[0], uhf ? P[1] : P[0]};
  if (uhf) {
    launch_axpby((long long)n2, 1.0, P[0], 0.0, Pt, stream);
    launch_axpby((long long)n2, 1.0, P[1], 1.0, Pt, stream);
  } else {
    Pt = P[0];
  }
  launch_zero(grad_dev, 3 * natoms * sizeof(double), stream);
  OneEGradArgs g1;
  g1.natoms = natoms;
  g1.atoms = atoms_dev;
  g1.boys_mode = opt.boys_mode;
  g1.P = Pt;
  g1.W = Wm;
  g1.nbf = nbf;
  g1.grad = grad_dev;
  g1.natoms_total = natoms;
  // one-electron terms once (shard 0); the two-electron term is sharded
  if (opt.shard_count <= 1 || opt.shard_rank == 0) launch_grad1e(shd, n1e, pairs1e, g1, num_sms, stream);
  launch_dmax(ns, bf_off_dev, nfun_dev, nbf, Pt, nullptr, nullptr, dmax, stream);
  GradArgs g2;
  g2.Pt = Pt;
  g2.Pa = uhf ? Ps[0] : Pt;
  g2.Pb = uhf ? Ps[1] : Pt;
  g2.dmax = opt.schwarz_thresh > 0 ? dmax : nullptr;
  g2.ns_ld = ns;
  // a mixed gradient screens its quartets at GRAD_SCREEN_MIXED (its FP32
  // half already carries errors well above what that drops)
  const bool gmix = opt.gradient_precision == PYFACC_PRECISION_MIXED ||
                    (opt.gradient_precision < 0 && opt.precision == PYFACC_PRECISION_MIXED);
  const double gthr = gmix ? std::max(opt.schwarz_thresh, GRAD_SCREEN_MIXED) : opt.schwarz_thresh;
  g2.thresh = gthr;
  g2.prim_thresh = gthr * PRIM_QUARTET_REL_GRAD * grad_prim_cut_scale(basis);
  g2.natoms_total = natoms;
  g2.uhf = uhf ? 1 : 0;
  g2.grad = grad_dev;
  unsigned long long* gstats = stats_dev;  // reuse the J/K counters' space
  PF_CUDA(cudaMemsetAsync(gstats, 0, 2 * NQCLASS * sizeof(unsigned long long), stream));
  g2.stats = gstats;
  // FP32 derivative integrals for the small quartets on request, or by
  // default in mixed mode (C20H42: 3.30 -> 3.18 ms, C100H202 80 -> 75 ms).  One
  // process splits at Q_ab Q_cd max|P| = gradient_fp32_thresh with lists
  // built on the device; shards use their static lists (split at fp32_thresh).
  const bool split = pd.primf != nullptr &&
                     (opt.gradient_precision == PYFACC_PRECISION_MIXED ||
                      (opt.gradient_precision < 0 && opt.precision == PYFACC_PRECISION_MIXED));
  const bool dyn_split = split && opt.shard_count <= 1;
  if (dyn_split)
    launch_dyn_tasks(pd, dmax, ns, gthr,
                     opt.gradient_fp32_thresh > 0 ? opt.gradient_fp32_thresh : opt.fp32_thresh, dyn, stream);
  // the FP64 and FP32 halves run on different streams, which swap from
  // class to class (an FP64 gradient keeps its classes on one stream: its
  // register-heavy kernels measured slower when two of them share the SMs)
  cudaStream_t s32 = ctx.side;
  PF_CUDA(cudaEventRecord(ctx.fork, stream));
  PF_CUDA(cudaStreamWaitEvent(ctx.side, ctx.fork, 0));
  int nth = 0;
  for (int bc = NCLASS - 1; bc >= 0; --bc)
    for (int kc = bc; kc >= 0; --kc, ++nth) {
      if (dyn_split) {
        const int qc = (bc == 0) ? 0 : (bc == 1 ? 1 + kc : 3 + kc);
        launch_grad2e(pd, dyn.lists[2 * qc], bc, kc, false, g2, num_sms, (nth & 1) ? s32 : stream);
        launch_grad2e(pd, dyn.lists[2 * qc + 1], bc, kc, true, g2, num_sms, (nth & 1) ? stream : s32);
      } else if (split) {
        launch_grad2e(pd, tasks[bc][kc][1], bc, kc, false, g2, num_sms, stream);
        launch_grad2e(pd, tasks[bc][kc][2], bc, kc, true, g2, num_sms, s32);
      } else {
        launch_grad2e(pd, tasks[bc][kc][0], bc, kc, false, g2, num_sms, stream);
      }
    }
  if (has_d)
    for (int bc = NCLASS; bc < NPAIRCLASS; ++bc)
      for (int kc = 0; kc <= bc; ++kc) launch_grad2e_d(pd, tasks[bc][kc][0], bc, kc, g2, num_sms, stream);
  PF_CUDA(cudaEventRecord(ctx.join, ctx.side));
  PF_CUDA(cudaStreamWaitEvent(stream, ctx.join, 0));
  if (reducer) reduce(grad_dev, 3LL * natoms);
  PF_CUDA(cudaEventRecord(a1, stream));
  std::vector<double> g(3 * natoms, 0.0);
  PF_CUDA(cudaMemcpyAsync(g.data(), grad_dev, 3 * natoms * sizeof(double), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  st.ms_grad = elapsed(a0, a1);
  unsigned long long cnt[2 * NQCLASS];
  PF_CUDA(cudaMemcpy(cnt, gstats, sizeof(cnt), cudaMemcpyDeviceToHost));
  st.flops_grad = 0.0;
  for (int q = 0; q < NQCLASS; ++q)
    st.flops_grad += (double)cnt[NQCLASS + q] * (class_flops(q).grad + prim_overhead_flops(q, false)) +
                       (double)cnt[q] * class_flops(q).gfin;
  nuclear_repulsion_gradient(g.data());
  grad_host = g;
  if (g_host) std::memcpy(g_host, g.data(), g.size() * sizeof(double));
  cudaEventDestroy(a0);
  cudaEventDestroy(a1);
}

static void copy_out(cudaStream_t s, double* host, const double* dev, size_t n) {
  if (host) PF_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
}

// Device matrices are symmetric (layout-free) except C, which is
// column-major (orbital j = column j) and is returned as such.
void System::fill_result(pyfacc_result* r) {
  const size_t n2 = (size_t)nbf * nbf;
  r->energy = st.energy;
  r->e_elec = st.e_elec;
  r->e_nuc = e_nuc;
  r->converged = st.converged ? 1 : 0;
  r->n_iter = st.n_iter;
  r->scf_type = uhf ? PYFACC_SCF_UHF : PYFACC_SCF_RHF;
  r->nbf = nbf;
  r->nshell = ns;
  r->n_fock_builds = st.n_fock;
  r->last_delta_e = st.last_de;
  r->last_diis_error = st.last_err;
  copy_out(stream, r->S, S, n2);
  copy_out(stream, r->T, T, n2);
  copy_out(stream, r->V, Vm, n2);
  if (r->P) {
    if (uhf) {
      launch_axpby((long long)n2, 1.0, P[0], 0.0, W1, stream);
      launch_axpby((long long)n2, 1.0, P[1], 1.0, W1, stream);
      copy_out(stream, r->P, W1, n2);
    } else {
      copy_out(stream, r->P, P[0], n2);
    }
  }
  if (r->C_alpha || r->C_beta || r->eps_alpha || r->eps_beta) final_orbitals();
  copy_out(stream, r->C_alpha, Cm[0], n2);
  copy_out(stream, r->C_beta, Cm[uhf ? 1 : 0], n2);
  copy_out(stream, r->eps_alpha, eps_dev, nbf);
  copy_out(stream, r->eps_beta, eps_dev + (uhf ? nbf : 0), nbf);
  PF_CUDA(cudaStreamSynchronize(stream));
  if (r->gradient && !grad_host.empty()) std::memcpy(r->gradient, grad_host.data(), grad_host.size() * sizeof(double));
  r->ms_total = st.ms_total;
  r->ms_one_electron = st.ms_1e;
  r->ms_fock = st.ms_fock;
  r->ms_diag = st.ms_diag;
  r->ms_gradient = st.ms_grad;
  r->quartets_fp64 = (long long)st.quartets[0];
  r->quartets_fp32 = (long long)st.quartets[1];
  r->flops_fock = st.flops_fock;
  r->flops_gradient = st.flops_grad;
  r->task_width = task_width;
}

void System::set_coords(const double* coords) {
  xyz.assign(coords, coords + 3 * natoms);
  for (auto& sh : basis.shells)
    for (int x = 0; x < 3; ++x) sh.c[x] = xyz[3 * sh.atom + x];
  e_nuc = nuclear_repulsion();
  upload_shells();
  build_pairs();
  st = ScfState();
  one_e_done = false;
  grad_host.clear();
}

}  // namespace pyfacc
