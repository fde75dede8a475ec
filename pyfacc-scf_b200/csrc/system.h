// The opaque pyfacc_system of the C ABI: one molecule resident on one GPU.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <string>
#include <vector>

#include "engine.h"
#include "pool.h"

namespace pyfacc {

struct ScfState {
  bool done = false;
  bool converged = false;
  int n_iter = 0;
  int n_fock = 0;
  double energy = 0.0, e_elec = 0.0;
  double last_de = 0.0, last_err = 0.0;
  double ms_total = 0, ms_1e = 0, ms_fock = 0, ms_diag = 0, ms_grad = 0;
  unsigned long long quartets[2] = {0, 0};
  double flops_fock = 0.0, flops_grad = 0.0;
};

struct System {
  System(const pyfacc_molecule& m, const pyfacc_options& o);
  ~System();
  System(const System&) = delete;
  System& operator=(const System&) = delete;

  // ---- configuration and molecule
  pyfacc_options opt;
  int device = 0, num_sms = 148;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  GpuContext ctx;
  int natoms = 0, charge = 0, nalpha = 0, nbeta = 0;
  bool uhf = false;
  std::vector<int> Z;
  std::vector<double> xyz;
  std::vector<std::string> species;
  std::string basis_name, basis_file;
  Basis basis;
  int nbf = 0, ns = 0;
  double e_nuc = 0.0;

  // ---- device data
  ShellDev shd;
  double4* atoms_dev = nullptr;
  int2* pairs1e[NPAIRCLASS] = {};  // per pair class ss, ps, pp, ds, dp, dd (l_a >= l_b)
  int n1e[NPAIRCLASS] = {};
  int* bf_off_dev = nullptr;
  int* nfun_dev = nullptr;
  PairData pd;
  // [bra class][ket class][full fp64 | mixed fp64 | mixed fp32]; the d
  // classes (3..5) use the full lists only (their quartets stay in FP64)
  TaskList tasks[NPAIRCLASS][NPAIRCLASS][3];
  bool has_d = false;  // the basis holds d shells
  DeviceBuf task_buf;
  long long quartets_total = 0;
  DynTaskSet dyn;          // per-build task lists (mixed precision)
  DeviceBuf dyn_buf;

  DeviceBuf mats;
  double *S = nullptr, *T = nullptr, *Vm = nullptr, *H = nullptr, *X = nullptr;
  double *F[2] = {nullptr, nullptr}, *J = nullptr, *K[2] = {nullptr, nullptr};
  double *P[2] = {nullptr, nullptr}, *Pbuilt[2] = {nullptr, nullptr}, *Pold[2] = {nullptr, nullptr};
  double *W1 = nullptr, *W2 = nullptr, *W3 = nullptr, *Err[2] = {nullptr, nullptr};
  double *Cm[2] = {nullptr, nullptr}, *Wm = nullptr, *small = nullptr;
  double* red_part = nullptr;  // partial sums of the DIIS / energy reductions
  double *Pu[4] = {nullptr, nullptr, nullptr, nullptr};  // purification work matrices
  double *Pp[2] = {nullptr, nullptr};  // projectors P' of the current density per spin (P = scale R^T P' R)
  double* pstate = nullptr;                      // TC2 state, two buffers of 8 (device)
  bool orbitals_ready = false;
  int task_width = TASK_WIDTH;  // kets per J/K task
  int purify_steps = 0, purify_fallbacks = 0;
  double purify_ms = 0.0;  // CUDA-event time of the TC2 graphs (verbose runs only)
  float* dmax = nullptr;
  std::vector<double*> diis_F, diis_E;
  double* eps_dev = nullptr;
  double* occ_dev = nullptr;   // atomic-occupation starting density (diagonal)
  double* pmin_dev = nullptr;  // smallest Cholesky pivot^2 of S
  int* info_dev = nullptr;
  unsigned long long* stats_dev = nullptr;
  const double** ptrs_dev = nullptr;
  double* grad_dev = nullptr;
  DeviceBuf syev_work;
  DeviceBuf small_buf;
  // four TC2 steps (cuBLAS DGEMM + update, ping-pong buffers) as one CUDA
  // graph per occupation number, replayed by purify() for nbf > 192
  std::vector<std::pair<int, cudaGraphExec_t>> tc2_graphs;
  std::vector<std::pair<int, int>> tc2_last;  // per occupation number: TC2 steps of the last purification
  cudaGraphExec_t tc2_graph(int nocc);
  int syev_lwork = 0;

  ScfState st;
  // pyfacc_system_jk_stats: ms, flops FP64/FP32, quartets FP64/FP32,
  // primitive quartets FP64/FP32, then per s/p quartet class: quartets
  // FP64, FP32, primitive quartets FP64, FP32 (NQCLASS each)
  static constexpr int JK_STATS_N = 7 + 4 * NQCLASS;
  double last_jk[JK_STATS_N] = {};
  // flops and counts of the J/K counters (stats_dev) for nk exchange densities
  void jk_counters(int nk, double out[6], double* per_class = nullptr);
  pyfacc_reduce_fn reducer = nullptr;   // sums shard results across processes
  void* reducer_ctx = nullptr;
  void reduce(double* data, long long count);
  bool one_e_done = false;
  std::vector<double> grad_host;

  // ---- setup (engine.cpp)
  static void spin_electrons(const std::vector<std::string>& sp, int chg, int* na, int* nb);
  double nuclear_repulsion() const;
  void nuclear_repulsion_gradient(double* g) const;
  void upload_shells();
  void build_pairs();
  void build_tasks();
  void alloc_matrices();
  void release_extra();
  void set_coords(const double* coords);

  // ---- operations (scf.cpp)
  void one_electron();
  // J = J[Dj], K[k] = K[Dk[k]] (precision 0 = fp64, 1 = mixed); screening by
  // Q_ab Q_cd max|D| with the density(ies) given.
  // fp32_thresh < 0: opt.fp32_thresh (mixed precision only)
  // out: JK_FULL (zeroed, then J = Jh + Jh^T), JK_HALF (zeroed, left as Jh)
  // or JK_ADD (added into an existing Jh; no reducer)
  void jk(const double* Dj, int nk, const double* const* Dk, double* Jo, double* const* Ko, int precision,
          bool dynamic = false, double thresh = -1.0, double fp32_thresh = -1.0, int out = 0);
  void eri_tensor(double* eri);
  void orthogonalizer();  // queued; its LINDEP status is read by check_overlap_factor after a later sync
  void check_overlap_factor();
  void diagonalize(const double* Fm, double* C, double* eps);
  void density_from(const double* C, int nocc, double scale, double* Pm);
  // P = scale * projector onto the nocc lowest eigenvectors of F (TC2
  // purification of X^T F X); false if it did not converge.
  // With Pp: also the projector P' of the orthonormal basis (P = scale
  // R^T P' R) into Pp.  density_step returns whether Pp was written (not
  // after an eigensolver fallback).
  bool purify(const double* Fm, int nocc, double scale, double* Pm, double* Pp = nullptr);
  bool density_step(const double* Fm, int nocc, double scale, double* Pm, double* C, double* eps,
                    double* Pp = nullptr);
  // The same from the orthonormal-basis Fock matrix F' = R F R^T.
  bool purify_orth(const double* Fp, int nocc, double scale, double* Pm, double* Pp);
  bool density_step_orth(const double* Fp, int nocc, double scale, double* Pm, double* C, double* eps,
                         double* Pp);
  void diagonalize_orth(const double* Fp, double* C, double* eps);
  bool purify_core(int nocc, double scale, double* Pm, double* Pp);
  void final_orbitals();
  // Diagonal starting density from atomic aufbau occupations of the
  // minimal-basis shells (total electrons, spread over 2 s / 6 p per shell).
  std::vector<double> atomic_occupations() const;
  void run_scf();
  void gradient(double* g_host);
  void fill_result(pyfacc_result* r);
  float elapsed(cudaEvent_t a, cudaEvent_t b);
};

}  // namespace pyfacc

struct pyfacc_system {
  pyfacc::System* impl;
};
