// C ABI of libpyfacc_b200.so (declared in include/pyfacc_b200.h).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>

#include <vector>

#include "batch.h"
#include "engine.h"
#include "system.h"

using pyfacc::Error;
using pyfacc::System;

namespace {

thread_local int g_last_status = PYFACC_OK;
thread_local std::string g_last_message;
thread_local pyfacc::BatchTiming g_batch_stats;

template <typename Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return PYFACC_OK;
  } catch (const Error& e) {
    g_last_message = e.what();
    if (std::getenv("PYFACC_VERBOSE")) std::fprintf(stderr, "pyfacc: %s\n", e.what());
    return e.status;
  } catch (const std::exception& e) {
    g_last_message = e.what();
    if (std::getenv("PYFACC_VERBOSE")) std::fprintf(stderr, "pyfacc: %s\n", e.what());
    return PYFACC_ERR_INVALID;
  }
}

int run_one(const pyfacc_molecule& m, const pyfacc_options& o, pyfacc_result* r) {
  std::unique_ptr<System> sys(new System(m, o));
  sys->run_scf();
  if (o.compute_gradient) sys->gradient(nullptr);
  if (r) sys->fill_result(r);
  return sys->st.converged ? PYFACC_OK : PYFACC_ERR_NOT_CONVERGED;
}

}  // namespace

namespace pyfacc {
void set_last_message(const std::string& m) { g_last_message = m; }
}  // namespace pyfacc

extern "C" {

const char* pyfacc_version(void) { return "pyfacc-b200 0.1 (sm_100a)"; }

const char* pyfacc_status_string(int s) {
  switch (s) {
    case PYFACC_OK: return "ok";
    case PYFACC_ERR_BASIS_NOT_FOUND: return "basis set file not found";
    case PYFACC_ERR_UNSUPPORTED_L: return "unsupported shell type (s and p only)";
    case PYFACC_ERR_NOT_CONVERGED: return "SCF not converged";
    case PYFACC_ERR_LINDEP: return "overlap matrix not positive definite";
    case PYFACC_ERR_CUDA: return "CUDA error";
    case PYFACC_ERR_TIMEOUT: return "device wait timed out";
    case PYFACC_ERR_INVALID: return "invalid argument";
    case PYFACC_ERR_ELEMENT: return "element without basis functions";
    case PYFACC_ERR_NO_DEVICE: return "no CUDA device";
    case PYFACC_ERR_NOT_READY: return "call order: run the SCF first";
    default: return "unknown status";
  }
}

int pyfacc_last_status(void) { return g_last_status; }

// Detail text of the most recent failure on this thread (extension).
const char* pyfacc_last_message(void) { return g_last_message.c_str(); }

void pyfacc_default_options(pyfacc_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->eps_energy = 1e-10;
  o->eps_diis = 1e-8;
  o->eps_density = 0.0;
  o->max_iter = 100;
  o->diis_size = 8;
  o->scf_type = PYFACC_SCF_AUTO;
  o->precision = PYFACC_PRECISION_FP64;
  o->boys_mode = PYFACC_BOYS_ACCURATE;
  o->schwarz_thresh = 1e-12;
  o->fp32_thresh = 1e-3;
  o->incremental = -1;
  o->rebuild_every = 12;
  o->compute_gradient = 0;
  o->device = -1;
  o->verbose = 0;
  o->shard_rank = 0;
  o->shard_count = 1;
  o->data_dir = nullptr;
  o->guess = PYFACC_GUESS_ATOMIC;
  o->incremental_thresh = 1e-11;
  o->task_width = 0;
  o->gradient_precision = -1;
  o->polish = 0;
  o->gradient_fp32_thresh = 1e-1;
  o->coarse_err = 1e-3;
}

// scf_interface.c:9-14 -> main.f90:15-64: species/coords/z in, energy out.
// The Fortran side stops at max_iter and returns the last energy (rscf.f90:
// 118-164); this engine does the same with DIIS, converging on |dE| < eps_scf
// and ||D - D_old||_F < eps_scf as rscf.f90:152-155 does.
// libint_overlap_c / libint_kinetic_c / libint_potential_c: the one-body
// shell-pair interface of the reference's Libint wrapper
// (src/cpp/libint_wrapper.cpp:16-105, 114-212, 220-327), same symbols and
// arguments, computed on the GPU.  Like the wrapper they return nothing; a
// failure (an l above 2, a contraction deeper than 32, no device) fills the
// block with NaN and leaves the status for pyfacc_last_status().
namespace {
void libint_block(int kind, int amA, int nA, const double* A, const double* alphaA, const double* cA, int amB,
                  int nB, const double* B, const double* alphaB, const double* cB, const double* C, double* out) {
  const int st = guarded([&] {
    pyfacc::libint_one_body(kind, amA, nA, A, alphaA, cA, amB, nB, B, alphaB, cB, C, out);
  });
  g_last_status = st;
  // the caller sized out as nint(amA) x nint(amB) (any l, as for Libint)
  if (st != PYFACC_OK && out && amA >= 0 && amB >= 0 && amA <= 20 && amB <= 20) {
    const int n = ((amA + 1) * (amA + 2) / 2) * ((amB + 1) * (amB + 2) / 2);
    for (int i = 0; i < n; ++i) out[i] = std::numeric_limits<double>::quiet_NaN();
  }
}
}  // namespace

void libint_overlap_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB, int contrdepthB,
                      double B[], double alphaB[], double cB[], double overlapAB[]) {
  libint_block(0, amA, contrdepthA, A, alphaA, cA, amB, contrdepthB, B, alphaB, cB, nullptr, overlapAB);
}

void libint_kinetic_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB, int contrdepthB,
                      double B[], double alphaB[], double cB[], double kineticAB[]) {
  libint_block(1, amA, contrdepthA, A, alphaA, cA, amB, contrdepthB, B, alphaB, cB, nullptr, kineticAB);
}

void libint_potential_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB, int contrdepthB,
                        double B[], double alphaB[], double cB[], double C[], double potAB[]) {
  libint_block(2, amA, contrdepthA, A, alphaA, cA, amB, contrdepthB, B, alphaB, cB, C, potAB);
}

void run_scf_c(int natoms, int nelectrons, int charge, int nalpha, int nbeta, const char* species, double* coords,
               double eps_scf, int max_iter, double* final_energy, const char* basis_set_c, int32_t* z_num) {
  (void)nelectrons;
  pyfacc_molecule m;
  m.natoms = natoms;
  m.z = z_num;
  m.coords = coords;
  m.species = species;
  m.charge = charge;
  m.nalpha = nalpha;
  m.nbeta = nbeta;
  m.basis = basis_set_c;
  pyfacc_options o;
  pyfacc_default_options(&o);
  o.eps_energy = eps_scf;
  o.eps_density = eps_scf;
  o.eps_diis = 1e300;  // the reference criterion is |dE| and ||dD|| only
  o.max_iter = max_iter;
  pyfacc_result r;
  std::memset(&r, 0, sizeof(r));
  int status = PYFACC_OK;
  const int st = guarded([&] { status = run_one(m, o, &r); });
  if (st != PYFACC_OK) status = st;
  g_last_status = status;
  if (final_energy) {
    // like the reference, a run that hit max_iter still returns its energy
    if (status == PYFACC_OK || status == PYFACC_ERR_NOT_CONVERGED) *final_energy = r.energy;
    else *final_energy = std::numeric_limits<double>::quiet_NaN();
  }
}

// main.f90:15-24, the bind(C) all-by-reference entry point.
void run_scf_interface_py(int32_t* natoms, int32_t* nelectrons, int32_t* charge, int32_t* nalpha, int32_t* nbeta,
                          const char* species, double* coords, double* eps_scf, int32_t* max_iter,
                          double* final_energy, const char* basis_set_c, int32_t* len_basis_set, int32_t* z_num) {
  std::string basis(basis_set_c, basis_set_c + (len_basis_set ? *len_basis_set : std::strlen(basis_set_c)));
  while (!basis.empty() && basis.back() == ' ') basis.pop_back();
  run_scf_c(*natoms, *nelectrons, *charge, *nalpha, *nbeta, species, coords, *eps_scf, *max_iter, final_energy,
            basis.c_str(), z_num);
}

int pyfacc_run(const pyfacc_molecule* mol, const pyfacc_options* opt, pyfacc_result* res) {
  if (!mol) return PYFACC_ERR_INVALID;
  pyfacc_options o;
  if (opt) o = *opt; else pyfacc_default_options(&o);
  int status = PYFACC_OK;
  const int st = guarded([&] { status = run_one(*mol, o, res); });
  return st != PYFACC_OK ? st : status;
}

// Closed-shell molecules of up to 160 basis functions run together in the
// batched engine (batch.h); open-shell or larger molecules, molecules whose
// results ask for matrices or orbitals, and any molecule whose batched
// purification or orthogonalisation did not converge run one by one through
// pyfacc_run.  The return value is the worst per-molecule status.
int pyfacc_run_batch(int nmol, const pyfacc_molecule* mols, const pyfacc_options* opt, pyfacc_result* res) {
  if (nmol < 0 || (nmol > 0 && !mols)) return PYFACC_ERR_INVALID;
  pyfacc_options o;
  if (opt) o = *opt; else pyfacc_default_options(&o);
  std::vector<int> status(nmol, PYFACC_OK), single, in_batch;
  std::vector<pyfacc::BatchMolHost> hosts;
  const auto tp0 = std::chrono::steady_clock::now();
  for (int i = 0; i < nmol; ++i) {
    pyfacc_result* r = res ? &res[i] : nullptr;
    const bool wants_matrices = r && (r->S || r->T || r->V || r->P || r->C_alpha || r->C_beta || r->eps_alpha ||
                                      r->eps_beta);
    bool uhf = false;
    pyfacc::BatchMolHost h;
    const int st = guarded([&] { h = pyfacc::batch_parse(mols[i], o, &uhf); });
    if (st != PYFACC_OK) {
      status[i] = st;
      if (r) r->energy = std::numeric_limits<double>::quiet_NaN();
      continue;
    }
    bool has_d = false;  // the batched kernels cover s/p shells; d molecules run on their own
    for (const auto& sh : h.basis.shells) has_d = has_d || sh.l > 1;
    if (uhf || wants_matrices || has_d || h.nbf > pyfacc::BATCH_NBF_MAX) {
      single.push_back(i);
    } else {
      in_batch.push_back(i);
      hosts.push_back(std::move(h));
    }
  }
  if (o.verbose)
    std::fprintf(stderr, "pyfacc batch parse (ms): %.2f\n",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp0).count());
  if (!hosts.empty()) {
    const int st = guarded([&] {
      pyfacc::Batch b(hosts, o);
      b.run(o.compute_gradient != 0);
      const pyfacc::BatchTiming& t = b.timing;
      g_batch_stats = t;
      for (size_t k = 0; k < in_batch.size(); ++k) {
        const int i = in_batch[k];
        if (b.failed((int)k)) {
          single.push_back(i);
          continue;
        }
        status[i] = b.converged((int)k) ? PYFACC_OK : PYFACC_ERR_NOT_CONVERGED;
        if (!res) continue;
        pyfacc_result* r = &res[i];
        const pyfacc::BatchMolHost& h = hosts[k];
        r->energy = b.energy((int)k);
        r->e_elec = r->energy - h.e_nuc;
        r->e_nuc = h.e_nuc;
        r->converged = b.converged((int)k) ? 1 : 0;
        r->n_iter = b.iterations((int)k);
        r->scf_type = PYFACC_SCF_RHF;
        r->nbf = h.nbf;
        r->nshell = h.ns;
        r->n_fock_builds = b.iterations((int)k) + (o.precision == PYFACC_PRECISION_MIXED ? 1 : 0);
        r->last_delta_e = b.last_delta_e((int)k);
        r->last_diis_error = b.last_error((int)k);
        if (r->gradient && o.compute_gradient)
          std::memcpy(r->gradient, b.gradient((int)k), 3 * (size_t)h.natoms * sizeof(double));
        // whole-batch statistics
        r->ms_total = t.ms_total;
        r->ms_one_electron = t.ms_1e;
        r->ms_fock = t.ms_scf + t.ms_polish;
        r->ms_diag = 0.0;
        r->ms_gradient = t.ms_grad;
        r->quartets_fp64 = (long long)t.quartets[0];
        r->quartets_fp32 = (long long)t.quartets[1];
        r->flops_fock = t.flops_fock;
        r->flops_gradient = t.flops_grad;
        r->task_width = t.width[pyfacc::NQCLASS - 1];
      }
    });
    if (st != PYFACC_OK)
      for (int i : in_batch) {
        status[i] = st;
        if (res) res[i].energy = std::numeric_limits<double>::quiet_NaN();
      }
  }
  for (int i : single) status[i] = pyfacc_run(&mols[i], &o, res ? &res[i] : nullptr);
  int worst = PYFACC_OK;
  for (int s : status)
    if (s != PYFACC_OK && (worst == PYFACC_OK || worst == PYFACC_ERR_NOT_CONVERGED)) worst = s;
  return worst;
}

// Statistics of the last batched run on this thread (extension).
int pyfacc_batch_last_stats(double* out, int n) {
  if (!out || n <= 0) return PYFACC_ERR_INVALID;
  const pyfacc::BatchTiming& b = g_batch_stats;
  const double v[] = {b.ms_total, b.ms_setup, b.ms_1e, b.ms_tune, b.ms_scf, b.ms_polish, b.ms_grad,
                      (double)b.iterations, b.flops_fock, b.flops_grad, (double)b.quartets[0],
                      (double)b.quartets[1], (double)b.width[0], (double)b.width[1], (double)b.width[2],
                      (double)b.width[3], (double)b.width[4], (double)b.width[5], (double)b.scf_graph_launches};
  const int nv = (int)(sizeof(v) / sizeof(v[0]));
  for (int k = 0; k < n; ++k) out[k] = k < nv ? v[k] : 0.0;
  return PYFACC_OK;
}

int pyfacc_system_create(const pyfacc_molecule* mol, const pyfacc_options* opt, pyfacc_system** out) {
  if (!mol || !out) return PYFACC_ERR_INVALID;
  *out = nullptr;
  pyfacc_options o;
  if (opt) o = *opt; else pyfacc_default_options(&o);
  return guarded([&] {
    std::unique_ptr<System> s(new System(*mol, o));
    *out = new pyfacc_system{s.release()};
  });
}

void pyfacc_system_destroy(pyfacc_system* sys) {
  if (!sys) return;
  delete sys->impl;
  delete sys;
}

int pyfacc_system_info(const pyfacc_system* sys, int* nbf, int* nshell, int* natoms, int* npairs) {
  if (!sys) return PYFACC_ERR_INVALID;
  if (nbf) *nbf = sys->impl->nbf;
  if (nshell) *nshell = sys->impl->ns;
  if (natoms) *natoms = sys->impl->natoms;
  if (npairs) *npairs = sys->impl->pd.npair;
  return PYFACC_OK;
}

int pyfacc_system_set_coords(pyfacc_system* sys, const double* coords) {
  if (!sys || !coords) return PYFACC_ERR_INVALID;
  return guarded([&] {
    PF_CUDA(cudaSetDevice(sys->impl->device));
    sys->impl->set_coords(coords);
  });
}

int pyfacc_system_one_electron(pyfacc_system* sys, double* S_dev, double* T_dev, double* V_dev) {
  if (!sys) return PYFACC_ERR_INVALID;
  return guarded([&] {
    System& s = *sys->impl;
    PF_CUDA(cudaSetDevice(s.device));
    s.one_electron();
    const size_t b = (size_t)s.nbf * s.nbf * sizeof(double);
    if (S_dev) PF_CUDA(cudaMemcpyAsync(S_dev, s.S, b, cudaMemcpyDeviceToDevice, s.stream));
    if (T_dev) PF_CUDA(cudaMemcpyAsync(T_dev, s.T, b, cudaMemcpyDeviceToDevice, s.stream));
    if (V_dev) PF_CUDA(cudaMemcpyAsync(V_dev, s.Vm, b, cudaMemcpyDeviceToDevice, s.stream));
    PF_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int pyfacc_system_jk(pyfacc_system* sys, const double* Dj_dev, int nk, const double* Dk_dev, double* J_dev,
                     double* K_dev, int precision) {
  if (!sys || !Dj_dev || !Dk_dev || !J_dev || !K_dev || nk < 1 || nk > 2) return PYFACC_ERR_INVALID;
  return guarded([&] {
    System& s = *sys->impl;
    PF_CUDA(cudaSetDevice(s.device));
    const size_t n2 = (size_t)s.nbf * s.nbf;
    const double* Dk[2] = {Dk_dev, Dk_dev + n2};
    double* Ko[2] = {K_dev, K_dev + n2};
    if (precision < PYFACC_PRECISION_FP64 || precision > PYFACC_PRECISION_FP32)
      throw Error(PYFACC_ERR_INVALID, "precision must be PYFACC_PRECISION_FP64, _MIXED or _FP32");
    PF_CUDA(cudaMemsetAsync(s.stats_dev, 0, sizeof(pyfacc::JkStats), s.stream));
    PF_CUDA(cudaEventRecord(s.ev0, s.stream));
    if (precision == PYFACC_PRECISION_FP32)  // every quartet in FP32, lists built on the device
      s.jk(Dj_dev, nk, Dk, J_dev, Ko, PYFACC_PRECISION_MIXED, true, -1.0, 1e300);
    else
      s.jk(Dj_dev, nk, Dk, J_dev, Ko, precision);
    PF_CUDA(cudaEventRecord(s.ev1, s.stream));
    PF_CUDA(cudaStreamSynchronize(s.stream));
    double c[6];
    s.jk_counters(nk, c, s.last_jk + 7);
    s.last_jk[0] = s.elapsed(s.ev0, s.ev1);
    for (int k = 0; k < 6; ++k) s.last_jk[1 + k] = c[k];
  });
}

int pyfacc_system_jk_stats(const pyfacc_system* sys, double* out, int n) {
  if (!sys || !out || n <= 0) return PYFACC_ERR_INVALID;
  for (int k = 0; k < n; ++k) out[k] = k < System::JK_STATS_N ? sys->impl->last_jk[k] : 0.0;
  return PYFACC_OK;
}

int pyfacc_system_eri_tensor(pyfacc_system* sys, double* eri_dev) {
  if (!sys || !eri_dev) return PYFACC_ERR_INVALID;
  return guarded([&] {
    System& s = *sys->impl;
    if (s.nbf > 64) throw Error(PYFACC_ERR_INVALID, "ERI tensor limited to nbf <= 64");
    PF_CUDA(cudaSetDevice(s.device));
    s.eri_tensor(eri_dev);
    PF_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int pyfacc_system_scf(pyfacc_system* sys, pyfacc_result* res) {
  if (!sys) return PYFACC_ERR_INVALID;
  int status = PYFACC_OK;
  const int st = guarded([&] {
    System& s = *sys->impl;
    PF_CUDA(cudaSetDevice(s.device));
    s.run_scf();
    if (s.opt.compute_gradient) s.gradient(nullptr);
    if (res) s.fill_result(res);
    status = s.st.converged ? PYFACC_OK : PYFACC_ERR_NOT_CONVERGED;
  });
  return st != PYFACC_OK ? st : status;
}

int pyfacc_system_gradient(pyfacc_system* sys, double* grad) {
  if (!sys) return PYFACC_ERR_INVALID;
  return guarded([&] {
    System& s = *sys->impl;
    PF_CUDA(cudaSetDevice(s.device));
    s.gradient(grad);
  });
}

int pyfacc_system_result(pyfacc_system* sys, pyfacc_result* res) {
  if (!sys || !res) return PYFACC_ERR_INVALID;
  return guarded([&] {
    System& s = *sys->impl;
    if (!s.st.done) throw Error(PYFACC_ERR_NOT_READY, "no SCF has run on this system");
    PF_CUDA(cudaSetDevice(s.device));
    s.fill_result(res);
  });
}

long long pyfacc_launch_count(void) { return pyfacc::launch_count(); }

int pyfacc_system_density_dev(pyfacc_system* sys, const double** P_dev) {
  if (!sys || !P_dev) return PYFACC_ERR_INVALID;
  *P_dev = sys->impl->P[0];
  return PYFACC_OK;
}

int pyfacc_boys_dev(int mode, int fp32, int mmax, int n, const double* x_dev, double* out_dev) {
  if (mmax < 0 || mmax > PYFACC_BOYS_MMAX || n < 0 || (n > 0 && (!x_dev || !out_dev))) return PYFACC_ERR_INVALID;
  return guarded([&] {
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    pyfacc::ensure_boys_tables(dev);
    pyfacc::launch_boys_test(mode, fp32, mmax, n, x_dev, out_dev, 0);
    PF_CUDA(cudaDeviceSynchronize());
  });
}

int pyfacc_dense_gemm_dev(int m, int n, int k, int ta, const double* A_dev, int tb, const double* B_dev,
                          double* C_dev, int sym, int asym_a) {
  if (m < 0 || n < 0 || k < 0 || (m * n > 0 && (!A_dev || !B_dev || !C_dev))) return PYFACC_ERR_INVALID;
  return guarded([&] {
    const int lda = ta ? m : k, ldb = tb ? k : n;
    pyfacc::launch_dgemm(m, n, k, ta != 0, A_dev, lda, tb != 0, B_dev, ldb, C_dev, n, 1.0, nullptr, n, 0.0, sym != 0,
                         asym_a != 0, 0);
    PF_CUDA(cudaDeviceSynchronize());
  });
}

int pyfacc_purify_dev(int n, int nocc, const double* F_dev, double* P_dev, int* steps) {
  if (n <= 0 || nocc < 0 || nocc > n || !F_dev || !P_dev || F_dev == P_dev) return PYFACC_ERR_INVALID;
  int status = PYFACC_OK;
  const int st = guarded([&] {
    const size_t n2 = (size_t)n * n;
    pyfacc::DeviceBuf work;
    work.ensure(2 * n2 * sizeof(double) + 64 * sizeof(double));
    double* Xb = work.as<double>();
    double* state = Xb + n2 + n2;
    // the projector is built in P_dev itself (the graph's X_a)
    cudaGraphExec_t g = pyfacc::build_tc2_graph(n, nocc, F_dev, P_dev, Xb, state, pyfacc::TC2_KMAX);
    const cudaError_t e = cudaGraphLaunch(g, 0);
    double ctl[8];
    cudaError_t e2 = e == cudaSuccess ? cudaMemcpy(ctl, state + 8, sizeof(ctl), cudaMemcpyDeviceToHost) : e;
    cudaGraphExecDestroy(g);
    PF_CUDA(e2);
    if (steps) *steps = (int)ctl[2];
    if (ctl[1] == 0.0 || ctl[4] != 0.0) status = PYFACC_ERR_NOT_CONVERGED;
  });
  return st != PYFACC_OK ? st : status;
}

int pyfacc_partition(int n, const double* cost, int parts, int* bounds) {
  if (n < 0 || parts < 1 || !bounds || (n > 0 && !cost)) return PYFACC_ERR_INVALID;
  pyfacc::partition_costs(n, cost, parts, bounds);
  return PYFACC_OK;
}

int pyfacc_system_set_reducer(pyfacc_system* sys, pyfacc_reduce_fn fn, void* ctx) {
  if (!sys) return PYFACC_ERR_INVALID;
  sys->impl->reducer = fn;
  sys->impl->reducer_ctx = ctx;
  return PYFACC_OK;
}

double pyfacc_probe_fp64_gflops(int device, double* fp32_gflops) {
  double r = -1.0;
  guarded([&] { r = pyfacc::probe_fp64(device, fp32_gflops); });
  return r;
}

}  // extern "C"
