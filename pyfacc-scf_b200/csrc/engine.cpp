// Host side of the B200 Hartree-Fock engine: one molecule on one GPU.
//
// SCF (rscf.f90:26-168 / uscf.f90:25-219 of PyFAcc-SCF, with the intended
// semantics: every 8-fold ERI image, RHF/UHF dispatch on n_alpha == n_beta,
// Pulay DIIS, convergence on |dE|, the DIIS commutator and optionally
// ||dD||_F):
//   S, T, V on the GPU; X = U s^-1/2 (la.f90:28-57, canonical, no
//   eigenvalue dropping) from cuSOLVER once; core guess; then per iteration
//   J/K digestion kernels (FP64, or mixed FP64/FP32 with incremental dP
//   builds), F = H + J - K/2 (RHF) or H + J - K_s (UHF), energy and DIIS
//   error reduced on the device, F' = X^T F X and C = X C' by cuBLAS DGEMM,
//   eigenvectors by cuSOLVER DSYEVD, D = 2 C_occ C_occ^T (RHF).
// Gradient: one- and two-electron derivative kernels contracted with P and
// W = sum_occ eps_i c_i c_i^T on the device, nuclear repulsion on the host.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "engine.h"
#include "pool.h"
#include "system.h"

namespace pyfacc {

void DeviceBuf::ensure(size_t b) {
  if (b <= bytes) return;
  release();
  size_t got = 0;
  p = pool_alloc(b, &got);
  bytes = got;
}
void DeviceBuf::release() {
  if (p) pool_free(p, bytes);
  p = nullptr;
  bytes = 0;
}

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

// ------------------------------------------------------------------ setup
// Argument checks shared by the single-molecule and batched engines, made
// before any device work so that bad input is reported the same way with
// or without a GPU.  The reference reads whatever the XYZ file holds
// (helper_functions.py:25-54); a NaN or infinite coordinate would reach the
// integrals there, here it is PYFACC_ERR_INVALID.
void validate_molecule(const pyfacc_molecule& m) {
  if (m.natoms <= 0 || !m.z || !m.coords || !m.basis) throw Error(PYFACC_ERR_INVALID, "empty molecule");
  for (int i = 0; i < 3 * m.natoms; ++i)
    if (!std::isfinite(m.coords[i]))
      throw Error(PYFACC_ERR_INVALID, "coordinate " + std::to_string(i % 3) + " of atom " + std::to_string(i / 3) +
                                          " is not finite");
}

System::System(const pyfacc_molecule& m, const pyfacc_options& o) : opt(o) {
  validate_molecule(m);
  if (opt.task_width != 0 && opt.task_width != 8 && opt.task_width != 16 && opt.task_width != 32)
    throw Error(PYFACC_ERR_INVALID, "task_width must be 0, 8, 16 or 32");
  if (opt.task_width) task_width = opt.task_width;
  if (opt.diis_size < 0 || opt.diis_size > MAX_DIIS)
    throw Error(PYFACC_ERR_INVALID, "diis_size must be 0.." + std::to_string(MAX_DIIS));
  // host-side parsing first: argument, element and basis errors are
  // reported before (and without) any device work
  natoms = m.natoms;
  Z.assign(m.z, m.z + natoms);
  xyz.assign(m.coords, m.coords + 3 * natoms);
  species.resize(natoms);
  for (int a = 0; a < natoms; ++a) {
    if (m.species) {
      std::string s(m.species + 2 * a, 2);
      while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
      species[a] = s;
    } else {
      species[a] = element_symbol(Z[a]);
    }
    if (species[a].empty() || element_z(species[a]) == 0)
      throw Error(PYFACC_ERR_ELEMENT, "unknown element at atom " + std::to_string(a));
  }
  charge = m.charge;
  if (m.nalpha >= 0 && m.nbeta >= 0) {
    nalpha = m.nalpha;
    nbeta = m.nbeta;
  } else {
    spin_electrons(species, charge, &nalpha, &nbeta);
  }
  basis_name = m.basis;
  basis_file = resolve_basis_file(basis_name, opt.data_dir);
  basis = build_basis(basis_file, species, xyz);
  nbf = basis.nbf;
  ns = (int)basis.shells.size();
  uhf = (opt.scf_type == PYFACC_SCF_UHF) || (opt.scf_type == PYFACC_SCF_AUTO && nalpha != nbeta);
  e_nuc = nuclear_repulsion();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(PYFACC_ERR_NO_DEVICE, "no CUDA device");
  if (opt.device >= 0) {
    device = opt.device;
    PF_CUDA(cudaSetDevice(device));
  } else {
    PF_CUDA(cudaGetDevice(&device));
  }
  PF_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  ensure_boys_tables(device);
  ctx = context_acquire(device);
  stream = ctx.stream;
  cublas = ctx.cublas;
  cusolver = ctx.cusolver;
  ev0 = ctx.ev0;
  ev1 = ctx.ev1;

  using clk = std::chrono::steady_clock;
  const auto c0 = clk::now();
  upload_shells();
  const auto c1 = clk::now();
  build_pairs();
  const auto c2 = clk::now();
  alloc_matrices();
  if (opt.verbose) {
    PF_CUDA(cudaStreamSynchronize(stream));
    const auto c3 = clk::now();
    auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    std::fprintf(stderr, "pyfacc setup (ms): shells %.3f  pairs + tasks %.3f  matrices %.3f\n", ms(c0, c1), ms(c1, c2),
                 ms(c2, c3));
  }
}

System::~System() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (auto& g : tc2_graphs) cudaGraphExecDestroy(g.second);
  release_extra();
  context_release(ctx);  // stream and handles go back to the per-device pool
}

// helper_functions.py:58-87: multiplicity 1 or 2, O2 -> 3, N2 -> 4.
void System::spin_electrons(const std::vector<std::string>& sp, int chg, int* na, int* nb) {
  int total = -chg;
  for (auto& s : sp) total += element_z(s);
  int mult = (total % 2 == 0) ? 1 : 2;
  bool all_same = std::all_of(sp.begin(), sp.end(), [&](const std::string& s) { return s == sp[0]; });
  if (all_same && sp.size() == 2 && sp[0] == "O") mult = 3;
  if (all_same && sp.size() == 2 && sp[0] == "N") mult = 4;
  const int twoS = mult - 1;
  if (total < 0) throw Error(PYFACC_ERR_INVALID, "charge exceeds the nuclear charge (negative electron count)");
  if ((total + twoS) % 2 != 0) throw Error(PYFACC_ERR_INVALID, "Inconsistent electron count and spin state.");
  *na = (total + twoS) / 2;
  *nb = total - *na;
}

// molecule.f90:31-52: sum_{i<j} Z_i Z_j / R_ij, pairs with R <= 1e-10 skipped.
double System::nuclear_repulsion() const {
  double e = 0.0;
  for (int i = 0; i < natoms; ++i)
    for (int j = i + 1; j < natoms; ++j) {
      double d2 = 0;
      for (int x = 0; x < 3; ++x) d2 += (xyz[3 * i + x] - xyz[3 * j + x]) * (xyz[3 * i + x] - xyz[3 * j + x]);
      const double r = std::sqrt(d2);
      if (r > 1.0e-10) e += (double)Z[i] * Z[j] / r;
    }
  return e;
}

void System::nuclear_repulsion_gradient(double* g) const {
  for (int i = 0; i < natoms; ++i)
    for (int j = 0; j < natoms; ++j) {
      if (i == j) continue;
      double d[3], r2 = 0;
      for (int x = 0; x < 3; ++x) {
        d[x] = xyz[3 * i + x] - xyz[3 * j + x];
        r2 += d[x] * d[x];
      }
      const double r = std::sqrt(r2);
      if (r <= 1.0e-10) continue;
      for (int x = 0; x < 3; ++x) g[3 * i + x] -= (double)Z[i] * Z[j] * d[x] / (r2 * r);
    }
}

void System::upload_shells() {
  std::vector<double4> cen(ns);
  std::vector<int4> desc(ns);
  std::vector<int> np(ns), nf(ns);
  std::vector<double> ex, co;
  std::vector<int> bfo(ns + 1);
  for (int s = 0; s < ns; ++s) {
    const Shell& sh = basis.shells[s];
    cen[s] = make_double4(sh.c[0], sh.c[1], sh.c[2], 0.0);
    desc[s] = make_int4(sh.l, sh.atom, basis.bf_off[s], (int)ex.size());
    np[s] = (int)sh.ex.size();
    nf[s] = (sh.l + 1) * (sh.l + 2) / 2;
    ex.insert(ex.end(), sh.ex.begin(), sh.ex.end());
    co.insert(co.end(), sh.co.begin(), sh.co.end());
    bfo[s] = basis.bf_off[s];
  }
  bfo[ns] = nbf;
  std::vector<double4> atoms(natoms);
  for (int a = 0; a < natoms; ++a) atoms[a] = make_double4(xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2], (double)Z[a]);
  // 1e pair lists: every pair a <= b of the upper triangle of S_overlap
  // (overlap.f90:292-329), per class, ordered so that l_a >= l_b, except
  // pairs on two atoms whose largest primitive-pair prefactor is below
  // ONE_E_PAIR_CUT: with mu_min from the two smallest exponents (mu grows
  // with both) and the largest |c N| of each shell, the test
  // mu_min R^2 > ln|cN|_a + ln|cN|_b - ln(cut) bounds every primitive pair
  std::vector<double> lcn(ns), amin(ns);
  for (int s = 0; s < ns; ++s) {
    const Shell& sh = basis.shells[s];
    double mx = 0.0, mn = 1e300;
    for (size_t k = 0; k < sh.ex.size(); ++k) {
      const double a = sh.ex[k];
      double nrm = std::pow(2.0 * a / 3.14159265358979323846, 0.75);
      if (sh.l == 1) nrm *= 2.0 * std::sqrt(a);
      if (sh.l == 2) nrm *= 4.0 * a;  // 4a / sqrt(3), times sqrt(3) for the mixed components
      mx = std::max(mx, std::fabs(sh.co[k] * nrm));
      mn = std::min(mn, a);
    }
    lcn[s] = std::log(std::max(mx, 1e-300));
    amin[s] = mn;
  }
  const double lcut = std::log(ONE_E_PAIR_CUT);
  std::vector<int2> p1[NPAIRCLASS];
  for (int a = 0; a < ns; ++a)
    for (int b = a; b < ns; ++b) {
      const Shell &sa = basis.shells[a], &sb = basis.shells[b];
      if (sa.atom != sb.atom) {
        double r2 = 0.0;
        for (int x = 0; x < 3; ++x) r2 += (sa.c[x] - sb.c[x]) * (sa.c[x] - sb.c[x]);
        const double mu = amin[a] * amin[b] / (amin[a] + amin[b]);
        if (mu * r2 > lcn[a] + lcn[b] - lcut) continue;
      }
      int x = a, y = b;
      if (basis.shells[x].l < basis.shells[y].l) std::swap(x, y);
      p1[pair_class(basis.shells[x].l, basis.shells[y].l)].push_back(make_int2(x, y));
    }
  int n1e_all = 0;
  for (int c = 0; c < NPAIRCLASS; ++c) n1e_all += n1e[c] = (int)p1[c].size();
  const size_t nex = std::max<size_t>(ex.size(), 1);
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_cen = carve(ns * sizeof(double4)), o_desc = carve(ns * sizeof(int4)), o_np = carve(ns * sizeof(int)),
               o_ex = carve(nex * sizeof(double)), o_co = carve(nex * sizeof(double)),
               o_atoms = carve(natoms * sizeof(double4)), o_p1 = carve((n1e_all + NPAIRCLASS) * sizeof(int2)),
               o_bfo = carve((ns + 1) * sizeof(int)), o_nf = carve(ns * sizeof(int));
  shd.buf.ensure(off);
  char* base = shd.buf.as<char>();
  shd.ns = ns;
  shd.cen = reinterpret_cast<double4*>(base + o_cen);
  shd.desc = reinterpret_cast<int4*>(base + o_desc);
  shd.nprim = reinterpret_cast<int*>(base + o_np);
  shd.ex = reinterpret_cast<double*>(base + o_ex);
  shd.co = reinterpret_cast<double*>(base + o_co);
  atoms_dev = reinterpret_cast<double4*>(base + o_atoms);
  pairs1e[0] = reinterpret_cast<int2*>(base + o_p1);
  for (int c = 1; c < NPAIRCLASS; ++c) pairs1e[c] = pairs1e[c - 1] + n1e[c - 1];
  bf_off_dev = reinterpret_cast<int*>(base + o_bfo);
  nfun_dev = reinterpret_cast<int*>(base + o_nf);
  PF_CUDA(cudaMemcpyAsync(shd.cen, cen.data(), ns * sizeof(double4), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(shd.desc, desc.data(), ns * sizeof(int4), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(shd.nprim, np.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(shd.ex, ex.data(), ex.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(shd.co, co.data(), co.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(atoms_dev, atoms.data(), natoms * sizeof(double4), cudaMemcpyHostToDevice, stream));
  for (int c = 0; c < NPAIRCLASS; ++c)
    if (n1e[c]) PF_CUDA(cudaMemcpyAsync(pairs1e[c], p1[c].data(), n1e[c] * sizeof(int2), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(bf_off_dev, bfo.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(nfun_dev, nf.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
}

// Largest |K| = |c_a N_a c_b N_b| sqrt(2) pi^(5/4) / p over primitive pairs of
// shells on one atom (|AB| = 0 maximises the Gaussian factor).
double max_prim_prefactor(const Basis& b) {
  double mx = 0.0;
  const double c0 = 5.9149671727956128778;
  auto nrm = [](int l, double a) {  // the x^l normalisation of gaussian.f90:80-98
    const double n = std::pow(2.0 * a / 3.14159265358979323846, 0.75);
    return l == 0 ? n : (l == 1 ? n * 2.0 * std::sqrt(a) : n * 4.0 * a / std::sqrt(3.0));
  };
  for (size_t i = 0; i < b.shells.size(); ++i)
    for (size_t j = 0; j <= i; ++j) {
      const Shell &A = b.shells[i], &B = b.shells[j];
      if (A.atom != B.atom) continue;
      for (size_t x = 0; x < A.ex.size(); ++x)
        for (size_t y = 0; y < B.ex.size(); ++y)
          mx = std::max(mx, std::fabs(A.co[x] * nrm(A.l, A.ex[x]) * B.co[y] * nrm(B.l, B.ex[y])) * c0 /
                                (A.ex[x] + B.ex[y]));
    }
  return mx;
}

// Canonical shell pairs grouped by class, Schwarz factors on the GPU, then
// sorted by Q (descending) inside each class; pairs that cannot reach the
// threshold against the largest Q are dropped.  Task lists per class pair.
void System::build_pairs() {
  using clk = std::chrono::steady_clock;
  clk::time_point tq[8];
  tq[0] = clk::now();
  std::vector<int4> pl0[NPAIRCLASS];
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      int a = i, b = j;
      if (basis.shells[a].l < basis.shells[b].l) std::swap(a, b);
      const int c = pair_class(basis.shells[a].l, basis.shells[b].l);
      pl0[c].push_back(make_int4(a, b, 0, 0));
    }
  has_d = false;
  for (int c = NCLASS; c < NPAIRCLASS; ++c) has_d = has_d || !pl0[c].empty();
  std::vector<int4> all0, all1;
  int off[NPAIRCLASS + 1] = {0, 0, 0, 0, 0, 0, 0};
  int nprim_tot = 0;
  for (int c = 0; c < NPAIRCLASS; ++c) {
    off[c + 1] = off[c] + (int)pl0[c].size();
    for (auto p : pl0[c]) {
      p.z = nprim_tot;
      nprim_tot += (int)(basis.shells[p.x].ex.size() * basis.shells[p.y].ex.size());
      all0.push_back(p);
      all1.push_back(make_int4(0, nbf, 0, 0));
    }
  }
  const int np_all = off[NPAIRCLASS];
  // scratch: unsorted records
  size_t o = 0;
  auto carve = [&](size_t bytes) {
    size_t r = o;
    o += (bytes + 255) / 256 * 256;
    return r;
  };
  const size_t s_pl0 = carve(np_all * sizeof(int4)), s_pl1 = carve(np_all * sizeof(int4)),
               s_i0 = carve(np_all * sizeof(int4)), s_i1 = carve(np_all * sizeof(int4)),
               s_i2 = carve(np_all * sizeof(int4)), s_g = carve(np_all * sizeof(double4)),
               s_pr = carve((size_t)std::max(nprim_tot, 1) * 3 * sizeof(double4)), s_q = carve(np_all * sizeof(double)),
               s_perm = carve(np_all * sizeof(int)), s_ps = carve(np_all * sizeof(int)),
               s_kept = carve(np_all * sizeof(int));
  tq[1] = clk::now();
  DeviceBuf scratch;
  scratch.ensure(o);
  tq[2] = clk::now();
  char* sb = scratch.as<char>();
  int4* d_pl0 = reinterpret_cast<int4*>(sb + s_pl0);
  int4* d_pl1 = reinterpret_cast<int4*>(sb + s_pl1);
  PairData tmp;
  tmp.info0 = reinterpret_cast<int4*>(sb + s_i0);
  tmp.info1 = reinterpret_cast<int4*>(sb + s_i1);
  tmp.info2 = reinterpret_cast<int4*>(sb + s_i2);
  tmp.geom = reinterpret_cast<double4*>(sb + s_g);
  tmp.prim = reinterpret_cast<double4*>(sb + s_pr);
  double* d_q = reinterpret_cast<double*>(sb + s_q);
  int* d_perm = reinterpret_cast<int*>(sb + s_perm);
  int* d_ps = reinterpret_cast<int*>(sb + s_ps);
  int* d_kept = reinterpret_cast<int*>(sb + s_kept);
  const double cut = PRIM_CUT_REL * max_prim_prefactor(basis);
  PF_CUDA(cudaMemcpyAsync(d_pl0, all0.data(), np_all * sizeof(int4), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(d_pl1, all1.data(), np_all * sizeof(int4), cudaMemcpyHostToDevice, stream));
  launch_build_pairs(shd, np_all, d_pl0, d_pl1, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, cut, d_kept,
                     stream);
  launch_schwarz(tmp, off, d_q, stream, ctx.side, ctx.fork, ctx.join);
  if (has_d) launch_schwarz_d(tmp, off, d_q, num_sms, stream);
  std::vector<double> q(np_all);
  std::vector<int> kept(np_all);
  PF_CUDA(cudaMemcpyAsync(q.data(), d_q, np_all * sizeof(double), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaMemcpyAsync(kept.data(), d_kept, np_all * sizeof(int), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  tq[3] = clk::now();
  const double qmax = np_all ? *std::max_element(q.begin(), q.end()) : 0.0;
  const double thr = opt.schwarz_thresh;
  std::vector<int> perm, new_ps;
  pd.class_off[0] = 0;
  int nprim_new = 0;
  pd.q_host.clear();
  pd.cls_host.clear();
  for (int c = 0; c < NPAIRCLASS; ++c) {
    std::vector<int> idx;
    for (int k = off[c]; k < off[c + 1]; ++k)
      if (thr <= 0 || q[k] * qmax >= thr) idx.push_back(k);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return q[x] > q[y]; });
    pd.class_maxprim[c] = 0;
    for (int k : idx) {
      pd.class_maxprim[c] = std::max(pd.class_maxprim[c], kept[k]);
      perm.push_back(k);
      new_ps.push_back(nprim_new);
      nprim_new += kept[k];
      pd.q_host.push_back(q[k]);
      pd.cls_host.push_back(c);
    }
    pd.class_off[c + 1] = (int)perm.size();
  }
  pd.npair = (int)perm.size();
  pd.nprim = nprim_new;
  // final records
  o = 0;
  const size_t f_i0 = carve(pd.npair * sizeof(int4)), f_i1 = carve(pd.npair * sizeof(int4)),
               f_i2 = carve(pd.npair * sizeof(int4)), f_g = carve(pd.npair * sizeof(double4)),
               f_pr = carve((size_t)std::max(nprim_new, 1) * 3 * sizeof(double4)),
               f_prf = carve((size_t)std::max(nprim_new, 1) * 3 * sizeof(float4));
  pd.buf.ensure(std::max<size_t>(o, 256));
  char* pb = pd.buf.as<char>();
  pd.info0 = reinterpret_cast<int4*>(pb + f_i0);
  pd.info1 = reinterpret_cast<int4*>(pb + f_i1);
  pd.info2 = reinterpret_cast<int4*>(pb + f_i2);
  pd.geom = reinterpret_cast<double4*>(pb + f_g);
  pd.prim = reinterpret_cast<double4*>(pb + f_pr);
  pd.primf = reinterpret_cast<float4*>(pb + f_prf);
  if (pd.npair > 0) {
    PF_CUDA(cudaMemcpyAsync(d_perm, perm.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, stream));
    PF_CUDA(cudaMemcpyAsync(d_ps, new_ps.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, stream));
    launch_gather_pairs(pd.npair, d_perm, d_ps, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, d_q, cut,
                        pd.info0, pd.info1, pd.info2, pd.geom, pd.prim, pd.primf, stream);
  }
  PF_CUDA(cudaStreamSynchronize(stream));
  tq[4] = clk::now();
  build_tasks();
  if (opt.verbose) {
    PF_CUDA(cudaStreamSynchronize(stream));
    tq[5] = clk::now();
    auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    std::fprintf(stderr, "pyfacc pairs (ms): host lists %.3f  scratch %.3f  records+Q %.3f  sort+gather %.3f  tasks %.3f\n",
                 ms(tq[0], tq[1]), ms(tq[1], tq[2]), ms(tq[2], tq[3]), ms(tq[3], tq[4]), ms(tq[4], tq[5]));
  }
}

// Contiguous ranges of n items with (as far as the granularity allows)
// equal total cost: range k ends at the first item whose cumulative cost
// reaches k/parts of the total.
void partition_costs(int n, const double* cost, int parts, int* bounds) {
  double total = 0.0;
  for (int i = 0; i < n; ++i) total += cost[i] > 0 ? cost[i] : 0.0;
  bounds[0] = 0;
  double acc = 0.0;
  int k = 1;
  for (int i = 0; i < n && k < parts; ++i) {
    acc += cost[i] > 0 ? cost[i] : 0.0;
    while (k < parts && acc >= total * k / parts) bounds[k++] = i + 1;
  }
  while (k <= parts) bounds[k++] = n;
}

// Ket ranges per bra: kets are the pairs of the ket class, sorted by Q; a
// bra reaches the prefix with Q_bra Q_ket >= thresh (and, in mixed mode, the
// FP64 part is the prefix with Q_bra Q_ket >= fp32_thresh).  For equal
// classes only kets up to the bra itself are canonical.
void System::build_tasks() {
  std::vector<int> hostbuf;
  struct Pending { int bc, kc, prec; size_t off; int nbra; };
  std::vector<Pending> pend;
  const double thr = std::max(opt.schwarz_thresh, 0.0);
  const double t32 = opt.fp32_thresh;
  quartets_total = 0;
  for (int bc = 0; bc < NPAIRCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int nb = pd.class_off[bc + 1] - pd.class_off[bc];
      const int nk = pd.class_off[kc + 1] - pd.class_off[kc];
      const double* qb = pd.q_host.data() + pd.class_off[bc];
      const double* qk = pd.q_host.data() + pd.class_off[kc];
      // kets with qb[i] * qk[j] >= t form a prefix of the ket list (qk
      // descending) that shrinks as i grows (qb descending): one pointer
      // walk per threshold over all bras
      std::vector<int> mfull(nb), m64v(nb);
      int pf = nk, p64 = nk;
      for (int i = 0; i < nb; ++i) {
        if (thr > 0)
          while (pf > 0 && !(qb[i] * qk[pf - 1] >= thr)) --pf;
        if (t32 > 0)
          while (p64 > 0 && !(qb[i] * qk[p64 - 1] >= t32)) --p64;
        int m = pf;
        if (bc == kc) m = std::min(m, i + 1);
        mfull[i] = m;
        m64v[i] = std::min(p64, m);
      }
      for (int prec = 0; prec < 3; ++prec) {
        Pending p{bc, kc, prec, hostbuf.size(), nb};
        std::vector<int> toff(nb + 1), lo(nb), hi(nb);
        long long quart = 0;
        int ntask = 0;
        for (int i = 0; i < nb; ++i) {
          const int m = mfull[i], m64 = m64v[i];
          int l = 0, h = m;
          if (prec == 1) h = m64;
          if (prec == 2) l = m64;
          lo[i] = l;
          hi[i] = h;
          toff[i] = ntask;
          ntask += (h - l + task_width - 1) / task_width;
          quart += h - l;
        }
        toff[nb] = ntask;
        if (prec == 0) quartets_total += quart;
        TaskList& tl = tasks[bc][kc][prec];
        tl.width = task_width;
        tl.nbra = nb;
        tl.ntasks = ntask;
        tl.nquartets = quart;
        hostbuf.insert(hostbuf.end(), toff.begin(), toff.end());
        hostbuf.insert(hostbuf.end(), lo.begin(), lo.end());
        hostbuf.insert(hostbuf.end(), hi.begin(), hi.end());
        pend.push_back(p);
      }
    }
  task_buf.ensure(std::max<size_t>(hostbuf.size() * sizeof(int), 256));
  int* d = task_buf.as<int>();
  // device-built lists: same shapes, filled per Fock build
  size_t dyn_ints = 2 * NQCLASS;
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) dyn_ints += 2 * (3 * (size_t)(pd.class_off[bc + 1] - pd.class_off[bc]) + 1);
  dyn_buf.ensure(dyn_ints * sizeof(int) + 256);
  int* dd = dyn_buf.as<int>();
  dyn.ntasks_dev = dd;
  dd += 2 * NQCLASS;
  dyn.dmax_global = reinterpret_cast<double*>(dyn_buf.as<char>() + dyn_ints * sizeof(int) + 128 - (dyn_ints * sizeof(int)) % 128);
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int qc = (bc == 0) ? 0 : (bc == 1 ? 1 + kc : 3 + kc);
      const int nb = pd.class_off[bc + 1] - pd.class_off[bc];
      for (int part = 0; part < 2; ++part) {
        TaskList& tl = dyn.lists[2 * qc + part];
        tl.width = task_width;
        tl.nbra = nb;
        tl.ntasks = std::max(1, tasks[bc][kc][0].ntasks);
        tl.task_off = dd;
        tl.ket_lo = dd + nb + 1;
        tl.ket_hi = dd + 2 * nb + 1;
        tl.ntasks_dev = dyn.ntasks_dev + 2 * qc + part;
        dd += 3 * nb + 1;
      }
    }
  PF_CUDA(cudaMemcpyAsync(d, hostbuf.data(), hostbuf.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
  const int nsh = std::max(opt.shard_count, 1), rank = std::min(std::max(opt.shard_rank, 0), nsh - 1);
  for (auto& p : pend) {
    TaskList& tl = tasks[p.bc][p.kc][p.prec];
    tl.task_off = d + p.off;
    tl.ket_lo = d + p.off + p.nbra + 1;
    tl.ket_hi = d + p.off + 2 * p.nbra + 1;
    if (nsh > 1) {
      // this shard's bra range of the list, balanced by task counts
      const int* toff = hostbuf.data() + p.off;
      std::vector<double> cost(p.nbra);
      for (int i = 0; i < p.nbra; ++i) cost[i] = toff[i + 1] - toff[i];
      std::vector<int> bounds(nsh + 1);
      partition_costs(p.nbra, cost.data(), nsh, bounds.data());
      const int b0 = bounds[rank], b1 = bounds[rank + 1];
      const int* lo = hostbuf.data() + p.off + p.nbra + 1;
      const int* hi = hostbuf.data() + p.off + 2 * p.nbra + 1;
      long long q = 0;
      for (int i = b0; i < b1; ++i) q += hi[i] - lo[i];
      tl.bra_offset = b0;
      tl.nbra = b1 - b0;
      tl.task_off += b0;
      tl.ket_lo += b0;
      tl.ket_hi += b0;
      tl.task_begin = toff[b0];
      tl.ntasks = toff[b1] - toff[b0];
      tl.nquartets = q;
    }
  }
  PF_CUDA(cudaStreamSynchronize(stream));
}

void System::alloc_matrices() {
  const size_t n2 = (size_t)nbf * nbf;
  const int nmat = 30 + 4 * std::max(opt.diis_size, 1);
  mats.ensure(nmat * n2 * sizeof(double) + 96 * sizeof(double) + ns * ns * sizeof(float) + 1024);
  double* m = mats.as<double>();
  auto take = [&]() { double* r = m; m += n2; return r; };
  S = take(); T = take(); Vm = take(); H = take(); X = take();
  F[0] = take(); F[1] = take(); J = take(); K[0] = take(); K[1] = take();
  P[0] = take(); P[1] = take(); Pbuilt[0] = take(); Pbuilt[1] = take(); Pold[0] = take(); Pold[1] = take();
  W1 = take(); W2 = take(); W3 = take(); Err[0] = take(); Err[1] = take(); Cm[0] = take(); Cm[1] = take();
  Wm = take();
  Pu[0] = take(); Pu[1] = take(); Pu[2] = take(); Pu[3] = take();
  Pp[0] = take(); Pp[1] = take();
  const int nd = std::max(opt.diis_size, 1);
  for (int i = 0; i < nd; ++i) {
    diis_F.push_back(m); m += 2 * n2;
    diis_E.push_back(m); m += 2 * n2;
  }
  small = m; m += 48;
  pstate = m; m += 48;  // purification graph state (24 doubles used)
  dmax = reinterpret_cast<float*>(m);
  const size_t red_bytes = (size_t)RED_BLOCKS * (nd + 3) * sizeof(double);
  small_buf.ensure(2 * nbf * sizeof(double) + 256 + sizeof(JkStats) + 256 + 64 * sizeof(double*) + 256 +
                   3 * natoms * sizeof(double) + 256 + 256 + red_bytes + 256 + nbf * sizeof(double) + 256 + 256);
  {
    char* b = small_buf.as<char>();
    size_t o = 0;
    auto take = [&](size_t n) { char* r = b + o; o += (n + 255) / 256 * 256; return r; };
    eps_dev = reinterpret_cast<double*>(take(2 * nbf * sizeof(double)));
    info_dev = reinterpret_cast<int*>(take(sizeof(int)));
    stats_dev = reinterpret_cast<unsigned long long*>(take(sizeof(JkStats)));
    ptrs_dev = reinterpret_cast<const double**>(take(64 * sizeof(double*)));
    grad_dev = reinterpret_cast<double*>(take(3 * natoms * sizeof(double)));
    red_part = reinterpret_cast<double*>(take(red_bytes));
    occ_dev = reinterpret_cast<double*>(take(nbf * sizeof(double)));
    pmin_dev = reinterpret_cast<double*>(take(sizeof(double)));
  }
  {
    const std::vector<double> occ = atomic_occupations();
    PF_CUDA(cudaMemcpy(occ_dev, occ.data(), nbf * sizeof(double), cudaMemcpyHostToDevice));
  }
  int lwork = 0;
  PF_CUSOLVER(cusolverDnDsyevd_bufferSize(cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nbf, W1, nbf,
                                          eps_dev, &lwork));
  syev_work.ensure(std::max<size_t>((size_t)lwork * sizeof(double), 256));
  syev_lwork = lwork;
}

void System::release_extra() {
  small_buf.release();
  eps_dev = nullptr;
  info_dev = nullptr;
  stats_dev = nullptr;
  ptrs_dev = nullptr;
  grad_dev = nullptr;
  red_part = nullptr;
  occ_dev = nullptr;
  pmin_dev = nullptr;
}

}  // namespace pyfacc
