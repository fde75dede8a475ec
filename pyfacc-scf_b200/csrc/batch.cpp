// Host side of the batched engine: packing of many molecules into one set
// of shells, pairs, task lists and matrices; the per-class task-width
// autotuner; the CUDA-graph SCF loop; the batched gradient.
#include "batch.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>

#include "system.h"

namespace pyfacc {

static double wall_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// f(0) .. f(n - 1) on up to 16 host threads (f must not throw).
template <typename F>
static void parallel_for(int n, F&& f) {
  int nt = (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  nt = std::min(nt, n / 8);
  if (nt <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&] {
      for (int i; (i = next.fetch_add(1)) < n;) f(i);
    });
  for (auto& x : th) x.join();
}

static int qclass_index(int bc, int kc) { return (bc == 0) ? 0 : (bc == 1 ? 1 + kc : 3 + kc); }
static const int kWidths[3] = {32, 16, 8};

BatchMolHost batch_parse(const pyfacc_molecule& m, const pyfacc_options& o, bool* uhf) {
  validate_molecule(m);
  BatchMolHost h;
  h.natoms = m.natoms;
  h.Z.assign(m.z, m.z + m.natoms);
  h.xyz.assign(m.coords, m.coords + 3 * m.natoms);
  h.species.resize(m.natoms);
  for (int a = 0; a < m.natoms; ++a) {
    if (m.species) {
      std::string s(m.species + 2 * a, 2);
      while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
      h.species[a] = s;
    } else {
      h.species[a] = element_symbol(h.Z[a]);
    }
    if (h.species[a].empty() || element_z(h.species[a]) == 0)
      throw Error(PYFACC_ERR_ELEMENT, "unknown element at atom " + std::to_string(a));
  }
  if (m.nalpha >= 0 && m.nbeta >= 0) {
    h.nalpha = m.nalpha;
    h.nbeta = m.nbeta;
  } else {
    System::spin_electrons(h.species, m.charge, &h.nalpha, &h.nbeta);
  }
  *uhf = (o.scf_type == PYFACC_SCF_UHF) || (o.scf_type == PYFACC_SCF_AUTO && h.nalpha != h.nbeta);
  h.nocc = (h.nalpha + h.nbeta + 1) / 2;  // rscf.f90:54-55
  h.basis = build_basis(resolve_basis_file(m.basis, o.data_dir), h.species, h.xyz);
  h.nbf = h.basis.nbf;
  h.ns = (int)h.basis.shells.size();
  // molecule.f90:31-52
  for (int i = 0; i < h.natoms; ++i)
    for (int j = i + 1; j < h.natoms; ++j) {
      double d2 = 0.0;
      for (int x = 0; x < 3; ++x) d2 += (h.xyz[3 * i + x] - h.xyz[3 * j + x]) * (h.xyz[3 * i + x] - h.xyz[3 * j + x]);
      const double r = std::sqrt(d2);
      if (r > 1.0e-10) h.e_nuc += (double)h.Z[i] * h.Z[j] / r;
    }
  return h;
}

Batch::Batch(const std::vector<BatchMolHost>& ms, const pyfacc_options& o) : opt(o), mols(ms) {
  const double t0 = wall_ms();
  nmol = (int)mols.size();
  if (nmol > 65535) throw Error(PYFACC_ERR_INVALID, "at most 65535 molecules per batch");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(PYFACC_ERR_NO_DEVICE, "no CUDA device");
  if (opt.device >= 0) {
    device = opt.device;
    PF_CUDA(cudaSetDevice(device));
  } else {
    PF_CUDA(cudaGetDevice(&device));
  }
  PF_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  if (opt.task_width != 0 && opt.task_width != 8 && opt.task_width != 16 && opt.task_width != 32)
    throw Error(PYFACC_ERR_INVALID, "task_width must be 0, 8, 16 or 32");
  ensure_boys_tables(device);
  ctx = context_acquire(device);
  stream = ctx.stream;
  const int nd = std::min(std::max(opt.diis_size, 0), BATCH_DIIS_MAX);
  long long mo = 0, dofs = 0;
  int aoff = 0, soff = 0;
  for (auto& m : mols) {
    if (m.nbf > BATCH_NBF_MAX) throw Error(PYFACC_ERR_INVALID, "molecule too large for the batched engine");
    m.atom_off = aoff;
    m.shell_off = soff;
    m.mat_off = mo;
    m.diis_off = dofs;
    aoff += m.natoms;
    soff += m.ns;
    mo += (long long)m.nbf * m.nbf;
    dofs += 2LL * nd * m.nbf * m.nbf;
    ns_max = std::max(ns_max, m.ns);
    nbf_max = std::max(nbf_max, m.nbf);
  }
  natoms_tot = aoff;
  ns_tot = soff;
  mtot = mo;
  if (mtot >= (1LL << 31) || (long long)nmol * ns_max * ns_max >= (1LL << 31))
    throw Error(PYFACC_ERR_INVALID, "batch too large: split it into several calls");
  const double t1 = wall_ms();
  upload();
  const double t2 = wall_ms();
  build_pairs();
  const double t3 = wall_ms();
  build_tasks();
  const double t4 = wall_ms();
  alloc();
  timing.ms_setup = wall_ms() - t0;
  if (opt.verbose)
    std::fprintf(stderr, "pyfacc batch setup (ms): context %.2f  shells %.2f  pairs %.2f  tasks %.2f  matrices %.2f\n",
                 t1 - t0, t2 - t1, t3 - t2, t4 - t3, wall_ms() - t4);
}

Batch::~Batch() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (auto& g : graphs)
    if (g) cudaGraphExecDestroy(g);
  if (scf_graph) cudaGraphExecDestroy(scf_graph);
  context_release(ctx);
}

double Batch::energy(int m) const { return st_host[m].E_final + mols[m].e_nuc; }

// Shells of all molecules (atoms and matrix offsets per shell), 1e pair
// lists inside each molecule, per-molecule shell tables.
void Batch::upload() {
  std::vector<double4> cen(ns_tot);
  std::vector<int4> desc(ns_tot), molt(ns_tot), mt(nmol);
  std::vector<int> np(ns_tot), nf(ns_tot), bfo(ns_tot);
  std::vector<double> ex, co;
  std::vector<double4> atoms(natoms_tot);
  std::vector<int2> p1[NCLASS];
  for (int m = 0; m < nmol; ++m) {
    const BatchMolHost& M = mols[m];
    for (int s = 0; s < M.ns; ++s) {
      const Shell& sh = M.basis.shells[s];
      const int g = M.shell_off + s;
      cen[g] = make_double4(sh.c[0], sh.c[1], sh.c[2], 0.0);
      desc[g] = make_int4(sh.l, M.atom_off + sh.atom, M.basis.bf_off[s], (int)ex.size());
      molt[g] = make_int4(M.atom_off, M.natoms, (int)M.mat_off, M.nbf);
      np[g] = (int)sh.ex.size();
      nf[g] = (sh.l + 1) * (sh.l + 2) / 2;
      bfo[g] = M.basis.bf_off[s];
      ex.insert(ex.end(), sh.ex.begin(), sh.ex.end());
      co.insert(co.end(), sh.co.begin(), sh.co.end());
    }
    for (int a = 0; a < M.natoms; ++a)
      atoms[M.atom_off + a] = make_double4(M.xyz[3 * a], M.xyz[3 * a + 1], M.xyz[3 * a + 2], (double)M.Z[a]);
    for (int a = 0; a < M.ns; ++a)
      for (int b = a; b < M.ns; ++b) {
        int x = a, y = b;
        if (M.basis.shells[x].l < M.basis.shells[y].l) std::swap(x, y);
        p1[M.basis.shells[x].l + M.basis.shells[y].l].push_back(make_int2(M.shell_off + x, M.shell_off + y));
      }
    mt[m] = make_int4(M.shell_off, M.ns, (int)M.mat_off, M.nbf);
  }
  for (int c = 0; c < NCLASS; ++c) n1e[c] = (int)p1[c].size();
  const size_t nex = std::max<size_t>(ex.size(), 1);
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_cen = carve(ns_tot * sizeof(double4)), o_desc = carve(ns_tot * sizeof(int4)),
               o_np = carve(ns_tot * sizeof(int)), o_ex = carve(nex * sizeof(double)), o_co = carve(nex * sizeof(double)),
               o_atoms = carve(natoms_tot * sizeof(double4)),
               o_p1 = carve((n1e[0] + n1e[1] + n1e[2] + 3) * sizeof(int2)), o_bfo = carve(ns_tot * sizeof(int)),
               o_nf = carve(ns_tot * sizeof(int)), o_molt = carve(ns_tot * sizeof(int4)),
               o_mt = carve(nmol * sizeof(int4));
  shd.buf.ensure(off);
  char* base = shd.buf.as<char>();
  shd.ns = ns_tot;
  shd.cen = reinterpret_cast<double4*>(base + o_cen);
  shd.desc = reinterpret_cast<int4*>(base + o_desc);
  shd.nprim = reinterpret_cast<int*>(base + o_np);
  shd.ex = reinterpret_cast<double*>(base + o_ex);
  shd.co = reinterpret_cast<double*>(base + o_co);
  shd.mol = reinterpret_cast<int4*>(base + o_molt);
  atoms_dev = reinterpret_cast<double4*>(base + o_atoms);
  pairs1e[0] = reinterpret_cast<int2*>(base + o_p1);
  pairs1e[1] = pairs1e[0] + n1e[0];
  pairs1e[2] = pairs1e[1] + n1e[1];
  bf_off_dev = reinterpret_cast<int*>(base + o_bfo);
  nfun_dev = reinterpret_cast<int*>(base + o_nf);
  mt_dev = reinterpret_cast<int4*>(base + o_mt);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) PF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
  };
  up(shd.cen, cen.data(), ns_tot * sizeof(double4));
  up(shd.desc, desc.data(), ns_tot * sizeof(int4));
  up(shd.nprim, np.data(), ns_tot * sizeof(int));
  up(shd.ex, ex.data(), ex.size() * sizeof(double));
  up(shd.co, co.data(), co.size() * sizeof(double));
  up(shd.mol, molt.data(), ns_tot * sizeof(int4));
  up(atoms_dev, atoms.data(), natoms_tot * sizeof(double4));
  for (int c = 0; c < NCLASS; ++c) up(pairs1e[c], p1[c].data(), n1e[c] * sizeof(int2));
  up(bf_off_dev, bfo.data(), ns_tot * sizeof(int));
  up(nfun_dev, nf.data(), ns_tot * sizeof(int));
  up(mt_dev, mt.data(), nmol * sizeof(int4));
  PF_CUDA(cudaStreamSynchronize(stream));
}

// Canonical pairs of every molecule, Schwarz factors on the GPU, then per
// class sorted by (molecule, Q descending); pairs that cannot reach the
// threshold against the largest Q of their molecule are dropped.
void Batch::build_pairs() {
  double tp[8];
  tp[0] = wall_ms();
  // pairs of class c of molecule m occupy [moff[c][m], moff[c][m + 1]) of
  // the class-major list, in (i, j <= i) shell order (as one molecule's
  // engine lists them); every molecule fills its own ranges
  std::vector<int> moff[NCLASS];
  int off[NCLASS + 1] = {0, 0, 0, 0};
  for (int c = 0; c < NCLASS; ++c) moff[c].assign(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    int nl[2] = {0, 0};
    for (const auto& sh : mols[m].basis.shells) nl[sh.l > 0 ? 1 : 0]++;
    moff[0][m + 1] = nl[0] * (nl[0] + 1) / 2;
    moff[1][m + 1] = nl[0] * nl[1];
    moff[2][m + 1] = nl[1] * (nl[1] + 1) / 2;
  }
  for (int c = 0; c < NCLASS; ++c) {
    moff[c][0] = off[c];
    for (int m = 0; m < nmol; ++m) moff[c][m + 1] += moff[c][m];
    off[c + 1] = moff[c][nmol];
  }
  const int np_all = off[NCLASS];
  std::vector<int4> all0(np_all), all1(np_all);
  std::vector<int> allm(np_all);
  std::vector<long long> np_of(np_all);  // primitive pairs of each pair
  parallel_for(nmol, [&](int m) {
    const BatchMolHost& M = mols[m];
    int pos[NCLASS] = {moff[0][m], moff[1][m], moff[2][m]};
    for (int i = 0; i < M.ns; ++i)
      for (int j = 0; j <= i; ++j) {
        int a = i, b = j;
        if (M.basis.shells[a].l < M.basis.shells[b].l) std::swap(a, b);
        const int c = M.basis.shells[a].l + M.basis.shells[b].l;
        const int k = pos[c]++;
        all0[k] = make_int4(M.shell_off + a, M.shell_off + b, 0, M.shell_off);
        all1[k] = make_int4((int)M.mat_off, M.nbf, m, m * ns_max * ns_max);
        allm[k] = m;
        np_of[k] = (long long)M.basis.shells[a].ex.size() * (long long)M.basis.shells[b].ex.size();
      }
  });
  long long nprim_tot = 0;
  for (int k = 0; k < np_all; ++k) {
    all0[k].z = (int)std::min<long long>(nprim_tot, INT32_MAX);
    nprim_tot += np_of[k];
  }
  if (nprim_tot >= (1LL << 31)) throw Error(PYFACC_ERR_INVALID, "batch too large: split it into several calls");
  size_t o = 0;
  auto carve = [&](size_t bytes) {
    size_t r = o;
    o += (bytes + 255) / 256 * 256;
    return r;
  };
  tp[1] = wall_ms();
  const size_t s_pl0 = carve(np_all * sizeof(int4)), s_pl1 = carve(np_all * sizeof(int4)),
               s_i0 = carve(np_all * sizeof(int4)), s_i1 = carve(np_all * sizeof(int4)),
               s_i2 = carve(np_all * sizeof(int4)), s_g = carve(np_all * sizeof(double4)),
               s_pr = carve((size_t)std::max<long long>(nprim_tot, 1) * 3 * sizeof(double4)),
               s_q = carve(np_all * sizeof(double)), s_perm = carve(np_all * sizeof(int)),
               s_ps = carve(np_all * sizeof(int)), s_kept = carve(np_all * sizeof(int));
  DeviceBuf scratch;
  scratch.ensure(o);
  const double scratch_mb = (double)o / 1048576.0;
  tp[2] = wall_ms();
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
  double maxpref = 0.0;
  for (const auto& m : mols) maxpref = std::max(maxpref, max_prim_prefactor(m.basis));
  const double cut = PRIM_CUT_REL * maxpref;
  PF_CUDA(cudaMemcpyAsync(d_pl0, all0.data(), np_all * sizeof(int4), cudaMemcpyHostToDevice, stream));
  PF_CUDA(cudaMemcpyAsync(d_pl1, all1.data(), np_all * sizeof(int4), cudaMemcpyHostToDevice, stream));
  launch_build_pairs(shd, np_all, d_pl0, d_pl1, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, cut, d_kept,
                     stream);
  launch_schwarz(tmp, off, d_q, stream);
  std::vector<double> q(np_all);
  std::vector<int> kept(np_all);
  PF_CUDA(cudaMemcpyAsync(q.data(), d_q, np_all * sizeof(double), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaMemcpyAsync(kept.data(), d_kept, np_all * sizeof(int), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  tp[3] = wall_ms();
  std::vector<double> qmax(nmol, 0.0);
  for (int k = 0; k < np_all; ++k) qmax[allm[k]] = std::max(qmax[allm[k]], q[k]);
  const double thr = opt.schwarz_thresh;
  // every (class, molecule) segment: the pairs that pass the screening,
  // sorted by Q (descending; ties by index, deterministic), then the
  // segments concatenated class by class, molecule by molecule
  const int nseg = NCLASS * nmol;
  std::vector<int> sorted(np_all), cnt(nseg);
  std::vector<long long> psum(nseg);
  parallel_for(nseg, [&](int g) {
    const int c = g / nmol, m = g % nmol;
    int* out = sorted.data() + moff[c][m];
    int n = 0;
    for (int k = moff[c][m]; k < moff[c][m + 1]; ++k)
      if (thr <= 0 || q[k] * qmax[m] >= thr) out[n++] = k;
    std::sort(out, out + n, [&](int x, int y) { return q[x] > q[y] || (q[x] == q[y] && x < y); });
    long long ps = 0;
    for (int i = 0; i < n; ++i) ps += kept[out[i]];
    cnt[g] = n;
    psum[g] = ps;
  });
  std::vector<int> pos(nseg + 1, 0);
  std::vector<long long> ppos(nseg + 1, 0);
  for (int g = 0; g < nseg; ++g) {
    pos[g + 1] = pos[g] + cnt[g];
    ppos[g + 1] = ppos[g] + psum[g];
  }
  for (int c = 0; c < NCLASS; ++c) {
    pd.class_off[c] = pos[c * nmol];
    seg[c].assign(nmol + 1, 0);
    for (int m = 0; m <= nmol; ++m) seg[c][m] = pos[c * nmol + m] - pos[c * nmol];
  }
  pd.class_off[NCLASS] = pos[nseg];
  std::vector<int> perm(pos[nseg]), new_ps(pos[nseg]);
  parallel_for(nseg, [&](int g) {
    const int c = g / nmol, m = g % nmol;
    const int* in = sorted.data() + moff[c][m];
    long long pp = ppos[g];
    for (int i = 0; i < cnt[g]; ++i) {
      perm[pos[g] + i] = in[i];
      new_ps[pos[g] + i] = (int)pp;
      pp += kept[in[i]];
    }
  });
  const long long nprim_new = ppos[nseg];
  for (int c = 0; c < NPAIRCLASS; ++c) pd.class_maxprim[c] = 0;
  for (int c = 0; c < NCLASS; ++c)
    for (int i = pd.class_off[c]; i < pd.class_off[c + 1]; ++i)
      pd.class_maxprim[c] = std::max(pd.class_maxprim[c], kept[perm[i]]);
  pd.q_host.clear();
  pd.cls_host.clear();
  pd.mol_host.clear();
  pd.npair = (int)perm.size();
  pd.nprim = (int)nprim_new;
  tp[4] = wall_ms();
  o = 0;
  const size_t f_i0 = carve(pd.npair * sizeof(int4)), f_i1 = carve(pd.npair * sizeof(int4)),
               f_i2 = carve(pd.npair * sizeof(int4)), f_g = carve(pd.npair * sizeof(double4)),
               f_pr = carve((size_t)std::max<long long>(nprim_new, 1) * 3 * sizeof(double4)),
               f_prf = carve((size_t)std::max<long long>(nprim_new, 1) * 3 * sizeof(float4));
  pd.buf.ensure(std::max<size_t>(o, 256));
  char* pb = pd.buf.as<char>();
  pd.info0 = reinterpret_cast<int4*>(pb + f_i0);
  pd.info1 = reinterpret_cast<int4*>(pb + f_i1);
  pd.info2 = reinterpret_cast<int4*>(pb + f_i2);
  pd.geom = reinterpret_cast<double4*>(pb + f_g);
  pd.prim = reinterpret_cast<double4*>(pb + f_pr);
  pd.primf = reinterpret_cast<float4*>(pb + f_prf);
  tp[5] = wall_ms();
  if (pd.npair > 0) {
    PF_CUDA(cudaMemcpyAsync(d_perm, perm.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, stream));
    PF_CUDA(cudaMemcpyAsync(d_ps, new_ps.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, stream));
    launch_gather_pairs(pd.npair, d_perm, d_ps, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, d_q, cut,
                        pd.info0, pd.info1, pd.info2, pd.geom, pd.prim, pd.primf, stream);
  }
  PF_CUDA(cudaStreamSynchronize(stream));
  tp[6] = wall_ms();
  scratch.release();
  tp[7] = wall_ms();
  if (opt.verbose)
    std::fprintf(stderr,
                 "pyfacc batch pairs (ms): host lists %.2f  scratch alloc %.2f (%.0f MB)  records+Q %.2f  sort %.2f"
                 "  buffer alloc %.2f (%.0f MB)  gather %.2f  free %.2f\n",
                 tp[1] - tp[0], tp[2] - tp[1], scratch_mb, tp[3] - tp[2], tp[4] - tp[3], tp[5] - tp[4],
                 (double)pd.buf.bytes / 1048576.0, tp[6] - tp[5], tp[7] - tp[6]);
}

// Task lists of every (bra class, ket class) combination, precision part
// and wanted task width, built on the device (batch_tasks.cu): ket ranges
// inside the bra's molecule, then per width the task offsets.  The host
// reads back only the task and quartet counts.
void Batch::build_tasks() {
  const double tt0 = wall_ms();
  // which task widths are needed per class: all three for the tuner, else
  // the fixed width or the cached tuner result
  std::array<int, NQCLASS> fixed{};
  bool have = false;
  if (opt.task_width) {
    fixed.fill(opt.task_width);
    have = true;
  } else {
    have = tuned_widths(&fixed);
  }
  auto wanted = [&](int q, int wi) { return !have || fixed[q] == kWidths[wi]; };
  // device layout: class segments, then per combination 3 x (lo, hi), then
  // the task offsets of each wanted (precision, width)
  size_t n = 0;
  size_t seg_off[NCLASS];
  for (int c = 0; c < NCLASS; ++c) {
    seg_off[c] = n;
    n += (size_t)nmol + 1;
  }
  struct Range { int bc, kc, nb; size_t lo[BATCH_NPARTS], hi[BATCH_NPARTS]; };
  struct Scan { int bc, kc, prec, wi; size_t toff; };
  std::vector<Range> ranges;
  std::vector<Scan> scans;
  int nb_max = 0;
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int nb = pd.class_off[bc + 1] - pd.class_off[bc];
      for (int wi = 0; wi < 3; ++wi)
        for (int prec = 0; prec < BATCH_NPARTS; ++prec) tasks_w[wi][bc][kc][prec] = TaskList();
      if (nb == 0) continue;
      Range r{bc, kc, nb, {}, {}};
      for (int p = 0; p < BATCH_NPARTS; ++p) {
        r.lo[p] = n;
        n += nb;
        r.hi[p] = n;
        n += nb;
      }
      ranges.push_back(r);
      nb_max = std::max(nb_max, nb);
      for (int p = 0; p < BATCH_NPARTS; ++p)
        for (int wi = 0; wi < 3; ++wi) {
          if (!wanted(qclass_index(bc, kc), wi)) continue;
          scans.push_back(Scan{bc, kc, p, wi, n});
          n += (size_t)nb + 1;
        }
    }
  const size_t cnt_off = (n * sizeof(int) + 255) / 256 * 256;
  const size_t bytes = cnt_off + scans.size() * (sizeof(int) + sizeof(long long)) + 256;
  task_buf.ensure(std::max<size_t>(bytes, 256));
  int* d = task_buf.as<int>();
  int* d_nt = reinterpret_cast<int*>(task_buf.as<char>() + cnt_off);
  long long* d_nq = reinterpret_cast<long long*>(task_buf.as<char>() + cnt_off +
                                                 (scans.size() * sizeof(int) + 7) / 8 * 8);
  std::vector<int> segs((size_t)NCLASS * (nmol + 1));
  for (int c = 0; c < NCLASS; ++c) std::copy(seg[c].begin(), seg[c].end(), segs.begin() + (size_t)c * (nmol + 1));
  PF_CUDA(cudaMemcpyAsync(d, segs.data(), segs.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
  const double tt1 = wall_ms();
  BatchRangeArgs ra{};
  ra.geom = pd.geom;
  ra.info2 = pd.info2;
  ra.thresh = std::max(opt.schwarz_thresh, 0.0);
  ra.fp32_thresh = opt.fp32_thresh;
  ra.grad_fp32_thresh = opt.gradient_fp32_thresh > 0 ? opt.gradient_fp32_thresh : opt.fp32_thresh;
  for (size_t k = 0; k < ranges.size(); ++k) {
    const Range& r = ranges[k];
    BatchRangeList& L = ra.l[k];
    L.bra_base = pd.class_off[r.bc];
    L.ket_base = pd.class_off[r.kc];
    L.nb = r.nb;
    L.same = r.bc == r.kc;
    L.seg_b = d + seg_off[r.bc];
    L.seg_k = d + seg_off[r.kc];
    for (int p = 0; p < BATCH_NPARTS; ++p) {
      L.lo[p] = d + r.lo[p];
      L.hi[p] = d + r.hi[p];
    }
  }
  launch_batch_ranges(ra, (int)ranges.size(), nb_max, stream);
  BatchScanArgs sa{};
  sa.ntasks = d_nt;
  sa.nquartets = d_nq;
  auto range_of = [&](int bc, int kc) -> const Range& {
    for (const auto& r : ranges)
      if (r.bc == bc && r.kc == kc) return r;
    throw Error(PYFACC_ERR_INVALID, "internal: missing task range");
  };
  for (size_t k = 0; k < scans.size(); ++k) {
    const Scan& sc = scans[k];
    const Range& r = range_of(sc.bc, sc.kc);
    sa.l[k] = BatchScanList{d + r.lo[sc.prec], d + r.hi[sc.prec], d + sc.toff, r.nb, kWidths[sc.wi]};
  }
  launch_batch_scans(sa, (int)scans.size(), stream);
  std::vector<int> nt(scans.size());
  std::vector<long long> nq(scans.size());
  if (!scans.empty()) {
    PF_CUDA(cudaMemcpyAsync(nt.data(), d_nt, nt.size() * sizeof(int), cudaMemcpyDeviceToHost, stream));
    PF_CUDA(cudaMemcpyAsync(nq.data(), d_nq, nq.size() * sizeof(long long), cudaMemcpyDeviceToHost, stream));
  }
  PF_CUDA(cudaStreamSynchronize(stream));
  for (size_t k = 0; k < scans.size(); ++k) {
    const Scan& sc = scans[k];
    const Range& r = range_of(sc.bc, sc.kc);
    TaskList& tl = tasks_w[sc.wi][sc.bc][sc.kc][sc.prec];
    tl.width = kWidths[sc.wi];
    tl.nbra = r.nb;
    tl.ntasks = nt[k];
    tl.nquartets = nq[k];
    tl.ket_lo = d + r.lo[sc.prec];
    tl.ket_hi = d + r.hi[sc.prec];
    tl.task_off = d + sc.toff;
  }
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int q = qclass_index(bc, kc);
      const int w = have ? fixed[q] : 32;
      const int wi = w == 32 ? 0 : (w == 16 ? 1 : 2);
      for (int p = 0; p < BATCH_NPARTS; ++p) tasks[bc][kc][p] = tasks_w[wi][bc][kc][p];
      timing.width[q] = w;
    }
  if (opt.verbose)
    std::fprintf(stderr, "pyfacc batch tasks (ms): layout %.2f  device build %.2f (%.1f MB, %zu lists)\n", tt1 - tt0,
                 wall_ms() - tt1, (double)bytes / 1048576.0, scans.size());
}

void Batch::alloc() {
  const int nd = std::min(std::max(opt.diis_size, 0), BATCH_DIIS_MAX);
  const size_t m8 = (size_t)mtot * sizeof(double);
  constexpr size_t nmat = 16;
  size_t o = 0;
  auto carve = [&](size_t bytes) {
    size_t r = o;
    o += (bytes + 255) / 256 * 256;
    return r;
  };
  size_t om[nmat];
  for (size_t k = 0; k < nmat; ++k) om[k] = carve(m8);
  const size_t o_diis = carve(std::max<size_t>(2 * nd * m8, 8));
  const size_t o_dmax = carve((size_t)nmol * ns_max * ns_max * sizeof(float));
  const size_t o_stats = carve(sizeof(JkStats) + 2 * NQCLASS * sizeof(unsigned long long));
  const size_t o_grad = carve(3 * (size_t)natoms_tot * sizeof(double));
  const size_t o_act = carve(sizeof(StepReport));
  const size_t o_ctl = carve(sizeof(BatchScfCtl));
  mats.ensure(o);
  char* b = mats.as<char>();
  double* mp[nmat];
  for (size_t k = 0; k < nmat; ++k) mp[k] = reinterpret_cast<double*>(b + om[k]);
  S = mp[0];
  T = mp[1];
  V = mp[2];
  W = mp[15];
  dmax = reinterpret_cast<float*>(b + o_dmax);
  stats_dev = reinterpret_cast<unsigned long long*>(b + o_stats);
  grad_dev = reinterpret_cast<double*>(b + o_grad);
  active_dev = reinterpret_cast<int*>(b + o_act);
  ctl_dev = reinterpret_cast<BatchScfCtl*>(b + o_ctl);
  const size_t st_bytes = (nmol * sizeof(BatchMolState) + 255) / 256 * 256;
  state_buf.ensure(st_bytes + nmol * sizeof(BatchMolDev) + 256);
  BatchMolState* st = state_buf.as<BatchMolState>();
  BatchMolDev* md = reinterpret_cast<BatchMolDev*>(state_buf.as<char>() + st_bytes);
  std::vector<BatchMolDev> mdh(nmol);
  int occ_off = 0;
  occ_host.clear();
  for (int m = 0; m < nmol; ++m) {
    const BatchMolHost& M = mols[m];
    mdh[m] = BatchMolDev{M.nbf, M.nocc, M.ns, M.natoms, occ_off, 0, M.mat_off, M.diis_off};
    const std::vector<double> occ = atomic_occupations(M.basis, M.Z, M.nalpha + M.nbeta);
    occ_host.insert(occ_host.end(), occ.begin(), occ.end());
    occ_off += M.nbf;
  }
  PF_CUDA(cudaMemcpyAsync(md, mdh.data(), nmol * sizeof(BatchMolDev), cudaMemcpyHostToDevice, stream));
  occ_buf.ensure(std::max<size_t>(occ_host.size() * sizeof(double), 256));
  PF_CUDA(cudaMemcpyAsync(occ_buf.as<double>(), occ_host.data(), occ_host.size() * sizeof(double),
                          cudaMemcpyHostToDevice, stream));
  BatchDenseArgs& a = dargs;
  a.mol = md;
  a.st = st;
  a.S = mp[0];
  a.H = mp[3];
  a.X = mp[4];
  a.F = mp[5];
  a.J = mp[6];
  a.K = mp[7];
  a.Jd = mp[8];
  a.Kd = mp[9];
  a.P = mp[10];
  a.Db = mp[11];
  a.T1 = mp[12];
  a.T2 = mp[13];
  a.T3 = mp[14];
  a.diis = reinterpret_cast<double*>(b + o_diis);
  a.ndiis = nd;
  a.max_iter = std::max(opt.max_iter, 1);
  a.rebuild_every = std::max(opt.rebuild_every, 1);
  const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
  a.incremental = (opt.incremental < 0 ? mixed : (opt.incremental != 0)) ? 1 : 0;
  a.e_tol = mixed ? std::max(opt.eps_energy, 1e-8) : opt.eps_energy;
  a.eps_diis = opt.eps_diis;
  a.eps_density = opt.eps_density;
  a.active = active_dev;
  a.max_err = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(active_dev) +
                                                    offsetof(StepReport, max_err));
  a.built_full = 1;
  a.coarse = 0;
  a.smem_nmax = nbf_max;  // nbf <= 160: at most 200 KB of shared memory
  batch_set_smem(a);
  PF_CUDA(cudaStreamSynchronize(stream));
}

void Batch::fock_build(bool mixed_lists, double thresh, unsigned long long* stats, bool all_fp32, bool overlap) {
  launch_batch_dmax(nmol, ns_max, mt_dev, bf_off_dev, nfun_dev, dargs.Db, dmax, stream);
  JkArgs a;
  a.Dj = dargs.Db;
  a.Dk0 = dargs.Db;
  a.Dk1 = dargs.Db;
  a.J = dargs.Jd;
  a.K0 = dargs.Kd;
  a.K1 = dargs.Kd;
  a.dmax = thresh > 0 ? dmax : nullptr;
  a.ns_ld = ns_max;
  a.thresh = thresh;
  a.stats = stats;
  a.prim_thresh = thresh * PRIM_QUARTET_REL;
  const bool fork = overlap;
  cudaStream_t s32 = stream;
  if (fork) {
    PF_CUDA(cudaEventRecord(ctx.fork, stream));
    PF_CUDA(cudaStreamWaitEvent(ctx.side, ctx.fork, 0));
    s32 = ctx.side;
  }
  int nth = 0;
  for (int bc = NCLASS - 1; bc >= 0; --bc)
    for (int kc = bc; kc >= 0; --kc, ++nth) {
      // the two halves swap streams from class to class
      // (single-precision lists: the classes alternate between the streams)
      const bool swap = fork && (nth & 1);
      if (all_fp32) {
        launch_jk(pd, tasks[bc][kc][0], bc, kc, true, 1, a, num_sms, swap ? s32 : stream);
      } else if (mixed_lists) {
        launch_jk(pd, tasks[bc][kc][1], bc, kc, false, 1, a, num_sms, swap ? s32 : stream);
        launch_jk(pd, tasks[bc][kc][2], bc, kc, true, 1, a, num_sms, swap ? stream : s32);
      } else {
        launch_jk(pd, tasks[bc][kc][0], bc, kc, false, 1, a, num_sms, swap ? s32 : stream);
      }
    }
  if (fork) {
    PF_CUDA(cudaEventRecord(ctx.join, ctx.side));
    PF_CUDA(cudaStreamWaitEvent(stream, ctx.join, 0));
  }
}

// Task-width autotuner: every quartet class is timed with tasks of 32, 16
// and 8 kets on the first (full) build of this batch, and the fastest width
// is kept per class.  Results are cached per batch shape (precision and the
// molecules' sizes), so repeated batches of the same shape skip the timing.
static std::mutex g_tune_mu;
static std::map<std::string, std::array<int, NQCLASS>> g_tune_cache;

std::string Batch::tune_key() const {
  std::ostringstream key;
  key << device << ':' << (opt.precision == PYFACC_PRECISION_MIXED ? 'm' : 'd') << ':' << opt.schwarz_thresh << ':'
      << opt.fp32_thresh;
  for (const auto& m : mols) key << ',' << m.nbf << '/' << m.natoms;
  return key.str();
}

bool Batch::tuned_widths(std::array<int, NQCLASS>* w) const {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_cache.find(tune_key());
  if (it == g_tune_cache.end()) return false;
  *w = it->second;
  return true;
}

void Batch::tune() {
  const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
  std::array<int, NQCLASS> best{};
  const bool have = tuned_widths(&best);
  if (!have) {
    const double t0 = wall_ms();
    launch_batch_dmax(nmol, ns_max, mt_dev, bf_off_dev, nfun_dev, dargs.Db, dmax, stream);
    JkArgs a;
    a.Dj = a.Dk0 = a.Dk1 = dargs.Db;
    a.J = dargs.Jd;
    a.K0 = a.K1 = dargs.Kd;
    a.dmax = opt.schwarz_thresh > 0 ? dmax : nullptr;
    a.ns_ld = ns_max;
    a.thresh = opt.schwarz_thresh;
    a.stats = nullptr;
    a.prim_thresh = opt.schwarz_thresh * PRIM_QUARTET_REL;
    cudaEvent_t e0 = ctx.ev0, e1 = ctx.ev1;
    auto run_class = [&](int wi, int bc, int kc) {
      if (mixed) {
        launch_jk(pd, tasks_w[wi][bc][kc][1], bc, kc, false, 1, a, num_sms, stream);
        launch_jk(pd, tasks_w[wi][bc][kc][2], bc, kc, true, 1, a, num_sms, stream);
      } else {
        launch_jk(pd, tasks_w[wi][bc][kc][0], bc, kc, false, 1, a, num_sms, stream);
      }
    };
    for (int bc = 0; bc < NCLASS; ++bc)
      for (int kc = 0; kc <= bc; ++kc) {
        const int q = qclass_index(bc, kc);
        run_class(0, bc, kc);  // warm-up
        float tbest = 0.0f;
        best[q] = kWidths[0];
        for (int wi = 0; wi < 3; ++wi) {
          PF_CUDA(cudaEventRecord(e0, stream));
          run_class(wi, bc, kc);
          PF_CUDA(cudaEventRecord(e1, stream));
          PF_CUDA(cudaEventSynchronize(e1));
          float ms = 0.0f;
          PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          // a narrower tile has to win by 3% to replace a wider one
          if (wi == 0 || ms < 0.97f * tbest) {
            tbest = ms;
            best[q] = kWidths[wi];
          }
        }
      }
    launch_zero(dargs.Jd, (size_t)mtot * sizeof(double), stream);
    launch_zero(dargs.Kd, (size_t)mtot * sizeof(double), stream);
    PF_CUDA(cudaStreamSynchronize(stream));
    timing.ms_tune = wall_ms() - t0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key()] = best;
  }
  for (int bc = 0; bc < NCLASS; ++bc)
    for (int kc = 0; kc <= bc; ++kc) {
      const int q = qclass_index(bc, kc);
      const int wi = best[q] == 32 ? 0 : (best[q] == 16 ? 1 : 2);
      for (int p = 0; p < BATCH_NPARTS; ++p) tasks[bc][kc][p] = tasks_w[wi][bc][kc][p];
      timing.width[q] = best[q];
    }
}

// One SCF iteration of the batch as a CUDA graph: density maxima of Db, the
// J/K class kernels (full builds screen at schwarz_thresh, incremental ones
// at incremental_thresh), the count reset and the dense step.
void Batch::capture_into(cudaGraph_t graph, int variant, bool reset_report, long long* launches) {
  const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
  const double inc_thresh = (mixed && opt.incremental_thresh > 0)
                                ? std::max(opt.incremental_thresh, opt.schwarz_thresh)
                                : opt.schwarz_thresh;
  const bool full = variant == G_FULL || variant == G_CFULL;
  const bool coarse = variant == G_CFULL || variant == G_CINC;
  BatchDenseArgs da = dargs;
  da.built_full = full ? 1 : 0;
  da.coarse = coarse ? 1 : 0;
  const double thresh =
      coarse ? std::max(COARSE_SCREEN, opt.schwarz_thresh) : (full ? opt.schwarz_thresh : inc_thresh);
  const long long c0 = launch_count();
  PF_CUDA(cudaStreamBeginCaptureToGraph(stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  try {
    // a full rebuild of an incremental run builds P itself (the previous
    // step left P_new - P in Db); the first full build has Db = P already
    if (variant == G_FULL && dargs.incremental) launch_batch_full_density(nmol, da, stream);
    fock_build(mixed, thresh, stats_dev, coarse, true);
    if (reset_report) PF_CUDA(cudaMemsetAsync(active_dev, 0, sizeof(StepReport), stream));
    launch_batch_step(nmol, da, stream);
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(stream, &g);
    throw;
  }
  cudaGraph_t g = nullptr;
  PF_CUDA(cudaStreamEndCapture(stream, &g));
  *launches = launch_count() - c0;
}

cudaGraphExec_t Batch::capture(int variant, long long* launches) {
  cudaGraph_t g = nullptr;
  PF_CUDA(cudaGraphCreate(&g, 0));
  try {
    capture_into(g, variant, true, launches);
  } catch (...) {
    cudaGraphDestroy(g);
    throw;
  }
  cudaGraphExec_t e = nullptr;
  const cudaError_t rc = cudaGraphInstantiate(&e, g, 0);
  cudaGraphDestroy(g);
  if (rc != cudaSuccess) throw Error(PYFACC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(rc));
  return e;
}

// The whole SCF of the batch as one graph: WHILE { select kernel (clears
// the step report, sets the SWITCH value from the control state), SWITCH
// over the four iteration variants, update kernel (counts, convergence of
// the batch, next variant, WHILE condition) }.  The host launches it once
// and reads the control state when it is done.
cudaGraphExec_t Batch::build_scf_graph() {
  cudaGraph_t g = nullptr;
  PF_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphExec_t exec = nullptr;
  try {
    cudaGraphConditionalHandle hloop, hvar;
    PF_CUDA(cudaGraphConditionalHandleCreate(&hloop, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hloop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wn = nullptr;
    PF_CUDA(cudaGraphAddNode(&wn, g, nullptr, 0, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    PF_CUDA(cudaGraphConditionalHandleCreate(&hvar, body, 0, 0));
    cudaGraphNode_t sel = nullptr, sw = nullptr, upd = nullptr;
    add_batch_select_node(body, &sel, ctl_dev, active_dev, hvar);
    cudaGraphNodeParams sp{};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = hvar;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = G_N;
    PF_CUDA(cudaGraphAddNode(&sw, body, &sel, 1, &sp));
    const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
    const bool coarse = mixed && dargs.incremental && opt.coarse_err > 0;
    for (int v = 0; v < G_N; ++v) {
      const bool used = v == G_FULL || (v == G_INC && dargs.incremental) || ((v == G_CFULL || v == G_CINC) && coarse);
      if (!used) continue;  // an empty branch
      capture_into(sp.conditional.phGraph_out[v], v, false, &graph_launches[v]);
    }
    add_batch_update_node(body, &upd, &sw, ctl_dev, active_dev, hloop);
    const cudaError_t rc = cudaGraphInstantiate(&exec, g, 0);
    if (rc != cudaSuccess)
      throw Error(PYFACC_ERR_CUDA, std::string("cudaGraphInstantiate (SCF graph): ") + cudaGetErrorString(rc));
  } catch (...) {
    cudaGraphDestroy(g);
    throw;
  }
  cudaGraphDestroy(g);
  return exec;
}

void Batch::run(bool gradient) {
  const bool mixed = opt.precision == PYFACC_PRECISION_MIXED;
  const double t0 = wall_ms();
  cudaEvent_t e0 = ctx.ev0, e1 = ctx.ev1;
  PF_CUDA(cudaMemsetAsync(dargs.st, 0, nmol * sizeof(BatchMolState), stream));
  PF_CUDA(cudaMemsetAsync(stats_dev, 0, sizeof(JkStats), stream));
  // ---- one-electron integrals, orthogonaliser, starting density
  PF_CUDA(cudaEventRecord(e0, stream));
  OneEArgs oa;
  oa.natoms = 0;
  oa.atoms = atoms_dev;
  oa.boys_mode = opt.boys_mode;
  oa.S = S;
  oa.T = T;
  oa.V = V;
  oa.nbf = 0;
  launch_one_electron(shd, n1e, pairs1e, oa, stream);
  double* H = const_cast<double*>(dargs.H);
  launch_axpby(mtot, 1.0, T, 0.0, H, stream);
  launch_axpby(mtot, 1.0, V, 1.0, H, stream);
  launch_batch_lowdin(nmol, dargs, const_cast<double*>(dargs.X), stream);
  const bool core = opt.guess == PYFACC_GUESS_CORE;
  if (!core) launch_batch_guess(nmol, dargs, occ_buf.as<double>(), stream);
  launch_batch_init(nmol, dargs, core ? 1 : 0, stream);
  PF_CUDA(cudaEventRecord(e1, stream));
  PF_CUDA(cudaEventSynchronize(e1));
  float ms = 0.0f;
  PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  timing.ms_1e = ms;
  // ---- task widths, graphs
  if (opt.task_width == 0) tune();
  const double ts = wall_ms();
  // Mixed precision starts with all-FP32 builds while the largest DIIS error
  // of the batch is above coarse_err (dynamic precision, as the single-
  // molecule engine); the next build is a full mixed one, which restarts the
  // incremental chain.
  bool coarse = mixed && dargs.incremental && opt.coarse_err > 0;
  int it = 0;
  if (!scf_graph && !scf_graph_failed) {
    try {
      scf_graph = build_scf_graph();
    } catch (const Error& e) {
      // a driver without conditional graph nodes: one graph launch per
      // iteration instead (below)
      scf_graph_failed = true;
      if (opt.verbose) std::fprintf(stderr, "pyfacc batch: whole-SCF graph unavailable (%s)\n", e.what());
    }
  }
  if (scf_graph) {
    BatchScfCtl c{};
    c.coarse = coarse ? 1 : 0;
    c.variant = coarse ? G_CFULL : G_FULL;
    c.incremental = dargs.incremental;
    c.rebuild_every = dargs.rebuild_every;
    c.max_iter = dargs.max_iter;
    c.coarse_max_iter = COARSE_MAX_ITER;
    c.coarse_err = opt.coarse_err;
    PF_CUDA(cudaMemcpyAsync(ctl_dev, &c, sizeof(c), cudaMemcpyHostToDevice, stream));
    PF_CUDA(cudaGraphLaunch(scf_graph, stream));
    PF_CUDA(cudaMemcpyAsync(&c, ctl_dev, sizeof(c), cudaMemcpyDeviceToHost, stream));
    PF_CUDA(cudaStreamSynchronize(stream));
    long long nl = 2LL * c.it;  // select + update kernels
    for (int v = 0; v < G_N; ++v) nl += c.counts[v] * graph_launches[v];
    count_launches(nl);
    it = c.it;
    timing.iterations = std::min(it, dargs.max_iter);
    scf_launches_last = 1;
  } else {
    if (!graphs[G_FULL]) graphs[G_FULL] = capture(G_FULL, &graph_launches[G_FULL]);
    if (dargs.incremental && !graphs[G_INC]) graphs[G_INC] = capture(G_INC, &graph_launches[G_INC]);
    if (coarse && !graphs[G_CFULL]) graphs[G_CFULL] = capture(G_CFULL, &graph_launches[G_CFULL]);
    if (coarse && !graphs[G_CINC]) graphs[G_CINC] = capture(G_CINC, &graph_launches[G_CINC]);
    int since_full = 0;
    bool restart = false;
    scf_launches_last = 0;
    for (it = 1; it <= dargs.max_iter; ++it) {
      int v;
      if (coarse) {
        v = it == 1 ? G_CFULL : G_CINC;
      } else {
        const bool full = !dargs.incremental || it == 1 || restart || since_full + 1 >= dargs.rebuild_every;
        v = full ? G_FULL : G_INC;
        since_full = full ? 0 : since_full + 1;
        restart = false;
      }
      PF_CUDA(cudaGraphLaunch(graphs[v], stream));
      count_launches(graph_launches[v]);
      ++scf_launches_last;
      PF_CUDA(cudaMemcpyAsync(&report, active_dev, sizeof(StepReport), cudaMemcpyDeviceToHost, stream));
      PF_CUDA(cudaStreamSynchronize(stream));
      if (report.active == 0) break;
      if (coarse) {
        double err;
        std::memcpy(&err, &report.max_err, sizeof(err));
        if (err < opt.coarse_err || it >= COARSE_MAX_ITER) {
          coarse = false;
          restart = true;
        }
      }
    }
    timing.iterations = std::min(it, dargs.max_iter);
  }
  timing.ms_scf = wall_ms() - ts;
  timing.scf_graph_launches = scf_launches_last;
  // ---- FP64 polish of mixed precision: F and E of the final densities
  if (mixed && opt.polish) {
    const double tp = wall_ms();
    launch_batch_polish_density(nmol, dargs, stream);
    fock_build(false, opt.schwarz_thresh, stats_dev);
    launch_batch_polish(nmol, dargs, stream);
    PF_CUDA(cudaStreamSynchronize(stream));
    timing.ms_polish = wall_ms() - tp;
  }
  st_host.resize(nmol);
  PF_CUDA(cudaMemcpyAsync(st_host.data(), dargs.st, nmol * sizeof(BatchMolState), cudaMemcpyDeviceToHost, stream));
  JkStats js;
  PF_CUDA(cudaMemcpyAsync(&js, stats_dev, sizeof(JkStats), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  timing.quartets[0] = timing.quartets[1] = 0;
  timing.flops_fock = 0.0;
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < NQCLASS; ++q) {
      timing.quartets[p] += js.quartets[p][q];
      const ClassFlops& cf = class_flops(q);
      timing.flops_fock += (double)js.prims[p][q] * (cf.vrr + prim_overhead_flops(q, p == 1)) +
                           (double)js.quartets[p][q] * (cf.hrr + digest_flops(q, 1));
    }
  if (gradient) gradient_run();
  timing.ms_total = wall_ms() - t0;
}

// dE/dR = sum P dH - sum W dS + 1/2 sum Gamma d(mn|ls) + dV_nn for every
// molecule: one batched W = 1/2 P F P, the batched one-electron gradient
// kernel and the two-electron gradient over the FP64 task lists.
void Batch::gradient_run() {
  const double t0 = wall_ms();
  cudaEvent_t ev[4];
  for (auto& e : ev) PF_CUDA(cudaEventCreate(&e));
  PF_CUDA(cudaEventRecord(ev[0], stream));
  launch_batch_wdens(nmol, dargs, W, stream);
  launch_batch_dmax(nmol, ns_max, mt_dev, bf_off_dev, nfun_dev, dargs.P, dmax, stream);
  launch_zero(grad_dev, 3 * (size_t)natoms_tot * sizeof(double), stream);
  OneEGradArgs g1;
  g1.natoms = 0;
  g1.atoms = atoms_dev;
  g1.boys_mode = opt.boys_mode;
  g1.P = dargs.P;
  g1.W = W;
  g1.nbf = 0;
  g1.grad = grad_dev;
  g1.natoms_total = natoms_tot;
  PF_CUDA(cudaEventRecord(ev[1], stream));
  launch_grad1e(shd, n1e, pairs1e, g1, num_sms, stream);
  PF_CUDA(cudaEventRecord(ev[2], stream));
  unsigned long long* gstats = stats_dev + sizeof(JkStats) / sizeof(unsigned long long);
  PF_CUDA(cudaMemsetAsync(gstats, 0, 2 * NQCLASS * sizeof(unsigned long long), stream));
  GradArgs g2;
  g2.Pt = dargs.P;
  g2.Pa = dargs.P;
  g2.Pb = dargs.P;
  g2.dmax = opt.schwarz_thresh > 0 ? dmax : nullptr;
  g2.ns_ld = ns_max;
  g2.thresh = opt.schwarz_thresh;
  double cut_scale = 1.0;
  for (const auto& m : mols) cut_scale = std::min(cut_scale, grad_prim_cut_scale(m.basis));
  g2.prim_thresh = opt.schwarz_thresh * PRIM_QUARTET_REL_GRAD * cut_scale;
  g2.natoms_total = natoms_tot;
  g2.uhf = 0;
  g2.grad = grad_dev;
  g2.stats = gstats;
  // FP32 derivative integrals for the quartets with Q_ab Q_cd below
  // gradient_fp32_thresh: on request, and by default in mixed mode (the
  // batch's launches are large enough for the split to pay at any molecule
  // size: 256 water clusters 104 -> 74 ms, max |dg| unchanged at 6e-9)
  const bool split = pd.primf != nullptr &&
                     (opt.gradient_precision == PYFACC_PRECISION_MIXED ||
                      (opt.gradient_precision < 0 && opt.precision == PYFACC_PRECISION_MIXED));
  if (split) {  // the FP32 half on the side stream, overlapping the FP64 half
    PF_CUDA(cudaEventRecord(ctx.fork, stream));
    PF_CUDA(cudaStreamWaitEvent(ctx.side, ctx.fork, 0));
  }
  int nth = 0;
  for (int bc = NCLASS - 1; bc >= 0; --bc)
    for (int kc = bc; kc >= 0; --kc, ++nth) {
      if (split) {  // the two halves swap streams from class to class
        launch_grad2e(pd, tasks[bc][kc][3], bc, kc, false, g2, num_sms, (nth & 1) ? ctx.side : stream);
        launch_grad2e(pd, tasks[bc][kc][4], bc, kc, true, g2, num_sms, (nth & 1) ? stream : ctx.side);
      } else {
        launch_grad2e(pd, tasks[bc][kc][0], bc, kc, false, g2, num_sms, stream);
      }
    }
  if (split) {
    PF_CUDA(cudaEventRecord(ctx.join, ctx.side));
    PF_CUDA(cudaStreamWaitEvent(stream, ctx.join, 0));
  }
  PF_CUDA(cudaEventRecord(ev[3], stream));
  grad_host.assign(3 * (size_t)natoms_tot, 0.0);
  PF_CUDA(cudaMemcpyAsync(grad_host.data(), grad_dev, grad_host.size() * sizeof(double), cudaMemcpyDeviceToHost,
                          stream));
  unsigned long long cnt[2 * NQCLASS];
  PF_CUDA(cudaMemcpyAsync(cnt, gstats, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
  PF_CUDA(cudaStreamSynchronize(stream));
  if (opt.verbose) {
    float a = 0, b = 0, c = 0;
    PF_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
    PF_CUDA(cudaEventElapsedTime(&b, ev[1], ev[2]));
    PF_CUDA(cudaEventElapsedTime(&c, ev[2], ev[3]));
    std::fprintf(stderr, "pyfacc batch gradient (ms): W + dmax %.3f  one-electron %.3f  two-electron %.3f\n", a, b, c);
  }
  for (auto& e : ev) cudaEventDestroy(e);
  timing.flops_grad = 0.0;
  for (int q = 0; q < NQCLASS; ++q)
    timing.flops_grad += (double)cnt[NQCLASS + q] * (class_flops(q).grad + prim_overhead_flops(q, false)) +
                       (double)cnt[q] * class_flops(q).gfin;
  // nuclear repulsion (molecule.f90:31-52 differentiated)
  for (const auto& M : mols)
    for (int i = 0; i < M.natoms; ++i)
      for (int j = 0; j < M.natoms; ++j) {
        if (i == j) continue;
        double d[3], r2 = 0.0;
        for (int x = 0; x < 3; ++x) {
          d[x] = M.xyz[3 * i + x] - M.xyz[3 * j + x];
          r2 += d[x] * d[x];
        }
        const double r = std::sqrt(r2);
        if (r <= 1.0e-10) continue;
        for (int x = 0; x < 3; ++x)
          grad_host[3 * (size_t)(M.atom_off + i) + x] -= (double)M.Z[i] * M.Z[j] * d[x] / (r2 * r);
      }
  timing.ms_grad = wall_ms() - t0;
}

}  // namespace pyfacc
