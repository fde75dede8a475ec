// pyfacc_jk_noalloc: Coulomb and exchange matrices of one molecule without
// any device allocation.
//
// Who needs this: programs that hand all of a GPU's memory to their own
// allocator at start-up -- a deep-learning framework whose caching allocator
// reserves most of HBM, or a long-running service that sizes a memory pool
// once and forbids allocations afterwards.  In such a process a library that
// calls cudaMalloc for its working buffers either fails or punches holes in
// the caller's pool.  This entry point touches no allocator: the caller
// passes the density and the J/K outputs (device memory it owns), and every
// intermediate buffer -- shells, shell-pair records, primitive pairs,
// Schwarz factors, task lists and density block maxima -- lives in one fixed
// array below, reserved statically in this library's device image.
//
// The array: PYFACC_NOALLOC_SCRATCH_BYTES (64 MiB) on every GPU on which the
// library is loaded, held until the process exits.  A molecule whose working
// set does not fit is rejected with PYFACC_ERR_INVALID before any device work
// (pyfacc_last_message() gives the bytes needed); STO-3G alkanes up to about
// C70 fit.  Other failures are reported the same way, as status codes.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory) and
// uploads the Boys tables.  That first call should come before any stream
// capture on the device.
//
// Stream: the work runs on the legacy default stream, which waits for the
// caller's blocking streams but not for streams created non-blocking (torch's
// side streams, for instance).  Whatever writes D_dev on such a stream must
// have finished (stream or event synchronised) before the call; J_dev and
// K_dev are complete when it returns.
//
// Sharing: every call uses the same array and leaves the last call's data in
// it.  Two calls whose work overlapped on the GPU would race on it, so calls
// from this process take a lock and return only after their kernels have
// finished.  Everything read from the array is written earlier in the same
// call; J and K are cleared before the atomic accumulation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"

#define PYFACC_NOALLOC_SCRATCH_BYTES (64u << 20)

namespace {

static __device__ __align__(256) unsigned char g_jk_scratch[PYFACC_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
std::vector<void*> g_scratch_addr;  // per device, from cudaGetSymbolAddress

unsigned char* scratch_on(int dev) {
  if ((int)g_scratch_addr.size() <= dev) g_scratch_addr.resize(dev + 1, nullptr);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_jk_scratch);
    if (e != cudaSuccess || !p)
      throw pyfacc::Error(PYFACC_ERR_CUDA, std::string("cudaGetSymbolAddress(g_jk_scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

// Bump carving of the static array.
struct Carver {
  unsigned char* base;
  size_t off = 0;
  template <typename T> T* take(size_t n) {
    T* p = reinterpret_cast<T*>(base + off);
    off += (std::max<size_t>(n, 1) * sizeof(T) + 255) / 256 * 256;
    return p;
  }
};

}  // namespace

using pyfacc::Error;

extern "C" int pyfacc_jk_noalloc(const pyfacc_molecule* mol, const char* data_dir, double schwarz_thresh,
                                 const double* D_dev, double* J_dev, double* K_dev) {
  if (!mol || !D_dev || !J_dev || !K_dev || mol->natoms <= 0 || !mol->z || !mol->coords || !mol->basis)
    return PYFACC_ERR_INVALID;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  try {
    using namespace pyfacc;
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = 0;  // the legacy default stream (see the header comment)

    // ---- basis (host)
    const int natoms = mol->natoms;
    std::vector<std::string> species(natoms);
    std::vector<double> xyz(mol->coords, mol->coords + 3 * natoms);
    for (int a = 0; a < natoms; ++a) {
      if (mol->species) {
        std::string t(mol->species + 2 * a, 2);
        while (!t.empty() && (t.back() == ' ' || t.back() == '\0')) t.pop_back();
        species[a] = t;
      } else {
        species[a] = element_symbol(mol->z[a]);
      }
      if (element_z(species[a]) == 0) throw Error(PYFACC_ERR_ELEMENT, "unknown element at atom " + std::to_string(a));
    }
    const Basis B = build_basis(resolve_basis_file(mol->basis, data_dir), species, xyz);
    const int ns = (int)B.shells.size(), nbf = B.nbf;
    for (const Shell& sh : B.shells)
      if (sh.l > 1) throw Error(PYFACC_ERR_UNSUPPORTED_L, "pyfacc_jk_noalloc covers s and p shells only");

    // ---- shells and the canonical pair list grouped by class (host)
    std::vector<double4> cen(ns);
    std::vector<int4> desc(ns);
    std::vector<int> np(ns), nf(ns), bfo(ns + 1);
    std::vector<double> ex, co;
    for (int i = 0; i < ns; ++i) {
      const Shell& sh = B.shells[i];
      cen[i] = make_double4(sh.c[0], sh.c[1], sh.c[2], 0.0);
      desc[i] = make_int4(sh.l, sh.atom, B.bf_off[i], (int)ex.size());
      np[i] = (int)sh.ex.size();
      nf[i] = (sh.l + 1) * (sh.l + 2) / 2;
      bfo[i] = B.bf_off[i];
      ex.insert(ex.end(), sh.ex.begin(), sh.ex.end());
      co.insert(co.end(), sh.co.begin(), sh.co.end());
    }
    bfo[ns] = nbf;
    std::vector<int4> pl0, pl1;
    int off[NCLASS + 1] = {0, 0, 0, 0};
    int nprim = 0;
    for (int c = 0; c < NCLASS; ++c) {
      for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) {
          int a = i, b = j;
          if (B.shells[a].l < B.shells[b].l) std::swap(a, b);
          if (B.shells[a].l + B.shells[b].l != c) continue;
          pl0.push_back(make_int4(a, b, nprim, 0));
          pl1.push_back(make_int4(0, nbf, 0, 0));
          nprim += np[a] * np[b];
        }
      off[c + 1] = (int)pl0.size();
    }
    const int npair = off[NCLASS];

    // ---- size check before any device work
    auto need = [&](size_t ntask_ints) {
      Carver c{nullptr};
      c.take<double4>(ns); c.take<int4>(ns); c.take<int>(ns); c.take<double>(ex.size()); c.take<double>(co.size());
      c.take<int>(ns + 1); c.take<int>(ns);
      c.take<int4>(npair); c.take<int4>(npair);                       // pair list
      for (int k = 0; k < 2; ++k) {                                   // unsorted + sorted records
        c.take<int4>(npair); c.take<int4>(npair); c.take<int4>(npair); c.take<double4>(npair);
        c.take<double4>((size_t)3 * nprim);
      }
      c.take<double>(npair); c.take<int>(npair); c.take<int>(npair); c.take<int>(npair);
      c.take<float>((size_t)ns * ns);
      c.take<int>(ntask_ints);
      return c.off;
    };
    // task ints are at most 3 * (npair + number of class pairs)
    const size_t worst = need((size_t)3 * (npair + 6) * NCLASS);
    if (worst > PYFACC_NOALLOC_SCRATCH_BYTES)
      throw Error(PYFACC_ERR_INVALID, "pyfacc_jk_noalloc: molecule needs " + std::to_string(worst) +
                                          " bytes of scratch, the static array holds " +
                                          std::to_string((size_t)PYFACC_NOALLOC_SCRATCH_BYTES));

    // ---- device set-up (first call on this device) and carving of the array
    unsigned char* base = scratch_on(dev);
    ensure_boys_tables(dev);
    Carver cv{base};
    ShellDev shd;
    shd.ns = ns;
    shd.cen = cv.take<double4>(ns);
    shd.desc = cv.take<int4>(ns);
    shd.nprim = cv.take<int>(ns);
    shd.ex = cv.take<double>(ex.size());
    shd.co = cv.take<double>(co.size());
    int* d_bfo = cv.take<int>(ns + 1);
    int* d_nf = cv.take<int>(ns);
    int4* d_pl0 = cv.take<int4>(npair);
    int4* d_pl1 = cv.take<int4>(npair);
    PairData tmp;
    tmp.info0 = cv.take<int4>(npair);
    tmp.info1 = cv.take<int4>(npair);
    tmp.info2 = cv.take<int4>(npair);
    tmp.geom = cv.take<double4>(npair);
    tmp.prim = cv.take<double4>((size_t)3 * nprim);
    PairData pd;
    pd.info0 = cv.take<int4>(npair);
    pd.info1 = cv.take<int4>(npair);
    pd.info2 = cv.take<int4>(npair);
    pd.geom = cv.take<double4>(npair);
    pd.prim = cv.take<double4>((size_t)3 * nprim);
    double* d_q = cv.take<double>(npair);
    int* d_perm = cv.take<int>(npair);
    int* d_ps = cv.take<int>(npair);
    int* d_kept = cv.take<int>(npair);
    const double cut = PRIM_CUT_REL * max_prim_prefactor(B);
    float* d_dmax = cv.take<float>((size_t)ns * ns);
    int* d_tasks = cv.take<int>((size_t)3 * (npair + 6) * NCLASS);

    PF_CUDA(cudaMemcpyAsync(shd.cen, cen.data(), ns * sizeof(double4), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(shd.desc, desc.data(), ns * sizeof(int4), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(shd.nprim, np.data(), ns * sizeof(int), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(shd.ex, ex.data(), ex.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(shd.co, co.data(), co.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d_bfo, bfo.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d_nf, nf.data(), ns * sizeof(int), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d_pl0, pl0.data(), npair * sizeof(int4), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d_pl1, pl1.data(), npair * sizeof(int4), cudaMemcpyHostToDevice, s));

    // ---- pair records and Schwarz factors, then sort by Q inside each class
    launch_build_pairs(shd, npair, d_pl0, d_pl1, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, cut, d_kept, s);
    launch_schwarz(tmp, off, d_q, s);
    std::vector<double> q(npair);
    std::vector<int> kept(npair);
    PF_CUDA(cudaMemcpyAsync(q.data(), d_q, npair * sizeof(double), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaMemcpyAsync(kept.data(), d_kept, npair * sizeof(int), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    const double qmax = npair ? *std::max_element(q.begin(), q.end()) : 0.0;
    std::vector<int> perm, new_ps;
    std::vector<double> qs;
    int nprim_new = 0;
    pd.class_off[0] = 0;
    for (int c = 0; c < NCLASS; ++c) {
      std::vector<int> idx;
      for (int k = off[c]; k < off[c + 1]; ++k)
        if (schwarz_thresh <= 0 || q[k] * qmax >= schwarz_thresh) idx.push_back(k);
      std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return q[x] > q[y]; });
      for (int k : idx) {
        perm.push_back(k);
        new_ps.push_back(nprim_new);
        nprim_new += kept[k];
        qs.push_back(q[k]);
      }
      pd.class_off[c + 1] = (int)perm.size();
    }
    pd.npair = (int)perm.size();
    if (pd.npair > 0) {
      PF_CUDA(cudaMemcpyAsync(d_perm, perm.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, s));
      PF_CUDA(cudaMemcpyAsync(d_ps, new_ps.data(), pd.npair * sizeof(int), cudaMemcpyHostToDevice, s));
      launch_gather_pairs(pd.npair, d_perm, d_ps, tmp.info0, tmp.info1, tmp.info2, tmp.geom, tmp.prim, d_q, cut,
                          pd.info0, pd.info1, pd.info2, pd.geom, pd.prim, nullptr, s);
    }

    // ---- task lists (FP64, Schwarz only)
    std::vector<int> hostbuf;
    struct Item { int bc, kc; size_t at; int nbra; int ntask; };
    std::vector<Item> items;
    const double thr = std::max(schwarz_thresh, 0.0);
    for (int bc = 0; bc < NCLASS; ++bc)
      for (int kc = 0; kc <= bc; ++kc) {
        const int nb = pd.class_off[bc + 1] - pd.class_off[bc];
        const int nk = pd.class_off[kc + 1] - pd.class_off[kc];
        const double* qb = qs.data() + pd.class_off[bc];
        const double* qk = qs.data() + pd.class_off[kc];
        std::vector<int> toff(nb + 1), lo(nb, 0), hi(nb);
        int ntask = 0;
        for (int i = 0; i < nb; ++i) {
          int m = nk;
          if (thr > 0) {
            int a = 0, b = nk;
            while (a < b) {
              const int mid = (a + b) / 2;
              if (qb[i] * qk[mid] >= thr) a = mid + 1; else b = mid;
            }
            m = a;
          }
          if (bc == kc) m = std::min(m, i + 1);
          hi[i] = m;
          toff[i] = ntask;
          ntask += (m + TASK_WIDTH - 1) / TASK_WIDTH;
        }
        toff[nb] = ntask;
        items.push_back({bc, kc, hostbuf.size(), nb, ntask});
        hostbuf.insert(hostbuf.end(), toff.begin(), toff.end());
        hostbuf.insert(hostbuf.end(), lo.begin(), lo.end());
        hostbuf.insert(hostbuf.end(), hi.begin(), hi.end());
      }
    if (!hostbuf.empty())
      PF_CUDA(cudaMemcpyAsync(d_tasks, hostbuf.data(), hostbuf.size() * sizeof(int), cudaMemcpyHostToDevice, s));

    // ---- J/K: clear the accumulators, block maxima, class kernels, J + J^T
    const size_t n2 = (size_t)nbf * nbf;
    PF_CUDA(cudaMemsetAsync(J_dev, 0, n2 * sizeof(double), s));
    PF_CUDA(cudaMemsetAsync(K_dev, 0, n2 * sizeof(double), s));
    launch_dmax(ns, d_bfo, d_nf, nbf, D_dev, nullptr, nullptr, d_dmax, s);
    JkArgs a;
    a.Dj = D_dev;
    a.Dk0 = D_dev;
    a.Dk1 = D_dev;
    a.J = J_dev;
    a.K0 = K_dev;
    a.K1 = K_dev;
    a.dmax = schwarz_thresh > 0 ? d_dmax : nullptr;
    a.ns_ld = ns;
    a.thresh = schwarz_thresh;
    a.stats = nullptr;
    int num_sms = 148;
    PF_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    for (const Item& it : items) {
      TaskList tl;
      tl.nbra = it.nbra;
      tl.ntasks = it.ntask;
      tl.task_off = d_tasks + it.at;
      tl.ket_lo = d_tasks + it.at + it.nbra + 1;
      tl.ket_hi = d_tasks + it.at + 2 * it.nbra + 1;
      launch_jk(pd, tl, it.bc, it.kc, false, 1, a, num_sms, s);
    }
    launch_symmetrize_add(nbf, J_dev, s);
    launch_symmetrize_add(nbf, K_dev, s);
    PF_CUDA(cudaStreamSynchronize(s));
    return PYFACC_OK;
  } catch (const Error& e) {
    pyfacc::set_last_message(e.what());
    return e.status;
  } catch (const std::exception& e) {
    pyfacc::set_last_message(e.what());
    return PYFACC_ERR_INVALID;
  }
}
