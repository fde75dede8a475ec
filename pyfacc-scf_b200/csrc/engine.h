// Internal declarations of the B200 Hartree-Fock engine.
//
// Device data layout (one molecule, or a batch of molecules packed together):
//  * shells       SoA: centre (double4), l, atom, bf offset, primitive range
//  * shell pairs  canonical pairs (a, b) with l_a >= l_b, grouped by class
//                 ss | ps | pp and sorted by Schwarz factor Q_ab (descending)
//                 inside a class:  info0 = {bf_a, bf_b, prim_start, n_prim},
//                 info1 = {shell_a, shell_b, atom_a, atom_b},
//                 info2 = {matrix offset (lo, hi), ld, molecule},
//                 geom = {A-B, Q_ab}
//  * prim pairs   3 x double4 per primitive pair:
//                 {p, 1/(2p), K, alpha}, {P, 0}, {P-A, 0} with
//                 K = c_a c_b N_a N_b exp(-alpha beta/p |AB|^2) sqrt(2) pi^(5/4) / p
//                 so that a primitive quartet prefactor is K_ab K_cd / sqrt(p+q);
//                 primitive pairs with |K| < 1e-16 max|K| are left out.
//  * tasks        per (bra class, ket class, precision): for bra pair i the
//                 ket range [ket_lo[i], ket_hi[i]) in chunks of 32 (one warp,
//                 one ket per lane); task_off is the exclusive prefix sum.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include <stdexcept>
#include "pyfacc_b200.h"

namespace pyfacc {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define PF_CUDA(x)                                                                          \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess)                                                                  \
      throw ::pyfacc::Error(PYFACC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int NCLASS = 3;        // ss, ps, pp: the pair classes of the straight-line kernels
constexpr int NQCLASS = 6;       // (ss|ss) (ps|ss) (ps|ps) (pp|ss) (pp|ps) (pp|pp)
// With d shells three more pair classes follow: ds, dp, dd (l_a >= l_b);
// their quartets run in the warp-cooperative kernels of kernels_d.cu.
constexpr int NPAIRCLASS = 6;
constexpr int NDQCLASS = 15;     // quartet classes with a d pair: bra class >= ket class
inline int pair_class(int la, int lb) { return la == 0 ? 0 : (la == 1 ? 1 + lb : 3 + lb); }  // la >= lb
// index of the d quartet class (bra pair class bc in 3..5, ket class kc <= bc)
inline int dclass_index(int bc, int kc) { return bc == 3 ? kc : (bc == 4 ? 4 + kc : 9 + kc); }
// primitive-quartet cut relative to the quartet screening threshold:
// |K_ab K_cd| max|D| < PRIM_QUARTET_REL * thresh skips a primitive quartet
// (its integral is at most ~1.5 |K_ab K_cd|, as F_m <= 1 and p + q > 0.4
// for STO-nG exponents).  1e-2 moves FP64 energies of C20H42..C100H202 by
// 2e-11..1e-10 Ha; 1 moves them by ~1e-8 and stalls the incremental builds
// of mixed precision.
constexpr double PRIM_QUARTET_REL = 1e-2;
// the same for derivative integrals (factors 2 alpha <= ~200 for STO-nG
// exponents): the screening threshold itself moves the gradient of
// C20H42..C100H202 by ~1e-9 Ha/bohr and leaves it translationally invariant
// (the fourth centre is minus the sum of the other three)
constexpr double PRIM_QUARTET_REL_GRAD = 1.0;
// The derivative factor 2 alpha grows with the tightest primitive: above an
// exponent of 100 (core shells of P and heavier atoms, the STO-6G carbon 1s)
// the gradient cut shrinks by 100 / alpha_max (grad_prim_cut_scale below),
// so that the bound on a skipped derivative integral stays where it is for
// the light atoms.
constexpr double GRAD_CUT_ALPHA = 100.0;
// quartet screening threshold of the all-FP32 builds of the first mixed
// iterations (their error is discarded by the full build that ends them);
// 1e-8 costs C100H202 an extra iteration
constexpr double COARSE_SCREEN = 1e-9;
// ... and how many times looser it may be while the DIIS error is still
// far above coarse_err (it scales with err / coarse_err, capped here).
// 100: C40H82 mixed step 30.0 -> 28.8 ms, C100H202 170 -> 162 ms at the
// same iteration counts; 1000 costs C40H82 an iteration, 10000 C100H202
// three.
constexpr double COARSE_SCREEN_SPAN = 100.0;
// the all-FP32 phase ends after this many builds even if the DIIS error
// stays above coarse_err (an oscillating start must still reach the
// mixed builds, on which alone the SCF may converge)
constexpr int COARSE_MAX_ITER = 20;
// one-electron pair screen: a shell pair on two atoms is left out of the
// S/T/V and one-electron-gradient lists when every primitive pair has
// |c_a N_a c_b N_b| exp(-mu R^2) below this.  The remaining factors (overlap
// volume, kinetic terms, 2 pi/p sum Z for the nuclei, p-function and
// derivative polynomials) stay below ~1e9 for STO-nG exponents and
// molecules of up to ~2000 atoms, so a left-out entry is below 1e-16.
constexpr double ONE_E_PAIR_CUT = 1e-25;
// smallest Cholesky pivot L_ii^2 of the overlap matrix (unit diagonal) below
// which it counts as linearly dependent (PYFACC_ERR_LINDEP)
constexpr double LINDEP_PIVOT = 1e-10;
constexpr int TASK_WIDTH = 32;   // default kets per task = lanes per warp
// largest contraction depth of a shell in the libint_*_c one-body entry points
constexpr int LIBINT1E_MAX_PRIM = 32;

// ---------------------------------------------------------------- host basis
struct Shell {
  int l = 0, atom = 0;
  double c[3] = {0, 0, 0};
  std::vector<double> ex, co;
};

struct Basis {
  std::vector<Shell> shells;
  std::vector<int> bf_off;  // nshell + 1
  int nbf = 0;
};

// Scale of the gradient's primitive-quartet cut for a basis (min(1,
// GRAD_CUT_ALPHA / largest exponent)).
inline double grad_prim_cut_scale(const Basis& b) {
  double amax = 0.0;
  for (const Shell& s : b.shells)
    for (double a : s.ex) amax = a > amax ? a : amax;
  return amax > GRAD_CUT_ALPHA ? GRAD_CUT_ALPHA / amax : 1.0;
}

// Argument checks of a molecule (engine.cpp): pointers and finite
// coordinates; throws PYFACC_ERR_INVALID.
void validate_molecule(const pyfacc_molecule& m);

// Diagonal atomic-occupation guess of a minimal basis (scf.cpp).
std::vector<double> atomic_occupations(const Basis& basis, const std::vector<int>& Z, int nelec);

// basis.cpp
const char* element_symbol(int z);
int element_z(const std::string& sym);
std::string resolve_basis_file(const std::string& name, const char* data_dir);
// Shells in the order of basis.f90:9-190 for the given atoms.
Basis build_basis(const std::string& basis_file, const std::vector<std::string>& species,
                  const std::vector<double>& xyz);

// --------------------------------------------------------- device structures
struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t b);
  void release();
  ~DeviceBuf() { release(); }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct TaskList {
  int nbra = 0;
  long long nquartets = 0;
  int ntasks = 0;              // launch bound (the exact count for static lists)
  int* task_off = nullptr;     // device, nbra + 1
  int* ket_lo = nullptr;       // device, nbra
  int* ket_hi = nullptr;       // device, nbra
  const int* ntasks_dev = nullptr;  // device count of a list built on the GPU
  int bra_offset = 0;   // first bra of this (shard of the) list within its class
  int task_begin = 0;   // global index of the first task (task_off values are global)
  int width = TASK_WIDTH;  // kets per task: 32, 16 or 8 (a warp runs 32 / width tasks)
};

// Packed pair data of one molecule or of a batch (every pair stores the
// offset and leading dimension of its molecule's matrices).
struct PairData {
  int npair = 0;
  int class_off[NPAIRCLASS + 1] = {0, 0, 0, 0, 0, 0, 0};  // s/p classes, then ds, dp, dd
  int nprim = 0;
  int class_maxprim[NPAIRCLASS] = {0, 0, 0, 0, 0, 0};  // largest kept primitive-pair count per class
  int4* info0 = nullptr;     // {bf_a, bf_b, prim_start, n_prim}
  int4* info1 = nullptr;     // {shell_a, shell_b, atom_a, atom_b}
  int4* info2 = nullptr;     // {mat_off lo, mat_off hi, ld, molecule}
  double4* geom = nullptr;   // {ABx, ABy, ABz, Q}
  double4* prim = nullptr;   // 3 per primitive pair
  float4* primf = nullptr;   // the same records in float (FP32 quartets)
  std::vector<double> q_host;   // Q of the sorted pairs
  std::vector<int> cls_host;    // class of the sorted pairs
  std::vector<int> mol_host;    // molecule of the sorted pairs
  DeviceBuf buf;
};

struct JkStats {
  unsigned long long quartets[2][NQCLASS];  // [fp64, fp32][class]
  unsigned long long prims[2][NQCLASS];
};

// Algorithmic flop counts of the generated class routines (eri_classes.cuh).
// Generated operation counts of a class: J/K VRR per primitive quartet and
// HRR per contracted quartet; gradient per primitive quartet (grad) and per
// contracted quartet (gfin: the HRR after the primitive sum, 0 for the
// classes that contract per primitive).
struct ClassFlops { int L, nout, vrr, hrr, grad, gfin; };
const ClassFlops& class_flops(int qclass);
// Flops charged per primitive quartet outside the VRR (prefactors + Boys)
// and per contracted quartet for the J/K digestion.
double prim_overhead_flops(int qclass, bool fp32);
double digest_flops(int qclass, int nk);

// ------------------------------------------------------------- launchers
// Every kernel launch of this library is counted (pyfacc_launch_count).
void count_launch();
void count_launches(long long n);  // kernels of a replayed CUDA graph
long long launch_count();
void ensure_boys_tables(int device);
// The same FP64 Boys tables for the d-shell kernels' copy (kernels_d.cu),
// called by ensure_boys_tables on the current device.
void upload_boys_tables_d(const double* tl, size_t ntl, const double* ex, size_t nex);
void launch_boys_test(int mode, int fp32, int mmax, int n, const double* x, double* out, cudaStream_t s);

struct ShellDev {  // device copies of the shells (packed over a batch)
  int ns = 0;
  double4* cen = nullptr;   // {x, y, z, 0}
  int4* desc = nullptr;     // {l, atom, bf_off, prim_start}
  int* nprim = nullptr;
  double* ex = nullptr;
  double* co = nullptr;
  int4* mol = nullptr;      // batches: per shell {first atom, natoms, mat_off, ld} of its molecule
  DeviceBuf buf;
};

// Pair construction: canonical pair list -> records, then Schwarz factors.
// Primitive pairs with |K| < cut are dropped from the sorted records; kept[i]
// receives the number kept for pair i (may be null).
void launch_build_pairs(const ShellDev& sh, int npair, const int4* pl0, const int4* pl1, int4* info0,
                        int4* info1, int4* info2, double4* geom, double4* prim, double cut, int* kept,
                        cudaStream_t s);
// With a side stream and two events the (pp) class runs there, next to the
// other two classes (the caller's stream waits for it before returning).
void launch_schwarz(const PairData& pd, int npair_class_begin[NCLASS + 1], double* q, cudaStream_t s,
                    cudaStream_t side = nullptr, cudaEvent_t fork = nullptr, cudaEvent_t join = nullptr);
void launch_gather_pairs(int npair, const int* perm, const int* new_pstart, const int4* i0, const int4* i1,
                         const int4* i2, const double4* g, const double4* pr, const double* q, double cut,
                         int4* o0, int4* o1, int4* o2, double4* og, double4* opr, float4* oprf, cudaStream_t s);
// Largest primitive-pair prefactor |K| of a basis (reached at |AB| = 0) and
// the relative cut below which primitive pairs are dropped.
double max_prim_prefactor(const Basis& b);
constexpr double PRIM_CUT_REL = 1e-16;

struct JkArgs {
  const double* Dj;      // density for J
  const double* Dk0;     // densities for K
  const double* Dk1;
  double* J;
  double* K0;
  double* K1;
  const float* dmax;     // shell-block max |D|, ns x ns (or null)
  int ns_ld;             // leading dimension of dmax
  double thresh;         // density-weighted Schwarz threshold
  unsigned long long* stats;  // JkStats layout (device) or null
  // primitive quartets with |K_ab K_cd| max|D| below this are skipped (the
  // primitive pairs of a shell pair are sorted by |K|); 0 = none
  double prim_thresh = 0.0;
};
void launch_jk(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, bool fp32, int nk,
               const JkArgs& a, int num_sms, cudaStream_t s);

// Task lists rebuilt on the GPU for one Fock build from the density bound
// dmax (ns x ns): a bra pair i keeps the ket prefix with
// Q_i Q_j max|D| >= thresh, the FP64 part being the prefix with
// Q_i Q_j max|D| >= fp32_thresh (the rest runs in FP32).  lists[2*(combo)+p]
// for the six class combos (bra >= ket) and p = 0 (FP64), 1 (FP32).
struct DynTaskSet {
  TaskList lists[2 * NQCLASS];
  int* ntasks_dev = nullptr;   // 2 * NQCLASS counts
  double* dmax_global = nullptr;
};
void launch_dyn_tasks(const PairData& pd, const float* dmax, int ns, double thresh, double fp32_thresh,
                      DynTaskSet& dt, cudaStream_t s);

struct GradArgs {
  const double* Pt;
  const double* Pa;
  const double* Pb;
  const float* dmax;
  int ns_ld;
  double thresh;
  int uhf;
  double* grad;  // natoms*3 (packed over a batch via the pair's atom index)
  unsigned long long* stats;  // [0..5] quartets, [6..11] primitive quartets per class, or null
  double prim_thresh = 0.0;   // as JkArgs::prim_thresh
  int natoms_total = 0;       // length of grad / 3; per-block shared-memory sums when small
};
void launch_grad2e(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, bool fp32, const GradArgs& a,
                   int num_sms, cudaStream_t s);

void launch_eri_tensor(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, int nbf,
                       double* eri, cudaStream_t s);

// Quartets with a d pair (kernels_d.cu), FP64, one warp per quartet.
// Schwarz factors of the ds, dp, dd pairs (off: unsorted class offsets).
void launch_schwarz_d(const PairData& pd, const int* off, double* q, int num_sms, cudaStream_t s);
void launch_jk_d(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, int nk, const JkArgs& a,
                 int num_sms, cudaStream_t s);
void launch_grad2e_d(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, const GradArgs& a,
                     int num_sms, cudaStream_t s);
// Full ERI tensor images of a d-class list (tests, small systems).
void launch_eri_tensor_d(const PairData& pd, const TaskList& tl, int bra_class, int ket_class, int nbf, double* eri,
                         cudaStream_t s);

// One-electron integrals over canonical shell pairs of the shells in sh.
struct OneEArgs {
  int natoms;
  const double4* atoms;  // {x, y, z, Z}
  int boys_mode;
  double* S;
  double* T;
  double* V;
  int nbf;
};
// pairs[c]: the shell pairs (a, b) of class c = l_a + l_b with l_a >= l_b.
// One shell pair's overlap (kind 0), kinetic (1) or unit-charge potential
// at C (2) integrals with the caller's coefficients on unnormalised
// primitives, into out (host, nint(la) x nint(lb) row-major); synchronous,
// on the current device's legacy default stream (kernels.cu).
void libint_one_body(int kind, int la, int na, const double* A, const double* ea, const double* ca, int lb, int nb,
                     const double* B, const double* eb, const double* cb, const double* C, double* out);
void launch_one_electron(const ShellDev& sh, const int* npair, const int2* const* pairs, const OneEArgs& a,
                         cudaStream_t s);

struct OneEGradArgs {
  int natoms;
  const double4* atoms;
  int boys_mode;
  const double* P;
  const double* W;
  int nbf;
  double* grad;
  int natoms_total;  // length of grad / 3 (all molecules of a batch)
};
void launch_grad1e(const ShellDev& sh, const int* npair, const int2* const* pairs, const OneEGradArgs& a,
                   int num_sms, cudaStream_t s);

// Small dense helpers.
void launch_symmetrize_add(int n, double* A, cudaStream_t s);
void launch_set_diag(int n, const double* d, double f, double* A, cudaStream_t s);  // A = diag(f d)
void launch_min_diag_sq(int n, const double* L, double* out, cudaStream_t s);   // out = min_i L_ii^2
void launch_identity(int n, double* A, cudaStream_t s);                  // A = I (n x n)             // A = A + A^T
void launch_axpby(long long n, double a, const double* x, double b, double* y, cudaStream_t s);  // y = a x + b y
void launch_antisym(int n, const double* B, double* E, cudaStream_t s);  // E = B - B^T (n x n)
void launch_diff_update(long long n, const double* x, double* y, double* out, cudaStream_t s);  // out = x - y; y = x
void launch_fock_half(int n, const double* H, const double* Jh, double kf, const double* Kh, double* F,
                      cudaStream_t s);  // F = H + Jh + Jh^T - kf (Kh + Kh^T)
void launch_fock(long long n, const double* H, const double* J, double kf, const double* K, double* F,
                 cudaStream_t s);                                          // F = H + J - kf K
// Blocks of the DIIS / energy reductions (their partial sums are combined
// in a fixed order: the results do not depend on scheduling).
constexpr int RED_BLOCKS = 64;
constexpr int MAX_DIIS = 64;  // largest Pulay subspace (diis_size)
// System::jk output forms
constexpr int JK_FULL = 0, JK_HALF = 1, JK_ADD = 2;
// Screening threshold of a mixed-precision gradient's quartets (Q_ab Q_cd
// max|P|): 1e-10 instead of the 1e-12 of the SCF moved max |dg| vs FP64 by
// < 1e-7 Ha/bohr on C40H82, C100H202, C30H61/STO-6G UHF, rna1 and gly30,
// for 15-26% less gradient time
constexpr double GRAD_SCREEN_MIXED = 1e-10;
// part: scratch of RED_BLOCKS x (m + 3) doubles
void launch_dot_many(long long n, const double* x, int m, const double* const* ys, double* out, double* part,
                     cudaStream_t s);
// out = sum_k c[k] src[k] (m host-side pointers and coefficients, any m >= 1)
void launch_lincomb(long long n, int m, const double* const* src, const double* c, double* out, cudaStream_t s);
void launch_scf_reduce(long long n, int uhf, const double* H, const double* Pa, const double* Pb,
                       const double* Fa, const double* Fb, const double* Ea, const double* Eb,
                       const double* Pa_old, const double* Pb_old, double* out, double* part, cudaStream_t s,
                       long long nd = 0, const double* x = nullptr, int m = 0, const double* const* ys = nullptr,
                       double* out_dots = nullptr);  // with m > 0 also out_dots[k] = <x, ys[k]> (length nd)
void launch_dmax(int ns, const int* bf_off, const int* nfun, int nbf, const double* A, const double* B,
                 const double* C, float* dmax, cudaStream_t s);
void launch_zero(void* p, size_t bytes, cudaStream_t s);
// TC2 purification one step per launch (large matrices): state = l_min,
// l_max, Tr X, Tr X^2, converged, steps, remaining final steps.
void launch_gersh(int n, const double* F, double* state, cudaStream_t s);
void launch_tc2_init(int n, const double* F, const double* state, double* X, cudaStream_t s);
void launch_tc2_step(int n, double nocc, const double* Xin, const double* X2, double* Xout, const double* sin,
                     double* sout, cudaStream_t s);

// FP64 tensor-core products of row-major matrices (dense.cu):
// C = alpha op(A) op(B) + beta Y (Y may be null), op = transpose when ta/tb;
// sym: the result is symmetric, only its upper-triangle tiles are computed
// and mirrored; asym_a: op(A) = A - A^T (not with ta).
void launch_dgemm(int m, int n, int k, bool ta, const double* A, int lda, bool tb, const double* B, int ldb,
                  double* C, int ldc, double alpha, const double* Y, int ldy, double beta, bool sym, bool asym_a,
                  cudaStream_t s);
// TC2 purification of the n x n matrix Fp into the projector on its nocc
// lowest eigenvectors as one graph (bounds, X_0 into Xa, a conditional WHILE
// loop of fused steps Xa -> Xb -> Xa); st holds >= 24 doubles of state, of
// which st[9] (done), st[10] (steps) and st[12] (failed) give the outcome.
cudaGraphExec_t build_tc2_graph(int n, int nocc, const double* Fp, double* Xa, double* Xb, double* st, int kmax);
constexpr int TC2_KMAX = 200;
constexpr int TC2_BODY_STEPS = 4;  // TC2 steps per WHILE iteration (even: the result ends in Xa)

double probe_fp64(int device, double* fp32);

// Cost-balanced contiguous split of n weighted items into parts ranges
// (bounds[0..parts]); the host side of pyfacc_partition.
void partition_costs(int n, const double* cost, int parts, int* bounds);

// Detail text returned by pyfacc_last_message() (capi.cpp).
void set_last_message(const std::string& m);

}  // namespace pyfacc
