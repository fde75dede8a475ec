// Batched engine: many closed-shell molecules of uneven size converged
// together on one GPU.
//
// Layout in HBM: the shells, shell pairs and primitive-pair records of all
// molecules are packed into one ShellDev / PairData (pairs sorted by class,
// then molecule, then Schwarz factor, so the kets of a bra are a contiguous
// segment of its own molecule); every n x n matrix of molecule m lives at
// offset mat_off[m] = sum_{k<m} n_k^2 of a packed array with leading
// dimension n_m, and its shell-block density maxima at m * ns_max^2.
//
// One SCF iteration of the whole batch is one CUDA graph: the shell-block
// density maxima of the build density, the J/K class kernels over the
// quartets of all molecules, and one dense-step kernel with a thread block
// per molecule (Fock matrix, energy, DIIS, Loewdin-orthogonalised TC2
// purification and the next build density, all on chip).  Converged
// molecules get a zero build density, so later builds skip their quartets.
#pragma once
#include <array>
#include <cmath>
#include <string>
#include <vector>

#include "engine.h"
#include "pool.h"

namespace pyfacc {

constexpr int BATCH_DIIS_MAX = 8;
constexpr int BATCH_THREADS = 256;   // threads of a dense-step block
constexpr int BATCH_NBF_MAX = 160;   // larger molecules run on their own

struct BatchMolDev {
  int nbf, nocc, ns, natoms;
  int occ_off, pad;    // first diagonal entry of the molecule in the guess occupations
  long long mat_off;   // first element of the molecule's n x n blocks
  long long diis_off;  // first element of its DIIS history (ndiis F then ndiis errors)
};

struct BatchMolState {
  double E, E_prev, err, dD, E_final;
  double B[BATCH_DIIS_MAX * BATCH_DIIS_MAX];  // DIIS error overlaps
  int age[BATCH_DIIS_MAX];                    // iteration that filled a slot, -1 empty
  int iter, head, converged, done, failed, tc2_steps, pad[2];
};

struct BatchDenseArgs {
  const BatchMolDev* mol;
  BatchMolState* st;
  const double *S, *H, *X;
  double *F, *J, *K, *Jd, *Kd, *P, *Db, *T1, *T2, *T3;
  double *diis;
  int ndiis, max_iter, rebuild_every, incremental;
  double e_tol, eps_diis, eps_density;
  int* active;     // molecules still iterating after this step (atomic count)
  int smem_nmax;   // molecules with nbf <= smem_nmax keep the TC2 iterate in shared memory
  // per graph variant: the build just done was a full one (J, K replaced,
  // not accumulated); it was an all-FP32 build of the first iterations
  // (no molecule may converge on it)
  int built_full, coarse;
  unsigned long long* max_err;  // largest DIIS error of the step (bits of a non-negative double)
};

// Iteration-graph variants of a batched SCF: full and incremental builds,
// and the all-FP32 full and incremental builds of the first mixed iterations.
enum BatchVariant { G_FULL = 0, G_INC = 1, G_CFULL = 2, G_CINC = 3, G_N = 4 };

// Control state of a batched SCF run as one graph launch: the build variant
// of every iteration is chosen on the device by the rules the host loop used
// (coarse phase while the batch's largest DIIS error is above coarse_err,
// then a full build, then incremental builds with a full rebuild every
// rebuild_every iterations).
struct BatchScfCtl {
  int it;            // iterations done
  int since_full;    // incremental builds since the last full one
  int coarse;        // the all-FP32 builds still run
  int restart;       // the next build must be full (end of the coarse phase)
  int variant;       // BatchVariant of the iteration in flight
  int incremental, rebuild_every, max_iter, coarse_max_iter;
  int stop;          // the loop ended (no molecule active, or max_iter)
  double coarse_err;
  long long counts[G_N];  // iterations run per variant
};
// At the top of an iteration: clear the step report, select this
// iteration's variant (the SWITCH node that follows).
void add_batch_select_node(cudaGraph_t g, cudaGraphNode_t* node, BatchScfCtl* ctl, int* report,
                           cudaGraphConditionalHandle variant);
// After the dense step: count, decide the next variant and whether the
// WHILE loop goes on.
void add_batch_update_node(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* dep, BatchScfCtl* ctl,
                           const int* report, cudaGraphConditionalHandle loop);

// X = S^{-1/2} of every molecule (coupled Newton-Schulz), into Xout; F, T1..T3
// are work space.  A molecule whose iteration does not converge is marked failed.
void launch_batch_lowdin(int nmol, const BatchDenseArgs& a, double* Xout, cudaStream_t s);
// Dynamic shared memory of the dense-step kernels (the TC2 iterate of the
// molecules with nbf <= a.smem_nmax); called once before any launch/capture.
void batch_set_smem(const BatchDenseArgs& a);
// P = diag(occ[occ_off + i]) of every molecule (atomic-occupation guess).
void launch_batch_guess(int nmol, const BatchDenseArgs& a, const double* occ, cudaStream_t s);
// Density of F = H (core guess) or of the guess already in P: sets P,
// Db = P (the first build is full), resets the per-molecule state.
void launch_batch_init(int nmol, const BatchDenseArgs& a, int core_guess, cudaStream_t s);
// One SCF step after a J/K build of Db into Jd/Kd.
void launch_batch_step(int nmol, const BatchDenseArgs& a, cudaStream_t s);
// Db = P of every molecule still iterating (before a full rebuild).
void launch_batch_full_density(int nmol, const BatchDenseArgs& a, cudaStream_t s);
// Db = P of the finished molecules (0 for the others) before the FP64 polish build.
void launch_batch_polish_density(int nmol, const BatchDenseArgs& a, cudaStream_t s);
// F and E of the final density after a full FP64 build (mixed precision);
// E -> st.E_final.
void launch_batch_polish(int nmol, const BatchDenseArgs& a, cudaStream_t s);
// Energy-weighted density W = 1/2 P F P into out.
void launch_batch_wdens(int nmol, const BatchDenseArgs& a, double* out, cudaStream_t s);
// Shell-block maxima |D| of every molecule: dm[m * ns_max^2 + a * ns_max + b].
// mt[m] = {first shell, ns, mat_off, nbf} (mat_off below 2^31).
void launch_batch_dmax(int nmol, int ns_max, const int4* mt, const int* bf_off, const int* nfun, const double* D,
                       float* dm, cudaStream_t s);

// Device-built task lists (batch_tasks.cu).  A range list covers one
// (bra class, ket class) combination: per bra its ket range [lo, hi) for the
// full list (0), the FP64 part (1) and the FP32 part (2) of mixed precision
// (split at Q_bra Q_ket = fp32_thresh), and the FP64 (3) and FP32 (4) parts
// of the mixed-precision gradient (split at grad_fp32_thresh).
constexpr int BATCH_NPARTS = 5;
struct BatchRangeList {
  int bra_base, ket_base, nb, same;
  const int* seg_b;  // nmol + 1 offsets of the molecules' bra pairs (relative to the class start)
  const int* seg_k;  // the same for the ket class
  int* lo[BATCH_NPARTS];
  int* hi[BATCH_NPARTS];
};
struct BatchRangeArgs {
  BatchRangeList l[NQCLASS];
  const double4* geom;  // .w = Schwarz factor Q of the pair
  const int4* info2;    // .z = molecule of the pair
  double thresh, fp32_thresh, grad_fp32_thresh;
};
// One task list: offsets of ceil((hi - lo) / width) tasks per bra.
struct BatchScanList {
  const int* lo;
  const int* hi;
  int* toff;  // nb + 1
  int nb, width;
};
constexpr int BATCH_MAX_SCANS = NQCLASS * BATCH_NPARTS * 3;
struct BatchScanArgs {
  BatchScanList l[BATCH_MAX_SCANS];
  int* ntasks;           // per list
  long long* nquartets;  // per list
};
void launch_batch_ranges(const BatchRangeArgs& a, int nlists, int nb_max, cudaStream_t s);
void launch_batch_scans(const BatchScanArgs& a, int nlists, cudaStream_t s);

struct BatchMolHost {
  int natoms = 0, nbf = 0, ns = 0, nalpha = 0, nbeta = 0, nocc = 0;
  int atom_off = 0, shell_off = 0;
  long long mat_off = 0, diis_off = 0;
  double e_nuc = 0.0;
  std::vector<int> Z;
  std::vector<double> xyz;
  std::vector<std::string> species;
  Basis basis;
};

struct BatchTiming {
  double ms_total = 0, ms_setup = 0, ms_1e = 0, ms_tune = 0, ms_scf = 0, ms_polish = 0, ms_grad = 0;
  int iterations = 0;
  int scf_graph_launches = 0;  // graph launches of the SCF loop (1 = the whole-SCF graph)
  double flops_fock = 0.0, flops_grad = 0.0;
  unsigned long long quartets[2] = {0, 0};
  int width[NQCLASS] = {32, 32, 32, 32, 32, 32};
};

class Batch {
 public:
  // Closed-shell molecules with nbf <= BATCH_NBF_MAX.
  Batch(const std::vector<BatchMolHost>& mols, const pyfacc_options& o);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;
  void run(bool gradient);
  // per molecule: energy, iterations, convergence, failure, gradient (3 natoms)
  double energy(int m) const;
  int iterations(int m) const { return st_host[m].iter; }
  bool converged(int m) const { return st_host[m].converged != 0; }
  bool failed(int m) const { return st_host[m].failed != 0; }
  double last_delta_e(int m) const { return std::fabs(st_host[m].E - st_host[m].E_prev); }
  double last_error(int m) const { return st_host[m].err; }
  const double* gradient(int m) const { return grad_host.data() + 3 * (size_t)mols[m].atom_off; }
  BatchTiming timing;

 private:
  pyfacc_options opt;
  int device = 0, num_sms = 148;
  GpuContext ctx;
  cudaStream_t stream = nullptr;
  std::vector<BatchMolHost> mols;
  int nmol = 0, ns_tot = 0, natoms_tot = 0, ns_max = 0, nbf_max = 0;
  long long mtot = 0;
  ShellDev shd;
  double4* atoms_dev = nullptr;
  int2* pairs1e[NPAIRCLASS] = {};  // one-electron pair lists (no d shells in a batch)
  int n1e[NPAIRCLASS] = {};
  int* bf_off_dev = nullptr;
  int* nfun_dev = nullptr;
  int4* mt_dev = nullptr;
  PairData pd;
  std::vector<int> seg[NCLASS];   // per class: nmol + 1 pair offsets (relative to the class start)
  TaskList tasks_w[3][NCLASS][NCLASS][BATCH_NPARTS];  // per width (32, 16, 8)
  TaskList tasks[NCLASS][NCLASS][BATCH_NPARTS];       // the widths in use
  DeviceBuf task_buf;
  DeviceBuf mats, state_buf;
  BatchDenseArgs dargs{};
  double *S = nullptr, *T = nullptr, *V = nullptr, *W = nullptr;
  float* dmax = nullptr;
  unsigned long long* stats_dev = nullptr;
  double* grad_dev = nullptr;
  int* active_dev = nullptr;     // followed by the step's largest DIIS error (8 bytes further)
  struct StepReport {
    int active;                  // molecules still iterating after the step
    int pad;
    unsigned long long max_err;  // bits of the largest DIIS error
  } report{};
  // iteration graphs (BatchVariant), launched one by one only when the
  // whole-SCF graph cannot be built
  cudaGraphExec_t graphs[G_N] = {nullptr, nullptr, nullptr, nullptr};
  long long graph_launches[G_N] = {0, 0, 0, 0};  // kernels per replay
  // the whole SCF: WHILE { select, SWITCH { the four variants }, update }
  cudaGraphExec_t scf_graph = nullptr;
  bool scf_graph_failed = false;
  int scf_launches_last = 0;
  BatchScfCtl* ctl_dev = nullptr;
  cudaGraphExec_t build_scf_graph();
  std::vector<BatchMolState> st_host;
  std::vector<double> grad_host;
  std::vector<double> occ_host;          // atomic-occupation guess, all molecules' diagonals
  DeviceBuf occ_buf;

  void upload();
  void build_pairs();
  void build_tasks();
  void alloc();
  // J/K of Db into Jd/Kd: FP64 lists, or the FP64 + FP32 halves of mixed mode
  // (all_fp32: every quartet of the full lists in FP32, the coarse builds;
  // overlap: the side stream takes every other class (of mixed lists the
  // FP64 and FP32 halves swap streams from class to class), forked and
  // joined by events, as captured into the iteration graphs)
  void fock_build(bool mixed_lists, double thresh, unsigned long long* stats, bool all_fp32 = false,
                  bool overlap = false);
  bool tuned_widths(std::array<int, NQCLASS>* w) const;  // cached tuner result for this batch shape
  std::string tune_key() const;
  void tune();
  cudaGraphExec_t capture(int variant, long long* launches);
  // the work of one iteration of the given variant, captured into graph
  // (reset_report: clear the step report first, as a standalone graph must)
  void capture_into(cudaGraph_t graph, int variant, bool reset_report, long long* launches);
  void gradient_run();
};

// Molecule description -> host record (species, electrons, basis, E_nn);
// throws Error on bad input.  uhf is set when the molecule needs UHF under
// the options' scf_type.
BatchMolHost batch_parse(const pyfacc_molecule& m, const pyfacc_options& o, bool* uhf);

}  // namespace pyfacc
