/*
 * pyfacc_b200.h -- C ABI of libpyfacc_b200.so, the B200 Hartree-Fock engine
 * that stands in for PyFAcc-SCF's libscf.so.
 *
 * Plain C types only: host pointers unless a name says "_dev" (CUDA device
 * memory of the device the call runs on), sizes in elements.  Matrices are
 * nbf x nbf, row-major and symmetric.  Coordinates are in bohr, atom-major
 * (x1 y1 z1 x2 ...), the memory order PyFAcc-SCF's Python driver hands over
 * (src/python/helper_functions.py:110-111).
 */
#ifndef PYFACC_B200_H
#define PYFACC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes returned by every int-returning entry point ---------- */
#define PYFACC_OK                  0
#define PYFACC_ERR_BASIS_NOT_FOUND 1  /* basis file missing                 */
#define PYFACC_ERR_UNSUPPORTED_L   2  /* shell type other than S, P, SP     */
#define PYFACC_ERR_NOT_CONVERGED   3  /* SCF hit max_iter                   */
#define PYFACC_ERR_LINDEP          4  /* overlap matrix not positive        */
#define PYFACC_ERR_CUDA            5  /* CUDA / cuBLAS / cuSOLVER failure   */
#define PYFACC_ERR_TIMEOUT         6  /* a bounded device wait gave up;
                                           reserved: no kernel of this build
                                           waits on a flag, so none returns it */
#define PYFACC_ERR_INVALID         7  /* bad argument                       */
#define PYFACC_ERR_ELEMENT         8  /* element without basis functions    */
#define PYFACC_ERR_NO_DEVICE       9  /* no CUDA device                     */
#define PYFACC_ERR_NOT_READY      10  /* call order (e.g. gradient before SCF) */

/* ---- options ------------------------------------------------------------ */
#define PYFACC_BOYS_ACCURATE             0 /* tabulated Taylor + asymptotic  */
#define PYFACC_BOYS_REFERENCE_TRAPEZOID  1 /* boys.f90:9-43, used for V only */
#define PYFACC_PRECISION_FP64            0
#define PYFACC_PRECISION_MIXED           1 /* FP32 quartets below fp32_thresh */
#define PYFACC_PRECISION_FP32            2 /* pyfacc_system_jk only: every
                                              quartet in FP32 (the coarse
                                              builds of a mixed SCF)          */
#define PYFACC_SCF_AUTO                  0 /* RHF if nalpha == nbeta          */
#define PYFACC_SCF_RHF                   1
#define PYFACC_SCF_UHF                   2
#define PYFACC_GUESS_CORE                0 /* core Hamiltonian (rscf.f90:113) */
#define PYFACC_GUESS_ATOMIC              1 /* atomic aufbau occupations      */

typedef struct pyfacc_options {
  double eps_energy;        /* |E_n - E_{n-1}| < eps_energy          (1e-10) */
  double eps_diis;          /* max |X^T (FDS - SDF) X| < eps_diis     (1e-8)  */
  double eps_density;       /* ||D_n - D_{n-1}||_F < eps_density; <=0 off (0) */
  int max_iter;             /* (100)                                           */
  int diis_size;            /* Pulay subspace, 0..64; 0 = plain Roothaan (8) */
  int scf_type;             /* PYFACC_SCF_*                           (AUTO)  */
  int precision;            /* PYFACC_PRECISION_*                     (FP64)  */
  int boys_mode;            /* PYFACC_BOYS_* for the V matrix         (ACCURATE) */
  double schwarz_thresh;    /* skip quartets with Q_ab Q_cd D_max below (1e-12) */
  double fp32_thresh;       /* mixed: Q_ab Q_cd (max|D| of a single
                               molecule's builds) below this run in FP32 (1e-3) */
  int incremental;          /* build G[dP] and add; -1 = on for MIXED   (-1)  */
  int rebuild_every;        /* full rebuild period of incremental builds (12) */
  int compute_gradient;     /* fill result->gradient after the SCF      (0)   */
  int device;               /* CUDA ordinal; -1 = current device        (-1)  */
  int verbose;              /* iteration lines on stderr                (0)   */
  int shard_rank;           /* J/K work shard of this process           (0)   */
  int shard_count;          /* number of shards (1 = whole Fock build)  (1)   */
  const char *data_dir;     /* directory holding basis_set/; NULL = search    */
  int guess;                /* PYFACC_GUESS_*                        (ATOMIC) */
  double incremental_thresh;/* screening of the incremental dP builds of
                               mixed mode; <= 0: schwarz_thresh      (1e-11) */
  int task_width;           /* kets per J/K task (8, 16 or 32; a warp runs
                               32/task_width tasks); 0 = 32 for one molecule,
                               chosen by timing for a batch            (0)   */
  int gradient_precision;   /* PYFACC_PRECISION_* of the derivative
                               integrals; MIXED evaluates the quartets with
                               Q_ab Q_cd (max|P|) below gradient_fp32_thresh
                               in FP32; -1 = MIXED for a mixed-precision SCF
                               (single molecules and batches), else FP64
                                                                       (-1) */
  int polish;               /* mixed: energy and F of the converged density
                               from one more full FP64 build (1, |dE| vs
                               FP64 ~1e-12), or from the last incremental
                               mixed build (0, |dE| ~1e-8)              (0)   */
  double gradient_fp32_thresh; /* mixed gradient: derivative quartets with
                               Q_ab Q_cd max|P| (in a batch: Q_ab Q_cd)
                               below this run in FP32
                               (max |dG| vs FP64 ~1e-6 Ha/bohr at 1e-1,
                               ~1e-7 at 1e-2 for C40H82, C100H202, rna1,
                               gly30); <= 0: fp32_thresh              (1e-1) */
  double coarse_err;        /* mixed: while the DIIS error is above this every
                               quartet runs in FP32; the first build below it
                               is a full mixed build that restarts the
                               incremental chain; 0 = off             (1e-3) */
} pyfacc_options;

typedef struct pyfacc_molecule {
  int natoms;
  const int32_t *z;         /* atomic numbers [natoms]                        */
  const double *coords;     /* bohr, atom-major [natoms*3]                    */
  const char *species;      /* 2*natoms chars, space padded, not NUL-terminated;
                               NULL = derive the symbols from z              */
  int charge;
  int nalpha, nbeta;        /* < 0: derived as helper_functions.py:76-87     */
  const char *basis;        /* "sto-2g" ... "sto-6g", NUL-terminated         */
} pyfacc_molecule;

typedef struct pyfacc_result {
  double energy;            /* total energy, hartree                          */
  double e_elec, e_nuc;
  int converged, n_iter, scf_type, nbf, nshell, n_fock_builds;
  double last_delta_e, last_diis_error;
  /* caller-owned outputs, filled when non-NULL (host memory)                */
  double *gradient;         /* [natoms*3], needs compute_gradient            */
  double *S, *T, *V;        /* [nbf*nbf]                                     */
  double *P;                /* total density [nbf*nbf]                       */
  double *C_alpha, *C_beta; /* MO coefficients, column i = orbital i         */
  double *eps_alpha, *eps_beta; /* orbital energies [nbf]                    */
  /* statistics                                                              */
  double ms_total, ms_one_electron, ms_fock, ms_diag, ms_gradient;
  long long quartets_fp64, quartets_fp32;   /* contracted quartets evaluated */
  double flops_fock;        /* algorithmic flops of all Fock builds           */
  double flops_gradient;    /* algorithmic flops of the two-electron gradient */
  int task_width;           /* J/K task width used                           */
} pyfacc_result;

typedef struct pyfacc_system pyfacc_system;   /* opaque, one molecule on one GPU */

/* ---- drop-in entry points of PyFAcc-SCF --------------------------------- */

/* src/c/scf_interface.c:9-14.  Same arguments and meaning; species is
 * 2*natoms space-padded chars, coords atom-major bohr, basis_set_c a
 * NUL-terminated name resolved as ./data/basis_set/<name>.txt (main.f90:33).
 * void like the original: on failure *final_energy is NaN and the status is
 * kept for pyfacc_last_status(). */
void run_scf_c(int natoms, int nelectrons, int charge, int nalpha, int nbeta, const char *species,
               double *coords, double eps_scf, int max_iter, double *final_energy,
               const char *basis_set_c, int32_t *z_num);

/* src/fortran/main.f90:15-24 (bind(C) name run_scf_interface_py): the
 * all-by-reference form with an explicit basis-name length. */
void run_scf_interface_py(int32_t *natoms, int32_t *nelectrons, int32_t *charge, int32_t *nalpha,
                          int32_t *nbeta, const char *species, double *coords, double *eps_scf,
                          int32_t *max_iter, double *final_energy, const char *basis_set_c,
                          int32_t *len_basis_set, int32_t *z_num);

/* One-body integrals of one shell pair: src/cpp/libint_wrapper.cpp:16-105
 * (libint_overlap_c), :114-212 (libint_kinetic_c), :220-327
 * (libint_potential_c), same symbols and arguments.  am*: angular momentum
 * (0..2 here); contrdepth*: primitives (1..32); A, B (and C): bohr;
 * alpha*, c*: exponents and contraction coefficients, applied as given to
 * unnormalised Cartesian primitives x^i y^j z^k exp(-alpha r^2) (no
 * normalisation is added); the result is the nint(amA) x nint(amB) block,
 * row-major, components in x-descending-then-y order; the potential is that
 * of a unit positive charge at C, int phi_a phi_b / |r - C|.  Computed on
 * the current CUDA device, synchronously on the legacy default stream.
 * void like the originals: on failure the block is NaN and the status is
 * kept for pyfacc_last_status(). */
void libint_overlap_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB,
                      int contrdepthB, double B[], double alphaB[], double cB[], double overlapAB[]);
void libint_kinetic_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB,
                      int contrdepthB, double B[], double alphaB[], double cB[], double kineticAB[]);
void libint_potential_c(int amA, int contrdepthA, double A[], double alphaA[], double cA[], int amB,
                        int contrdepthB, double B[], double alphaB[], double cB[], double C[], double potAB[]);

/* Status of the last run_scf_c / run_scf_interface_py / libint_*_c call on
 * this thread (the originals return nothing; la.f90:22-25 only prints). */
int pyfacc_last_status(void);
const char *pyfacc_status_string(int status);
/* Text of the most recent failure on this thread (extension). */
const char *pyfacc_last_message(void);

/* ---- extended API (no counterpart in the reference) --------------------- */

void pyfacc_default_options(pyfacc_options *opt);

/* One molecule: SCF (RHF/UHF per scf_type) and optionally the analytic
 * nuclear gradient (rscf.f90:26-168 / uscf.f90:25-219 plus gradient). */
int pyfacc_run(const pyfacc_molecule *mol, const pyfacc_options *opt, pyfacc_result *res);

/* Many molecules of uneven size converged together on one GPU: the shell
 * quartets of all closed-shell molecules (up to 160 basis functions each)
 * run in the same J/K launches, the whole SCF of the batch is one CUDA graph
 * launch (a conditional WHILE loop whose body selects the build variant on
 * the device, then J/K class kernels + one dense-step kernel with a thread
 * block per molecule: Fock matrix, energy, DIIS, TC2 purification), and J/K task widths
 * are picked per quartet class by timing (options.task_width = 0).  Open-shell
 * or larger molecules, results that ask for matrices, and molecules whose
 * batched purification fails run through pyfacc_run.  res[i] as in
 * pyfacc_run (timings and counters are those of the whole batch); returns the
 * worst per-molecule status. */
int pyfacc_run_batch(int nmol, const pyfacc_molecule *mols, const pyfacc_options *opt,
                     pyfacc_result *res);
/* Statistics of the last batched run on this thread: out[0..n) =
 * {ms_total, ms_setup, ms_one_electron, ms_tune, ms_scf, ms_polish,
 *  ms_gradient, iterations, flops_fock, flops_gradient, quartets_fp64,
 *  quartets_fp32, task width of the six quartet classes (ss|ss) (ps|ss)
 *  (ps|ps) (pp|ss) (pp|ps) (pp|pp), graph launches of the SCF loop (1 when
 *  the whole SCF ran as one graph with a device-driven WHILE loop)}. */
int pyfacc_batch_last_stats(double *out, int n);

/* Handle API: basis, shell pairs and Schwarz factors stay resident on the
 * GPU between calls. */
int pyfacc_system_create(const pyfacc_molecule *mol, const pyfacc_options *opt, pyfacc_system **sys);
void pyfacc_system_destroy(pyfacc_system *sys);
int pyfacc_system_info(const pyfacc_system *sys, int *nbf, int *nshell, int *natoms, int *npairs);
/* Replace the coordinates (same atoms); pair data is rebuilt. */
int pyfacc_system_set_coords(pyfacc_system *sys, const double *coords);
/* S, T, V into device buffers (nbf*nbf each; any may be NULL). */
int pyfacc_system_one_electron(pyfacc_system *sys, double *S_dev, double *T_dev, double *V_dev);
/* J[D_j] and K[D_k] for nk in {1,2} exchange densities: J_dev = sum (mn|ls) Dj_ls,
 * K_dev[k] = sum (ml|ns) Dk[k]_ls.  precision: PYFACC_PRECISION_*.
 * Schwarz screening uses the density: Q_ab Q_cd max|D| < schwarz_thresh. */
int pyfacc_system_jk(pyfacc_system *sys, const double *Dj_dev, int nk, const double *Dk_dev,
                     double *J_dev, double *K_dev, int precision);
/* Statistics of the last pyfacc_system_jk call on this system:
 * out[0..n) = {ms (CUDA events on the engine stream around the build),
 * algorithmic flops of the FP64 quartets, of the FP32 quartets, contracted
 * quartets FP64, FP32, primitive quartets FP64, FP32}, then per s/p quartet
 * class in the order (ss|ss) (ps|ss) (ps|ps) (pp|ss) (pp|ps) (pp|pp):
 * out[7..13) quartets FP64, out[13..19) quartets FP32, out[19..25)
 * primitive quartets FP64, out[25..31) primitive quartets FP32.  Entries
 * beyond 31 are zero. */
int pyfacc_system_jk_stats(const pyfacc_system *sys, double *out, int n);
/* Full (nbf^4) ERI tensor on the device, small systems only (tests). */
int pyfacc_system_eri_tensor(pyfacc_system *sys, double *eri_dev);
/* SCF with the system's options; res as in pyfacc_run. */
int pyfacc_system_scf(pyfacc_system *sys, pyfacc_result *res);
/* Analytic gradient [natoms*3] (host) of the last converged SCF. */
int pyfacc_system_gradient(pyfacc_system *sys, double *grad);
/* Result of the last SCF (and gradient) on this system: energies, timings,
 * statistics and the requested output matrices, without recomputing. */
int pyfacc_system_result(pyfacc_system *sys, pyfacc_result *res);
/* Device pointer to the density of the last SCF (nbf*nbf; RHF total,
 * UHF alpha). */
int pyfacc_system_density_dev(pyfacc_system *sys, const double **P_dev);
/* Number of kernel launches this library has issued in this process. */
long long pyfacc_launch_count(void);

#define PYFACC_BOYS_MMAX 6
/* Boys function F_m(x), m = 0..mmax (mmax <= PYFACC_BOYS_MMAX), for n arguments (device buffers;
 * out_dev[i*(mmax+1)+m]).  mode: PYFACC_BOYS_*; fp32 != 0 uses the
 * single-precision path of mixed mode. */
int pyfacc_boys_dev(int mode, int fp32, int mmax, int n, const double *x_dev, double *out_dev);

/* Dense FP64 products on the tensor cores (the kernels of the SCF step),
 * row-major device matrices with leading dimensions m (A: m x k, or k x m
 * when ta), n (B: k x n, or n x k when tb) and n (C: m x n):
 * C = op(A) op(B), op = transpose when ta / tb; asym_a != 0 uses
 * op(A) = A - A^T (square A, ta = 0); sym != 0 computes a result known to be
 * symmetric from its upper triangle. */
int pyfacc_dense_gemm_dev(int m, int n, int k, int ta, const double *A_dev, int tb, const double *B_dev,
                          double *C_dev, int sym, int asym_a);
/* TC2 purification of a symmetric n x n device matrix F into the projector
 * onto its nocc lowest eigenvectors (P_dev, n x n, not aliasing F_dev);
 * *steps receives the
 * number of TC2 steps.  PYFACC_ERR_NOT_CONVERGED without a gap at nocc. */
int pyfacc_purify_dev(int n, int nocc, const double *F_dev, double *P_dev, int *steps);

/* Cost-balanced split of n weighted work items into `parts` contiguous
 * ranges: bounds[0..parts] (host only, no GPU needed). */
int pyfacc_partition(int n, const double *cost, int parts, int *bounds);

/* Sharded Fock builds across processes (one GPU each): a system created
 * with options.shard_rank / shard_count evaluates its share of every
 * quartet list; after each J/K build and after the two-electron gradient
 * the engine synchronises its stream and calls fn(ctx, data_dev, count),
 * which must sum the `count` doubles at data_dev over all shards in place
 * (e.g. an NCCL all-reduce) before returning 0. */
typedef int (*pyfacc_reduce_fn)(void *ctx, double *data_dev, long long count);
int pyfacc_system_set_reducer(pyfacc_system *sys, pyfacc_reduce_fn fn, void *ctx);

/* Sustained FP64 FMA rate of the current device, GFLOP/s (microbenchmark). */
double pyfacc_probe_fp64_gflops(int device, double *fp32_gflops);

const char *pyfacc_version(void);

/* J[D] and K[D] of one molecule for a density already in device memory,
 * with no device allocation at all.  No counterpart in the reference: it is
 * for programs whose device memory belongs to their own allocator (a
 * framework's caching allocator, a pool sized once at start-up), where a
 * library cudaMalloc would fail or fragment the pool.  D_dev, J_dev, K_dev are
 * nbf*nbf device buffers owned by the caller (J, K are overwritten); every
 * intermediate lives in a 64 MiB array reserved statically on each GPU that
 * loads the library, and a molecule that needs more is rejected with
 * PYFACC_ERR_INVALID (pyfacc_last_message() gives the size).  The first call
 * on a device sets that device up and should precede any stream capture.
 * Calls share the array; calls from one process are serialised and return
 * after their kernels finish.  The kernels run on the legacy default stream:
 * a density written on a non-blocking stream must be complete (that stream
 * synchronised) before the call. */
int pyfacc_jk_noalloc(const pyfacc_molecule *mol, const char *data_dir, double schwarz_thresh,
                      const double *D_dev, double *J_dev, double *K_dev);

#ifdef __cplusplus
}
#endif
#endif /* PYFACC_B200_H */
