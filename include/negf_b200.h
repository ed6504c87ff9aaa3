/*
 * negf_b200.h -- C ABI of the B200 block-tridiagonal NEGF library
 * (libnegf_b200.so, sm_100a CUDA).
 *
 * It is the drop-in boundary for LibNEGF.jl's hot path: every entry point
 * below replaces one reference interface, cited as file:line within the
 * LibNEGF.jl project.  A Julia backend (backend_nvidia.jl, beside
 * src/backend_cpu.jl) reaches these functions through ccall only.
 *
 * Conventions
 *  - Matrices are complex128 (two doubles, re then im; C99 `double _Complex`,
 *    Julia ComplexF64), column-major with a leading dimension, exactly as
 *    Julia stores a Matrix{ComplexF64}.
 *  - "dptr" arguments are DEVICE pointers (cudaMalloc / CuArray / torch);
 *    arrays of dptrs are HOST arrays of device pointers.  Functions that take
 *    host data say so.
 *  - `stream` is a cudaStream_t (NULL: the legacy default stream).  Sweep
 *    entry points synchronise the stream before returning so that they can
 *    report singular pivots; the plan API does not.
 *  - Every function returns NEGF_SUCCESS or an error code; negf_last_error()
 *    returns the message of the last failure on the calling thread.  The
 *    reference prints and calls exit() on a LAPACK failure
 *    (src/backend_cpu.jl:151-155); this library returns NEGF_ERR_SINGULAR.
 *  - There is no CPU fallback: without a usable CUDA device every call
 *    returns NEGF_ERR_CUDA.
 */
#ifndef NEGF_B200_H
#define NEGF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NEGF_SUCCESS 0
#define NEGF_ERR_INVALID 1   /* bad argument */
#define NEGF_ERR_CUDA 2      /* CUDA runtime error / no device */
#define NEGF_ERR_SINGULAR 3  /* zero pivot in a diagonal block */
#define NEGF_ERR_NOMEM 4     /* device allocation failed */
#define NEGF_ERR_TIMEOUT 5   /* a bounded wait ran out (negf_server_wait, tensor-core pipeline waits) */

/* Message of the last failure on this thread ("" when none). */
const char* negf_last_error(void);
/* Library version, 100 * major + minor. */
int negf_version(void);

/* ------------------------------------------------------------------------
 * Backend primitives (the be_* layer of src/backend_cpu.jl), batched.
 * ---------------------------------------------------------------------- */

/* One GEMM problem:  C = alpha * op(A) * op(B) + beta * Cin + diag * I.
 * op(A) is m x k, op(B) is k x n; Cin may equal C; k = 0 gives
 * C = beta * Cin + diag * I. */
typedef struct {
  const void* A; /* dptr */
  const void* B; /* dptr */
  const void* Cin; /* dptr or NULL */
  void* C;       /* dptr */
  int32_t m, n, k;
  int32_t lda, ldb, ldc, ldcin;
  double alpha[2], beta[2], diag[2];
} negf_zgemm_problem;

/* Batched be_gemm! (src/backend_cpu.jl:208-219): all problems share
 * opA, opB in {'N','T','C'}.  One launch on the FP64 tensor path. */
int negf_zgemm_batched(char opA, char opB, int32_t nprob, const negf_zgemm_problem* probs, void* stream);

/* negf_zgemm_batched in the MIXED precision mode (INT8 tensor cores with
 * digit splitting; see NEGF_PREC_MIXED).  Same problems; results agree with
 * the FP64 ones to ~1e-15 relative to |op(A)| |op(B)| (FP64-grade); k <= 1024. */
int negf_zgemm_batched_mixed(char opA, char opB, int32_t nprob, const negf_zgemm_problem* probs, void* stream);

/* Limit, in seconds, of each pipeline wait inside the mixed-precision product
 * kernel (its mbarrier waits on copies, tensor-core completion and
 * accumulator drains; seconds <= 0: the default, about 1 s).  A wait that
 * runs out ends the kernel's work early: it waits for its own copies and
 * tensor-core operations in flight, releases its tensor memory and returns,
 * and the call reports NEGF_ERR_TIMEOUT; the CUDA context stays usable.
 * Process-wide; applies to launches made after the call (a solver plan
 * replayed from a CUDA graph keeps the limit of its capture). */
int negf_set_tensor_wait_limit(double seconds);

/* Batched be_copy_in_hw! / be_ctranspose! (src/backend_cpu.jl:42-68):
 * C[i] = op(A[i]) with op 'N' (copy) or 'C' (conjugate transpose); C[i] is
 * m[i] x n[i] (A[i] is n[i] x m[i] for 'C'). */
int negf_zcopy_batched(char op, int32_t nprob, const int32_t* m, const int32_t* n, void* const* A,
                       const int32_t* lda, void* const* C, const int32_t* ldc, void* stream);

/* Batched be_fill! (src/backend_cpu.jl:86-88): every entry of C[i]
 * (m[i] x n[i]) set to value (re, im). */
int negf_zfill_batched(int32_t nprob, const int32_t* m, const int32_t* n, void* const* C, const int32_t* ldc,
                       const double* value, void* stream);

/* Batched inversion Ainv[i] = A[i]^{-1} by blocked Gauss-Jordan with partial
 * pivoting; replaces be_lu! + be_mldivide!(identity) / be_inv_from_lu!
 * (src/backend_cpu.jl:147-206).  A[i] is not modified.  n[i] <= 1024.
 * info (host, nprob entries, may be NULL) receives 0 or the first zero-pivot
 * column (1-based) per matrix. */
int negf_zinv_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* const* Ainv,
                      const int32_t* ldainv, int32_t* info, void* stream);

/* negf_zinv_batched without any device allocation.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot let the
 * library call cudaMalloc / cudaFree -- applications whose device memory all
 * comes from their own pool, or loops that cannot afford the device-wide
 * synchronisation of cudaFree.  Inputs, outputs and results are those of
 * negf_zinv_batched; all scratch (block copies, rank-nb update buffers,
 * pivots, flags, launch descriptors) lives in one fixed 64 MiB __device__
 * array that every GPU loading the library keeps until the process exits.
 * A request whose scratch exceeds 64 MiB (more than 51 blocks of 256 or 15 of 512
 * per call) is rejected with NEGF_ERR_INVALID.  The first call on a device
 * looks up the array's address and sets kernel attributes: make it before
 * any stream capture.  All calls share the array, so calls that overlap on
 * the GPU (different streams or threads on one device) race; calls in
 * sequence on one stream are safe. */
int negf_zinv_batched_noalloc(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda,
                              void* const* Ainv, const int32_t* ldainv, int32_t* info, void* stream);

/* Batched LU with partial pivoting, in place, LAPACK getrf semantics;
 * replaces be_lu! / be_getrf! (src/backend_cpu.jl:147-169, :255-265).
 * ipiv (dptrs, may be NULL entries) receives 1-based LAPACK pivots. */
int negf_zgetrf_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* const* ipiv,
                        int32_t* info, void* stream);

/* Batched triangular solve with the factors of negf_zgetrf_batched /
 * be_trsm! (src/backend_cpu.jl:241-253): B[i] = alpha * op(T)^{-1} B[i]
 * (side 'L') or alpha * B[i] op(T)^{-1} (side 'R'), T the upper ('U') or
 * unit/non-unit lower ('L') triangle of A[i]; trans 'N' only. */
int negf_ztrsm_batched(char side, char uplo, char trans, char diag, const double* alpha, int32_t nprob,
                       const int32_t* m, const int32_t* n, void* const* A, const int32_t* lda, void* const* B,
                       const int32_t* ldb, void* stream);

/* Batched be_getri! with identity pivots (src/backend_cpu.jl:229-239):
 * A[i] (holding L\U factors) is replaced by U^{-1} L^{-1}. */
int negf_zgetri_nopiv_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* stream);

/* ------------------------------------------------------------------------
 * Whole-sweep entry points (the reference's algorithm functions).
 * nsys independent systems of npl layers; block_sizes holds nsys*npl sizes
 * (system-major); block dptr tables are system-major: Md[s*npl + i] is
 * M[i,i] of system s, Mu[s*(npl-1)+i] is M[i,i+1], Ml[s*(npl-1)+i] is M[i+1,i].
 * Blocks are dense with ld = their row count.
 * ---------------------------------------------------------------------- */

/* Block tridiagonal of M^{-1} by RGF: bndiag_of_inv_rgf_local!
 * (src/matinvertndiag_rgf.jl:114-200).  Gu / Gl may be NULL.  With Gfull
 * (nsys*npl*npl dptrs, row-major block index i*npl+j, NULL entries skipped)
 * every block of the inverse is written (buildFullInv, rgf.jl:185-199). */
int negf_rgf(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
             void* const* Ml, void* const* Gd, void* const* Gu, void* const* Gl, void* const* Gfull, void* stream);

/* Block tridiagonal of G^n = M^{-1} S M^{-H} by recursive Keldysh:
 * keldyshndiag! (src/keldyshndiag.jl:120-317).  S is Hermitian, given as
 * diagonal blocks Sd (nsys*npl) and upper blocks Su (nsys*(npl-1)); it is
 * overwritten with G^n in the same storage (the reference's auxData.buffS). */
int negf_keldysh(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                 void* const* Ml, void* const* Sd, void* const* Su, void* stream);

/* Block n-diagonal (bandwidth w = (ndiag-1)/2) of M^{-1}:
 * bndiag_of_inv_general_rgf! (src/matinvertndiag_general_rgf.jl:31-146).
 * Mb holds nsys*npl*npl dptrs (row-major block index i*npl+j), non-NULL
 * exactly for |i-j| <= w; Gb likewise for the output.  Mb is not modified
 * (the reference overwrites Min, :86). */
int negf_general_rgf(int32_t nsys, int32_t npl, int32_t ndiag, const int32_t* block_sizes, void* const* Mb,
                     void* const* Gb, void* stream);

/* Selected inverse on a general block pattern: Block_factorization! then
 * Block_inverse! (src/selected_inverse.jl:9-55, :139-206).  Ab holds
 * npl*npl dptrs (row-major block index), NULL where the block is unassigned;
 * fill-in blocks created by the factorisation must be provided (pre-zeroed)
 * and flagged in fill (npl*npl bytes, 1 = fill-in).  All blocks have size b.
 * mode: 1 = factorisation only, 2 = inverse only (Ab holds factors),
 * 3 = both.  In place. */
int negf_selected_inverse(int32_t npl, int32_t b, void* const* Ab, const uint8_t* fill, int32_t mode, void* stream);

/* negf_selected_inverse over nsys systems at once (Block_factorization! /
 * Block_inverse!, src/selected_inverse.jl:9-206, one call per system in the
 * reference): Ab holds nsys*npl*npl dptrs (system-major, then row-major block
 * index); every system has system 0's block pattern; each step is one batched
 * launch over all systems.  pivoting = 1 factors each diagonal block as the
 * reference's be_getrf! does (LAPACK getrf, src/backend_cpu.jl:255-265, whose
 * row interchanges the reference then discards, so it is exact only for
 * blocks that need none); pivoting = 0 is lu(NoPivot()), the factorisation
 * selected_inverse.jl:17 names, exact for any blocks with non-zero leading
 * minors.  precision NEGF_PREC_MIXED runs the block products (the triangular
 * solves with the explicit factor inverses, the Schur updates and the
 * Block_inverse! products) on the INT8 tensor cores with FP64-grade digit
 * splitting; the diagonal-block LU and triangular inverses stay FP64. */
int negf_selected_inverse_batched(int32_t nsys, int32_t npl, int32_t b, void* const* Ab, const uint8_t* fill,
                                  int32_t mode, int32_t pivoting, int32_t precision, void* stream);

/* Domain-decomposed RGF: bndiag_of_inv_ddrgf! (src/matinvertndiag_ddrgf_core.jl:
 * 719-758) with one level and the reference's partition (separators of one
 * layer at t*(D1+1), src/matinvertndiag_ddrgf_utils.jl:278-312, :478-575);
 * the separator Schur complement is inverted by sequential RGF.
 * block_size_d1 <= 0 picks the interior size from the library's cost model.
 * Output as negf_rgf (Gu/Gl may be NULL). */
int negf_ddrgf(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
               void* const* Ml, int32_t block_size_d1, void* const* Gd, void* const* Gu, void* const* Gl,
               void* stream);

#define NEGF_DDRGF_MAX_LEVELS 6

/* Multi-level DDRGF: level k (k = 0 .. nlevels-1) partitions the separator
 * Schur complement of level k-1 (the original matrix for k = 0) with interior
 * size block_size_d1[k]; the last level's Schur complement is inverted by
 * sequential RGF.  This is the recursion of bndiag_of_inv_ddrgf! through
 * _inv_Schur_compl! (src/matinvertndiag_ddrgf_core.jl:656-680) over the
 * levels allocate_aux_data_DDRGF builds (src/matinvertndiag_ddrgf_setup.jl:
 * 4-51).  A level whose partition has a single task runs sequential RGF
 * (core.jl:726-729); an impossible partition (get_nr_tasks = -1) is
 * NEGF_ERR_INVALID.  nlevels = 0 picks the levels from the library's GPU cost
 * model (negf_ddrgf_choose_levels).  nlevels <= NEGF_DDRGF_MAX_LEVELS.  All
 * systems share npl; block sizes may differ per system.  Output as negf_rgf
 * (Gu/Gl may be NULL). */
int negf_ddrgf_levels(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                      void* const* Ml, int32_t nlevels, const int32_t* block_size_d1, void* const* Gd,
                      void* const* Gu, void* const* Gl, void* stream);
/* negf_ddrgf_levels with a precision mode: NEGF_PREC_MIXED runs every block
 * product of the sweep (domain RGF and full inverses, Schur complement, the
 * 12 / 21 / 11 assembly) on the INT8 tensor cores with FP64-grade digit
 * splitting; the diagonal-block inversions stay FP64. */
int negf_ddrgf_levels_ex(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                         void* const* Ml, int32_t nlevels, const int32_t* block_size_d1, void* const* Gd,
                         void* const* Gu, void* const* Gl, int32_t precision, void* stream);

/* The reference's partition helper (src/matinvertndiag_ddrgf_utils.jl:
 * 278-312): writes nr_tasks (-1: impossible) and the last interior size. */
int negf_ddrgf_get_nr_tasks(int32_t npl, int32_t block_size_d1, int32_t* nr_tasks, int32_t* last_d1);
/* One-level partition choice of the library's GPU cost model for npl layers
 * of size b (npl: sequential RGF is cheaper). */
int negf_ddrgf_choose_d1(int32_t npl, int32_t b, int32_t nsys, int32_t* block_size_d1);
/* Level choice of the library's GPU cost model: up to max_levels interior
 * sizes into block_size_d1 (nlevels = 0: sequential RGF is cheapest).  The
 * model weighs the serial launch depth of each level against its batched
 * GEMM work; host only. */
int negf_ddrgf_choose_levels(int32_t npl, int32_t b, int32_t nsys, int32_t max_levels, int32_t* nlevels,
                             int32_t* block_size_d1);
/* The reference's own partition search, restated: opt_params
 * (src/matinvertndiag_ddrgf_utils.jl:357-453) with cost_rgf / cost_ddrgf
 * (:221-276) and check_nr_threads (:455-465), for nr_threads CPU threads and
 * the measured ratios r_lu = t(LU)/t(GEMM), r_mldiv = t(solve)/t(GEMM),
 * damp_rgf = t(GEMM, 1 thread)/t(GEMM, all threads).  Writes nr_levels and,
 * per level, nr_tasks and block_size_d1 (arrays of NEGF_DDRGF_MAX_LEVELS) and
 * the model cost (may be NULL).  allocate_aux_data_DDRGF builds
 * max(1, nr_levels - 1) DDRGF levels from these (setup.jl:36-48).  Host only. */
int negf_ddrgf_opt_params(int32_t npl, int32_t nr_threads, double r_lu, double r_mldiv, double damp_rgf,
                          int32_t* nr_levels, int32_t* nr_tasks, int32_t* block_size_d1, double* cost);
/* The pieces of that search (host only): cost_rgf (src/matinvertndiag_ddrgf_
 * utils.jl:221-247; do_full needs L <= 4), cost_ddrgf (:249-276; D1 <= 4) and
 * bndiag_of_inv_ddrgf_check_nr_threads (:455-465: threads actually used,
 * tasks per thread, tasks of the last thread). */
int negf_ddrgf_cost_rgf(int32_t L, double r_lu, double r_mldiv, int32_t do_full, double* cost);
int negf_ddrgf_cost_ddrgf(double r_lu, double r_mldiv, int32_t nr_tasks, int32_t nr_threads, int32_t block_size_d1,
                          double* cost);
int negf_ddrgf_check_nr_threads(int32_t nr_threads, int32_t nr_tasks, int32_t* threads, int32_t* max_per_thread,
                                int32_t* last_per_thread);

/* ------------------------------------------------------------------------
 * Batched-energy NEGF solver (the reference has no energy loop; this is the
 * batched form of running RGF + keldyshndiag! per energy point).
 * M(E) = (E + i eta) I - H - Sigma, Sigma_L on layer 0, Sigma_R on layer
 * N-1; Gamma = i (Sigma - Sigma^H); Sigma^in = f_L Gamma_L (+) f_R Gamma_R;
 * G^< = i G^R Sigma^in G^A; T(E) = Re Tr[Gamma_L G^R_{1N} Gamma_R G^A_{N1}].
 * ---------------------------------------------------------------------- */
typedef struct negf_device_s* negf_device_t;

/* Upload one device: Hd[i] (npl host pointers, b_i x b_i), Hu[i]
 * (npl-1 host pointers, b_i x b_{i+1}, H_{i+1,i} = Hu[i]^H), sigL (b_0 x b_0),
 * sigR (b_{N-1} x b_{N-1}); all complex128 column-major host arrays. */
int negf_device_create(int32_t npl, const int32_t* block_sizes, const void* const* Hd, const void* const* Hu,
                       const void* sigL, const void* sigR, negf_device_t* out);
/* Re-upload H and the self-energies of an existing device (same sizes);
 * solvers built on the device stay valid. */
int negf_device_upload(negf_device_t dev, const void* const* Hd, const void* const* Hu, const void* sigL,
                       const void* sigR);
int negf_device_destroy(negf_device_t dev);
/* Overlap matrix S of a non-orthogonal basis (host blocks: Sd[i] b_i x b_i,
 * Su[i] = S_{i,i+1} b_i x b_{i+1}, S_{i+1,i} = Su[i]^H; a NULL array or entry
 * is the identity / zero).  Solvers created afterwards form
 * M(E) = (E + i eta) S - H - Sigma(E) per energy on the device, as the
 * reference's build_M_from_HS (src/matloader.jl:89-95). */
int negf_device_set_overlap(negf_device_t dev, const void* const* Sd, const void* const* Su);

typedef struct {
  double eta, mu_l, mu_r, kT;
  int32_t want_gr;   /* diagonal G^R blocks */
  int32_t want_gl;   /* diagonal G^< blocks */
  int32_t want_t;    /* transmission */
  int32_t max_chunk; /* energies per device-resident batch (0: by HBM budget) */
  double hbm_budget_gb; /* 0: 80% of free device memory */
  int32_t precision; /* NEGF_PREC_FP64 or NEGF_PREC_MIXED */
  /* Schedule knobs (0: library default); chosen per batch by the autotuner
   * of the Python layer (libnegf_b200.autotune): */
  int32_t gemm_form; /* FP64 complex products: 1 = four real products, 2 = 3M (Gauss, default) */
  int32_t gj_nb;     /* Gauss-Jordan panel width for blocks > 112: 8, 16 or 32 (must fit shared memory) */
  /* 1: the lead self-energies depend on the energy; solvers then take them per
   * energy from negf_solver_set_self_energies (replacing the device's
   * constant ones) and form Gamma(E) on the device. */
  int32_t sigma_per_energy;
  /* NEGF_PREC_MIXED only: the Gauss-Jordan rank-nb updates of the diagonal
   * inversions as INT8 digit products with 34 digit pairs (2; as accurate as
   * FP64 products) or as FP64 DMMA products (1); 0: the library default (1).
   * The inversion panels always run in FP64. */
  int32_t gj_update;
} negf_solve_opts;

/* Precision modes.  FP64: every product in FP64 on the DMMA tensor path.
 * MIXED: the Schur-complement products run on the INT8 tensor cores
 * (tcgen05) with FP64-accurate digit splitting (per row a 54-bit fixed-point
 * value as 7 base-256 digits, the 28 digit pairs of weight >= 2^-60 formed
 * with exact int32 accumulation: ~1e-15 relative to |op(A)| |op(B)| per
 * product); the inversion panels stay in FP64 and their rank-nb updates
 * follow negf_solve_opts.gj_update. */
#define NEGF_PREC_FP64 0
#define NEGF_PREC_MIXED 1

/* Solve nE energy points (energies: host array).  gr_out / gl_out receive
 * nE * sum_i b_i^2 complex128 values (energy-major, then layer, column-major
 * blocks); t_out receives nE doubles.  Outputs are HOST pointers unless
 * out_on_device != 0.  NULL outputs are skipped. */
int negf_solve(negf_device_t dev, int32_t nE, const double* energies, const negf_solve_opts* opts, void* gr_out,
               void* gl_out, double* t_out, int32_t out_on_device, void* stream);

/* Selected inverse of M(E) = (E + i eta) S - H - Sigma for nE energies: the
 * blocks (i,i), (i,i+1), (i+1,i) of G^R(E) = M(E)^{-1}, every recursion step
 * one batched launch over all energies of a device-resident chunk.  This is
 * the batched form of one reference call per energy point of
 *   method 0: bndiag_of_inv_rgf_local! (src/matinvertndiag_rgf.jl:114-200);
 *   method 1: bndiag_of_inv_ddrgf! (src/matinvertndiag_ddrgf_core.jl:719-758)
 *             with nlevels interior sizes block_size_d1 (nlevels = 0: the
 *             library's GPU cost model chooses);
 *   method 2: Block_factorization! + Block_inverse! (src/selected_inverse.jl:
 *             9-206) with lu(NoPivot()) diagonal factorisations (one block
 *             size).
 * opts: eta, precision (NEGF_PREC_MIXED: block products on the INT8 tensor
 * cores with FP64-grade digit splitting, inversion panels and LU in FP64),
 * max_chunk / hbm_budget_gb (energies per chunk), gemm_form, gj_nb,
 * gj_update; sigma_per_energy must
 * be 0.  Outputs (NULL: skipped), energy-major: gd_out nE * sum b_i^2; gu_out
 * (blocks (i,i+1), b_i x b_{i+1}) and gl_out (blocks (i+1,i), b_{i+1} x b_i)
 * nE * sum b_i b_{i+1}; column-major blocks.  HOST pointers unless
 * out_on_device != 0.  Synchronises the stream. */
int negf_device_selected_inverse(negf_device_t dev, int32_t nE, const double* energies, const negf_solve_opts* opts,
                                 int32_t method, int32_t nlevels, const int32_t* block_size_d1, void* gd_out,
                                 void* gu_out, void* gl_out, int32_t out_on_device, void* stream);
#define NEGF_METHOD_RGF 0
#define NEGF_METHOD_DDRGF 1
#define NEGF_METHOD_SELINV 2

/* Resident-plan form of negf_solve for repeated solves of a fixed number of
 * energies with inputs and outputs kept in device memory. */
typedef struct negf_solver_s* negf_solver_t;
int negf_solver_create(negf_device_t dev, int32_t nE, const negf_solve_opts* opts, negf_solver_t* out);
/* One resident plan for a batch of devices of different layer counts and
 * block sizes (nE[k] energies of devs[k]): every recursion step is one
 * batched launch over all (device, energy) pairs that reach it.  The energy
 * array of negf_solver_set_energies and the outputs are device-major: the
 * nE[0] energies of devs[0], then those of devs[1], ...; gr/gl hold, per
 * energy, the diagonal blocks of its device in layer order.  Transmission
 * needs equal first and last block sizes per device.  (The reference solves
 * one system and one energy per call; this is the batching of
 * src/matinvertndiag_rgf.jl:114-200 and src/keldyshndiag.jl:120-317 over
 * systems.) */
int negf_solver_create_batch(int32_t ndev, const negf_device_t* devs, const int32_t* nE,
                             const negf_solve_opts* opts, negf_solver_t* out);
/* Device bytes a batch solver of these devices / energy counts would
 * allocate (workspace and outputs, the estimate negf_solve uses to split an
 * energy list by its HBM budget); for admission control. */
int negf_batch_bytes(int32_t ndev, const negf_device_t* devs, const int32_t* nE, const negf_solve_opts* opts,
                     int64_t* bytes);
int negf_solver_destroy(negf_solver_t s);
/* Per-energy lead self-energies (host arrays of nE block pointers in the
 * solver's energy order; Sigma_L(E) b_0 x b_0, Sigma_R(E) b_{N-1} x b_{N-1})
 * for a solver created with opts.sigma_per_energy = 1; copied before return. */
int negf_solver_set_self_energies(negf_solver_t s, const void* const* sigL, const void* const* sigR, void* stream);
/* energies: host array of nE values (uploaded to a device parameter table). */
int negf_solver_set_energies(negf_solver_t s, const double* energies, void* stream);
/* One pass over all energies (captured into a CUDA graph on first use). */
int negf_solver_run(negf_solver_t s, void* stream);
/* Device pointers of the resident outputs (valid until destroy): gr/gl as in
 * negf_solve; t_dev holds 2*nE doubles (re, im of the trace per energy). */
int negf_solver_outputs(negf_solver_t s, void** gr_dev, void** gl_dev, double** t_dev);
/* Copy the resident outputs into host buffers (pinned for full speed) on
 * `stream` and wait: gr/gl as in negf_solve, t as 2*nE doubles (re, im). */
int negf_solver_download(negf_solver_t s, void* gr_host, void* gl_host, double* t_host, void* stream);
/* One pass with the downloads overlapped: each diagonal G^R block layer is
 * copied to the host as soon as the downward RGF pass has finished it, each
 * G^< layer as soon as the last RKD pass has, on a copy stream of the solver
 * that runs beside the remaining launches (the pass replays launch by launch
 * instead of as a graph).  Same outputs and layout as negf_solver_run +
 * negf_solver_download; waits for everything and checks the pivot flags
 * before returning.  Host buffers that are not pinned fall back to run, then
 * download. */
int negf_solver_run_download(negf_solver_t s, void* gr_host, void* gl_host, double* t_host, void* stream);
/* Synchronous check of the zero-pivot flags of the last run. */
int negf_solver_check(negf_solver_t s);
/* One pass launch by launch (no graph) with a CUDA event recorded after every
 * launch on `stream`; per-launch durations accumulate until read. */
int negf_solver_run_profiled(negf_solver_t s, void* stream);
/* Kernel kinds: 0 GEMM, 1 inversion panel, 2 inversion un-permute, 3 block
 * copies, 4 trace, 5 LU panel, 6 LU row swaps, 7 triangular diagonal blocks,
 * 8 INT8 digit split, 9 INT8 tensor-core product (mixed precision); the
 * arrays hold NEGF_PROFILE_KINDS entries. Synchronises and writes, per
 * kind, the summed milliseconds, real flops (for kind 8, the digit split,
 * its algorithmic bytes instead: operands read once, 21 digit bytes per
 * complex element and a scale per row written; for kind 9 the INT8
 * operations: 3 real products x digit pairs x 2mnk per complex product) and
 * launch counts of the
 * profiled passes since the last reset (reset != 0 starts a new
 * accumulation). */
#define NEGF_PROFILE_KINDS 10
int negf_solver_profile_read(negf_solver_t s, double* ms, double* flops, int64_t* launches, int32_t reset);
/* Real flops of one pass (8mnk per complex GEMM, 8n^3 per inversion),
 * number of kernel launches per pass and workspace bytes. */
int negf_solver_stats(negf_solver_t s, double* flops, int64_t* launches, int64_t* workspace_bytes);

/* ------------------------------------------------------------------------
 * Reference C ABI: src/c_interface/libnegf_c_interface.h:12-38.
 * Same struct layout and signature, so libnegf_c_example.c links unchanged.
 * Runs DDRGF (the reference's wrapper does, libnegf_c_interface.jl:119) on
 * the block n-diagonal band of the input CSC matrix; the returned arrays are
 * malloc'd and freed by the caller with free().  On failure the result has
 * m = n = nnz = 0 and NULL arrays (the reference has no error channel).
 * ---------------------------------------------------------------------- */
typedef struct {
  int32_t m;
  int32_t n;
  int32_t nnz;
  int32_t* colptr;
  int32_t* rowval;
  void* nzval; /* double complex* */
} CCscMatrix;

CCscMatrix run_bndiag_wrapper(int32_t m, int32_t n, int32_t nnz_in, int32_t* colptr_in, int32_t* rowval_in,
                              void* nzval_in, int32_t n_blocks, int32_t* block_sizes_in, int32_t n_dict,
                              const char** dict_keys_in, int32_t* dict_vals_in, int32_t is_hermitian);

/* Dense debug path: bndiag_of_inv_direct (src/matinvertndiag_direct.jl:17-61,
 * :78-85) -- the block n-diagonal part of M^{-1} through the whole inverse,
 * as a cross-check of the recursive methods on small systems.  M is an n x n
 * CSC matrix (0-based, rows sorted within each column, as from Julia's
 * SparseMatrixCSC), block_sizes the layers (sum n), ndiag_out the output
 * band (odd).  The CSC -> dense scatter, the inverse and the band extraction
 * run on the device.  Up to n = 1024 the inverse is one Gauss-Jordan
 * inversion with partial pivoting over all rows (LAPACK's inv does getrf +
 * getri); above, block elimination over the layers (no pivoting between
 * layers; every layer <= 1024).  The result is M with its out band replaced
 * by the inverse's, as the reference's in-place version leaves it: stored
 * entries of M outside the band are kept, exact zeros of the inverse inside
 * the band are not stored.  *result receives malloc'd arrays the caller
 * frees with free().  Device memory: 2 n^2 complex plus the inversion's
 * workspace. */
int negf_bndiag_of_inv_direct(int32_t n, int32_t nnz, const int32_t* colptr, const int32_t* rowval,
                              const void* nzval, int32_t n_blocks, const int32_t* block_sizes, int32_t ndiag_out,
                              CCscMatrix* result);

/* ------------------------------------------------------------------------
 * Device memory of finished plans.  The reference allocates per call through
 * Julia's GC; here the workspace of a destroyed plan (solver, sweep, server
 * group) stays with the library, per device, and is reused by the next plans
 * (at most half of the device's memory is kept; the library's own HBM budget
 * queries count it as free, and a failed allocation releases it and retries).
 * This call hands all of it back to the driver, for callers that allocate
 * device memory outside the library after a solve.
 * ---------------------------------------------------------------------- */
int negf_release_cached_memory(void);

/* ------------------------------------------------------------------------
 * Measurement helpers (roofline denominators measured on the device):
 * FP64 throughput of the tensor (mma.sync f64) and DFMA paths, TFLOP/s, for
 * the FP64 path; dense INT8 tcgen05 throughput, TOP/s, for the mixed path.
 * ---------------------------------------------------------------------- */
int negf_probe_fp64_peak(double* dmma_tflops, double* dfma_tflops);
int negf_probe_int8_peak(double* tops);
/* Whether FP64 arithmetic progresses beside INT8 tensor-core MMAs on one SM:
 * mean cycles of seven warps of DFMA chains alone, the same beside one thread
 * issuing back-to-back 128 x 256 x 32 kind::i8 MMAs, and the MMA stream
 * alone.  fp64_beside ~ fp64_alone + mma means the two do not overlap, so
 * the product kernel's FP64 drains cost their full time. */
int negf_probe_fp64_int8_overlap(double* fp64_alone_cycles, double* fp64_beside_mma_cycles, double* mma_cycles);

/* ------------------------------------------------------------------------
 * Request server.  The reference has no request loop (one system and one
 * energy per call); this batches whole NEGF solves (RGF + RKD +
 * transmission: src/matinvertndiag_rgf.jl:114-200, src/keldyshndiag.jl:
 * 120-317) submitted from any thread of any host language, continuously:
 * `lanes` worker threads, each with its own CUDA stream, admit queued
 * requests first in, first out, whenever the HBM budget (negf_batch_bytes
 * estimates; budget_gb <= 0: 80 % of the memory free at creation) has room
 * for them beside the groups already in flight, and solve each admitted group
 * as one batch plan.  A request that arrives while others are on the GPU
 * therefore starts as soon as memory allows and runs beside them.  A group
 * that fails to allocate is halved, one that fails otherwise is re-solved
 * request by request, and a single request above the budget goes through
 * negf_solve, which splits its energies.  opts gives eta, mu_l, mu_r, kT,
 * precision and the schedule knobs; the want_* flags follow each request's
 * non-NULL outputs; sigma_per_energy must be 0.  The server keeps a few bytes
 * per ticket (status, latency) until it is destroyed.
 * ---------------------------------------------------------------------- */
typedef struct negf_server_s* negf_server_t;
/* Two lanes. */
int negf_server_create(const negf_solve_opts* opts, double budget_gb, negf_server_t* out);
/* lanes in [1, 16] (1: one group at a time). */
int negf_server_create_ex(const negf_solve_opts* opts, double budget_gb, int32_t lanes, negf_server_t* out);
/* Upload the device (host blocks as negf_device_create; the caller may free
 * them on return) and queue nE energies.  gr_out / gl_out (nE * sum b_i^2
 * complex128, energy-major then layer, each block column-major) and t_out
 * (nE doubles) are host buffers, any of them NULL, that must stay valid until
 * the request is done.  Call with the server's device current. */
int negf_server_submit(negf_server_t srv, int32_t npl, const int32_t* block_sizes, const void* const* Hd,
                       const void* const* Hu, const void* sigL, const void* sigR, int32_t nE, const double* energies,
                       void* gr_out, void* gl_out, double* t_out, int64_t* ticket);
/* done = 1 once the request's outputs are written; the return value is then
 * the request's status (NEGF_SUCCESS while pending). */
int negf_server_poll(negf_server_t srv, int64_t ticket, int32_t* done);
/* Wait at most timeout_s seconds: the request's status, or NEGF_ERR_TIMEOUT;
 * latency_s (may be NULL) receives the seconds from the entry into
 * negf_server_submit to completion. */
int negf_server_wait(negf_server_t srv, int64_t ticket, double timeout_s, double* latency_s);
/* Completed requests, groups solved, and the p50 / p99 latency (seconds) of
 * the completed requests. */
int negf_server_stats(negf_server_t srv, int64_t* completed, int64_t* groups, double* p50_s, double* p99_s);
/* Requests waiting, groups on the GPU now, the most groups ever on the GPU at
 * once, and the byte estimate (GB) of the groups on the GPU. */
int negf_server_stats_ex(negf_server_t srv, int64_t* queued, int32_t* inflight_groups,
                         int32_t* peak_inflight_groups, double* inflight_gb);
/* Finish the queued requests, stop the lanes, free the server. */
int negf_server_destroy(negf_server_t srv);
/* The grouping rule for an idle server (host only): requests in order, each group as
 * many as fit budget bytes (a request above it alone); sizes receives the
 * group sizes (room for nreq), ngroups their count. */
int negf_server_group_sizes(int32_t nreq, const int64_t* bytes, double budget, int32_t* sizes, int32_t* ngroups);

#ifdef __cplusplus
}
#endif

#endif /* NEGF_B200_H */
