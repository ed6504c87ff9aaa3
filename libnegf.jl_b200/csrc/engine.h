// Host-side sweep planner of the B200 NEGF library.
//
// A sweep (RGF, RKD, general RGF, selected inverse, DDRGF, the batched-energy
// NEGF solve) is compiled once into a Plan: an ordered list of batched kernel
// launches whose problem descriptors live in one device buffer.  Every launch
// covers all independent systems (energies, devices, DDRGF domains) of one
// step of the recursion, so the serial dependency of the reference's loops is
// kept while each step fills the GPU.  A Plan is replayed with run(); with
// use_graph it is captured once into a CUDA graph and relaunched from there.
#pragma once

#include <string>
#include <functional>
#include <map>
#include <vector>
#include <cstddef>

#include "negf_common.cuh"

namespace negf {

// launchers (zgemm.cu, zinv.cu, zelem.cu)
cudaError_t launch_zgemm_batched(char opA, char opB, const ZGemmProblem* probs_dev, const int* tile_start_dev,
                                 int nprob, int total_tiles, cudaStream_t stream);
cudaError_t launch_zgemm_batched_ex(char opA, char opB, bool preload, const ZGemmProblem* probs_dev,
                                    const int* tile_start_dev, int nprob, int total_tiles, cudaStream_t stream,
                                    int form = 0, int uniform_tiles = 0);
bool zgemm_preload_ok(const ZGemmProblem& p);
int zgemm_tiles(int m, int n);
// small-K 3M kernel (32 x 64 tiles, two CTAs per SM) for steps with every
// k <= 32 in the 3M form; a step using it carries form 3 and counts its tiles
// with zgemm_tiles_smallk
bool zgemm_smallk_ok(int form, int max_k);
int zgemm_tiles_smallk(int m, int n);
size_t zgemm_smem_bytes();
cudaError_t zgemm_prepare(char opA, char opB);
size_t zgj_panel_smem_bytes(int n, int nb);
// max_n (the largest block of the batch) selects the register-resident panel
// kernel where it applies; 0 keeps the shared-memory one
cudaError_t launch_zgj_panel(const ZInvProblem* probs_dev, int nprob, int k0, int nb, int blocked, size_t smem,
                             cudaStream_t stream, int max_n = 0);
cudaError_t launch_zgj_unpermute(const ZInvProblem* probs_dev, int nprob, int max_n, cudaStream_t stream);
cudaError_t launch_zblockops(const ZBlockOp* ops_dev, int nops, int max_m, int max_n, cudaStream_t stream);
cudaError_t launch_ztrace_prod(const void* probs_dev, int nprob, cudaStream_t stream);
size_t zgetrf_panel_smem_bytes(int n, int nb);
size_t ztrtri_smem_bytes(int nb);
cudaError_t zlu_prepare(size_t panel_smem, size_t tri_smem);
cudaError_t launch_zgetrf_panel(const void* probs, int nprob, int k0, int nb, size_t smem, cudaStream_t st);
cudaError_t launch_zlaswp_copy(const void* probs, int nprob, int k0, int nb, int max_n, cudaStream_t st);
cudaError_t launch_ztrtri_diag(const void* probs, int nprob, int nb, int upper, int max_n, size_t smem,
                               cudaStream_t st);

// mixed-precision (Ozaki / INT8 tcgen05) complex GEMM, zgemm_ozaki.cu
struct OzSplitProblem;
struct OzMmaProblem;
size_t ozaki_mma_smem_bytes();
cudaError_t ozaki_prepare();
// dense INT8 tensor-core throughput of this device, TOP/s
cudaError_t ozaki_probe_int8(double* tops);
cudaError_t ozaki_probe_overlap(double* fp64_alone, double* fp64_beside_mma, double* mma_alone);
cudaError_t launch_ozaki_split(const void* probs, int nprob, int max_rows_pad, int max_k_pad, cudaStream_t st);
// CSC <-> band blocks on the device (csc.cu); block table slot 3 i + (j - i + 1)
cudaError_t launch_csc_scatter(int n, const int* colptr, const int* rowval, const cplx* nz, int nnz, const int* blk_of,
                               const int* off, const int* bsz, cplx* const* blocks, int hermitian, cudaStream_t st);
cudaError_t launch_csc_band_out(int pass, int n, int npl, int wout, const int* blk_of, const int* off, const int* bsz,
                                const cplx* const* res, const int* colptr_in, const int* rowval_in,
                                const cplx* nz_in, int nnz_in, int* counts, const int* colptr_out, int* rowval_out,
                                cplx* nz_out, cudaStream_t st);
cudaError_t launch_csc_full_scatter(int n, const int* colptr, const int* rowval, const cplx* nz, int nnz,
                                    const int* blk_of, const int* off, const int* bsz, cplx* const* table, int nb,
                                    cudaStream_t st);
cudaError_t launch_csc_direct_out(int pass, int n, int npl, int wout, const int* blk_of, const int* off,
                                  const int* iblk_of, const int* ioff, const int* ibsz, int nb, const cplx* const* res,
                                  const int* colptr_in, const int* rowval_in, const cplx* nz_in, int nnz_in,
                                  int* counts, const int* colptr_out, int* rowval_out, cplx* nz_out, cudaStream_t st);
// tile_map: per output tile an int4 (problem, m tile | n tile << 16,
// K chunks | m tiles << 16, n tiles)
// pairs: 34 (products as accurate as FP64) or 28 (within ~3x of the FP64 bound)
cudaError_t launch_ozaki_mma(const void* probs, const void* tile_map, int total_tiles, int* err, cudaStream_t st,
                             int pairs);
// pipeline wait limit (clock cycles) of product launches made from now on; <= 0: the default (~1 s)
void ozaki_set_wait_cycles(long long cycles);

// LU request (LAPACK getrf semantics, in place).  ipiv receives 0-based
// global pivot rows; ipiv_lapack (optional, device int32) 1-based ones.
struct LuSpec {
  cplx* A;
  int n, ld;
  int* ipiv;
  cplx* Linv;  // scratch nb x nb
  cplx* T;     // scratch nb x n
  int* info;
  bool nopiv = false;  // lu(A, NoPivot()): no row interchanges
};
// Triangular inverse request: X = inverse of the upper (non-unit) or unit
// lower triangle of the packed factors A; T is scratch n x nb.
struct TriSpec {
  const cplx* A;
  int n, lda;
  cplx* X;
  int ldx;
  cplx* T;
};
constexpr int kTriNb = 32;
int lu_panel_width(int max_n);

struct ZTraceProblemHost {
  const cplx* X;
  const cplx* Y;
  int n, ldx, ldy, pad_;
  double* out;
};

// Largest block size the Gauss-Jordan inversion supports (panel in shared memory).
constexpr int kMaxBlock = 1024;

// Panel width used for an inversion batch whose largest block is max_n
// (max_n itself when the whole block fits in shared memory).
int gj_panel_width(int max_n);

// Inversion request: W (n x n, ld) holds X and is destroyed; out receives X^{-1}.
struct InvSpec {
  cplx* W;
  int n, ld;
  cplx* out;
  int ldo;
  cplx* F;        // scratch n x nb
  cplx* Bbuf;     // scratch nb x n
  uint8_t* used;  // scratch n
  int* piv;       // scratch n
  int* info;
};

struct Step {
  enum Kind {
    GEMM = 0, GJ_PANEL = 1, GJ_UNPERMUTE = 2, BLOCKOP = 3, TRACE = 4, LU_PANEL = 5, LU_SWAP = 6, TRI_DIAG = 7,
    OZ_SPLIT = 8, OZ_MMA = 9
  } kind;
  char opA = 'N', opB = 'N';
  size_t off = 0;        // descriptor offset in the blob
  size_t tiles_off = 0;  // tile prefix-sum offset (GEMM)
  int count = 0, total_tiles = 0, max_m = 0, max_n = 0;
  int k0 = 0, nb = 0, blocked = 0;
  bool preload = false;  // GEMM: accumulators start from Cin (all problems alpha, beta = +-1)
  int form = 0;          // GEMM: 0 default, 1 four real products, 2 3M, 3 small-K 3M; OZ_MMA: digit pairs (34 or 28)
  int uniform_tiles = 0; // GEMM: tiles of every problem when all have the same count, else 0
  size_t smem = 0;
  double flops = 0.0;    // real flops of the step (8mnk per complex GEMM)
  double bytes = 0.0;    // OZ_SPLIT: algorithmic bytes (operands read once, digit slices and scales written)
};

class Plan {
 public:
  Plan() = default;
  ~Plan();
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;

  // device memory owned by the plan (workspace); zero-initialised, 256-byte
  // aligned, sub-allocated from a few large chunks
  void* alloc(size_t bytes);
  cplx* alloc_c(size_t n) { return static_cast<cplx*>(alloc(n * sizeof(cplx))); }

  // Complex GEMM step; with set_mixed(true) the products (k > 0) run on the
  // INT8 tensor cores with FP64-accurate Ozaki splitting.  The Gauss-Jordan
  // rank-nb updates issued by inv() follow set_gj_update.
  void gemm(char opA, char opB, const std::vector<ZGemmProblem>& probs);
  void gemm_fp64(char opA, char opB, const std::vector<ZGemmProblem>& probs);
  // pairs: 28 or 34 digit pairs for this step (0: the plan's count)
  void gemm_mixed(char opA, char opB, const std::vector<ZGemmProblem>& probs, int pairs = 0);
  // pairs: digit pairs of the INT8 products, 34 (as accurate as FP64
  // products) or 28 (within ~3x of the FP64 rounding bound, ~18 % fewer MMAs)
  void set_mixed(bool on, int pairs = 34) { mixed_ = on; oz_pairs_ = pairs == 28 ? 28 : 34; }
  int mixed_pairs() const { return oz_pairs_; }
  // schedule knobs: FP64 GEMM form (0 default, 1 four products, 2 3M) and the
  // Gauss-Jordan panel width for blocks > 112 (0 default)
  void set_schedule(int gemm_form, int gj_nb) { gemm_form_ = gemm_form; gj_nb_ = gj_nb; }
  // Gauss-Jordan rank-nb updates of a mixed plan: 1 FP64 DMMA products, 2
  // INT8 digit products with 34 pairs (as accurate as FP64 products), 0 the
  // default (1: at 256 x 32 layers both take the same time per pass, and the
  // FP64 form needs no digit split).  Plans without set_mixed(true) keep them
  // in FP64.
  void set_gj_update(int mode) { gj_update_ = mode; }
  bool gj_update_int8() const { return mixed_ && gj_update_ == 2; }
  int panel_width(int max_n) const;
  bool mixed() const { return mixed_; }
  int* error_flag() const { return err_; }
  void inv(const std::vector<InvSpec>& specs);
  void blockops(const std::vector<ZBlockOp>& ops);
  void trace(const std::vector<ZTraceProblemHost>& probs);
  void getrf(const std::vector<LuSpec>& specs);
  void trtri(const std::vector<TriSpec>& specs, bool upper);

  cudaError_t finalize();
  // Records a plan-owned event on s after work that uses the plan's memory
  // (every run does it; callers add it after their own uploads outside a
  // run).  The destructor waits for these events before the chunks are
  // reused: events stay valid after their streams are destroyed, and waiting
  // for them leaves other threads' graph captures alone.
  void fence(cudaStream_t s);
  cudaError_t run(cudaStream_t stream, bool use_graph);
  // Launch-by-launch replay with a CUDA event recorded after every launch
  // (events[0] before the first); events must hold steps.size() + 1 events.
  cudaError_t run_events(cudaStream_t stream, const std::vector<cudaEvent_t>& events);
  // Markers: mark(tag) notes that everything built so far is done at this
  // point of the pass; run_marked replays launch by launch (no graph) and
  // calls at_mark(tag) in stream order at every marker, so the caller can
  // record an event there and start work that depends on it.
  void mark(int tag) { marks_.push_back({steps.size(), tag}); }
  const std::vector<std::pair<size_t, int>>& marks() const { return marks_; }
  cudaError_t run_marked(cudaStream_t stream, const std::function<cudaError_t(int)>& at_mark);

  double flops() const;
  size_t num_launches() const;
  // device bytes the plan holds (its chunks)
  size_t workspace_bytes() const { return owned_bytes_; }
  std::vector<Step> steps;

 private:
  cudaError_t launch_step(const Step& s, const unsigned char* base, cudaStream_t stream);
  size_t push_bytes(const void* p, size_t n);
  void* raw_alloc(size_t bytes);
  std::vector<unsigned char> blob_;
  void* dblob_ = nullptr;
  std::vector<std::pair<void*, size_t>> owned_;  // chunks and their sizes
  std::vector<std::pair<cudaStream_t, cudaEvent_t>> fences_;  // last use of the memory per stream (fence)
  size_t owned_bytes_ = 0;
  std::vector<std::pair<size_t, int>> marks_;
  unsigned char* chunk_ = nullptr;  // bump pointer into the current chunk
  size_t chunk_left_ = 0, chunk_size_ = 0;
  bool finalized_ = false;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
  cudaStream_t graph_stream_ = nullptr;
  bool mixed_ = false;
  int oz_pairs_ = 34;
  int gemm_form_ = 0, gj_nb_ = 0, gj_update_ = 0;
  int* err_ = nullptr;            // tensor-core wait time-out flag (device int)
  unsigned char* oz_pool_ = nullptr;  // digit-slice scratch shared by all mixed steps
  size_t oz_pool_bytes_ = 0;
  // Digits of the previous mixed step, reusable by the next one when no other
  // step comes in between and its products did not write the operand: per
  // operand view (pointer, row and K strides, rows, cols, conj, side) its
  // slices, scales and padded sizes
  struct OzSplitDone {
    int8_t* slices;
    int* exps;
    int rpad, kpad;
  };
  std::map<std::vector<long long>, OzSplitDone> oz_prev_;
  std::vector<std::pair<const char*, const char*>> oz_prev_out_;  // byte ranges the previous step wrote
  size_t oz_prev_end_ = 0;        // pool bytes its digits occupy
  size_t oz_prev_steps_ = 0;      // steps.size() right after it
  unsigned char* oz_prev_pool_ = nullptr;
};

// ---------------------------------------------------------------------------
// Block-tridiagonal systems and the sweeps over them.

// View of one block-tridiagonal matrix M through its operand blocks:
//   M[i,i]   = dscale * D[i] + shift * I
//   M[i,i+1] = uscale * U[i]
//   M[i+1,i] = lscale * op(Lw[i]),  op = identity (lop 'N') or conjugate
//              transpose (lop 'C', Lw[i] then has the (i,i+1) shape).
// The NEGF device path uses D = H_ii (+Sigma), U = Lw = H_{i,i+1}, dscale =
// uscale = lscale = -1, shift = E + i*eta, lop = 'C'; the reference API path
// uses the M blocks themselves with unit scales.
struct TriSystem {
  std::vector<int> b;
  std::vector<const cplx*> D, U, Lw;
  std::vector<int> ldD, ldU, ldL;
  cplx dscale{1.0, 0.0}, shift{0.0, 0.0}, uscale{1.0, 0.0}, lscale{1.0, 0.0};
  const cplx* shift_ptr = nullptr;  // when set, the shift is read from device memory
  char lop = 'N';
  int* info = nullptr;  // device int, set on a zero pivot
  int npl() const { return static_cast<int>(b.size()); }
  int maxb() const;
};

// Workspace of the RGF upward pass of one system.
struct RgfWork {
  std::vector<cplx*> g;   // g[i] = X_i^{-1}          (b_i x b_i)
  std::vector<cplx*> R;   // R[i] = M[i,i+1] g[i+1]   (b_i x b_{i+1})
  std::vector<cplx*> L;   // L[i] = g[i+1] M[i+1,i]   (b_{i+1} x b_i), index i for L_{i+1}
  cplx* W = nullptr;      // inversion workspace (maxb^2)
  cplx* F = nullptr;
  cplx* Bbuf = nullptr;
  uint8_t* used = nullptr;
  int* piv = nullptr;
};

// Output block pointers of a tridiagonal result (null entries: not wanted).
struct TriOut {
  std::vector<cplx*> d, u, l;   // d[i] (i,i); u[i] (i,i+1); l[i] (i+1,i)
  std::vector<int> ldd, ldu, ldl;
};

void alloc_rgf_work(Plan& plan, const TriSystem& s, RgfWork& w);
// Upward pass (src/matinvertndiag_rgf.jl:143-162), all systems batched per layer.
void build_rgf_upward(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work);
// Downward pass (src/matinvertndiag_rgf.jl:166-182) writing the tridiagonal of
// M^{-1}; with full_rows/full_cols the whole inverse (rgf.jl:185-199) is
// written into full[s][i*npl+j] (null = skip).
// on_final(i), when given, is called once layer i's diagonal output is final
// for every system (in layer order).
void build_rgf_downward(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
                        std::vector<TriOut>& out, const std::function<void(int)>& on_final = {});
void build_rgf_full_inverse(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
                            std::vector<std::vector<cplx*>>& full);
// RKD passes (src/keldyshndiag.jl:221-317).  S holds the Hermitian middle
// operator (diagonal + upper blocks) on entry and G^n on exit.
struct HermBlocks {
  std::vector<cplx*> d, u;
  std::vector<int> ldd, ldu;
};
// on_final(i), when given, is called once G^n's diagonal block i is final
// (no later step of the pass reads or writes it) for every system.
void build_rkd(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
               std::vector<HermBlocks>& S, const std::function<void(int)>& on_final = {});

// Block selected inverse (selinv.cu): Block_factorization! and / or
// Block_inverse! (src/selected_inverse.jl:9-206, mode bit 1 / bit 2) in place
// on each system's npl x npl block table (row-major, null = unassigned; all
// systems share system 0's pattern; blocks b x b, ld b).  info points to npl
// ints per system (zero pivot of block i).  nopiv: lu(NoPivot()) for the
// diagonal blocks instead of the reference's getrf with discarded pivots.
struct SelInvSystem {
  std::vector<cplx*> A;
  int* info = nullptr;
};
int build_selected_inverse(Plan& plan, std::vector<SelInvSystem>& sys, int npl, int b, int mode, bool nopiv);

// Multi-level DDRGF (sweeps.cu) of systems with one layer count and unit
// scales (D, U, Lw are the M blocks themselves, lop 'N'); d1s[level] are the
// interior sizes, past the last level sequential RGF.
int build_ddrgf_level(Plan& plan, const std::vector<TriSystem>& sys, std::vector<TriOut>& out,
                      const std::vector<int>& d1s, size_t level);
// Levels of the library's GPU cost model for nsys systems of npl layers of b.
std::vector<int> choose_levels(int npl, int b, int nsys, int max_levels);

// Device chunks of destroyed plans are kept per device for the next plans
// (cudaFree of hundreds of chunks costs ~1 ms each and synchronises the
// device): cached_bytes() is memory the library holds but can hand out again,
// release_cached_memory() returns it to the driver.
size_t cached_bytes(int device);
void release_cached_memory();

std::string& last_error();
void set_error(const std::string& msg);

}  // namespace negf

struct negf_solver_s;
namespace negf {
// One pass of a solver launch by launch on `stream`, without graph capture
// (negf_api.cu): for one-off plans such as a request-server group's.
int solver_run_direct(negf_solver_s* s, cudaStream_t stream);

}  // namespace negf
