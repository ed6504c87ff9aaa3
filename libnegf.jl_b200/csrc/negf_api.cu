// extern "C" entry points of libnegf_b200.so (declared in include/negf_b200.h).
#include "../../include/negf_b200.h"
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

using namespace negf;

namespace {

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(NEGF_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define NEGF_TRY_CUDA(expr, where)                  \
  do {                                              \
    cudaError_t e__ = (expr);                       \
    if (e__ != cudaSuccess) return cuda_fail(e__, where); \
  } while (0)

int check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(NEGF_ERR_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
  return NEGF_SUCCESS;
}

inline cplx c2(const double* v) { return make_double2(v[0], v[1]); }

// Run a finished plan once, synchronously, and read the per-system info codes.
int run_plan_sync(Plan& plan, cudaStream_t st, int* dinfo, int nsys, const char* what) {
  cudaError_t e = plan.run(st, false);
  if (e != cudaSuccess) return cuda_fail(e, what);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, what);
  if (dinfo) {
    std::vector<int> info(nsys);
    e = cudaMemcpy(info.data(), dinfo, sizeof(int) * nsys, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, what);
    for (int s = 0; s < nsys; ++s)
      if (info[s] != 0) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "%s: zero pivot in system %d (column %d of a diagonal block)", what, s,
                      info[s]);
        return fail(NEGF_ERR_SINGULAR, buf);
      }
  }
  return NEGF_SUCCESS;
}

// Build the TriSystem list of the reference-API sweeps from pointer tables.
int make_systems(int nsys, int npl, const int32_t* bs, void* const* Md, void* const* Mu, void* const* Ml,
                 int* dinfo, std::vector<TriSystem>& sys) {
  if (nsys <= 0 || npl <= 0 || !bs || !Md) return fail(NEGF_ERR_INVALID, "nsys, npl, block_sizes and Md are required");
  if (npl > 1 && (!Mu || !Ml)) return fail(NEGF_ERR_INVALID, "Mu and Ml are required when npl > 1");
  sys.resize(nsys);
  for (int s = 0; s < nsys; ++s) {
    TriSystem& t = sys[s];
    t.b.assign(bs + (size_t)s * npl, bs + (size_t)(s + 1) * npl);
    for (int x : t.b)
      if (x <= 0 || x > kMaxBlock) return fail(NEGF_ERR_INVALID, "block sizes must be in [1, 1024]");
    for (int i = 0; i < npl; ++i) {
      t.D.push_back(static_cast<const cplx*>(Md[(size_t)s * npl + i]));
      t.ldD.push_back(t.b[i]);
      if (!t.D.back()) return fail(NEGF_ERR_INVALID, "NULL diagonal block");
    }
    for (int i = 0; i + 1 < npl; ++i) {
      t.U.push_back(static_cast<const cplx*>(Mu[(size_t)s * (npl - 1) + i]));
      t.ldU.push_back(t.b[i]);
      t.Lw.push_back(static_cast<const cplx*>(Ml[(size_t)s * (npl - 1) + i]));
      t.ldL.push_back(t.b[i + 1]);
      if (!t.U.back() || !t.Lw.back()) return fail(NEGF_ERR_INVALID, "NULL off-diagonal block");
    }
    t.info = dinfo + s;
  }
  return NEGF_SUCCESS;
}

// ---------------------------------------------------------------------------
// FP64 peak probe kernels (throughput loops, no memory traffic)
__global__ void probe_dmma(double* out, int iters) {
  double a0 = threadIdx.x * 1e-3, a1 = 1.0 + a0, b0 = 0.5 + a0;
  double c[4] = {0, 0, 0, 0}, d[4] = {0, 0, 0, 0};
  for (int i = 0; i < iters; ++i) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3]) : "d"(a0), "d"(a1), "d"(b0));
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3]) : "d"(a1), "d"(a0), "d"(b0));
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = c[0] + c[1] + c[2] + c[3] + d[0] + d[1] + d[2] + d[3];
}

__global__ void probe_dfma(double* out, int iters) {
  double x[8];
  for (int j = 0; j < 8; ++j) x[j] = threadIdx.x * 1e-3 + j;
  double y = 0.999999, z = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = fma(x[j], y, z);
  }
  double s = 0;
  for (int j = 0; j < 8; ++j) s += x[j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// ---------------------------------------------------------------------------
// Device object and resident solver of the batched-energy NEGF path.

struct negf_device_s {
  int npl = 0;
  std::vector<int> b;
  std::vector<cplx*> D;   // H_ii (+ Sigma_L on layer 0, + Sigma_R on layer N-1)
  std::vector<cplx*> Hu;  // H_{i,i+1}
  cplx* gamL = nullptr;
  cplx* gamR = nullptr;
  cplx* sigL = nullptr;
  cplx* sigR = nullptr;
  std::vector<cplx*> Sd, Su;       // overlap blocks (set by negf_device_set_overlap)
  bool has_S = false;
  std::unique_ptr<Plan> assemble;  // Sigma / Gamma assembly launches
  cudaStream_t stream = nullptr;
  std::vector<void*> owned;
  ~negf_device_s() {
    assemble.reset();
    if (stream) cudaStreamDestroy(stream);
    for (void* p : owned) cudaFree(p);
  }
};

struct negf_solver_s {
  negf_device_s* dev = nullptr;             // the first (or only) device
  std::vector<negf_device_s*> devs;         // devices of the batch, in order
  std::vector<int> dev_nE;                  // energies per device
  size_t out_total = 0;                     // elements of gr / gl (all devices and energies)
  int nE = 0;                               // energies of all devices
  negf_solve_opts opts{};
  std::unique_ptr<Plan> plan;
  cplx* params = nullptr;  // [shift (nE) | f_L (nE) | f_R (nE) | i (1)]
  cplx* gr = nullptr;      // nE * sum b_i^2
  cplx* gl = nullptr;
  double* t2 = nullptr;    // 2 * nE (re, im)
  int* info = nullptr;
  std::vector<cplx*> sigL_e, sigR_e;  // per-energy self-energies (opts.sigma_per_energy)
  std::vector<int> bL_e, bR_e;        // their sizes
  size_t per_energy = 0;   // sum b_i^2 (single-device solvers; 0 for a multi-device batch)
  std::vector<std::vector<cudaEvent_t>> ev_sets;  // one event set per profiled pass
  size_t ev_used = 0;
  cudaStream_t copy_stream = nullptr;  // overlapped downloads (negf_solver_run_download)
  cudaEvent_t mark_ev = nullptr, join_ev = nullptr;
  ~negf_solver_s() {
    // downloads on the copy stream read plan memory: done before the plan goes
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    for (auto& v : ev_sets)
      for (cudaEvent_t e : v) cudaEventDestroy(e);
    if (mark_ev) cudaEventDestroy(mark_ev);
    if (join_ev) cudaEventDestroy(join_ev);
    if (copy_stream) cudaStreamDestroy(copy_stream);
  }
};

// Plan marker tags of the solver pass: output layer i final.
constexpr int kMarkGR = 0, kMarkGL = 1 << 20;

namespace {

size_t solver_bytes_per_energy(const negf_device_s& d, const negf_solve_opts& o) {
  size_t n = d.npl, mb = 0, sb2 = 0, sbb = 0;
  for (int x : d.b) { mb = std::max<size_t>(mb, x); sb2 += (size_t)x * x; }
  for (size_t i = 0; i + 1 < n; ++i) sbb += (size_t)d.b[i] * d.b[i + 1];
  size_t nb = gj_panel_width((int)mb);
  size_t c = sb2 + 2 * sbb + mb * mb + 2 * mb * nb;  // RGF work
  if (o.want_gr) c += sb2 + 4 * mb * mb;              // G^R diagonal + rings
  if (o.want_gl) c += sb2 + sbb + 3 * n * mb * mb;    // G^n storage + RKD scratch
  if (o.want_t) c += 4 * mb * mb;
  if (d.has_S || o.sigma_per_energy) c += sb2 + 2 * sbb;  // per-energy M blocks
  if (o.sigma_per_energy) c += 2 * ((size_t)d.b.front() * d.b.front() + (size_t)d.b.back() * d.b.back());
  size_t bytes = c * sizeof(cplx) + 64;
  if (o.precision == NEGF_PREC_MIXED) {
    // digit slices of the INT8 products (21 bytes per padded element): the
    // widest steps (the Keldysh per-layer products of all layers at once)
    // split about three operands per layer
    const size_t pad = (mb + 127) / 128 * 128;
    bytes += 21 * 3 * n * pad * pad;
  }
  return bytes;
}

// Opt-in shared memory per block of the current device (bytes).
size_t max_panel_smem() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return (size_t)v;
}

// One plan for every (device, energy) item of the batch: the devices may differ
// in layer count and block sizes; each batched launch takes the items whose
// recursion reaches that step. Item e uses parameter slots e (shift), nE + e
// (f_L), 2 nE + e (f_R) and output blocks at offset off(e) in gr / gl
// (device-major, then energy, then layer).
int build_solver(negf_solver_s& S) {
  const int nE = S.nE;
  Plan& plan = *S.plan;
  struct Item {
    negf_device_s* d;
    size_t off;
  };
  std::vector<Item> items;
  size_t off = 0;
  for (size_t k = 0; k < S.devs.size(); ++k) {
    size_t pe = 0;
    for (int x : S.devs[k]->b) pe += (size_t)x * x;
    for (int e = 0; e < S.dev_nE[k]; ++e) {
      items.push_back({S.devs[k], off});
      off += pe;
    }
  }
  if ((int)items.size() != nE) return fail(NEGF_ERR_INVALID, "energy counts do not add up");
  S.out_total = off;
  S.per_energy = S.devs.size() == 1 ? off / (size_t)nE : 0;
  S.params = plan.alloc_c(3 * (size_t)nE + 1);
  S.info = static_cast<int*>(plan.alloc(sizeof(int) * nE));
  if (S.opts.want_gr) S.gr = plan.alloc_c(S.out_total);
  if (S.opts.want_gl) S.gl = plan.alloc_c(S.out_total);
  if (S.opts.want_t) S.t2 = static_cast<double*>(plan.alloc(sizeof(double) * 2 * nE));
  const cplx i_unit = make_double2(0.0, 1.0);
  NEGF_TRY_CUDA(cudaMemcpy(S.params + 3 * nE, &i_unit, sizeof(cplx), cudaMemcpyHostToDevice), "solver params");
  if (S.opts.precision != NEGF_PREC_FP64 && S.opts.precision != NEGF_PREC_MIXED)
    return fail(NEGF_ERR_INVALID, "precision must be NEGF_PREC_FP64 or NEGF_PREC_MIXED");
  for (negf_device_s* dv : S.devs) {
    for (int x : dv->b)
      if (S.opts.precision == NEGF_PREC_MIXED && x > 1024)
        return fail(NEGF_ERR_INVALID, "the mixed precision mode supports blocks up to 1024");
    if (S.opts.want_t && dv->b.front() != dv->b.back())
      return fail(NEGF_ERR_INVALID, "transmission needs equal first and last block sizes");
  }
  // the RGF / RKD products: 28 digit pairs (within ~3x of the FP64 rounding
  // bound per product; ~3e-11 per block at 256 x 32 layers against the truth)
  plan.set_mixed(S.opts.precision == NEGF_PREC_MIXED, 28);
  if (S.opts.gemm_form < 0 || S.opts.gemm_form > 2) return fail(NEGF_ERR_INVALID, "gemm_form must be 0, 1 or 2");
  if (S.opts.gj_nb != 0 && S.opts.gj_nb != 8 && S.opts.gj_nb != 16 && S.opts.gj_nb != 32)
    return fail(NEGF_ERR_INVALID, "gj_nb must be 0, 8, 16 or 32");
  for (negf_device_s* dv : S.devs)
    for (int x : dv->b)
      if (S.opts.gj_nb > 0 && x > 112 && zgj_panel_smem_bytes(x, S.opts.gj_nb) > max_panel_smem())
        return fail(NEGF_ERR_INVALID, "gj_nb too wide for the block size (shared memory)");
  if (S.opts.gj_update < 0 || S.opts.gj_update > 2) return fail(NEGF_ERR_INVALID, "gj_update must be 0, 1 or 2");
  plan.set_schedule(S.opts.gemm_form, S.opts.gj_nb);
  plan.set_gj_update(S.opts.gj_update);

  const bool sig_e = S.opts.sigma_per_energy != 0;
  std::vector<TriSystem> sys(nE);
  std::vector<RgfWork> work(nE);
  std::vector<cplx*> gamL_of(nE), gamR_of(nE);
  // per-energy M(E) = z S - H - Sigma(E) (z = E + i eta) when the device has an
  // overlap or the self-energies depend on the energy (build_M_from_HS,
  // src/matloader.jl:89-95); otherwise M is never formed (shift in the GEMM
  // epilogue, off-diagonal blocks shared)
  std::vector<ZBlockOp> asm_set, asm_add, asm_l1, asm_l2, asm_r1, asm_r2;
  auto op = [](ZOpKind k, const cplx* A, int lda, cplx* C, int ldc, int m, int n2, cplx alpha, cplx beta,
               const cplx* alpha_ptr = nullptr) {
    ZBlockOp o{};
    o.A = A; o.lda = lda; o.C = C; o.ldc = ldc; o.m = m; o.n = n2; o.kind = k;
    o.alpha = alpha; o.beta = beta; o.alpha_ptr = alpha_ptr;
    return o;
  };
  const cplx P1 = make_double2(1.0, 0.0), M1 = make_double2(-1.0, 0.0), Z0 = make_double2(0.0, 0.0);
  if (sig_e) {
    S.sigL_e.assign(nE, nullptr);
    S.sigR_e.assign(nE, nullptr);
    S.bL_e.assign(nE, 0);
    S.bR_e.assign(nE, 0);
  }
  for (int e = 0; e < nE; ++e) {
    const negf_device_s& d = *items[e].d;
    const int n = d.npl;
    TriSystem& t = sys[e];
    t.b = d.b;
    t.info = S.info + e;
    gamL_of[e] = d.gamL;
    gamR_of[e] = d.gamR;
    if (sig_e || d.has_S) {
      const cplx* z = S.params + e;
      std::vector<cplx*> md(n);
      for (int i = 0; i < n; ++i) {
        cplx* m = md[i] = plan.alloc_c((size_t)d.b[i] * d.b[i]);
        t.D.push_back(m); t.ldD.push_back(d.b[i]);
        asm_set.push_back(op(ZOP_AXPBY, d.D[i], d.b[i], m, d.b[i], d.b[i], d.b[i], M1, Z0));
        if (d.has_S) asm_add.push_back(op(ZOP_AXPBY, d.Sd[i], d.b[i], m, d.b[i], d.b[i], d.b[i], P1, P1, z));
        else asm_add.push_back(op(ZOP_ADD_DIAG, nullptr, 1, m, d.b[i], d.b[i], d.b[i], P1, P1, z));
      }
      for (int i = 0; i + 1 < n; ++i) {
        const int bi = d.b[i], bj = d.b[i + 1];
        cplx* u = plan.alloc_c((size_t)bi * bj);
        cplx* l = plan.alloc_c((size_t)bi * bj);
        t.U.push_back(u); t.ldU.push_back(bi);
        t.Lw.push_back(l); t.ldL.push_back(bj);
        asm_set.push_back(op(ZOP_AXPBY, d.Hu[i], bi, u, bi, bi, bj, M1, Z0));
        asm_set.push_back(op(ZOP_CTRANS_AXPBY, d.Hu[i], bi, l, bj, bj, bi, M1, Z0));
        if (d.has_S) {
          asm_add.push_back(op(ZOP_AXPBY, d.Su[i], bi, u, bi, bi, bj, P1, P1, z));
          asm_add.push_back(op(ZOP_CTRANS_AXPBY, d.Su[i], bi, l, bj, bj, bi, P1, P1, z));
        }
      }
      t.dscale = P1; t.uscale = P1; t.lscale = P1;
      t.lop = 'N';
      t.shift_ptr = nullptr;
      if (sig_e) {
        // Sigma(E) replaces the device's constant self-energy (already in D[0], D[N-1])
        const int b0 = d.b.front(), bN = d.b.back();
        S.bL_e[e] = b0; S.bR_e[e] = bN;
        S.sigL_e[e] = plan.alloc_c((size_t)b0 * b0);
        S.sigR_e[e] = plan.alloc_c((size_t)bN * bN);
        gamL_of[e] = plan.alloc_c((size_t)b0 * b0);
        gamR_of[e] = plan.alloc_c((size_t)bN * bN);
        asm_set.push_back(op(ZOP_GAMMA, S.sigL_e[e], b0, gamL_of[e], b0, b0, b0, P1, Z0));
        asm_set.push_back(op(ZOP_GAMMA, S.sigR_e[e], bN, gamR_of[e], bN, bN, bN, P1, Z0));
        asm_l1.push_back(op(ZOP_AXPBY, d.sigL, b0, md[0], b0, b0, b0, P1, P1));
        asm_l2.push_back(op(ZOP_AXPBY, S.sigL_e[e], b0, md[0], b0, b0, b0, M1, P1));
        asm_r1.push_back(op(ZOP_AXPBY, d.sigR, bN, md[n - 1], bN, bN, bN, P1, P1));
        asm_r2.push_back(op(ZOP_AXPBY, S.sigR_e[e], bN, md[n - 1], bN, bN, bN, M1, P1));
      }
    } else {
      for (int i = 0; i < n; ++i) { t.D.push_back(d.D[i]); t.ldD.push_back(d.b[i]); }
      for (int i = 0; i + 1 < n; ++i) {
        t.U.push_back(d.Hu[i]); t.ldU.push_back(d.b[i]);
        t.Lw.push_back(d.Hu[i]); t.ldL.push_back(d.b[i]);
      }
      t.dscale = make_double2(-1.0, 0.0);
      t.uscale = make_double2(-1.0, 0.0);
      t.lscale = make_double2(-1.0, 0.0);
      t.lop = 'C';
      t.shift_ptr = S.params + e;
    }
    alloc_rgf_work(plan, t, work[e]);
  }
  // one launch per list: every block is written at most once per launch
  plan.blockops(asm_set);
  plan.blockops(asm_add);
  plan.blockops(asm_l1);
  plan.blockops(asm_l2);
  plan.blockops(asm_r1);
  plan.blockops(asm_r2);
  // block pointers inside the output arrays
  auto out_blocks = [&](cplx* base, int e) {
    const negf_device_s& d = *items[e].d;
    std::vector<cplx*> v;
    size_t o = items[e].off;
    for (int i = 0; i < d.npl; ++i) { v.push_back(base + o); o += (size_t)d.b[i] * d.b[i]; }
    return v;
  };
  std::vector<HermBlocks> herm(nE);
  if (S.opts.want_gl) {
    // Sigma^in = f_L Gamma_L (+) f_R Gamma_R in Hermitian storage
    std::vector<ZBlockOp> zero, setL, addR;
    for (int e = 0; e < nE; ++e) {
      const negf_device_s& d = *items[e].d;
      const int n = d.npl;
      HermBlocks& h = herm[e];
      h.d = out_blocks(S.gl, e);
      for (int i = 0; i < n; ++i) h.ldd.push_back(d.b[i]);
      for (int i = 0; i + 1 < n; ++i) {
        h.u.push_back(plan.alloc_c((size_t)d.b[i] * d.b[i + 1]));
        h.ldu.push_back(d.b[i]);
      }
      // every pass starts from Sigma^in: zero all diagonal and upper blocks
      for (int i = 0; i < n; ++i) {
        ZBlockOp z{}; z.C = h.d[i]; z.ldc = d.b[i]; z.m = z.n = d.b[i]; z.kind = ZOP_FILL;
        zero.push_back(z);
      }
      for (int i = 0; i + 1 < n; ++i) {
        ZBlockOp z{}; z.C = h.u[i]; z.ldc = d.b[i]; z.m = d.b[i]; z.n = d.b[i + 1]; z.kind = ZOP_FILL;
        zero.push_back(z);
      }
      ZBlockOp l{}; l.A = gamL_of[e]; l.lda = d.b[0]; l.C = h.d[0]; l.ldc = d.b[0]; l.m = l.n = d.b[0];
      l.kind = ZOP_AXPBY; l.alpha_ptr = S.params + nE + e; l.beta = make_double2(1.0, 0.0);
      setL.push_back(l);
      ZBlockOp r{}; r.A = gamR_of[e]; r.lda = d.b[n - 1]; r.C = h.d[n - 1]; r.ldc = d.b[n - 1];
      r.m = r.n = d.b[n - 1]; r.kind = ZOP_AXPBY; r.alpha_ptr = S.params + 2 * nE + e; r.beta = make_double2(1.0, 0.0);
      addR.push_back(r);
    }
    plan.blockops(zero);
    plan.blockops(setL);
    plan.blockops(addR);
  }
  build_rgf_upward(plan, sys, work);
  if (S.opts.want_gr) {
    std::vector<TriOut> out(nE);
    for (int e = 0; e < nE; ++e) {
      const negf_device_s& d = *items[e].d;
      TriOut& o = out[e];
      o.d = out_blocks(S.gr, e);
      for (int i = 0; i < d.npl; ++i) o.ldd.push_back(d.b[i]);
      int mb = sys[e].maxb();
      cplx* ring = plan.alloc_c(4 * (size_t)mb * mb);
      for (int i = 0; i + 1 < d.npl; ++i) {
        o.u.push_back(ring + (size_t)(i % 2) * mb * mb);
        o.l.push_back(ring + (size_t)(2 + i % 2) * mb * mb);
        o.ldu.push_back(d.b[i]);
        o.ldl.push_back(d.b[i + 1]);
      }
    }
    build_rgf_downward(plan, sys, work, out, [&](int i) { plan.mark(kMarkGR + i); });
  }
  if (S.opts.want_gl) {
    // G^< = i G^n, layer by layer as soon as G^n's layer is final
    build_rkd(plan, sys, work, herm, [&](int i) {
      std::vector<ZBlockOp> sc;
      for (int e = 0; e < nE; ++e) {
        const negf_device_s& d = *items[e].d;
        if (i >= d.npl) continue;
        ZBlockOp o{}; o.A = herm[e].d[i]; o.lda = d.b[i]; o.C = herm[e].d[i]; o.ldc = d.b[i];
        o.m = o.n = d.b[i]; o.kind = ZOP_AXPBY; o.alpha_ptr = S.params + 3 * nE; o.beta = make_double2(0.0, 0.0);
        sc.push_back(o);
      }
      plan.blockops(sc);
      plan.mark(kMarkGL + i);
    });
  }
  if (S.opts.want_t) {
    // G^R_{1N} by G_{1,j} = -G_{1,j-1} R_{j-1}, G_{1,1} = g_1 (rgf.jl:169, :185-199)
    std::vector<std::vector<cplx*>> Y(nE);
    std::vector<cplx*> P(nE), Q(nE);
    int maxN = 0;
    for (int e = 0; e < nE; ++e) {
      const int mb = sys[e].maxb();
      maxN = std::max(maxN, items[e].d->npl);
      cplx* a = plan.alloc_c(4 * (size_t)mb * mb);
      Y[e] = {a, a + (size_t)mb * mb};
      P[e] = a + 2 * (size_t)mb * mb;
      Q[e] = a + 3 * (size_t)mb * mb;
    }
    auto ycur = [&](int e, int j) -> const cplx* { return j == 0 ? work[e].g[0] : Y[e][j % 2]; };
    for (int j = 1; j < maxN; ++j) {
      std::vector<ZGemmProblem> pr;
      for (int e = 0; e < nE; ++e) {
        const negf_device_s& d = *items[e].d;
        if (j >= d.npl) continue;
        const int b0 = d.b[0];
        ZGemmProblem p{};
        p.A = ycur(e, j - 1); p.lda = b0;
        p.B = work[e].R[j - 1]; p.ldb = d.b[j - 1];
        p.C = Y[e][j % 2]; p.ldc = b0; p.ldcin = 1;
        p.m = b0; p.n = d.b[j]; p.k = d.b[j - 1];
        p.alpha = make_double2(-1.0, 0.0);
        pr.push_back(p);
      }
      plan.gemm('N', 'N', pr);
    }
    std::vector<ZGemmProblem> p1, p2;
    std::vector<ZTraceProblemHost> tr;
    for (int e = 0; e < nE; ++e) {
      const negf_device_s& d = *items[e].d;
      const int n = d.npl, b0 = d.b[0], bN = d.b[n - 1];
      const cplx* G1N = ycur(e, n - 1);
      ZGemmProblem a{};  // P = Gamma_L G1N  (b0 x bN)
      a.A = gamL_of[e]; a.lda = b0; a.B = G1N; a.ldb = b0; a.C = P[e]; a.ldc = b0; a.ldcin = 1;
      a.m = b0; a.n = bN; a.k = b0; a.alpha = make_double2(1.0, 0.0);
      p1.push_back(a);
      ZGemmProblem c{};  // Q = Gamma_R G1N^H  (bN x b0)
      c.A = gamR_of[e]; c.lda = bN; c.B = G1N; c.ldb = b0; c.C = Q[e]; c.ldc = bN; c.ldcin = 1;
      c.m = bN; c.n = b0; c.k = bN; c.alpha = make_double2(1.0, 0.0);
      p2.push_back(c);
      ZTraceProblemHost t{};
      t.X = P[e]; t.ldx = b0; t.Y = Q[e]; t.ldy = bN; t.n = b0; t.out = S.t2 + 2 * e;
      tr.push_back(t);
    }
    plan.gemm('N', 'N', p1);
    plan.gemm('N', 'C', p2);
    plan.trace(tr);
  }
  NEGF_TRY_CUDA(plan.finalize(), "solver finalize");
  return NEGF_SUCCESS;
}

}  // namespace

extern "C" {

const char* negf_last_error(void) { return last_error().c_str(); }

int negf_version(void) { return 100; }

int negf_zgemm_batched(char opA, char opB, int32_t nprob, const negf_zgemm_problem* probs, void* stream) {
  if (int r = check_device()) return r;
  if (nprob < 0 || (nprob > 0 && !probs)) return fail(NEGF_ERR_INVALID, "bad problem list");
  auto okop = [](char c) { return c == 'N' || c == 'T' || c == 'C'; };
  if (!okop(opA) || !okop(opB)) return fail(NEGF_ERR_INVALID, "op must be N, T or C");
  try {
    Plan plan;
    std::vector<ZGemmProblem> v(nprob);
    for (int i = 0; i < nprob; ++i) {
      const negf_zgemm_problem& q = probs[i];
      if (q.m < 0 || q.n < 0 || q.k < 0) return fail(NEGF_ERR_INVALID, "negative dimension");
      ZGemmProblem& p = v[i];
      p.A = static_cast<const cplx*>(q.A); p.B = static_cast<const cplx*>(q.B);
      p.Cin = static_cast<const cplx*>(q.Cin); p.C = static_cast<cplx*>(q.C); p.diag_ptr = nullptr;
      p.m = q.m; p.n = q.n; p.k = q.k;
      p.lda = std::max(1, q.lda); p.ldb = std::max(1, q.ldb); p.ldc = std::max(1, q.ldc);
      p.ldcin = std::max(1, q.ldcin); p.pad_ = 0;
      p.alpha = c2(q.alpha); p.beta = c2(q.beta); p.diag = c2(q.diag);
      if (p.m > 0 && p.n > 0 && !p.C) return fail(NEGF_ERR_INVALID, "NULL C");
      if (p.k > 0 && (!p.A || !p.B)) return fail(NEGF_ERR_INVALID, "NULL A or B");
    }
    plan.gemm(opA, opB, v);
    return run_plan_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_zgemm_batched");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_set_tensor_wait_limit(double seconds) {
  if (!(seconds == seconds)) return fail(NEGF_ERR_INVALID, "negf_set_tensor_wait_limit: NaN");
  // clock64() runs at the SM clock (<= ~2 GHz on B200)
  ozaki_set_wait_cycles(seconds > 0.0 ? std::max(64LL, (long long)std::min(seconds * 2e9, 4e18)) : 0LL);
  return NEGF_SUCCESS;
}

int negf_zgemm_batched_mixed(char opA, char opB, int32_t nprob, const negf_zgemm_problem* probs, void* stream) {
  if (int r = check_device()) return r;
  if (nprob < 0 || (nprob > 0 && !probs)) return fail(NEGF_ERR_INVALID, "bad problem list");
  auto okop = [](char c) { return c == 'N' || c == 'T' || c == 'C'; };
  if (!okop(opA) || !okop(opB)) return fail(NEGF_ERR_INVALID, "op must be N, T or C");
  try {
    Plan plan;
    plan.set_mixed(true);
    std::vector<ZGemmProblem> v(nprob);
    for (int i = 0; i < nprob; ++i) {
      const negf_zgemm_problem& q = probs[i];
      if (q.m < 0 || q.n < 0 || q.k < 0 || q.k > 1024)
        return fail(NEGF_ERR_INVALID, "dimensions must be >= 0 and k <= 1024");
      ZGemmProblem& p = v[i];
      p.A = static_cast<const cplx*>(q.A); p.B = static_cast<const cplx*>(q.B);
      p.Cin = static_cast<const cplx*>(q.Cin); p.C = static_cast<cplx*>(q.C); p.diag_ptr = nullptr;
      p.m = q.m; p.n = q.n; p.k = q.k;
      p.lda = std::max(1, q.lda); p.ldb = std::max(1, q.ldb); p.ldc = std::max(1, q.ldc);
      p.ldcin = std::max(1, q.ldcin); p.pad_ = 0;
      p.alpha = c2(q.alpha); p.beta = c2(q.beta); p.diag = c2(q.diag);
      if (p.m > 0 && p.n > 0 && !p.C) return fail(NEGF_ERR_INVALID, "NULL C");
      if (p.k > 0 && (!p.A || !p.B)) return fail(NEGF_ERR_INVALID, "NULL A or B");
    }
    plan.gemm(opA, opB, v);
    int rc = run_plan_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_zgemm_batched_mixed");
    if (rc) return rc;
    if (plan.error_flag()) {
      int h = 0;
      NEGF_TRY_CUDA(cudaMemcpy(&h, plan.error_flag(), sizeof(int), cudaMemcpyDeviceToHost), "mixed gemm");
      if (h) return fail(NEGF_ERR_TIMEOUT, "negf_zgemm_batched_mixed: tensor-core completion wait timed out");
    }
    return NEGF_SUCCESS;
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_zcopy_batched(char op, int32_t nprob, const int32_t* m, const int32_t* n, void* const* A,
                       const int32_t* lda, void* const* C, const int32_t* ldc, void* stream) {
  if (int r = check_device()) return r;
  if (op != 'N' && op != 'C') return fail(NEGF_ERR_INVALID, "op must be N or C");
  if (nprob < 0 || (nprob > 0 && (!m || !n || !A || !lda || !C || !ldc))) return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    std::vector<ZBlockOp> ops;
    for (int i = 0; i < nprob; ++i) {
      if (m[i] <= 0 || n[i] <= 0) continue;
      ZBlockOp o{};
      o.A = static_cast<const cplx*>(A[i]); o.lda = std::max(1, lda[i]);
      o.C = static_cast<cplx*>(C[i]); o.ldc = std::max(1, ldc[i]);
      o.m = m[i]; o.n = n[i]; o.kind = op == 'N' ? ZOP_COPY : ZOP_CTRANSPOSE;
      ops.push_back(o);
    }
    plan.blockops(ops);
    return run_plan_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_zcopy_batched");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_zfill_batched(int32_t nprob, const int32_t* m, const int32_t* n, void* const* C, const int32_t* ldc,
                       const double* value, void* stream) {
  if (int r = check_device()) return r;
  if (!value || nprob < 0 || (nprob > 0 && (!m || !n || !C || !ldc))) return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    std::vector<ZBlockOp> ops;
    for (int i = 0; i < nprob; ++i) {
      if (m[i] <= 0 || n[i] <= 0) continue;
      ZBlockOp o{};
      o.C = static_cast<cplx*>(C[i]); o.ldc = std::max(1, ldc[i]);
      o.m = m[i]; o.n = n[i]; o.kind = ZOP_FILL; o.alpha = make_double2(value[0], value[1]);
      ops.push_back(o);
    }
    plan.blockops(ops);
    return run_plan_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_zfill_batched");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_zinv_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* const* Ainv,
                      const int32_t* ldainv, int32_t* info, void* stream) {
  if (int r = check_device()) return r;
  if (nprob < 0 || (nprob > 0 && (!n || !A || !lda || !Ainv || !ldainv))) return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * std::max(1, nprob)));
    std::vector<ZBlockOp> copies;
    std::vector<InvSpec> specs;
    for (int i = 0; i < nprob; ++i) {
      if (n[i] < 0 || n[i] > kMaxBlock) return fail(NEGF_ERR_INVALID, "n must be in [0, 1024]");
      if (n[i] == 0) continue;
      int mb = n[i], nb = gj_panel_width(mb);
      InvSpec sp;
      sp.W = plan.alloc_c((size_t)mb * mb);
      sp.n = mb; sp.ld = mb; sp.out = static_cast<cplx*>(Ainv[i]); sp.ldo = ldainv[i];
      sp.F = plan.alloc_c((size_t)mb * nb);
      sp.Bbuf = plan.alloc_c((size_t)mb * nb);
      sp.used = static_cast<uint8_t*>(plan.alloc(mb));
      sp.piv = static_cast<int*>(plan.alloc(sizeof(int) * mb));
      sp.info = dinfo + i;
      specs.push_back(sp);
      ZBlockOp o{}; o.A = static_cast<const cplx*>(A[i]); o.lda = lda[i]; o.C = sp.W; o.ldc = mb;
      o.m = o.n = mb; o.kind = ZOP_COPY;
      copies.push_back(o);
    }
    plan.blockops(copies);
    plan.inv(specs);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = plan.run(st, false);
    if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched");
    NEGF_TRY_CUDA(cudaStreamSynchronize(st), "negf_zinv_batched");
    std::vector<int> h(std::max(1, nprob));
    NEGF_TRY_CUDA(cudaMemcpy(h.data(), dinfo, sizeof(int) * std::max(1, nprob), cudaMemcpyDeviceToHost),
                  "negf_zinv_batched");
    int bad = -1;
    for (int i = 0; i < nprob; ++i) {
      if (info) info[i] = h[i];
      if (h[i] && bad < 0) bad = i;
    }
    if (bad >= 0) {
      char buf[128];
      std::snprintf(buf, sizeof buf, "negf_zinv_batched: matrix %d is singular (zero pivot in column %d)", bad, h[bad]);
      return fail(NEGF_ERR_SINGULAR, buf);
    }
    return NEGF_SUCCESS;
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_rgf(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
             void* const* Ml, void* const* Gd, void* const* Gu, void* const* Gl, void* const* Gfull, void* stream) {
  if (int r = check_device()) return r;
  if (!Gd && !Gfull) return fail(NEGF_ERR_INVALID, "Gd or Gfull is required");
  try {
    Plan plan;
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * nsys));
    std::vector<TriSystem> sys;
    if (int r = make_systems(nsys, npl, block_sizes, Md, Mu, Ml, dinfo, sys)) return r;
    std::vector<RgfWork> work(nsys);
    for (int s = 0; s < nsys; ++s) alloc_rgf_work(plan, sys[s], work[s]);
    build_rgf_upward(plan, sys, work);
    std::vector<TriOut> out(nsys);
    std::vector<std::vector<cplx*>> full(nsys);
    for (int s = 0; s < nsys; ++s) {
      const TriSystem& t = sys[s];
      TriOut& o = out[s];
      auto pick = [&](void* const* tab, size_t idx, int i, int j) -> cplx* {
        if (Gfull) return static_cast<cplx*>(Gfull[(size_t)s * npl * npl + (size_t)i * npl + j]);
        return tab ? static_cast<cplx*>(tab[idx]) : nullptr;
      };
      for (int i = 0; i < npl; ++i) {
        cplx* p = pick(Gd, (size_t)s * npl + i, i, i);
        if (!p) return fail(NEGF_ERR_INVALID, "NULL diagonal output block");
        o.d.push_back(p);
        o.ldd.push_back(t.b[i]);
      }
      for (int i = 0; i + 1 < npl; ++i) {
        cplx* u = pick(Gu, (size_t)s * (npl - 1) + i, i, i + 1);
        cplx* l = pick(Gl, (size_t)s * (npl - 1) + i, i + 1, i);
        if (!u) u = plan.alloc_c((size_t)t.b[i] * t.b[i + 1]);
        if (!l) l = plan.alloc_c((size_t)t.b[i] * t.b[i + 1]);
        o.u.push_back(u); o.ldu.push_back(t.b[i]);
        o.l.push_back(l); o.ldl.push_back(t.b[i + 1]);
      }
      if (Gfull) {
        full[s].assign((size_t)npl * npl, nullptr);
        for (int i = 0; i < npl; ++i)
          for (int j = 0; j < npl; ++j)
            full[s][(size_t)i * npl + j] = static_cast<cplx*>(Gfull[(size_t)s * npl * npl + (size_t)i * npl + j]);
        for (int i = 0; i < npl; ++i) full[s][(size_t)i * npl + i] = o.d[i];
        for (int i = 0; i + 1 < npl; ++i) {
          full[s][(size_t)i * npl + i + 1] = o.u[i];
          full[s][(size_t)(i + 1) * npl + i] = o.l[i];
        }
      }
    }
    build_rgf_downward(plan, sys, work, out);
    if (Gfull) build_rgf_full_inverse(plan, sys, work, full);
    return run_plan_sync(plan, static_cast<cudaStream_t>(stream), dinfo, nsys, "negf_rgf");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_keldysh(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                 void* const* Ml, void* const* Sd, void* const* Su, void* stream) {
  if (int r = check_device()) return r;
  if (!Sd || (npl > 1 && !Su)) return fail(NEGF_ERR_INVALID, "Sd and Su are required");
  try {
    Plan plan;
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * nsys));
    std::vector<TriSystem> sys;
    if (int r = make_systems(nsys, npl, block_sizes, Md, Mu, Ml, dinfo, sys)) return r;
    std::vector<RgfWork> work(nsys);
    std::vector<HermBlocks> herm(nsys);
    for (int s = 0; s < nsys; ++s) {
      alloc_rgf_work(plan, sys[s], work[s]);
      for (int i = 0; i < npl; ++i) {
        herm[s].d.push_back(static_cast<cplx*>(Sd[(size_t)s * npl + i]));
        herm[s].ldd.push_back(sys[s].b[i]);
      }
      for (int i = 0; i + 1 < npl; ++i) {
        herm[s].u.push_back(static_cast<cplx*>(Su[(size_t)s * (npl - 1) + i]));
        herm[s].ldu.push_back(sys[s].b[i]);
      }
    }
    build_rgf_upward(plan, sys, work);
    build_rkd(plan, sys, work, herm);
    return run_plan_sync(plan, static_cast<cudaStream_t>(stream), dinfo, nsys, "negf_keldysh");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

// --- batched-energy NEGF solver ---------------------------------------------

int negf_device_create(int32_t npl, const int32_t* block_sizes, const void* const* Hd, const void* const* Hu,
                       const void* sigL, const void* sigR, negf_device_t* out) {
  if (int r = check_device()) return r;
  if (!out || npl <= 0 || !block_sizes || !Hd || (npl > 1 && !Hu) || !sigL || !sigR)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  std::unique_ptr<negf_device_s> d(new negf_device_s);
  d->npl = npl;
  d->b.assign(block_sizes, block_sizes + npl);
  for (int x : d->b)
    if (x <= 0 || x > kMaxBlock) return fail(NEGF_ERR_INVALID, "block sizes must be in [1, 1024]");
  auto dalloc = [&](size_t elems) -> cplx* {
    void* p = nullptr;
    if (cudaMalloc(&p, elems * sizeof(cplx)) != cudaSuccess) return nullptr;
    d->owned.push_back(p);
    return static_cast<cplx*>(p);
  };
  for (int i = 0; i < npl; ++i) {
    cplx* p = dalloc((size_t)d->b[i] * d->b[i]);
    if (!p) return fail(NEGF_ERR_NOMEM, "device allocation failed");
    d->D.push_back(p);
  }
  for (int i = 0; i + 1 < npl; ++i) {
    cplx* p = dalloc((size_t)d->b[i] * d->b[i + 1]);
    if (!p) return fail(NEGF_ERR_NOMEM, "device allocation failed");
    d->Hu.push_back(p);
  }
  const int b0 = d->b[0], bN = d->b[npl - 1];
  d->gamL = dalloc((size_t)b0 * b0);
  d->gamR = dalloc((size_t)bN * bN);
  d->sigL = dalloc((size_t)b0 * b0);
  d->sigR = dalloc((size_t)bN * bN);
  if (!d->gamL || !d->gamR || !d->sigL || !d->sigR) return fail(NEGF_ERR_NOMEM, "device allocation failed");
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(NEGF_ERR_CUDA, "stream creation failed");
  try {
    d->assemble.reset(new Plan);
    auto axpy = [](const cplx* A, cplx* C, int b) {
      ZBlockOp o{};
      o.A = A; o.lda = b; o.C = C; o.ldc = b; o.m = o.n = b; o.kind = ZOP_AXPBY;
      o.alpha = make_double2(1.0, 0.0); o.beta = make_double2(1.0, 0.0);
      return o;
    };
    auto gam = [](const cplx* A, cplx* C, int b) {
      ZBlockOp o{};
      o.A = A; o.lda = b; o.C = C; o.ldc = b; o.m = o.n = b; o.kind = ZOP_GAMMA;
      return o;
    };
    // two launches so that npl == 1 (both self-energies on one block) stays race-free
    d->assemble->blockops({axpy(d->sigL, d->D[0], b0), gam(d->sigL, d->gamL, b0), gam(d->sigR, d->gamR, bN)});
    d->assemble->blockops({axpy(d->sigR, d->D[npl - 1], bN)});
    if (d->assemble->finalize() != cudaSuccess) return fail(NEGF_ERR_CUDA, "device assembly plan");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
  negf_device_t h = d.release();
  return negf_device_upload(h, Hd, Hu, sigL, sigR) == NEGF_SUCCESS ? (*out = h, NEGF_SUCCESS)
                                                                   : (delete h, NEGF_ERR_CUDA);
}

int negf_device_set_overlap(negf_device_t d, const void* const* Sd, const void* const* Su) {
  if (!d) return fail(NEGF_ERR_INVALID, "NULL device");
  const int n = d->npl;
  auto dalloc = [&](size_t elems) -> cplx* {
    void* p = nullptr;
    if (cudaMalloc(&p, elems * sizeof(cplx)) != cudaSuccess) return nullptr;
    d->owned.push_back(p);
    return static_cast<cplx*>(p);
  };
  if (d->Sd.empty()) {
    for (int i = 0; i < n; ++i) {
      cplx* p = dalloc((size_t)d->b[i] * d->b[i]);
      if (!p) return fail(NEGF_ERR_NOMEM, "device allocation failed");
      d->Sd.push_back(p);
    }
    for (int i = 0; i + 1 < n; ++i) {
      cplx* p = dalloc((size_t)d->b[i] * d->b[i + 1]);
      if (!p) return fail(NEGF_ERR_NOMEM, "device allocation failed");
      d->Su.push_back(p);
    }
  }
  for (int i = 0; i < n; ++i) {
    const size_t cnt = (size_t)d->b[i] * d->b[i];
    if (Sd && Sd[i]) {
      NEGF_TRY_CUDA(cudaMemcpy(d->Sd[i], Sd[i], cnt * sizeof(cplx), cudaMemcpyHostToDevice), "set overlap");
    } else {
      std::vector<cplx> eye(cnt, make_double2(0.0, 0.0));
      for (int r = 0; r < d->b[i]; ++r) eye[r + (size_t)r * d->b[i]] = make_double2(1.0, 0.0);
      NEGF_TRY_CUDA(cudaMemcpy(d->Sd[i], eye.data(), cnt * sizeof(cplx), cudaMemcpyHostToDevice), "set overlap");
    }
  }
  for (int i = 0; i + 1 < n; ++i) {
    const size_t cnt = (size_t)d->b[i] * d->b[i + 1];
    if (Su && Su[i]) {
      NEGF_TRY_CUDA(cudaMemcpy(d->Su[i], Su[i], cnt * sizeof(cplx), cudaMemcpyHostToDevice), "set overlap");
    } else {
      NEGF_TRY_CUDA(cudaMemset(d->Su[i], 0, cnt * sizeof(cplx)), "set overlap");
    }
  }
  d->has_S = true;
  return NEGF_SUCCESS;
}

int negf_solver_set_self_energies(negf_solver_t s, const void* const* sigL, const void* const* sigR, void* stream) {
  if (!s || !sigL || !sigR) return fail(NEGF_ERR_INVALID, "bad arguments");
  if (!s->opts.sigma_per_energy)
    return fail(NEGF_ERR_INVALID, "the solver was not created with opts.sigma_per_energy");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int e = 0; e < s->nE; ++e) {
    if (!sigL[e] || !sigR[e]) return fail(NEGF_ERR_INVALID, "NULL self-energy block");
    NEGF_TRY_CUDA(cudaMemcpyAsync(s->sigL_e[e], sigL[e], sizeof(cplx) * s->bL_e[e] * s->bL_e[e],
                                  cudaMemcpyHostToDevice, st), "set self-energies");
    NEGF_TRY_CUDA(cudaMemcpyAsync(s->sigR_e[e], sigR[e], sizeof(cplx) * s->bR_e[e] * s->bR_e[e],
                                  cudaMemcpyHostToDevice, st), "set self-energies");
  }
  NEGF_TRY_CUDA(cudaStreamSynchronize(st), "set self-energies");
  return NEGF_SUCCESS;
}

int negf_device_upload(negf_device_t d, const void* const* Hd, const void* const* Hu, const void* sigL,
                       const void* sigR) {
  if (!d) return fail(NEGF_ERR_INVALID, "NULL device");
  const int n = d->npl;
  // copies straight from the caller's buffers (pinned ones go at full PCIe rate)
  for (int i = 0; i < n; ++i)
    NEGF_TRY_CUDA(cudaMemcpyAsync(d->D[i], Hd[i], (size_t)d->b[i] * d->b[i] * sizeof(cplx), cudaMemcpyHostToDevice,
                                  d->stream), "device upload");
  for (int i = 0; i + 1 < n; ++i)
    NEGF_TRY_CUDA(cudaMemcpyAsync(d->Hu[i], Hu[i], (size_t)d->b[i] * d->b[i + 1] * sizeof(cplx),
                                  cudaMemcpyHostToDevice, d->stream), "device upload");
  NEGF_TRY_CUDA(cudaMemcpyAsync(d->sigL, sigL, (size_t)d->b[0] * d->b[0] * sizeof(cplx), cudaMemcpyHostToDevice,
                                d->stream), "device upload");
  NEGF_TRY_CUDA(cudaMemcpyAsync(d->sigR, sigR, (size_t)d->b[n - 1] * d->b[n - 1] * sizeof(cplx),
                                cudaMemcpyHostToDevice, d->stream), "device upload");
  // device-side assembly: D_0 += Sigma_L, D_{N-1} += Sigma_R, Gamma = i (Sigma - Sigma^H)
  NEGF_TRY_CUDA(d->assemble->run(d->stream, false), "device upload");
  NEGF_TRY_CUDA(cudaStreamSynchronize(d->stream), "device upload");
  return NEGF_SUCCESS;
}

int negf_device_destroy(negf_device_t dev) {
  delete dev;
  return NEGF_SUCCESS;
}

int negf_solver_create(negf_device_t dev, int32_t nE, const negf_solve_opts* opts, negf_solver_t* out) {
  if (int r = check_device()) return r;
  if (!dev || nE <= 0 || !opts || !out) return fail(NEGF_ERR_INVALID, "bad arguments");
  std::unique_ptr<negf_solver_s> s(new negf_solver_s);
  s->dev = dev;
  s->devs = {dev};
  s->dev_nE = {nE};
  s->nE = nE;
  s->opts = *opts;
  s->plan.reset(new Plan);
  try {
    if (int r = build_solver(*s)) return r;
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed (reduce the number of energies per batch)");
  }
  *out = s.release();
  return NEGF_SUCCESS;
}

int negf_solver_create_batch(int32_t ndev, const negf_device_t* devs, const int32_t* nE,
                             const negf_solve_opts* opts, negf_solver_t* out) {
  if (int r = check_device()) return r;
  if (ndev <= 0 || !devs || !nE || !opts || !out) return fail(NEGF_ERR_INVALID, "bad arguments");
  std::unique_ptr<negf_solver_s> s(new negf_solver_s);
  for (int k = 0; k < ndev; ++k) {
    if (!devs[k] || nE[k] <= 0) return fail(NEGF_ERR_INVALID, "every device needs a handle and nE > 0");
    s->devs.push_back(devs[k]);
    s->dev_nE.push_back(nE[k]);
    s->nE += nE[k];
  }
  s->dev = devs[0];
  s->opts = *opts;
  s->plan.reset(new Plan);
  try {
    if (int r = build_solver(*s)) return r;
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed (split the batch)");
  }
  *out = s.release();
  return NEGF_SUCCESS;
}

int negf_batch_bytes(int32_t ndev, const negf_device_t* devs, const int32_t* nE, const negf_solve_opts* opts,
                     int64_t* bytes) {
  if (ndev < 0 || (ndev > 0 && (!devs || !nE)) || !opts || !bytes) return fail(NEGF_ERR_INVALID, "bad arguments");
  size_t total = 0;
  for (int k = 0; k < ndev; ++k) {
    if (!devs[k] || nE[k] < 0) return fail(NEGF_ERR_INVALID, "bad device or energy count");
    total += (size_t)nE[k] * solver_bytes_per_energy(*devs[k], *opts);
  }
  *bytes = (int64_t)total;
  return NEGF_SUCCESS;
}

int negf_solver_destroy(negf_solver_t s) {
  delete s;
  return NEGF_SUCCESS;
}

int negf_solver_set_energies(negf_solver_t s, const double* energies, void* stream) {
  if (!s || !energies) return fail(NEGF_ERR_INVALID, "bad arguments");
  const int nE = s->nE;
  std::vector<cplx> p(3 * (size_t)nE);
  const negf_solve_opts& o = s->opts;
  for (int e = 0; e < nE; ++e) {
    double E = energies[e];
    p[e] = make_double2(E, o.eta);
    p[nE + e] = make_double2(1.0 / (1.0 + std::exp((E - o.mu_l) / o.kT)), 0.0);
    p[2 * nE + e] = make_double2(1.0 / (1.0 + std::exp((E - o.mu_r) / o.kT)), 0.0);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NEGF_TRY_CUDA(cudaMemcpyAsync(s->params, p.data(), p.size() * sizeof(cplx), cudaMemcpyHostToDevice, st),
                "set energies");
  NEGF_TRY_CUDA(cudaMemsetAsync(s->info, 0, sizeof(int) * nE, st), "set energies");
  s->plan->fence(st);
  return NEGF_SUCCESS;
}

int negf_solver_run(negf_solver_t s, void* stream) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  // the legacy NULL stream cannot be captured: replay the launches directly there
  cudaError_t e = s->plan->run(static_cast<cudaStream_t>(stream), stream != nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "negf_solver_run");
  return NEGF_SUCCESS;
}

extern "C++" {
namespace negf {
// One pass launch by launch on `stream` (no graph capture: for one-off plans
// such as a server group's).
int solver_run_direct(negf_solver_s* s, cudaStream_t stream) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  cudaError_t e = s->plan->run(stream, false);
  if (e != cudaSuccess) return cuda_fail(e, "negf_solver_run");
  return NEGF_SUCCESS;
}
}  // namespace negf
}  // extern "C++"

int negf_solver_run_profiled(negf_solver_t s, void* stream) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  const size_t need = s->plan->steps.size() + 1;
  if (s->ev_used == s->ev_sets.size()) {
    std::vector<cudaEvent_t> v(need);
    for (auto& e : v) NEGF_TRY_CUDA(cudaEventCreate(&e), "profiled run");
    s->ev_sets.push_back(std::move(v));
  }
  cudaError_t e = s->plan->run_events(static_cast<cudaStream_t>(stream), s->ev_sets[s->ev_used]);
  if (e != cudaSuccess) return cuda_fail(e, "negf_solver_run_profiled");
  ++s->ev_used;
  return NEGF_SUCCESS;
}

int negf_solver_profile_read(negf_solver_t s, double* ms, double* flops, int64_t* launches, int32_t reset) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  const int K = NEGF_PROFILE_KINDS;
  std::vector<double> t(K, 0.0), f(K, 0.0);
  std::vector<int64_t> n(K, 0);
  const auto& steps = s->plan->steps;
  for (size_t p = 0; p < s->ev_used; ++p) {
    const auto& ev = s->ev_sets[p];
    NEGF_TRY_CUDA(cudaEventSynchronize(ev.back()), "profile read");
    for (size_t i = 0; i < steps.size(); ++i) {
      float x = 0.f;
      NEGF_TRY_CUDA(cudaEventElapsedTime(&x, ev[i], ev[i + 1]), "profile read");
      int k = static_cast<int>(steps[i].kind);
      t[k] += x;
      // kind 8: algorithmic bytes; kind 9: INT8 operations, 3 real products
      // x digit pairs x 2mnk per complex product (8mnk flops)
      f[k] += steps[i].kind == Step::OZ_SPLIT  ? steps[i].bytes
              : steps[i].kind == Step::OZ_MMA ? steps[i].flops * (6.0 * steps[i].form / 8.0)
                                              : steps[i].flops;
      n[k] += 1;
    }
  }
  for (int k = 0; k < K; ++k) {
    if (ms) ms[k] = t[k];
    if (flops) flops[k] = f[k];
    if (launches) launches[k] = n[k];
  }
  if (reset) s->ev_used = 0;
  return NEGF_SUCCESS;
}

int negf_solver_download(negf_solver_t s, void* gr_host, void* gl_host, double* t_host, void* stream) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t bytes = s->out_total * sizeof(cplx);
  if (gr_host && s->gr) NEGF_TRY_CUDA(cudaMemcpyAsync(gr_host, s->gr, bytes, cudaMemcpyDeviceToHost, st), "download");
  if (gl_host && s->gl) NEGF_TRY_CUDA(cudaMemcpyAsync(gl_host, s->gl, bytes, cudaMemcpyDeviceToHost, st), "download");
  if (t_host && s->t2)
    NEGF_TRY_CUDA(cudaMemcpyAsync(t_host, s->t2, 2 * sizeof(double) * s->nE, cudaMemcpyDeviceToHost, st), "download");
  NEGF_TRY_CUDA(cudaStreamSynchronize(st), "download");
  return NEGF_SUCCESS;
}

int negf_solver_run_download(negf_solver_t s, void* gr_host, void* gl_host, double* t_host, void* stream) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // copies into pageable memory would block the host between launches: then
  // run the pass and download after it
  auto pinned = [](const void* p) {
    cudaPointerAttributes a{};
    return p == nullptr || (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost);
  };
  if (!pinned(gr_host) || !pinned(gl_host)) {
    cudaGetLastError();  // clear a lookup error of an unregistered pointer
    if (int r = negf_solver_run(s, stream)) return r;
    if (int r = negf_solver_download(s, gr_host, gl_host, t_host, stream)) return r;
    return negf_solver_check(s);
  }
  if (!s->copy_stream) {
    NEGF_TRY_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking), "run_download");
    NEGF_TRY_CUDA(cudaEventCreateWithFlags(&s->mark_ev, cudaEventDisableTiming), "run_download");
    NEGF_TRY_CUDA(cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming), "run_download");
  }
  // energies are device-major: one pitched copy per (device group, layer)
  struct Group { const negf_device_s* d; size_t base, per; int count; std::vector<size_t> off; };
  std::vector<Group> groups;
  {
    size_t base = 0;
    for (size_t k = 0; k < s->devs.size(); ++k) {
      Group g{s->devs[k], base, 0, s->dev_nE[k], {}};
      for (int x : g.d->b) { g.off.push_back(g.per); g.per += (size_t)x * x; }
      base += g.per * (size_t)g.count;
      if (g.count > 0) groups.push_back(std::move(g));
    }
  }
  auto at_mark = [&](int tag) -> cudaError_t {
    const bool gl = tag >= kMarkGL;
    const int layer = gl ? tag - kMarkGL : tag - kMarkGR;
    char* host = static_cast<char*>(gl ? gl_host : gr_host);
    const cplx* dev = gl ? s->gl : s->gr;
    if (!host || !dev) return cudaSuccess;
    cudaError_t e = cudaEventRecord(s->mark_ev, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_stream, s->mark_ev, 0);
    for (const Group& g : groups) {
      if (e != cudaSuccess || layer >= g.d->npl) continue;
      const size_t o = (g.base + g.off[layer]) * sizeof(cplx), pitch = g.per * sizeof(cplx);
      const size_t width = (size_t)g.d->b[layer] * g.d->b[layer] * sizeof(cplx);
      e = cudaMemcpy2DAsync(host + o, pitch, reinterpret_cast<const char*>(dev) + o, pitch, width, g.count,
                            cudaMemcpyDeviceToHost, s->copy_stream);
    }
    return e;
  };
  NEGF_TRY_CUDA(s->plan->run_marked(st, at_mark), "run_download");
  if (t_host && s->t2)
    NEGF_TRY_CUDA(cudaMemcpyAsync(t_host, s->t2, 2 * sizeof(double) * s->nE, cudaMemcpyDeviceToHost, st),
                  "run_download");
  NEGF_TRY_CUDA(cudaEventRecord(s->join_ev, s->copy_stream), "run_download");
  NEGF_TRY_CUDA(cudaStreamWaitEvent(st, s->join_ev, 0), "run_download");
  NEGF_TRY_CUDA(cudaStreamSynchronize(st), "run_download");
  return negf_solver_check(s);
}

int negf_solver_outputs(negf_solver_t s, void** gr_dev, void** gl_dev, double** t_dev) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  if (gr_dev) *gr_dev = s->gr;
  if (gl_dev) *gl_dev = s->gl;
  if (t_dev) *t_dev = s->t2;
  return NEGF_SUCCESS;
}

int negf_solver_stats(negf_solver_t s, double* flops, int64_t* launches, int64_t* workspace_bytes) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  if (flops) *flops = s->plan->flops();
  if (launches) *launches = (int64_t)s->plan->num_launches();
  if (workspace_bytes) *workspace_bytes = (int64_t)s->plan->workspace_bytes();
  return NEGF_SUCCESS;
}

int negf_solver_check(negf_solver_t s) {
  if (!s) return fail(NEGF_ERR_INVALID, "NULL solver");
  std::vector<int> h(s->nE);
  NEGF_TRY_CUDA(cudaMemcpy(h.data(), s->info, sizeof(int) * s->nE, cudaMemcpyDeviceToHost), "solver check");
  if (s->plan->error_flag()) {
    int fl = 0;
    NEGF_TRY_CUDA(cudaMemcpy(&fl, s->plan->error_flag(), sizeof(int), cudaMemcpyDeviceToHost), "solver check");
    if (fl) return fail(NEGF_ERR_TIMEOUT, "tensor-core completion wait timed out in the mixed-precision products");
  }
  for (int e = 0; e < s->nE; ++e)
    if (h[e]) {
      char buf[128];
      std::snprintf(buf, sizeof buf, "energy %d: zero pivot (column %d of a diagonal block)", e, h[e]);
      return fail(NEGF_ERR_SINGULAR, buf);
    }
  return NEGF_SUCCESS;
}

int negf_solve(negf_device_t dev, int32_t nE, const double* energies, const negf_solve_opts* opts, void* gr_out,
               void* gl_out, double* t_out, int32_t out_on_device, void* stream) {
  if (opts && opts->sigma_per_energy)
    return fail(NEGF_ERR_INVALID, "negf_solve has no per-energy self-energies; use a solver and "
                                  "negf_solver_set_self_energies");
  if (int r = check_device()) return r;
  if (!dev || nE <= 0 || !energies || !opts) return fail(NEGF_ERR_INVALID, "bad arguments");
  negf_solve_opts o = *opts;
  o.want_gr = gr_out != nullptr;
  o.want_gl = gl_out != nullptr;
  o.want_t = t_out != nullptr;
  int chunk = o.max_chunk > 0 ? std::min(o.max_chunk, nE) : nE;
  if (o.max_chunk <= 0) {
    size_t fr = 0, tot = 0;
    NEGF_TRY_CUDA(cudaMemGetInfo(&fr, &tot), "negf_solve");
    { int d = 0; cudaGetDevice(&d); fr += cached_bytes(d); }  // the library's cached chunks are free to it
    double budget = o.hbm_budget_gb > 0 ? o.hbm_budget_gb * 1e9 : 0.8 * (double)fr;
    size_t per = solver_bytes_per_energy(*dev, o);
    int fit = (int)std::max(1.0, std::floor(budget / (double)per));
    chunk = std::min(nE, fit);
  }
  negf_solver_t s = nullptr;
  if (int r = negf_solver_create(dev, chunk, &o, &s)) return r;
  std::unique_ptr<negf_solver_s> guard(s);
  cudaStream_t own = nullptr;
  if (!stream) {
    NEGF_TRY_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "negf_solve");
    stream = own;
  }
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { if (s) cudaStreamDestroy(s); }
  } sg{own};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t per = s->per_energy;
  std::vector<double> eb(chunk);
  std::vector<double> t2(2 * (size_t)chunk);
  cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int e0 = 0; e0 < nE; e0 += chunk) {
    int cnt = std::min(chunk, nE - e0);
    for (int e = 0; e < chunk; ++e) eb[e] = energies[e0 + std::min(e, cnt - 1)];
    if (int r = negf_solver_set_energies(s, eb.data(), stream)) return r;
    if (!out_on_device && cnt == chunk) {
      // host outputs of a full chunk: downloads overlap the pass
      if (int r = negf_solver_run_download(s, gr_out ? static_cast<cplx*>(gr_out) + (size_t)e0 * per : nullptr,
                                           gl_out ? static_cast<cplx*>(gl_out) + (size_t)e0 * per : nullptr,
                                           t_out ? t2.data() : nullptr, stream))
        return r;
      if (t_out)
        for (int e = 0; e < cnt; ++e) t_out[e0 + e] = t2[2 * e];
      continue;
    }
    if (int r = negf_solver_run(s, stream)) return r;
    if (gr_out)
      NEGF_TRY_CUDA(cudaMemcpyAsync(static_cast<cplx*>(gr_out) + (size_t)e0 * per, s->gr, (size_t)cnt * per * sizeof(cplx),
                                    kind, st), "negf_solve output");
    if (gl_out)
      NEGF_TRY_CUDA(cudaMemcpyAsync(static_cast<cplx*>(gl_out) + (size_t)e0 * per, s->gl, (size_t)cnt * per * sizeof(cplx),
                                    kind, st), "negf_solve output");
    if (t_out) {
      NEGF_TRY_CUDA(cudaMemcpyAsync(t2.data(), s->t2, 2 * (size_t)cnt * sizeof(double), cudaMemcpyDeviceToHost, st),
                    "negf_solve output");
    }
    NEGF_TRY_CUDA(cudaStreamSynchronize(st), "negf_solve");
    if (int r = negf_solver_check(s)) return r;
    if (t_out) {
      if (out_on_device) {
        std::vector<double> tr(cnt);
        for (int e = 0; e < cnt; ++e) tr[e] = t2[2 * e];
        NEGF_TRY_CUDA(cudaMemcpy(t_out + e0, tr.data(), cnt * sizeof(double), cudaMemcpyHostToDevice), "negf_solve");
      } else {
        for (int e = 0; e < cnt; ++e) t_out[e0 + e] = t2[2 * e];
      }
    }
  }
  return NEGF_SUCCESS;
}

// Selected inverse of M(E) for a list of energies (the batched form of one
// bndiag_of_inv_rgf_local! / bndiag_of_inv_ddrgf! / Block_factorization! +
// Block_inverse! call per energy point).
namespace {

// Device bytes of one energy of negf_device_selected_inverse (inputs,
// workspace, device outputs of a host-output call, digit slices).
size_t selinv_bytes_per_energy(const negf_device_s& d, int method, int d1, bool mixed, bool host_out) {
  const size_t n = d.npl;
  size_t mb = 0, sd = 0, su = 0;
  for (int x : d.b) { mb = std::max<size_t>(mb, x); sd += (size_t)x * x; }
  for (size_t i = 0; i + 1 < n; ++i) su += (size_t)d.b[i] * d.b[i + 1];
  size_t c = sd + (d.has_S ? 2 * su : 0);                  // M(E) diagonal (+ off-diagonal) blocks
  if (host_out || method == 2) c += sd + 2 * su;            // output blocks (in place for method 2)
  size_t ops = 3;                                           // operands per layer of the widest mixed step
  if (method == 0) {
    c += sd + 2 * su + mb * mb + 64 * mb;                   // RGF work
  } else if (method == 1) {
    const size_t D1 = (size_t)std::max(1, d1);
    c += sd + 2 * su + mb * mb + 64 * mb;                   // domain RGF work
    c += D1 * sd;                                           // domain full inverses: D1 blocks per layer
    c += 10 * sd;                                           // Schur complement and 12 / 21 / 11 temporaries
    ops = 6;
  } else {
    c += 2 * sd + (2 * n + 2) * mb * mb + 64 * mb * n;      // factor inverses, scratch, LU / trtri scratch
  }
  size_t bytes = c * sizeof(cplx) + 64 * n;
  if (mixed) {
    const size_t pad = (mb + 127) / 128 * 128;
    bytes += 21 * ops * n * pad * pad;
  }
  return bytes;
}

}  // namespace

int negf_device_selected_inverse(negf_device_t dev, int32_t nE, const double* energies, const negf_solve_opts* opts,
                                 int32_t method, int32_t nlevels, const int32_t* block_size_d1, void* gd_out,
                                 void* gu_out, void* gl_out, int32_t out_on_device, void* stream) {
  if (int r = check_device()) return r;
  if (!dev || nE <= 0 || !energies || !opts || method < 0 || method > 2 || nlevels < 0 ||
      nlevels > NEGF_DDRGF_MAX_LEVELS || (nlevels > 0 && !block_size_d1) ||
      (opts->precision != NEGF_PREC_FP64 && opts->precision != NEGF_PREC_MIXED) || opts->gj_update < 0 ||
      opts->gj_update > 2)
    return fail(NEGF_ERR_INVALID, "negf_device_selected_inverse: bad arguments");
  if (opts->sigma_per_energy)
    return fail(NEGF_ERR_INVALID, "negf_device_selected_inverse: the device's constant self-energies are used");
  const negf_device_s& d = *dev;
  const int n = d.npl;
  int mb = 0;
  for (int x : d.b) mb = std::max(mb, x);
  if (method == 2)
    for (int x : d.b)
      if (x != d.b[0]) return fail(NEGF_ERR_INVALID, "negf_device_selected_inverse: the block selected inverse "
                                                     "needs one block size");
  std::vector<size_t> od(n), ou(std::max(n - 1, 0));
  size_t sd = 0, su = 0;
  for (int i = 0; i < n; ++i) { od[i] = sd; sd += (size_t)d.b[i] * d.b[i]; }
  for (int i = 0; i + 1 < n; ++i) { ou[i] = su; su += (size_t)d.b[i] * d.b[i + 1]; }
  const bool mixed = opts->precision == NEGF_PREC_MIXED;
  std::vector<int> fixed_d1s;
  if (nlevels > 0) {
    fixed_d1s.assign(block_size_d1, block_size_d1 + nlevels);
    for (int x : fixed_d1s)
      if (x <= 0) return fail(NEGF_ERR_INVALID, "negf_device_selected_inverse: interior sizes must be positive");
  }
  int chunk = opts->max_chunk > 0 ? std::min<int>(opts->max_chunk, nE) : nE;
  if (opts->max_chunk <= 0) {
    size_t fr = 0, tot = 0;
    NEGF_TRY_CUDA(cudaMemGetInfo(&fr, &tot), "negf_device_selected_inverse");
    { int d = 0; cudaGetDevice(&d); fr += cached_bytes(d); }
    const double budget = opts->hbm_budget_gb > 0 ? opts->hbm_budget_gb * 1e9 : 0.8 * (double)fr;
    const int d1 = nlevels > 0 ? fixed_d1s[0] : 16;
    const size_t per = selinv_bytes_per_energy(d, method, d1, mixed, !out_on_device);
    chunk = std::min<int>(nE, (int)std::max(1.0, std::floor(budget / (double)per)));
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const cudaMemcpyKind kind = cudaMemcpyDeviceToHost;
  static constexpr cplx ONE{1.0, 0.0}, MONE{-1.0, 0.0}, ZERO{0.0, 0.0};
  auto kzero = [](cplx* C, int ldc, int m, int nn, const cplx* Cin, cplx beta, cplx diag) {
    ZGemmProblem p{};
    p.C = C; p.Cin = Cin; p.m = m; p.n = nn; p.k = 0;
    p.lda = p.ldb = 1; p.ldc = ldc; p.ldcin = ldc;
    p.alpha = ZERO; p.beta = beta; p.diag = diag;
    return p;
  };
  auto bop = [](int kindop, const cplx* A, int lda, cplx* C, int ldc, int m, int nn, cplx alpha, cplx beta) {
    ZBlockOp o{};
    o.A = A; o.lda = lda; o.C = C; o.ldc = ldc; o.m = m; o.n = nn; o.kind = kindop; o.alpha = alpha; o.beta = beta;
    return o;
  };
  for (int e0 = 0; e0 < nE;) {
    const int cnt = std::min(chunk, nE - e0);
    try {
      Plan plan;
      // DDRGF's interior-domain inverses and the block LU amplify product
      // errors more than RGF does: FP64-grade products (34 digit pairs) there
      plan.set_mixed(mixed, method == 0 ? 28 : 34);
      plan.set_schedule(opts->gemm_form, opts->gj_nb);
      plan.set_gj_update(opts->gj_update);
      int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * (size_t)cnt * n));
      // output blocks of this chunk: the caller's device buffers, or plan memory
      // downloaded afterwards (every sweep writes all three kinds)
      auto out_base = [&](void* user, size_t per) -> cplx* {
        if (user && out_on_device) return static_cast<cplx*>(user) + (size_t)e0 * per;
        return plan.alloc_c((size_t)cnt * std::max<size_t>(per, 1));
      };
      cplx* GD = out_base(gd_out, sd);
      cplx* GU = (n > 1) ? out_base(gu_out, su) : nullptr;
      cplx* GL = (n > 1) ? out_base(gl_out, su) : nullptr;
      // M(E) = (E + i eta) S - H - Sigma: diagonal blocks per energy; the
      // off-diagonal blocks are shared by all energies unless S couples layers
      std::vector<ZGemmProblem> asm_g;
      std::vector<ZBlockOp> asm_o1, asm_o2;
      std::vector<cplx*> Mu_sh(std::max(n - 1, 0)), Ml_sh(std::max(n - 1, 0));
      if (!d.has_S && method != 2)
        for (int i = 0; i + 1 < n; ++i) {
          Mu_sh[i] = plan.alloc_c((size_t)d.b[i] * d.b[i + 1]);
          Ml_sh[i] = plan.alloc_c((size_t)d.b[i] * d.b[i + 1]);
          asm_g.push_back(kzero(Mu_sh[i], d.b[i], d.b[i], d.b[i + 1], d.Hu[i], MONE, ZERO));
          asm_o1.push_back(bop(ZOP_CTRANS_AXPBY, d.Hu[i], d.b[i], Ml_sh[i], d.b[i + 1], d.b[i + 1], d.b[i], MONE, ZERO));
        }
      std::vector<TriSystem> sys(cnt);
      std::vector<TriOut> out(cnt);
      std::vector<SelInvSystem> ssys(method == 2 ? cnt : 0);
      for (int e = 0; e < cnt; ++e) {
        const cplx z = make_double2(energies[e0 + e], opts->eta);
        TriSystem& ts = sys[e];
        TriOut& o = out[e];
        ts.info = dinfo + (size_t)e * n;
        std::vector<cplx*> Md(n), Mu(std::max(n - 1, 0)), Ml(std::max(n - 1, 0));
        for (int i = 0; i < n; ++i) {
          const int bi = d.b[i];
          Md[i] = method == 2 ? GD + (size_t)e * sd + od[i] : plan.alloc_c((size_t)bi * bi);
          asm_g.push_back(kzero(Md[i], bi, bi, bi, d.D[i], MONE, d.has_S ? ZERO : z));
          if (d.has_S) asm_o1.push_back(bop(ZOP_AXPBY, d.Sd[i], bi, Md[i], bi, bi, bi, z, ONE));
        }
        for (int i = 0; i + 1 < n; ++i) {
          const int bi = d.b[i], bj = d.b[i + 1];
          if (method == 2) {
            Mu[i] = GU + (size_t)e * su + ou[i];
            Ml[i] = GL + (size_t)e * su + ou[i];
          } else if (d.has_S) {
            Mu[i] = plan.alloc_c((size_t)bi * bj);
            Ml[i] = plan.alloc_c((size_t)bi * bj);
          } else {
            Mu[i] = Mu_sh[i];
            Ml[i] = Ml_sh[i];
          }
          if (method == 2 || d.has_S) {
            asm_g.push_back(kzero(Mu[i], bi, bi, bj, d.Hu[i], MONE, ZERO));
            asm_o1.push_back(bop(ZOP_CTRANS_AXPBY, d.Hu[i], bi, Ml[i], bj, bj, bi, MONE, ZERO));
            if (d.has_S) {
              asm_o2.push_back(bop(ZOP_AXPBY, d.Su[i], bi, Mu[i], bi, bi, bj, z, ONE));
              asm_o2.push_back(bop(ZOP_CTRANS_AXPBY, d.Su[i], bi, Ml[i], bj, bj, bi, z, ONE));
            }
          }
        }
        if (method == 2) {
          SelInvSystem& ss = ssys[e];
          ss.A.assign((size_t)n * n, nullptr);
          ss.info = ts.info;
          for (int i = 0; i < n; ++i) ss.A[(size_t)i * n + i] = Md[i];
          for (int i = 0; i + 1 < n; ++i) {
            ss.A[(size_t)i * n + i + 1] = Mu[i];
            ss.A[(size_t)(i + 1) * n + i] = Ml[i];
          }
          continue;
        }
        for (int i = 0; i < n; ++i) {
          ts.b.push_back(d.b[i]);
          ts.D.push_back(Md[i]); ts.ldD.push_back(d.b[i]);
          o.d.push_back(GD + (size_t)e * sd + od[i]); o.ldd.push_back(d.b[i]);
        }
        for (int i = 0; i + 1 < n; ++i) {
          ts.U.push_back(Mu[i]); ts.ldU.push_back(d.b[i]);
          ts.Lw.push_back(Ml[i]); ts.ldL.push_back(d.b[i + 1]);
          o.u.push_back(GU + (size_t)e * su + ou[i]); o.ldu.push_back(d.b[i]);
          o.l.push_back(GL + (size_t)e * su + ou[i]); o.ldl.push_back(d.b[i + 1]);
        }
      }
      plan.gemm_fp64('N', 'N', asm_g);  // k = 0: C = -Cin (+ z I)
      plan.blockops(asm_o1);
      plan.blockops(asm_o2);
      if (method == 0) {
        std::vector<RgfWork> w(cnt);
        for (int e = 0; e < cnt; ++e) alloc_rgf_work(plan, sys[e], w[e]);
        build_rgf_upward(plan, sys, w);
        build_rgf_downward(plan, sys, w, out);
      } else if (method == 1) {
        const std::vector<int> d1s = nlevels > 0 ? fixed_d1s : choose_levels(n, mb, cnt, NEGF_DDRGF_MAX_LEVELS);
        if (int r = build_ddrgf_level(plan, sys, out, d1s, 0)) return r;
      } else {
        if (int r = build_selected_inverse(plan, ssys, n, d.b[0], 3, true)) return r;
      }
      NEGF_TRY_CUDA(plan.run(st, false), "negf_device_selected_inverse");
      if (!out_on_device) {
        if (gd_out)
          NEGF_TRY_CUDA(cudaMemcpyAsync(static_cast<cplx*>(gd_out) + (size_t)e0 * sd, GD, (size_t)cnt * sd * sizeof(cplx),
                                        kind, st), "negf_device_selected_inverse output");
        if (gu_out && n > 1)
          NEGF_TRY_CUDA(cudaMemcpyAsync(static_cast<cplx*>(gu_out) + (size_t)e0 * su, GU, (size_t)cnt * su * sizeof(cplx),
                                        kind, st), "negf_device_selected_inverse output");
        if (gl_out && n > 1)
          NEGF_TRY_CUDA(cudaMemcpyAsync(static_cast<cplx*>(gl_out) + (size_t)e0 * su, GL, (size_t)cnt * su * sizeof(cplx),
                                        kind, st), "negf_device_selected_inverse output");
      }
      NEGF_TRY_CUDA(cudaStreamSynchronize(st), "negf_device_selected_inverse");
      if (plan.error_flag()) {
        int h = 0;
        NEGF_TRY_CUDA(cudaMemcpy(&h, plan.error_flag(), sizeof(int), cudaMemcpyDeviceToHost), "negf_device_selected_inverse");
        if (h) return fail(NEGF_ERR_TIMEOUT, "negf_device_selected_inverse: a tensor-core wait timed out");
      }
      std::vector<int> info((size_t)cnt * n);
      NEGF_TRY_CUDA(cudaMemcpy(info.data(), dinfo, sizeof(int) * info.size(), cudaMemcpyDeviceToHost),
                    "negf_device_selected_inverse");
      for (int e = 0; e < cnt; ++e)
        for (int i = 0; i < n; ++i)
          if (info[(size_t)e * n + i]) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "negf_device_selected_inverse: energy %d is singular (block %d)", e0 + e, i);
            return fail(NEGF_ERR_SINGULAR, buf);
          }
    } catch (const std::bad_alloc&) {
      if (chunk == 1) return fail(NEGF_ERR_NOMEM, "negf_device_selected_inverse: device allocation failed");
      chunk = std::max(1, chunk / 2);  // retry this chunk with half as many energies
      continue;
    }
    e0 += cnt;
  }
  return NEGF_SUCCESS;
}

int negf_probe_fp64_peak(double* dmma_tflops, double* dfma_tflops) {
  if (int r = check_device()) return r;
  int dev = 0, sms = 0;
  NEGF_TRY_CUDA(cudaGetDevice(&dev), "probe");
  NEGF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "probe");
  const int blocks = sms * 4, threads = 256, iters = 20000;
  double* out = nullptr;
  NEGF_TRY_CUDA(cudaMalloc(&out, sizeof(double) * blocks * threads), "probe");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float ms = 0.f;
  probe_dmma<<<blocks, threads>>>(out, 100);
  cudaEventRecord(a);
  probe_dmma<<<blocks, threads>>>(out, iters);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  if (dmma_tflops) *dmma_tflops = 2.0 * 16 * 8 * 4 * 2.0 * iters * blocks * (threads / 32) / (ms * 1e9);
  probe_dfma<<<blocks, threads>>>(out, 100);
  cudaEventRecord(a);
  probe_dfma<<<blocks, threads>>>(out, iters);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  if (dfma_tflops) *dfma_tflops = 2.0 * 8 * iters * (double)blocks * threads / (ms * 1e9);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaError_t e = cudaGetLastError();
  cudaFree(out);
  if (e != cudaSuccess) return cuda_fail(e, "probe");
  return NEGF_SUCCESS;
}

int negf_release_cached_memory(void) {
  negf::release_cached_memory();
  return NEGF_SUCCESS;
}

int negf_probe_int8_peak(double* tops) {
  if (int r = check_device()) return r;
  cudaError_t e = ozaki_probe_int8(tops);
  if (e != cudaSuccess) return cuda_fail(e, "int8 probe");
  return NEGF_SUCCESS;
}

int negf_probe_fp64_int8_overlap(double* fp64_alone_cycles, double* fp64_beside_mma_cycles, double* mma_cycles) {
  if (int r = check_device()) return r;
  cudaError_t e = ozaki_probe_overlap(fp64_alone_cycles, fp64_beside_mma_cycles, mma_cycles);
  if (e != cudaSuccess) return cuda_fail(e, "overlap probe");
  return NEGF_SUCCESS;
}

}  // extern "C"
