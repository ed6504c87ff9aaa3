// Batched block inversion that allocates no device memory.
//
// negf_zinv_batched (negf_api.cu) takes its scratch -- a working copy of each
// block, the rank-nb update buffers, pivot rows, flags and the launch
// descriptors -- from cudaMalloc.  Some callers cannot allow that: an
// application that hands out all device memory from its own pool (a Julia or
// Python framework allocator, a fixed arena in a long-running solver service)
// must not see side allocations, and cudaMalloc / cudaFree synchronise the
// device, which a latency-sensitive loop cannot afford.  This entry point runs
// the same kernels with all scratch placed in one file-scope __device__ array
// of fixed size; the caller still passes the input and output blocks.
//
// Properties (also stated in include/negf_b200.h):
//  * every GPU that loads the library reserves kNoAllocScratchBytes (64 MiB)
//    for the array until the process exits;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and raises the kernels'
//    shared-memory limits; make that first call before any stream capture;
//  * all calls share the array: calls that overlap on the GPU (other streams,
//    other host threads on the same device) race on it; consecutive calls on
//    one stream are safe, each call clears what must start at zero;
//  * requests whose scratch does not fit are rejected with NEGF_ERR_INVALID.
#include "../../include/negf_b200.h"
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

namespace negf {
cudaError_t zgj_prepare(size_t smem);  // zinv.cu
}

using namespace negf;

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;

// The scratch array.  In host code this name is a host-side stand-in, not a
// device address: host code only ever uses the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 128;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(NEGF_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Once per device, with that device current: the device address of the
// scratch array and the kernels' dynamic shared-memory limits.
int setup_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(NEGF_ERR_INVALID, "negf_zinv_batched_noalloc: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e, "negf_zinv_batched_noalloc: cudaGetSymbolAddress");
    e = zgemm_prepare('N', 'N');
    if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: GEMM kernel attributes");
    e = zgj_prepare(zgj_panel_smem_bytes(112, 112));
    if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: panel kernel attributes");
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return NEGF_SUCCESS;
}

// Bump layout inside the scratch array (256-byte aligned pieces).
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = (off + 255) & ~size_t(255);
    off = o + bytes;
    return o;
  }
};

}  // namespace

extern "C" int negf_zinv_batched_noalloc(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda,
                                         void* const* Ainv, const int32_t* ldainv, int32_t* info, void* stream) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(NEGF_ERR_CUDA, "negf_zinv_batched_noalloc: no usable CUDA device");
  if (nprob < 0 || (nprob > 0 && (!n || !A || !lda || !Ainv || !ldainv)))
    return fail(NEGF_ERR_INVALID, "negf_zinv_batched_noalloc: bad arguments");
  if (nprob == 0) return NEGF_SUCCESS;
  int max_n = 0;
  for (int i = 0; i < nprob; ++i) {
    if (n[i] < 0 || n[i] > kMaxBlock) return fail(NEGF_ERR_INVALID, "negf_zinv_batched_noalloc: n must be in [0, 1024]");
    max_n = std::max(max_n, n[i]);
  }
  if (max_n == 0) return NEGF_SUCCESS;
  const int nb = gj_panel_width(max_n);
  const bool blocked = nb < max_n;
  const int npanels = blocked ? (max_n + nb - 1) / nb : 1;

  // scratch layout (sizes only; the device address is known after set-up)
  Layout L;
  const size_t o_info = L.take(sizeof(int) * nprob);
  std::vector<size_t> o_W(nprob), o_F(nprob), o_B(nprob), o_used(nprob), o_piv(nprob);
  for (int i = 0; i < nprob; ++i) {
    const size_t m = (size_t)std::max(n[i], 1);
    o_W[i] = L.take(m * m * sizeof(cplx));
    o_F[i] = L.take(m * nb * sizeof(cplx));
    o_B[i] = L.take(m * nb * sizeof(cplx));
    o_used[i] = L.take(m);
    o_piv[i] = L.take(m * sizeof(int));
  }
  const size_t o_ops = L.take(sizeof(ZBlockOp) * nprob);
  const size_t o_inv = L.take(sizeof(ZInvProblem) * nprob);
  std::vector<size_t> o_gp(npanels), o_ts(npanels);
  for (int p = 0; p < npanels; ++p) {
    o_gp[p] = L.take(sizeof(ZGemmProblem) * nprob);
    o_ts[p] = L.take(sizeof(int) * nprob);
  }
  if (L.off > kNoAllocScratchBytes) {
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "negf_zinv_batched_noalloc: the request needs %zu bytes of scratch, more than the fixed %zu "
                  "(at most 51 blocks of 256 or 15 blocks of 512 per call)",
                  L.off, kNoAllocScratchBytes);
    return fail(NEGF_ERR_INVALID, buf);
  }

  unsigned char* base = nullptr;
  if (int r = setup_device(&base)) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  auto at = [&](size_t off) { return base + off; };

  // descriptors
  std::vector<ZBlockOp> ops;
  std::vector<ZInvProblem> inv;
  for (int i = 0; i < nprob; ++i) {
    if (n[i] == 0) continue;
    ZInvProblem p;
    p.W = reinterpret_cast<cplx*>(at(o_W[i]));
    p.F = reinterpret_cast<cplx*>(at(o_F[i]));
    p.Bbuf = reinterpret_cast<cplx*>(at(o_B[i]));
    p.used = at(o_used[i]);
    p.piv = reinterpret_cast<int*>(at(o_piv[i]));
    p.out = static_cast<cplx*>(Ainv[i]);
    p.info = reinterpret_cast<int*>(at(o_info)) + i;
    p.n = n[i]; p.ld = n[i]; p.ldo = ldainv[i]; p.pad_ = 0;
    inv.push_back(p);
    ZBlockOp o{};
    o.A = static_cast<const cplx*>(A[i]); o.lda = lda[i]; o.C = p.W; o.ldc = n[i];
    o.m = o.n = n[i]; o.kind = ZOP_COPY;
    ops.push_back(o);
  }
  const int cnt = static_cast<int>(inv.size());
  cudaError_t e = cudaMemsetAsync(at(o_info), 0, sizeof(int) * nprob, st);  // info starts at zero
  if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_ops), ops.data(), sizeof(ZBlockOp) * cnt, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_inv), inv.data(), sizeof(ZInvProblem) * cnt, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: descriptors");
  e = launch_zblockops(reinterpret_cast<const ZBlockOp*>(at(o_ops)), cnt, max_n, max_n, st);
  if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: copy");
  const ZInvProblem* dinv = reinterpret_cast<const ZInvProblem*>(at(o_inv));
  if (!blocked) {
    e = launch_zgj_panel(dinv, cnt, 0, nb, 0, zgj_panel_smem_bytes(max_n, nb), st);
    if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: panel");
  } else {
    for (int p = 0; p < npanels; ++p) {
      const int k0 = p * nb;
      e = launch_zgj_panel(dinv, cnt, k0, nb, 1, zgj_panel_smem_bytes(max_n, nb), st);
      if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: panel");
      std::vector<ZGemmProblem> g;
      std::vector<int> ts;
      int tiles = 0;
      for (const auto& q : inv) {
        if (q.n <= k0) continue;
        const int w = std::min(nb, q.n - k0);
        ZGemmProblem gp{};
        gp.A = q.F; gp.lda = q.n; gp.B = q.Bbuf; gp.ldb = w; gp.Cin = q.W; gp.ldcin = q.ld; gp.C = q.W;
        gp.ldc = q.ld; gp.m = q.n; gp.n = q.n; gp.k = w;
        gp.alpha = make_double2(1.0, 0.0); gp.beta = make_double2(1.0, 0.0); gp.diag = make_double2(0.0, 0.0);
        gp.diag_ptr = nullptr;
        ts.push_back(tiles);
        tiles += zgemm_tiles(q.n, q.n);
        g.push_back(gp);
      }
      if (g.empty()) continue;
      e = cudaMemcpyAsync(at(o_gp[p]), g.data(), sizeof(ZGemmProblem) * g.size(), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(at(o_ts[p]), ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = launch_zgemm_batched('N', 'N', reinterpret_cast<const ZGemmProblem*>(at(o_gp[p])),
                                 reinterpret_cast<const int*>(at(o_ts[p])), (int)g.size(), tiles, st);
      if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: update");
    }
    e = launch_zgj_unpermute(dinv, cnt, max_n, st);
    if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc: un-permute");
  }
  std::vector<int> h(nprob, 0);
  e = cudaMemcpyAsync(h.data(), at(o_info), sizeof(int) * nprob, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "negf_zinv_batched_noalloc");
  int bad = -1;
  for (int i = 0; i < nprob; ++i) {
    if (info) info[i] = h[i];
    if (h[i] && bad < 0) bad = i;
  }
  if (bad >= 0) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "negf_zinv_batched_noalloc: matrix %d is singular (zero pivot in column %d)", bad,
                  h[bad]);
    return fail(NEGF_ERR_SINGULAR, buf);
  }
  return NEGF_SUCCESS;
}
