// Batched complex FP64 block inversion by blocked Gauss-Jordan with partial
// pivoting.
//
// The reference factors every diagonal Schur complement with zgetrf and then
// applies X^{-1} through zgetrs (be_lu! / be_mldivide!, src/backend_cpu.jl:
// 147-206); the downward pass needs X^{-1} explicitly anyway
// (src/matinvertndiag_rgf.jl:169,180).  Here X^{-1} is formed once, so every
// later use is a tensor-core GEMM.
//
// Algorithm (per matrix, n x n, panel width nb):
//   for each panel K = [k0, k0+nb):
//     * panel kernel (one CTA per matrix): the n x nb slab W[:,K] is held in
//       shared memory; for each column c: warp-level arg-max of |re|+|im| over
//       rows not yet used as pivots (LAPACK's izamax rule, ties to the lowest
//       row), then the in-place Gauss-Jordan step on the slab.  No rows are
//       swapped; the pivot row of column c is recorded in piv[c].  The kernel
//       writes the slab back and prepares the rank-nb update
//         F = slab - E_P (E_P has 1 at (piv[k0+i], i)),  Bbuf = W[P, :] with
//         the K columns zeroed;
//     * a batched GEMM applies W += F * Bbuf (the same kernel as all other
//       products).
//   Finally inv(X)[r, piv[c]] = W[piv[r], c]; a gather kernel writes the
//   un-permuted inverse to its destination.
// When n * n fits in shared memory the whole matrix is one panel and no GEMM
// is needed.
#include "negf_common.cuh"

namespace negf {

constexpr int GJ_THREADS = 512;

struct GjPanelArgs {
  int k0;      // first column of this panel
  int nb;      // panel width (columns)
  int blocked; // 1: write F/Bbuf for the trailing GEMM; 0: whole matrix in one panel
};

__device__ __forceinline__ void argmax_merge(double& v, int& r, double v2, int r2) {
  if (v2 > v || (v2 == v && r2 >= 0 && (r < 0 || r2 < r))) { v = v2; r = r2; }
}

__global__ void __launch_bounds__(GJ_THREADS)
    zgj_panel_kernel(const ZInvProblem* __restrict__ probs, GjPanelArgs args) {
  const ZInvProblem p = probs[blockIdx.x];
  const int n = p.n;
  const int k0 = args.k0;
  if (n <= 0 || k0 >= n) return;
  const int w = min(args.nb, n - k0);
  constexpr int NW = GJ_THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* S = reinterpret_cast<cplx*>(smem_raw);  // n x w, column-major
  cplx* colbuf = S + (size_t)n * w;               // n
  cplx* rowbuf = colbuf + n;                       // w
  double* redv = reinterpret_cast<double*>(rowbuf + w);  // NW (pivot value of the column, as complex below)
  int* redr = reinterpret_cast<int*>(redv + NW);   // NW
  int* sh_piv = redr + NW;                          // w
  uint8_t* used = reinterpret_cast<uint8_t*>(sh_piv + w);  // n
  cplx* sh_pv = reinterpret_cast<cplx*>(redv);      // reuses redv[0..1]: the scaled pivot inverse

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // column-per-warp, row-per-lane loops (no integer division)
  for (int j = warp; j < w; j += NW)
    for (int r = lane; r < n; r += 32) S[(size_t)j * n + r] = p.W[r + (size_t)(k0 + j) * p.ld];
  for (int r = tid; r < n; r += GJ_THREADS) used[r] = (k0 == 0) ? 0 : p.used[r];
  __syncthreads();

  for (int c = 0; c < w; ++c) {
    if (warp == 0) {
      // pivot search over unused rows, then stage column c and the scaled pivot row
      double bv = -1.0;
      int br = -1;
      for (int r = lane; r < n; r += 32)
        if (!used[r]) argmax_merge(bv, br, cabs1(S[(size_t)c * n + r]), r);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
        int r2 = __shfl_xor_sync(0xffffffffu, br, off);
        argmax_merge(bv, br, v2, r2);
      }
      const int pr = br;  // identical in every lane after the xor reduction
      if (lane == 0) {
        sh_piv[c] = pr;
        if (pr < 0 || bv == 0.0) {
          if (p.info) atomicCAS(p.info, 0, k0 + c + 1);
        }
        if (pr >= 0) used[pr] = 1;
      }
      if (pr >= 0) {
        cplx pivv = S[(size_t)c * n + pr];
        cplx pv = (pivv.x == 0.0 && pivv.y == 0.0) ? make_double2(0.0, 0.0) : cinv(pivv);
        for (int r = lane; r < n; r += 32) colbuf[r] = S[(size_t)c * n + r];
        for (int j = lane; j < w; j += 32) rowbuf[j] = (j == c) ? pv : cmul(S[(size_t)j * n + pr], pv);
        if (lane == 0) *sh_pv = pv;
      }
    }
    __syncthreads();
    const int pr = sh_piv[c];
    if (pr < 0) break;  // no candidate row: the host reports the info code
    const cplx pv = *sh_pv;
    for (int j = warp; j < w; j += NW) {
      const cplx rj = rowbuf[j];
      cplx* Sj = S + (size_t)j * n;
      if (j == c) {
        for (int r = lane; r < n; r += 32) Sj[r] = (r == pr) ? rj : cneg(cmul(colbuf[r], pv));
      } else {
        for (int r = lane; r < n; r += 32) Sj[r] = (r == pr) ? rj : cfms(Sj[r], colbuf[r], rj);
      }
    }
    __syncthreads();
  }

  if (!args.blocked) {
    // whole matrix in one panel: write the un-permuted inverse directly,
    // out[r, piv[c]] = S[piv[r], c]
    bool ok = true;
    for (int c = 0; c < w; ++c) ok = ok && sh_piv[c] >= 0;
    if (!ok) return;  // singular: info is set, out is left untouched
    for (int c = warp; c < n; c += NW) {
      cplx* o = p.out + (size_t)sh_piv[c] * p.ldo;
      const cplx* Sc = S + (size_t)c * n;
      for (int r = lane; r < n; r += 32) o[r] = Sc[sh_piv[r]];
    }
    return;
  }
  // write back slab, pivots and used flags
  for (int j = warp; j < w; j += NW)
    for (int r = lane; r < n; r += 32) p.W[r + (size_t)(k0 + j) * p.ld] = S[(size_t)j * n + r];
  for (int c = tid; c < w; c += GJ_THREADS) p.piv[k0 + c] = sh_piv[c];
  for (int r = tid; r < n; r += GJ_THREADS) p.used[r] = used[r];
  // F = slab - E_P  (n x w, ld n)
  for (int j = warp; j < w; j += NW) {
    const int pj = sh_piv[j];
    for (int r = lane; r < n; r += 32) {
      cplx v = S[(size_t)j * n + r];
      if (r == pj) v.x -= 1.0;
      p.F[r + (size_t)j * n] = v;
    }
  }
  // Bbuf = W[P, :] with panel columns zeroed  (w x n, ld w); the non-panel
  // columns of W are not modified by this kernel, so these are old values
  for (int j = warp; j < n; j += NW) {
    const bool inK = (j >= k0 && j < k0 + w);
    for (int c = lane; c < w; c += 32) {
      cplx v = make_double2(0.0, 0.0);
      if (!inK) v = p.W[sh_piv[c] + (size_t)j * p.ld];
      p.Bbuf[c + (size_t)j * w] = v;
    }
  }
}

// out[r, j] = W[piv[r], q[j]] with q the inverse permutation of piv:
// out[r, piv[c]] = W[piv[r], c].
__global__ void zgj_unpermute_kernel(const ZInvProblem* __restrict__ probs) {
  const ZInvProblem p = probs[blockIdx.y];
  const int n = p.n;
  // one thread per (r, c) element of W's column c -> output column piv[c]
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    int c = idx / n, r = idx - c * n;
    int pc = p.piv[c], pr = p.piv[r];
    if (pc < 0 || pr < 0) continue;
    p.out[r + (size_t)pc * p.ldo] = p.W[pr + (size_t)c * p.ld];
  }
}

size_t zgj_panel_smem_bytes(int n, int nb) {
  int w = nb < n ? nb : n;
  size_t b = (size_t)n * w * sizeof(cplx) + (size_t)n * sizeof(cplx) + (size_t)w * sizeof(cplx);
  b += (GJ_THREADS / 32) * (sizeof(double) + sizeof(int)) + (size_t)w * sizeof(int) + (size_t)n;
  return (b + 15) & ~size_t(15);
}

cudaError_t launch_zgj_panel(const ZInvProblem* probs_dev, int nprob, int k0, int nb, int blocked, size_t smem,
                             cudaStream_t stream) {
  if (nprob <= 0) return cudaSuccess;
  GjPanelArgs a{k0, nb, blocked};
  zgj_panel_kernel<<<nprob, GJ_THREADS, smem, stream>>>(probs_dev, a);
  return cudaGetLastError();
}

// Raise the dynamic shared-memory limit of the panel kernel (outside capture).
// The attribute is process-wide, so it is always set to the device's opt-in
// maximum: a later, smaller request never lowers the limit another live plan
// relies on.
cudaError_t zgj_prepare(size_t smem) {
  int dev = 0, mx = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)mx) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(zgj_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}

cudaError_t launch_zgj_unpermute(const ZInvProblem* probs_dev, int nprob, int max_n, cudaStream_t stream) {
  if (nprob <= 0) return cudaSuccess;
  int per = max_n * max_n;
  int bx = (per + 255) / 256;
  if (bx > 64) bx = 64;
  dim3 grid(bx, nprob);
  zgj_unpermute_kernel<<<grid, 256, 0, stream>>>(probs_dev);
  return cudaGetLastError();
}

}  // namespace negf
