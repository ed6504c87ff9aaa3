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

// The same panel step with the slab in registers, for blocked panels of
// n <= 256 RT rows and nb <= 2 CT columns (RT * CT = 16 values per thread):
// thread t owns rows r = (t >> 1) + 256 k (k < RT) and panel columns
// (t & 1) CT .. (t & 1) CT + CT - 1.  The threads of the half that holds the
// pivot column rotate their register columns by one after every step, so the
// pivot column is always register column 0 (every register index is a
// compile-time one); register column j of half h holds panel column
// h CT + (j + rot) mod CT.  Per column: each warp reduces the arg-max of its
// rows, every thread merges the 16 warp results (one barrier), the two threads
// of the pivot row publish the scaled pivot row (a second barrier), and every
// thread updates its 16 values, taking its row's pivot column value from its
// partner lane.  Shared memory holds only the 16 partials and the pivot row;
// the arithmetic and the pivot rule are those of zgj_panel_kernel, so the
// results are identical.
template <int RT, int CT>
__global__ void __launch_bounds__(GJ_THREADS, 1)
    zgj_panel_reg_kernel(const ZInvProblem* __restrict__ probs, GjPanelArgs args) {
  static_assert(GJ_THREADS == 512 && RT * CT == 16, "register panel layout");
  // fields are read where needed (not held in registers across the column loop)
  const ZInvProblem* __restrict__ pp = probs + blockIdx.x;
  const int n = pp->n;
  const int k0 = args.k0;
  if (n <= 0 || k0 >= n) return;
  const int w = min(args.nb, n - k0);
  constexpr int NW = GJ_THREADS / 32;
  __shared__ double part_v[NW];
  __shared__ int part_r[NW];
  __shared__ cplx rowbuf[2 * CT];
  __shared__ cplx sh_pv;
  __shared__ int sh_piv[2 * CT];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, h = tid & 1, rr = tid >> 1;
  if (tid < 2 * CT) sh_piv[tid] = 0;  // valid row indices even if the column loop stops early

  cplx a[RT][CT];
  bool used[RT];
  {
    const cplx* W = pp->W;
    const int ld = pp->ld;
#pragma unroll
    for (int k = 0; k < RT; ++k) {
      const int r = rr + 256 * k;
      used[k] = r >= n || (k0 > 0 && pp->used[r]);
#pragma unroll
      for (int j = 0; j < CT; ++j) {
        const int col = h * CT + j;
        a[k][j] = (r < n && col < w) ? W[r + (size_t)(k0 + col) * ld] : make_double2(0.0, 0.0);
      }
    }
  }

  int rot = 0;  // rotations of this thread's register columns
  for (int c = 0; c < w; ++c) {
    const bool mine = h == (c >= CT ? 1 : 0);
    // 1. arg-max of |re| + |im| over this thread's unused rows of column c
    double bv = -1.0;
    int br = -1;
    if (mine)
#pragma unroll
      for (int k = 0; k < RT; ++k)
        if (!used[k]) argmax_merge(bv, br, cabs1(a[k][0]), rr + 256 * k);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
      const int r2 = __shfl_xor_sync(0xffffffffu, br, off);
      argmax_merge(bv, br, v2, r2);
    }
    if (lane == 0) {
      part_v[warp] = bv;
      part_r[warp] = br;
    }
    __syncthreads();
    // 2. every thread merges the warp results (one order for all): one pivot
    bv = part_v[0];
    br = part_r[0];
#pragma unroll
    for (int q = 1; q < NW; ++q) argmax_merge(bv, br, part_v[q], part_r[q]);
    const int pr = br;
    if (pr < 0 || bv == 0.0) {
      if (tid == 0 && pp->info) atomicCAS(pp->info, 0, k0 + c + 1);
      if (pr < 0) break;  // uniform: the host reports the info code
    }
    // 3. the pivot column value of each of this thread's rows (register column
    //    0 of the partner that holds column c), then the two threads of row pr
    //    publish the pivot inverse and the scaled pivot row
    const int kp = pr >> 8;
    cplx cv[RT];
#pragma unroll
    for (int k = 0; k < RT; ++k) {
      cplx o;
      o.x = __shfl_xor_sync(0xffffffffu, a[k][0].x, 1);
      o.y = __shfl_xor_sync(0xffffffffu, a[k][0].y, 1);
      cv[k] = mine ? a[k][0] : o;
    }
    if (rr == (pr & 255)) {
      cplx pivv = cv[0];
#pragma unroll
      for (int k = 1; k < RT; ++k)
        if (k == kp) pivv = cv[k];
      const cplx pv = (pivv.x == 0.0 && pivv.y == 0.0) ? make_double2(0.0, 0.0) : cinv(pivv);
#pragma unroll
      for (int j = 0; j < CT; ++j) {
        cplx sj = a[0][j];
#pragma unroll
        for (int k = 1; k < RT; ++k)
          if (k == kp) sj = a[k][j];
        const int jj = j + rot < CT ? j + rot : j + rot - CT;
        rowbuf[h * CT + jj] = (mine && j == 0) ? pv : cmul(sj, pv);
      }
      if (mine) {
        sh_pv = pv;
        sh_piv[c] = pr;
      }
#pragma unroll
      for (int k = 0; k < RT; ++k)
        if (k == kp) used[k] = true;
    }
    __syncthreads();
    // 4. the Gauss-Jordan step on this thread's values (the pivot row is read
    //    element by element, so its values are not all held in registers)
    const cplx pv = sh_pv;
    const volatile double* rb = reinterpret_cast<const volatile double*>(rowbuf + h * CT);
#pragma unroll
    for (int k = 0; k < RT; ++k) {
      const bool prow = rr + 256 * k == pr;
#pragma unroll
      for (int j = 0; j < CT; ++j) {
        const int jj = j + rot < CT ? j + rot : j + rot - CT;
        const cplx rj = make_double2(rb[2 * jj], rb[2 * jj + 1]);
        if (prow) a[k][j] = rj;
        else if (mine && j == 0) a[k][j] = cneg(cmul(cv[k], pv));
        else a[k][j] = cfms(a[k][j], cv[k], rj);
      }
    }
    // 5. the pivot half brings its next column to register column 0
    if (mine) {
#pragma unroll
      for (int k = 0; k < RT; ++k) {
        const cplx t = a[k][0];
#pragma unroll
        for (int j = 0; j + 1 < CT; ++j) a[k][j] = a[k][j + 1];
        a[k][CT - 1] = t;
      }
      rot = rot + 1 == CT ? 0 : rot + 1;
    }
    // the next column's partials overwrite part_v only after every thread
    // passed the barrier above, and rowbuf only after the next one
  }
  __syncthreads();
  // write back slab, pivots, used flags and F = slab - E_P (n x w, ld n)
  {
    cplx* W = pp->W;
    cplx* F = pp->F;
    const int ld = pp->ld;
#pragma unroll
    for (int k = 0; k < RT; ++k) {
      const int r = rr + 256 * k;
      if (r >= n) continue;
#pragma unroll
      for (int j = 0; j < CT; ++j) {
        const int jj = j + rot < CT ? j + rot : j + rot - CT;
        const int col = h * CT + jj;
        if (col >= w) continue;
        cplx v = a[k][j];
        W[r + (size_t)(k0 + col) * ld] = v;
        if (r == sh_piv[col]) v.x -= 1.0;
        F[r + (size_t)col * n] = v;
      }
      if (h == 0) pp->used[r] = used[k] ? 1 : 0;
    }
  }
  for (int c = tid; c < w; c += GJ_THREADS) pp->piv[k0 + c] = sh_piv[c];
  // Bbuf = W[P, :] with panel columns zeroed  (w x n, ld w): element e = c +
  // j w is W[piv_c, j]; the pivot rows are scattered, so every thread keeps
  // GU gathers in flight before it stores them
  {
    const cplx* W = pp->W;
    cplx* Bbuf = pp->Bbuf;
    const int ld = pp->ld;
    const int total = w * n;
    constexpr int GU = 8;
    for (int e0 = tid; e0 < total; e0 += GU * GJ_THREADS) {
      cplx v[GU];
#pragma unroll
      for (int u = 0; u < GU; ++u) {
        const int e = e0 + u * GJ_THREADS;
        v[u] = make_double2(0.0, 0.0);
        if (e < total) {
          const int c = e % w, j = e / w;
          if (j < k0 || j >= k0 + w) v[u] = W[sh_piv[c] + (size_t)j * ld];
        }
      }
#pragma unroll
      for (int u = 0; u < GU; ++u) {
        const int e = e0 + u * GJ_THREADS;
        if (e < total) Bbuf[e] = v[u];
      }
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
                             cudaStream_t stream, int max_n) {
  if (nprob <= 0) return cudaSuccess;
  GjPanelArgs a{k0, nb, blocked};
  // blocked panels of up to 256 rows x 32 columns or 512 rows x 16 columns:
  // the slab in registers
  if (blocked && max_n > 0 && max_n <= 256 && nb <= 32)
    zgj_panel_reg_kernel<1, 16><<<nprob, GJ_THREADS, 0, stream>>>(probs_dev, a);
  else if (blocked && max_n > 0 && max_n <= 512 && nb <= 16)
    zgj_panel_reg_kernel<2, 8><<<nprob, GJ_THREADS, 0, stream>>>(probs_dev, a);
  else
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
