// Batched complex FP64 LU with partial pivoting (LAPACK getrf semantics) or
// without row interchanges (lu(A, NoPivot())), and triangular inverses of the
// factors.
//
// Used by the selected inverse (the reference's be_getrf! / be_trsm! /
// be_getri!, src/backend_cpu.jl:229-265, called from
// src/selected_inverse.jl:9-206): every triangular solve with a factor is
// applied as a tensor-core GEMM with the factor's explicit inverse.
//
// LU (right-looking, panel width nb):
//   panel kernel: rows [k0, n) x columns [k0, k0+w) in shared memory, pivot
//     search per column (|re|+|im|, first maximum, as izamax), row swaps and
//     rank-1 updates inside the panel; writes ipiv (0-based, global) and the
//     inverse of the unit-lower w x w block L11 into scratch;
//   swap kernel: applies the panel's row interchanges to all other columns
//     (LAPACK's zlaswp on both sides) and copies A12 into scratch;
//   GEMMs (engine): A12 = L11^{-1} A12,  A22 -= A21 A12.
// Triangular inverse (blocked by nb): diagonal blocks inverted in shared
// memory here, off-diagonal blocks by GEMM recurrences in the engine.
#include "negf_common.cuh"

namespace negf {

constexpr int LU_THREADS = 256;

__global__ void __launch_bounds__(LU_THREADS)
    zgetrf_panel_kernel(const ZLuProblem* __restrict__ probs, int k0, int nb) {
  const ZLuProblem p = probs[blockIdx.x];
  const int n = p.n;
  if (k0 >= n) return;
  const int w = min(nb, n - k0);
  const int h = n - k0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* S = reinterpret_cast<cplx*>(smem_raw);   // h x w, column-major
  double* redv = reinterpret_cast<double*>(S + (size_t)h * w);
  int* redr = reinterpret_cast<int*>(redv + LU_THREADS / 32);
  int* sp = redr + LU_THREADS / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int idx = tid; idx < h * w; idx += LU_THREADS) {
    int c = idx / h, r = idx - c * h;
    S[idx] = p.A[(k0 + r) + (size_t)(k0 + c) * p.ld];
  }
  __syncthreads();
  for (int c = 0; c < w; ++c) {
    if (p.nopiv) {  // block-uniform branch: lu(A, NoPivot())
      if (tid == 0) {
        *sp = c;
        if (cabs1(S[(size_t)c * h + c]) <= 0.0 && p.info) atomicCAS(p.info, 0, k0 + c + 1);
      }
      __syncthreads();
    } else {
    double bv = -1.0;
    int br = -1;
    for (int r = c + tid; r < h; r += LU_THREADS) {
      double v = cabs1(S[(size_t)c * h + r]);
      if (v > bv) { bv = v; br = r; }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double v2 = __shfl_down_sync(0xffffffffu, bv, off);
      int r2 = __shfl_down_sync(0xffffffffu, br, off);
      if (v2 > bv || (v2 == bv && r2 >= 0 && (br < 0 || r2 < br))) { bv = v2; br = r2; }
    }
    if (lane == 0) { redv[warp] = bv; redr[warp] = br; }
    __syncthreads();
    if (warp == 0) {
      bv = lane < LU_THREADS / 32 ? redv[lane] : -1.0;
      br = lane < LU_THREADS / 32 ? redr[lane] : -1;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double v2 = __shfl_down_sync(0xffffffffu, bv, off);
        int r2 = __shfl_down_sync(0xffffffffu, br, off);
        if (v2 > bv || (v2 == bv && r2 >= 0 && (br < 0 || r2 < br))) { bv = v2; br = r2; }
      }
      if (lane == 0) {
        if (br < 0) br = c;
        *sp = br;
        if (bv <= 0.0 && p.info) atomicCAS(p.info, 0, k0 + c + 1);
      }
    }
    __syncthreads();
    }
    const int pr = *sp;
    if (tid == 0) p.ipiv[k0 + c] = k0 + pr;
    if (pr != c)
      for (int j = tid; j < w; j += LU_THREADS) {
        cplx t = S[(size_t)j * h + c];
        S[(size_t)j * h + c] = S[(size_t)j * h + pr];
        S[(size_t)j * h + pr] = t;
      }
    __syncthreads();
    cplx piv = S[(size_t)c * h + c];
    cplx inv = (piv.x == 0.0 && piv.y == 0.0) ? make_double2(0.0, 0.0) : cinv(piv);
    for (int r = c + 1 + tid; r < h; r += LU_THREADS) S[(size_t)c * h + r] = cmul(S[(size_t)c * h + r], inv);
    __syncthreads();
    const int rows = h - c - 1, cols = w - c - 1;
    for (int idx = tid; idx < rows * cols; idx += LU_THREADS) {
      int j = c + 1 + idx / rows, r = c + 1 + idx % rows;
      S[(size_t)j * h + r] = cfms(S[(size_t)j * h + r], S[(size_t)c * h + r], S[(size_t)j * h + c]);
    }
    __syncthreads();
  }
  for (int idx = tid; idx < h * w; idx += LU_THREADS) {
    int c = idx / h, r = idx - c * h;
    p.A[(k0 + r) + (size_t)(k0 + c) * p.ld] = S[idx];
  }
  // inverse of the unit lower w x w block (forward substitution per column)
  if (p.Linv && w < n) {
    for (int j = tid; j < w; j += LU_THREADS) {
      for (int i = 0; i < w; ++i) {
        cplx v;
        if (i < j) v = make_double2(0.0, 0.0);
        else if (i == j) v = make_double2(1.0, 0.0);
        else {
          v = make_double2(0.0, 0.0);
          for (int k = j; k < i; ++k) v = cfms(v, S[(size_t)k * h + i], p.Linv[k + (size_t)j * w]);
        }
        p.Linv[i + (size_t)j * w] = v;
      }
    }
  }
}

// Row interchanges of panel [k0, k0+w) on every column outside the panel,
// then T = A[k0:k0+w, k0+w:n] (w x (n-k0-w), ld w).
__global__ void zlaswp_copy_kernel(const ZLuProblem* __restrict__ probs, int k0, int nb) {
  const ZLuProblem p = probs[blockIdx.y];
  const int n = p.n;
  if (k0 >= n) return;
  const int w = min(nb, n - k0);
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    if (col >= k0 && col < k0 + w) continue;
    cplx* a = p.A + (size_t)col * p.ld;
    for (int c = 0; c < w; ++c) {
      int r1 = k0 + c, r2 = p.ipiv[k0 + c];
      if (r1 != r2) {
        cplx t = a[r1];
        a[r1] = a[r2];
        a[r2] = t;
      }
    }
    if (col >= k0 + w)
      for (int c = 0; c < w; ++c) p.T[c + (size_t)(col - k0 - w) * w] = a[k0 + c];
  }
}

// Inverse of one nb x nb diagonal block of the packed L\U factors:
// upper -> inverse of the non-unit upper triangle, else the inverse of the
// unit lower triangle.  X is the n x n output (zero elsewhere beforehand).
__global__ void ztrtri_diag_kernel(const ZTriProblem* __restrict__ probs, int nb, int upper) {
  const ZTriProblem p = probs[blockIdx.y];
  const int j0 = blockIdx.x * nb;
  if (j0 >= p.n) return;
  const int w = min(nb, p.n - j0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* S = reinterpret_cast<cplx*>(smem_raw);  // w x w block
  cplx* X = S + (size_t)w * w;                   // w x w inverse
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    int c = idx / w, r = idx - c * w;
    S[idx] = p.A[(j0 + r) + (size_t)(j0 + c) * p.lda];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < w; j += blockDim.x) {
    if (upper) {
      // X[:,j]: back substitution, X[i,j] = -(sum_{k=i+1..j} U[i,k] X[k,j]) / U[i,i]
      for (int i = w - 1; i >= 0; --i) {
        cplx v;
        if (i > j) v = make_double2(0.0, 0.0);
        else {
          cplx acc = (i == j) ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0);
          for (int k = i + 1; k <= j; ++k) acc = cfms(acc, S[i + (size_t)k * w], X[k + (size_t)j * w]);
          cplx d = S[i + (size_t)i * w];
          v = (d.x == 0.0 && d.y == 0.0) ? make_double2(0.0, 0.0) : cmul(acc, cinv(d));
        }
        X[i + (size_t)j * w] = v;
      }
    } else {
      for (int i = 0; i < w; ++i) {
        cplx v;
        if (i < j) v = make_double2(0.0, 0.0);
        else if (i == j) v = make_double2(1.0, 0.0);
        else {
          v = make_double2(0.0, 0.0);
          for (int k = j; k < i; ++k) v = cfms(v, S[i + (size_t)k * w], X[k + (size_t)j * w]);
        }
        X[i + (size_t)j * w] = v;
      }
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    int c = idx / w, r = idx - c * w;
    p.X[(j0 + r) + (size_t)(j0 + c) * p.ldx] = X[idx];
  }
}

size_t zgetrf_panel_smem_bytes(int n, int nb) {
  int w = nb < n ? nb : n;
  return ((size_t)n * w * sizeof(cplx) + (LU_THREADS / 32) * (sizeof(double) + sizeof(int)) + 16 + 15) & ~size_t(15);
}

size_t ztrtri_smem_bytes(int nb) { return 2 * (size_t)nb * nb * sizeof(cplx); }

// The shared-memory attributes are process-wide: set them to the device's
// opt-in maximum so that no later plan lowers a limit another one relies on.
cudaError_t zlu_prepare(size_t panel_smem, size_t tri_smem) {
  int dev = 0, mx = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (panel_smem > (size_t)mx || tri_smem > (size_t)mx) return cudaErrorInvalidValue;
  if (panel_smem) e = cudaFuncSetAttribute(zgetrf_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  if (e == cudaSuccess && tri_smem)
    e = cudaFuncSetAttribute(ztrtri_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  return e;
}

cudaError_t launch_zgetrf_panel(const void* probs, int nprob, int k0, int nb, size_t smem, cudaStream_t st) {
  if (nprob <= 0) return cudaSuccess;
  zgetrf_panel_kernel<<<nprob, LU_THREADS, smem, st>>>(static_cast<const ZLuProblem*>(probs), k0, nb);
  return cudaGetLastError();
}

cudaError_t launch_zlaswp_copy(const void* probs, int nprob, int k0, int nb, int max_n, cudaStream_t st) {
  if (nprob <= 0) return cudaSuccess;
  dim3 grid((max_n + 127) / 128, nprob);
  zlaswp_copy_kernel<<<grid, 128, 0, st>>>(static_cast<const ZLuProblem*>(probs), k0, nb);
  return cudaGetLastError();
}

cudaError_t launch_ztrtri_diag(const void* probs, int nprob, int nb, int upper, int max_n, size_t smem,
                               cudaStream_t st) {
  if (nprob <= 0) return cudaSuccess;
  dim3 grid((max_n + nb - 1) / nb, nprob);
  ztrtri_diag_kernel<<<grid, 64, smem, st>>>(static_cast<const ZTriProblem*>(probs), nb, upper);
  return cudaGetLastError();
}

}  // namespace negf
