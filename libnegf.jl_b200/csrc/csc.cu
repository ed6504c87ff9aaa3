// Sparse (CSC) <-> block conversions on the device for run_bndiag_wrapper:
// the reference converts on the host (bm_convert, src/blockmatrix.jl:34-72
// sparse -> blocks, :82-127 blocks -> sparse; called from
// src/c_interface/libnegf_c_interface.jl:85-142).
#include "negf_common.cuh"

namespace negf {

// Block (i, j) of the tridiagonal band, j - i in {-1, 0, 1}: table[3 i + j - i + 1].
__device__ __forceinline__ int band_slot(int bi, int bj) { return 3 * bi + (bj - bi + 1); }

// One thread per column: scatter the column's nonzeros into the band blocks
// (diagonal and upper only when hermitian; the lower blocks are conjugate
// transposes made afterwards).  Entries outside the band are ignored, as the
// reference's conversion of a tridiagonal pattern does.
__global__ void csc_scatter_kernel(int n, const int* __restrict__ colptr, const int* __restrict__ rowval,
                                   const cplx* __restrict__ nz, int nnz, const int* __restrict__ blk_of,
                                   const int* __restrict__ off, const int* __restrict__ bsz, cplx* const* blocks,
                                   int hermitian) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int bj = blk_of[c];
  const int p0 = max(0, colptr[c]), p1 = min(nnz, colptr[c + 1]);
  for (int p = p0; p < p1; ++p) {
    const int r = rowval[p];
    if (r < 0 || r >= n) continue;
    const int bi = blk_of[r];
    if (bi - bj > 1 || bj - bi > 1) continue;
    if (hermitian && bi > bj) continue;
    cplx* B = blocks[band_slot(bi, bj)];
    B[(r - off[bi]) + (size_t)(c - off[bj]) * bsz[bi]] = nz[p];
  }
}

// value (r, c) of the input CSC (rows sorted within a column), 0 if absent
__device__ __forceinline__ cplx csc_at(const int* colptr, const int* rowval, const cplx* nz, int nnz, int r, int c) {
  int lo = max(0, colptr[c]), hi = min(nnz, colptr[c + 1]) - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = rowval[mid];
    if (v == r) return nz[mid];
    if (v < r) lo = mid + 1; else hi = mid - 1;
  }
  return make_double2(0.0, 0.0);
}

// Output band of width wout (blocks |bi - bj| <= wout): the tridiagonal from the
// result blocks, the rest from the input.  pass 0 counts the nonzeros of every
// column, pass 1 writes them at the column's offset.
__global__ void csc_band_out_kernel(int pass, int n, int npl, int wout, const int* __restrict__ blk_of,
                                    const int* __restrict__ off, const int* __restrict__ bsz, const cplx* const* res,
                                    const int* __restrict__ colptr_in, const int* __restrict__ rowval_in,
                                    const cplx* __restrict__ nz_in, int nnz_in, int* __restrict__ counts,
                                    const int* __restrict__ colptr_out, int* __restrict__ rowval_out,
                                    cplx* __restrict__ nz_out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int bj = blk_of[c];
  int cnt = 0;
  const int q0 = pass ? colptr_out[c] : 0;
  for (int bi = max(0, bj - wout); bi <= min(npl - 1, bj + wout); ++bi) {
    const bool tri = bi - bj <= 1 && bj - bi <= 1;
    const cplx* R = tri ? res[band_slot(bi, bj)] : nullptr;
    for (int r = off[bi]; r < off[bi + 1]; ++r) {
      const cplx v = tri ? R[(r - off[bi]) + (size_t)(c - off[bj]) * bsz[bi]]
                         : csc_at(colptr_in, rowval_in, nz_in, nnz_in, r, c);
      if (v.x == 0.0 && v.y == 0.0) continue;
      if (pass) {
        rowval_out[q0 + cnt] = r;
        nz_out[q0 + cnt] = v;
      }
      ++cnt;
    }
  }
  if (!pass) counts[c] = cnt;
}

cudaError_t launch_csc_scatter(int n, const int* colptr, const int* rowval, const cplx* nz, int nnz, const int* blk_of,
                               const int* off, const int* bsz, cplx* const* blocks, int hermitian, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  csc_scatter_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, colptr, rowval, nz, nnz, blk_of, off, bsz, blocks,
                                                       hermitian);
  return cudaGetLastError();
}

cudaError_t launch_csc_band_out(int pass, int n, int npl, int wout, const int* blk_of, const int* off, const int* bsz,
                                const cplx* const* res, const int* colptr_in, const int* rowval_in,
                                const cplx* nz_in, int nnz_in, int* counts, const int* colptr_out, int* rowval_out,
                                cplx* nz_out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  csc_band_out_kernel<<<(n + 127) / 128, 128, 0, st>>>(pass, n, npl, wout, blk_of, off, bsz, res, colptr_in,
                                                        rowval_in, nz_in, nnz_in, counts, colptr_out, rowval_out,
                                                        nz_out);
  return cudaGetLastError();
}

}  // namespace negf
