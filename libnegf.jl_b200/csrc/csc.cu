// Sparse (CSC) <-> block conversions on the device for run_bndiag_wrapper and
// the dense debug path negf_bndiag_of_inv_direct:
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

// Dense debug path (bndiag_of_inv_direct!, src/matinvertndiag_direct.jl:17-61).
// One warp per column; lanes take consecutive nonzeros, so the writes of a
// column into its (column-major) blocks are coalesced.  table[bi * nb + bj]
// is block (bi, bj) of an nb-layer partition, every slot present.
__global__ void csc_full_scatter_kernel(int n, const int* __restrict__ colptr, const int* __restrict__ rowval,
                                        const cplx* __restrict__ nz, int nnz, const int* __restrict__ blk_of,
                                        const int* __restrict__ off, const int* __restrict__ bsz, cplx* const* table,
                                        int nb) {
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (c >= n) return;
  const int bj = blk_of[c];
  const int p0 = max(0, colptr[c]), p1 = min(nnz, colptr[c + 1]);
  for (int p = p0 + lane; p < p1; p += 32) {
    const int r = rowval[p];
    if (r < 0 || r >= n) continue;
    const int bi = blk_of[r];
    table[bi * nb + bj][(r - off[bi]) + (size_t)(c - off[bj]) * bsz[bi]] = nz[p];
  }
}

// Output of the dense path, column by column as the reference leaves it: M's
// stored entries above the out band (rows < lo), the inverse's band rows
// [lo, hi) (exact zeros dropped), M's stored entries below it (rows >= hi).
// Rows come out sorted when M's are.  One warp per column; a ballot orders
// each 32-row chunk.  pass 0 counts, pass 1 writes at colptr_out[c].
__global__ void csc_direct_out_kernel(int pass, int n, int npl, int wout, const int* __restrict__ blk_of,
                                      const int* __restrict__ off, const int* __restrict__ iblk_of,
                                      const int* __restrict__ ioff, const int* __restrict__ ibsz, int nb,
                                      const cplx* const* res, const int* __restrict__ colptr_in,
                                      const int* __restrict__ rowval_in, const cplx* __restrict__ nz_in, int nnz_in,
                                      int* __restrict__ counts, const int* __restrict__ colptr_out,
                                      int* __restrict__ rowval_out, cplx* __restrict__ nz_out) {
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (c >= n) return;
  const unsigned below = (1u << lane) - 1u;
  const int bj = blk_of[c];
  const int lo = off[max(0, bj - wout)], hi = off[min(npl - 1, bj + wout) + 1];
  const int p0 = max(0, colptr_in[c]), p1 = min(nnz_in, colptr_in[c + 1]);
  const int base = pass ? colptr_out[c] : 0;
  int cnt = 0;
  auto emit = [&](bool keep, int r, cplx v) {
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (pass && keep) {
      const int q = base + cnt + __popc(m & below);
      rowval_out[q] = r;
      nz_out[q] = v;
    }
    cnt += __popc(m);
  };
  for (int q = p0; q < p1; q += 32) {  // stored entries above the band
    const int p = q + lane;
    const int r = p < p1 ? rowval_in[p] : -1;
    const bool keep = r >= 0 && r < lo;
    emit(keep, r, keep ? nz_in[p] : make_double2(0.0, 0.0));
  }
  const int jb = iblk_of[c];
  for (int r0 = lo; r0 < hi; r0 += 32) {  // the band of the inverse
    const int r = r0 + lane;
    cplx v = make_double2(0.0, 0.0);
    if (r < hi) {
      const int ib = iblk_of[r];
      v = res[ib * nb + jb][(r - ioff[ib]) + (size_t)(c - ioff[jb]) * ibsz[ib]];
    }
    emit(r < hi && (v.x != 0.0 || v.y != 0.0), r, v);
  }
  for (int q = p0; q < p1; q += 32) {  // stored entries below the band
    const int p = q + lane;
    const int r = p < p1 ? rowval_in[p] : -1;
    const bool keep = r >= hi && r < n;
    emit(keep, r, keep ? nz_in[p] : make_double2(0.0, 0.0));
  }
  if (!pass && lane == 0) counts[c] = cnt;
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

cudaError_t launch_csc_full_scatter(int n, const int* colptr, const int* rowval, const cplx* nz, int nnz,
                                    const int* blk_of, const int* off, const int* bsz, cplx* const* table, int nb,
                                    cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  csc_full_scatter_kernel<<<(n + 7) / 8, 256, 0, st>>>(n, colptr, rowval, nz, nnz, blk_of, off, bsz, table, nb);
  return cudaGetLastError();
}

cudaError_t launch_csc_direct_out(int pass, int n, int npl, int wout, const int* blk_of, const int* off,
                                  const int* iblk_of, const int* ioff, const int* ibsz, int nb, const cplx* const* res,
                                  const int* colptr_in, const int* rowval_in, const cplx* nz_in, int nnz_in,
                                  int* counts, const int* colptr_out, int* rowval_out, cplx* nz_out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  csc_direct_out_kernel<<<(n + 7) / 8, 256, 0, st>>>(pass, n, npl, wout, blk_of, off, iblk_of, ioff, ibsz, nb, res,
                                                      colptr_in, rowval_in, nz_in, nnz_in, counts, colptr_out,
                                                      rowval_out, nz_out);
  return cudaGetLastError();
}

}  // namespace negf
