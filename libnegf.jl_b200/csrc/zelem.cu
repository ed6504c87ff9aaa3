// Batched elementwise block operations: the reference's be_copy_in_hw!,
// be_ctranspose!, be_fill!, be_identity and axpby!/axpy!
// (src/backend_cpu.jl:42-88, src/selected_inverse.jl:185-199), one launch per
// list of blocks.  The conjugate transpose stages 32x32 tiles through shared
// memory so both the read and the write are coalesced.
#include "negf_common.cuh"

namespace negf {

constexpr int EL_TILE = 32;

__global__ void zblockop_kernel(const ZBlockOp* __restrict__ ops) {
  ZBlockOp o = ops[blockIdx.z];
  if (o.alpha_ptr) o.alpha = *o.alpha_ptr;
  __shared__ cplx tile[EL_TILE][EL_TILE + 1];
  const int tilesm = (o.m + EL_TILE - 1) / EL_TILE;
  const int tilesn = (o.n + EL_TILE - 1) / EL_TILE;
  for (int t = blockIdx.x; t < tilesm * tilesn; t += gridDim.x) {
    const int r0 = (t % tilesm) * EL_TILE, c0 = (t / tilesm) * EL_TILE;
    if (o.kind == ZOP_CTRANSPOSE || o.kind == ZOP_HERM_PART || o.kind == ZOP_GAMMA || o.kind == ZOP_CTRANS_AXPBY) {
      // A is n x m here (C = A^H is m x n); read A tile (c0.., r0..) coalesced along its rows
      for (int i = threadIdx.y; i < EL_TILE; i += blockDim.y) {
        int ar = c0 + threadIdx.x, ac = r0 + i;  // element A[ar, ac], ar < n, ac < m
        if (ar < o.n && ac < o.m) tile[i][threadIdx.x] = o.A[ar + (size_t)ac * o.lda];
      }
      __syncthreads();
      for (int i = threadIdx.y; i < EL_TILE; i += blockDim.y) {
        int r = r0 + threadIdx.x, c = c0 + i;
        if (r < o.m && c < o.n) {
          cplx v = cconj(tile[threadIdx.x][i]);  // A[c, r]^*
          if (o.kind == ZOP_HERM_PART) {
            cplx a = o.A[r + (size_t)c * o.lda];
            v = make_double2(0.5 * (a.x + v.x), 0.5 * (a.y + v.y));
          } else if (o.kind == ZOP_GAMMA) {
            cplx a = o.A[r + (size_t)c * o.lda];
            cplx d = make_double2(a.x - v.x, a.y - v.y);  // A - A^H
            v = make_double2(-d.y, d.x);                  // i * d
          } else if (o.kind == ZOP_CTRANS_AXPBY) {
            v = cmul(o.alpha, v);
            if (o.beta.x != 0.0 || o.beta.y != 0.0) v = cadd(v, cmul(o.beta, o.C[r + (size_t)c * o.ldc]));
          }
          o.C[r + (size_t)c * o.ldc] = v;
        }
      }
      __syncthreads();
    } else {
      for (int i = threadIdx.y; i < EL_TILE; i += blockDim.y) {
        int r = r0 + threadIdx.x, c = c0 + i;
        if (r >= o.m || c >= o.n) continue;
        size_t ci = r + (size_t)c * o.ldc;
        cplx v;
        switch (o.kind) {
          case ZOP_COPY: v = o.A[r + (size_t)c * o.lda]; break;
          case ZOP_AXPBY: {  // beta = 0 does not read C (BLAS semantics)
            cplx a = o.A[r + (size_t)c * o.lda];
            v = cmul(o.alpha, a);
            if (o.beta.x != 0.0 || o.beta.y != 0.0) v = cadd(v, cmul(o.beta, o.C[ci]));
            break;
          }
          case ZOP_ADD_DIAG:
            if (r != c) continue;
            v = cadd(o.C[ci], o.alpha);
            break;
          case ZOP_FILL: v = o.alpha; break;
          case ZOP_IDENTITY: v = (r == c) ? o.alpha : make_double2(0.0, 0.0); break;
          default: v = make_double2(0.0, 0.0); break;
        }
        o.C[ci] = v;
      }
    }
  }
}

cudaError_t launch_zblockops(const ZBlockOp* ops_dev, int nops, int max_m, int max_n, cudaStream_t stream) {
  if (nops <= 0) return cudaSuccess;
  int tiles = ((max_m + EL_TILE - 1) / EL_TILE) * ((max_n + EL_TILE - 1) / EL_TILE);
  if (tiles > 64) tiles = 64;
  if (tiles < 1) tiles = 1;
  // grid.z is limited to 65535: chunk the op list
  for (int base = 0; base < nops; base += 65535) {
    int cnt = nops - base < 65535 ? nops - base : 65535;
    dim3 grid(tiles, 1, cnt);
    zblockop_kernel<<<grid, dim3(EL_TILE, 8), 0, stream>>>(ops_dev + base);
  }
  return cudaGetLastError();
}

// Transmission T = Re Tr[GamL * G1N * GamR * G1N^H] needs only the trace of a
// product of two b x b matrices: Tr[X * Y] = sum_{r,c} X[r,c] Y[c,r].
// One block per problem; the result is written to out[i] (real part) and
// out_im[i] (imaginary part).
struct ZTraceProblem {
  const cplx* X;
  const cplx* Y;
  int n, ldx, ldy, pad_;
  double* out;
};

__global__ void ztrace_prod_kernel(const ZTraceProblem* __restrict__ probs) {
  const ZTraceProblem p = probs[blockIdx.x];
  double sr = 0.0, si = 0.0;
  for (int idx = threadIdx.x; idx < p.n * p.n; idx += blockDim.x) {
    int c = idx / p.n, r = idx - c * p.n;
    cplx x = p.X[r + (size_t)c * p.ldx];
    cplx y = p.Y[c + (size_t)r * p.ldy];
    sr += x.x * y.x - x.y * y.y;
    si += x.x * y.y + x.y * y.x;
  }
  __shared__ double red[2][32];
  for (int off = 16; off > 0; off >>= 1) {
    sr += __shfl_down_sync(0xffffffffu, sr, off);
    si += __shfl_down_sync(0xffffffffu, si, off);
  }
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[0][warp] = sr; red[1][warp] = si; }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    sr = lane < nw ? red[0][lane] : 0.0;
    si = lane < nw ? red[1][lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, off);
      si += __shfl_down_sync(0xffffffffu, si, off);
    }
    if (lane == 0) { p.out[0] = sr; p.out[1] = si; }
  }
}

cudaError_t launch_ztrace_prod(const void* probs_dev, int nprob, cudaStream_t stream) {
  if (nprob <= 0) return cudaSuccess;
  ztrace_prod_kernel<<<nprob, 256, 0, stream>>>(static_cast<const ZTraceProblem*>(probs_dev));
  return cudaGetLastError();
}

}  // namespace negf
