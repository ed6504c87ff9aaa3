// Batched complex FP64 GEMM on the sm_100a FP64 tensor path (DMMA).
//
// Every Schur-complement product of the RGF / RKD / selected-inverse / DDRGF
// sweeps (the reference's be_gemm!, src/backend_cpu.jl:208-219, and the
// getrs-with-explicit-inverse products that replace be_mldivide!) runs here.
//
// Design:
//  * one launch covers a whole list of independent problems of arbitrary
//    (m, n, k) -- all energies x all blocks of one sweep step; CTAs map to
//    (problem, 64x64 output tile) through a prefix sum of tile counts;
//  * a CTA computes a 64x64 complex tile with 4 warps (2x2 of 32x32); the
//    K loop stages 64x16 complex A and 16x64 complex B tiles through a
//    3-stage cp.async pipeline (each complex double is one 16-byte cp.async,
//    so transposed / conjugated operands are handled on the copy);
//  * the complex product uses four real mma.sync m16n8k4 f64 products
//    (re += Ar*Br - Ai*Bi, im += Ar*Bi + Ai*Br); FP64 has no tcgen05 kind,
//    and on B200 mma.sync f64 and DFMA both peak near 37 TFLOP/s (measured
//    by negf_probe_fp64_peak), so DMMA is the FP64 tensor path;
//  * epilogue: C = alpha*acc + beta*Cin + diag*I, bounds-checked.
#include "negf_common.cuh"

#include <cstdlib>

namespace negf {

namespace gemm {
constexpr int BM = 64, BN = 64, BK = 16;
constexpr int THREADS = 128;
constexpr int STAGES = 3;
constexpr int AS_LD = BM + 1;  // As[k][m]
constexpr int BS_LD = BK + 1;  // Bs[n][k]
constexpr int AS_SIZE = BK * AS_LD;
constexpr int BS_SIZE = BN * BS_LD;
constexpr int STAGE_SIZE = AS_SIZE + BS_SIZE;  // complex elements per stage
constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE_SIZE * sizeof(cplx);
}  // namespace gemm

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma16x8x4(double& c0, double& c1, double& c2, double& c3, double a0, double a1,
                                           double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
      : "d"(a0), "d"(a1), "d"(b0));
}

// CTA -> (problem, tile).  nprob > 0: binary search over the exclusive
// prefix sum tile_start; nprob < 0: every problem has -nprob tiles (the
// host's uniform batches), so the problem is a division away and the CTA
// skips the chain of dependent loads of the search.
__device__ __forceinline__ void zgemm_locate(int bid, const int* __restrict__ tile_start, int nprob, int& prob,
                                             int& tile) {
  if (nprob < 0) {
    const int T = -nprob;
    prob = bid / T;
    tile = bid - prob * T;
    return;
  }
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= bid) lo = mid; else hi = mid - 1;
  }
  prob = lo;
  tile = bid - tile_start[lo];
}

// Stage one K-slab of A (BM x BK of op(A)) and B (BK x BN of op(B)).
template <bool TA, bool TB>
__device__ __forceinline__ void load_stage(cplx* As, cplx* Bs, const ZGemmProblem& p, int m0, int n0, int k0,
                                           int tid) {
  using namespace gemm;
  // A tile: element (r, kk) of op(A)
#pragma unroll
  for (int i = 0; i < (BM * BK) / THREADS; ++i) {
    int idx = tid + i * THREADS;
    int r, kk;
    if (!TA) { r = idx % BM; kk = idx / BM; }   // contiguous in r for column-major A
    else     { kk = idx % BK; r = idx / BK; }   // contiguous in k for A^T / A^H
    int gr = m0 + r, gk = k0 + kk;
    bool ok = gr < p.m && gk < p.k;
    const cplx* src = p.A;
    if (ok) src = TA ? (p.A + gk + (size_t)gr * p.lda) : (p.A + gr + (size_t)gk * p.lda);
    cp_async16(&As[kk * AS_LD + r], src, ok);
  }
  // B tile: element (kk, c) of op(B)
#pragma unroll
  for (int i = 0; i < (BN * BK) / THREADS; ++i) {
    int idx = tid + i * THREADS;
    int c, kk;
    if (!TB) { kk = idx % BK; c = idx / BK; }   // contiguous in k for column-major B
    else     { c = idx % BN; kk = idx / BN; }   // contiguous in n for B^T / B^H
    int gc = n0 + c, gk = k0 + kk;
    bool ok = gc < p.n && gk < p.k;
    const cplx* src = p.B;
    if (ok) src = TB ? (p.B + gc + (size_t)gk * p.ldb) : (p.B + gk + (size_t)gc * p.ldb);
    cp_async16(&Bs[c * BS_LD + kk], src, ok);
  }
}

template <bool TA, bool CA, bool TB, bool CB, bool PRE>
__global__ void __launch_bounds__(gemm::THREADS, 2)
    zgemm_batched_kernel(const ZGemmProblem* __restrict__ probs, const int* __restrict__ tile_start, int nprob) {
  using namespace gemm;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);

  int lo, t;
  zgemm_locate(blockIdx.x, tile_start, nprob, lo, t);
  const ZGemmProblem p = probs[lo];
  int tiles_m = (p.m + BM - 1) / BM;
  int m0 = (t % tiles_m) * BM;
  int n0 = (t / tiles_m) * BN;

  int tid = threadIdx.x;
  int warp = tid >> 5, lane = tid & 31;
  int g = lane >> 2, tq = lane & 3;
  int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

  // PRE (chosen per launch by the host when every problem has alpha, beta in
  // {1, -1} and a Cin): in-place updates C = +-A*B +- C, i.e. every Schur
  // update of the sweeps, start the accumulators from Cin, so the loads are
  // issued before the main loop and overlap the first operand copies instead
  // of stalling the epilogue.
  const bool preload = PRE && p.k > 0 && p.Cin != nullptr;
  const double pre_sign = p.alpha.x * p.beta.x;  // beta / alpha for alpha, beta in {1, -1}

  double acc_re[2][4][4], acc_im[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        acc_re[a][b][c] = 0.0;
        acc_im[a][b][c] = 0.0;
        if (preload) {
          int r = m0 + wm + a * 16 + g + ((c >> 1) << 3);
          int cc = n0 + wn + b * 8 + 2 * tq + (c & 1);
          if (r < p.m && cc < p.n) {
            cplx v = p.Cin[r + (size_t)cc * p.ldcin];
            acc_re[a][b][c] = pre_sign * v.x;
            acc_im[a][b][c] = pre_sign * v.y;
          }
        }
      }

  int nk = (p.k + BK - 1) / BK;
  // prologue
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, s * BK, tid);
    cp_async_commit();
  }

  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    // prefetch the slab STAGES-1 ahead into the buffer freed last iteration
    int kn = kt + STAGES - 1;
    if (kn < nk) {
      int s = kn % STAGES;
      load_stage<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, kn * BK, tid);
    }
    cp_async_commit();

    const cplx* As = smem + (kt % STAGES) * STAGE_SIZE;
    const cplx* Bs = As + AS_SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[2][2], ai[2][2], br[4], bi[4], nbi[4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        cplx x0 = As[(kk + tq) * AS_LD + wm + mi * 16 + g];
        cplx x1 = As[(kk + tq) * AS_LD + wm + mi * 16 + g + 8];
        ar[mi][0] = x0.x; ai[mi][0] = CA ? -x0.y : x0.y;
        ar[mi][1] = x1.x; ai[mi][1] = CA ? -x1.y : x1.y;
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        cplx y = Bs[(wn + ni * 8 + g) * BS_LD + kk + tq];
        br[ni] = y.x;
        bi[ni] = CB ? -y.y : y.y;
        nbi[ni] = -bi[ni];
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          double* cr = acc_re[mi][ni];
          double* ci = acc_im[mi][ni];
          dmma16x8x4(cr[0], cr[1], cr[2], cr[3], ar[mi][0], ar[mi][1], br[ni]);
          dmma16x8x4(cr[0], cr[1], cr[2], cr[3], ai[mi][0], ai[mi][1], nbi[ni]);
          dmma16x8x4(ci[0], ci[1], ci[2], ci[3], ar[mi][0], ar[mi][1], bi[ni]);
          dmma16x8x4(ci[0], ci[1], ci[2], ci[3], ai[mi][0], ai[mi][1], br[ni]);
        }
    }
  }
  cp_async_wait<0>();

  // epilogue
  const bool has_ab = p.k > 0;
  const bool has_cin = (p.beta.x != 0.0 || p.beta.y != 0.0) && p.Cin != nullptr && !preload;
  const cplx dg = p.diag_ptr ? *p.diag_ptr : p.diag;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int r = m0 + wm + mi * 16 + g + ((e >> 1) << 3);
        int c = n0 + wn + ni * 8 + 2 * tq + (e & 1);
        if (r < p.m && c < p.n) {
          cplx v = make_double2(0.0, 0.0);
          if (has_ab) {
            double xr = acc_re[mi][ni][e], xi = acc_im[mi][ni][e];
            v.x = p.alpha.x * xr - p.alpha.y * xi;
            v.y = p.alpha.x * xi + p.alpha.y * xr;
          }
          if (has_cin) {
            cplx ci = p.Cin[r + (size_t)c * p.ldcin];
            v.x += p.beta.x * ci.x - p.beta.y * ci.y;
            v.y += p.beta.x * ci.y + p.beta.y * ci.x;
          }
          if (r == c) { v.x += dg.x; v.y += dg.y; }
          p.C[r + (size_t)c * p.ldc] = v;
        }
      }
}

// ---------------------------------------------------------------------------
// 3M variant (Gauss's complex product): three real DMMA products per complex
// product instead of four,
//   P1 = Ar Br,  P2 = Ai Bi,  P3 = (Ar + Ai)(Br + Bi),
//   Re C = P1 - P2,  Im C = P3 - P1 - P2,
// the scheme of zgemm3m (normwise stable; the imaginary part carries an
// absolute error of a few ulps of |A||B| instead of |Im C|).  Same 64x64
// tile and staging as the 4M kernel; 8 warps of 32x16 so that the three
// accumulator sets fit the register file.
namespace gemm3m {
constexpr int THREADS = 256;
}

template <bool TA, bool CA, bool TB, bool CB, bool PRE>
__global__ void __launch_bounds__(gemm3m::THREADS, 1)
    zgemm3m_batched_kernel(const ZGemmProblem* __restrict__ probs, const int* __restrict__ tile_start, int nprob) {
  using namespace gemm;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  int lo, t;
  zgemm_locate(blockIdx.x, tile_start, nprob, lo, t);
  const ZGemmProblem p = probs[lo];
  const int tiles_m = (p.m + BM - 1) / BM;
  const int m0 = (t % tiles_m) * BM;
  const int n0 = (t / tiles_m) * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;

  const bool preload = PRE && p.k > 0 && p.Cin != nullptr;
  const double pre_sign = p.alpha.x * p.beta.x;
  double P1[2][2][4], P2[2][2][4], P3[2][2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        P1[a][b][c] = 0.0; P2[a][b][c] = 0.0; P3[a][b][c] = 0.0;
        if (preload) {
          // Re = P1 - P2 = s Cr,  Im = P3 - P1 - P2 = s Ci
          int r = m0 + wm + a * 16 + g + ((c >> 1) << 3);
          int cc = n0 + wn + b * 8 + 2 * tq + (c & 1);
          if (r < p.m && cc < p.n) {
            cplx v = p.Cin[r + (size_t)cc * p.ldcin];
            P1[a][b][c] = pre_sign * v.x;
            P3[a][b][c] = pre_sign * v.x + pre_sign * v.y;
          }
        }
      }

  const int nk = (p.k + BK - 1) / BK;
  // the loader is written for 128 threads: the first four warps stage each slab
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk && tid < THREADS)
      load_stage<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, s * BK, tid);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    int kn = kt + STAGES - 1;
    if (kn < nk && tid < THREADS) {
      int s = kn % STAGES;
      load_stage<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, kn * BK, tid);
    }
    cp_async_commit();
    const cplx* As = smem + (kt % STAGES) * STAGE_SIZE;
    const cplx* Bs = As + AS_SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[2][2], ai[2][2], as[2][2], br[2], bi[2], bs[2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        cplx x0 = As[(kk + tq) * AS_LD + wm + mi * 16 + g];
        cplx x1 = As[(kk + tq) * AS_LD + wm + mi * 16 + g + 8];
        ar[mi][0] = x0.x; ai[mi][0] = CA ? -x0.y : x0.y; as[mi][0] = ar[mi][0] + ai[mi][0];
        ar[mi][1] = x1.x; ai[mi][1] = CA ? -x1.y : x1.y; as[mi][1] = ar[mi][1] + ai[mi][1];
      }
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
        cplx y = Bs[(wn + ni * 8 + g) * BS_LD + kk + tq];
        br[ni] = y.x;
        bi[ni] = CB ? -y.y : y.y;
        bs[ni] = br[ni] + bi[ni];
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) {
          double* p1 = P1[mi][ni];
          double* p2 = P2[mi][ni];
          double* p3 = P3[mi][ni];
          dmma16x8x4(p1[0], p1[1], p1[2], p1[3], ar[mi][0], ar[mi][1], br[ni]);
          dmma16x8x4(p2[0], p2[1], p2[2], p2[3], ai[mi][0], ai[mi][1], bi[ni]);
          dmma16x8x4(p3[0], p3[1], p3[2], p3[3], as[mi][0], as[mi][1], bs[ni]);
        }
    }
  }
  cp_async_wait<0>();

  const bool has_ab = p.k > 0;
  const bool has_cin = (p.beta.x != 0.0 || p.beta.y != 0.0) && p.Cin != nullptr && !preload;
  const cplx dg = p.diag_ptr ? *p.diag_ptr : p.diag;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int r = m0 + wm + mi * 16 + g + ((e >> 1) << 3);
        int c = n0 + wn + ni * 8 + 2 * tq + (e & 1);
        if (r < p.m && c < p.n) {
          cplx v = make_double2(0.0, 0.0);
          if (has_ab) {
            double xr = P1[mi][ni][e] - P2[mi][ni][e];
            double xi = P3[mi][ni][e] - P1[mi][ni][e] - P2[mi][ni][e];
            v.x = p.alpha.x * xr - p.alpha.y * xi;
            v.y = p.alpha.x * xi + p.alpha.y * xr;
          }
          if (has_cin) {
            cplx ci = p.Cin[r + (size_t)c * p.ldcin];
            v.x += p.beta.x * ci.x - p.beta.y * ci.y;
            v.y += p.beta.x * ci.y + p.beta.y * ci.x;
          }
          if (r == c) { v.x += dg.x; v.y += dg.y; }
          p.C[r + (size_t)c * p.ldc] = v;
        }
      }
}

// ---------------------------------------------------------------------------
// Small-K 3M variant for products with k <= 32 (the Gauss-Jordan rank-nb
// updates W += F Bbuf and other thin products).  Such a tile has one or two
// K slabs, so the 64 x 64 kernel (one CTA per SM at 246 registers) spends
// most of its time waiting for its operand and Cin loads with nothing to
// overlap them.  Here a CTA computes a 32 x 64 tile with 8 warps of 16 x 16
// (24 accumulator doubles per thread), small enough for two CTAs per SM, so
// one CTA's loads overlap the other's DMMA products.  Same staging scheme
// (3-stage cp.async ring, 16 K per slab), same arithmetic as the 3M kernel.
namespace gemm_sk {
constexpr int BM = 32, BN = 64, BK = 16;
constexpr int THREADS = 256;
constexpr int STAGES = 3;
constexpr int AS_LD = BM + 1;  // As[k][m]
constexpr int BS_LD = BK + 1;  // Bs[n][k]
constexpr int AS_SIZE = BK * AS_LD;
constexpr int BS_SIZE = BN * BS_LD;
constexpr int STAGE_SIZE = AS_SIZE + BS_SIZE;
constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE_SIZE * sizeof(cplx);
}  // namespace gemm_sk

template <bool TA, bool TB>
__device__ __forceinline__ void load_stage_sk(cplx* As, cplx* Bs, const ZGemmProblem& p, int m0, int n0, int k0,
                                              int tid) {
  using namespace gemm_sk;
#pragma unroll
  for (int i = 0; i < (BM * BK) / THREADS; ++i) {
    const int idx = tid + i * THREADS;
    int r, kk;
    if (!TA) { r = idx % BM; kk = idx / BM; }
    else     { kk = idx % BK; r = idx / BK; }
    const int gr = m0 + r, gk = k0 + kk;
    const bool ok = gr < p.m && gk < p.k;
    const cplx* src = p.A;
    if (ok) src = TA ? (p.A + gk + (size_t)gr * p.lda) : (p.A + gr + (size_t)gk * p.lda);
    cp_async16(&As[kk * AS_LD + r], src, ok);
  }
#pragma unroll
  for (int i = 0; i < (BN * BK) / THREADS; ++i) {
    const int idx = tid + i * THREADS;
    int c, kk;
    if (!TB) { kk = idx % BK; c = idx / BK; }
    else     { c = idx % BN; kk = idx / BN; }
    const int gc = n0 + c, gk = k0 + kk;
    const bool ok = gc < p.n && gk < p.k;
    const cplx* src = p.B;
    if (ok) src = TB ? (p.B + gc + (size_t)gk * p.ldb) : (p.B + gk + (size_t)gc * p.ldb);
    cp_async16(&Bs[c * BS_LD + kk], src, ok);
  }
}

template <bool TA, bool CA, bool TB, bool CB, bool PRE>
__global__ void __launch_bounds__(gemm_sk::THREADS, 2)
    zgemm3m_smallk_kernel(const ZGemmProblem* __restrict__ probs, const int* __restrict__ tile_start, int nprob) {
  using namespace gemm_sk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  int lo, t;
  zgemm_locate(blockIdx.x, tile_start, nprob, lo, t);
  const ZGemmProblem p = probs[lo];
  const int tiles_m = (p.m + BM - 1) / BM;
  const int m0 = (t % tiles_m) * BM;
  const int n0 = (t / tiles_m) * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp & 1) * 16, wn = (warp >> 1) * 16;

  const bool preload = PRE && p.k > 0 && p.Cin != nullptr;
  const double pre_sign = p.alpha.x * p.beta.x;
  double P1[2][4], P2[2][4], P3[2][4];
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      P1[b][c] = 0.0; P2[b][c] = 0.0; P3[b][c] = 0.0;
      if (preload) {
        const int r = m0 + wm + g + ((c >> 1) << 3);
        const int cc = n0 + wn + b * 8 + 2 * tq + (c & 1);
        if (r < p.m && cc < p.n) {
          const cplx v = p.Cin[r + (size_t)cc * p.ldcin];
          P1[b][c] = pre_sign * v.x;
          P3[b][c] = pre_sign * v.x + pre_sign * v.y;
        }
      }
    }

  const int nk = (p.k + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage_sk<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, s * BK, tid);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int kn = kt + STAGES - 1;
    if (kn < nk) {
      const int s = kn % STAGES;
      load_stage_sk<TA, TB>(smem + s * STAGE_SIZE, smem + s * STAGE_SIZE + AS_SIZE, p, m0, n0, kn * BK, tid);
    }
    cp_async_commit();
    const cplx* As = smem + (kt % STAGES) * STAGE_SIZE;
    const cplx* Bs = As + AS_SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[2], ai[2], as[2], br[2], bi[2], bs[2];
      const cplx x0 = As[(kk + tq) * AS_LD + wm + g];
      const cplx x1 = As[(kk + tq) * AS_LD + wm + g + 8];
      ar[0] = x0.x; ai[0] = CA ? -x0.y : x0.y; as[0] = ar[0] + ai[0];
      ar[1] = x1.x; ai[1] = CA ? -x1.y : x1.y; as[1] = ar[1] + ai[1];
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
        const cplx y = Bs[(wn + ni * 8 + g) * BS_LD + kk + tq];
        br[ni] = y.x;
        bi[ni] = CB ? -y.y : y.y;
        bs[ni] = br[ni] + bi[ni];
      }
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
        double* p1 = P1[ni];
        double* p2 = P2[ni];
        double* p3 = P3[ni];
        dmma16x8x4(p1[0], p1[1], p1[2], p1[3], ar[0], ar[1], br[ni]);
        dmma16x8x4(p2[0], p2[1], p2[2], p2[3], ai[0], ai[1], bi[ni]);
        dmma16x8x4(p3[0], p3[1], p3[2], p3[3], as[0], as[1], bs[ni]);
      }
    }
  }
  cp_async_wait<0>();

  const bool has_ab = p.k > 0;
  const bool has_cin = (p.beta.x != 0.0 || p.beta.y != 0.0) && p.Cin != nullptr && !preload;
  const cplx dg = p.diag_ptr ? *p.diag_ptr : p.diag;
#pragma unroll
  for (int ni = 0; ni < 2; ++ni)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = m0 + wm + g + ((e >> 1) << 3);
      const int c = n0 + wn + ni * 8 + 2 * tq + (e & 1);
      if (r < p.m && c < p.n) {
        cplx v = make_double2(0.0, 0.0);
        if (has_ab) {
          const double xr = P1[ni][e] - P2[ni][e];
          const double xi = P3[ni][e] - P1[ni][e] - P2[ni][e];
          v.x = p.alpha.x * xr - p.alpha.y * xi;
          v.y = p.alpha.x * xi + p.alpha.y * xr;
        }
        if (has_cin) {
          const cplx ci = p.Cin[r + (size_t)c * p.ldcin];
          v.x += p.beta.x * ci.x - p.beta.y * ci.y;
          v.y += p.beta.x * ci.y + p.beta.y * ci.x;
        }
        if (r == c) { v.x += dg.x; v.y += dg.y; }
        p.C[r + (size_t)c * p.ldc] = v;
      }
    }
}

using ZGemmKernel = void (*)(const ZGemmProblem*, const int*, int);

template <bool PRE, bool G3M>
static ZGemmKernel pick_kernel_t(int ia, int ib) {
#define NEGF_K(TA, CA, TB, CB) \
  (G3M ? zgemm3m_batched_kernel<TA, CA, TB, CB, PRE> : zgemm_batched_kernel<TA, CA, TB, CB, PRE>)
  switch (ia * 3 + ib) {
    case 0: return NEGF_K(false, false, false, false);
    case 1: return NEGF_K(false, false, true, false);
    case 2: return NEGF_K(false, false, true, true);
    case 3: return NEGF_K(true, false, false, false);
    case 4: return NEGF_K(true, false, true, false);
    case 5: return NEGF_K(true, false, true, true);
    case 6: return NEGF_K(true, true, false, false);
    case 7: return NEGF_K(true, true, true, false);
    default: return NEGF_K(true, true, true, true);
  }
#undef NEGF_K
}

// The 3M kernel is the default; NEGF_ZGEMM=4m selects the four-product kernel.
static bool use_3m() {
  static const bool v = [] {
    const char* e = std::getenv("NEGF_ZGEMM");
    return !(e && (e[0] == '4'));
  }();
  return v;
}

template <bool PRE>
static ZGemmKernel pick_smallk_t(int ia, int ib) {
  switch (ia * 3 + ib) {
    case 0: return zgemm3m_smallk_kernel<false, false, false, false, PRE>;
    case 1: return zgemm3m_smallk_kernel<false, false, true, false, PRE>;
    case 2: return zgemm3m_smallk_kernel<false, false, true, true, PRE>;
    case 3: return zgemm3m_smallk_kernel<true, false, false, false, PRE>;
    case 4: return zgemm3m_smallk_kernel<true, false, true, false, PRE>;
    case 5: return zgemm3m_smallk_kernel<true, false, true, true, PRE>;
    case 6: return zgemm3m_smallk_kernel<true, true, false, false, PRE>;
    case 7: return zgemm3m_smallk_kernel<true, true, true, false, PRE>;
    default: return zgemm3m_smallk_kernel<true, true, true, true, PRE>;
  }
}

static ZGemmKernel pick_smallk(char opA, char opB, bool pre) {
  const int ia = opA == 'N' ? 0 : (opA == 'T' ? 1 : 2);
  const int ib = opB == 'N' ? 0 : (opB == 'T' ? 1 : 2);
  return pre ? pick_smallk_t<true>(ia, ib) : pick_smallk_t<false>(ia, ib);
}

static ZGemmKernel pick_kernel(char opA, char opB, bool pre, bool g3m) {
  int ia = opA == 'N' ? 0 : (opA == 'T' ? 1 : 2);
  int ib = opB == 'N' ? 0 : (opB == 'T' ? 1 : 2);
  if (g3m) return pre ? pick_kernel_t<true, true>(ia, ib) : pick_kernel_t<false, true>(ia, ib);
  return pre ? pick_kernel_t<true, false>(ia, ib) : pick_kernel_t<false, false>(ia, ib);
}

size_t zgemm_smem_bytes() { return gemm::SMEM_BYTES; }

// Raise the dynamic shared-memory limit of one op variant (both accumulator
// initialisations) on the current device; done when a plan is finalised,
// outside any stream capture.
cudaError_t zgemm_prepare(char opA, char opB) {
  for (int v = 0; v < 4; ++v) {
    cudaError_t e = cudaFuncSetAttribute(pick_kernel(opA, opB, v & 1, v & 2), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)gemm::SMEM_BYTES);
    if (e != cudaSuccess) return e;
  }
  for (int v = 0; v < 2; ++v) {
    cudaError_t e = cudaFuncSetAttribute(pick_smallk(opA, opB, v & 1), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)gemm_sk::SMEM_BYTES);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The small-K kernel serves steps whose problems all have k <= 32 when the
// 3M form is in use (form 2, or the default without NEGF_ZGEMM=4m);
// NEGF_ZGEMM_SMALLK=0 keeps them on the 64 x 64 kernel.
bool zgemm_smallk_ok(int form, int max_k) {
  static const bool on = [] {
    const char* e = std::getenv("NEGF_ZGEMM_SMALLK");
    return !(e && e[0] == '0');
  }();
  return on && max_k <= 32 && (form == 2 || (form == 0 && use_3m()));
}

int zgemm_tiles_smallk(int m, int n) {
  if (m <= 0 || n <= 0) return 0;
  return ((m + gemm_sk::BM - 1) / gemm_sk::BM) * ((n + gemm_sk::BN - 1) / gemm_sk::BN);
}

// True when the problem qualifies for the accumulator preload variant.
bool zgemm_preload_ok(const ZGemmProblem& p) {
  return p.k > 0 && p.Cin != nullptr && p.alpha.y == 0.0 && p.beta.y == 0.0 &&
         (p.alpha.x == 1.0 || p.alpha.x == -1.0) && (p.beta.x == 1.0 || p.beta.x == -1.0);
}

// Host launchers.  probs_dev / tile_start_dev are device arrays prepared by
// the caller (tile_start has nprob entries, exclusive prefix sum of tile
// counts).  preload may only be set when zgemm_preload_ok holds for every
// problem of the launch.
cudaError_t launch_zgemm_batched_ex(char opA, char opB, bool preload, const ZGemmProblem* probs_dev,
                                    const int* tile_start_dev, int nprob, int total_tiles, cudaStream_t stream,
                                    int form, int uniform_tiles) {
  if (nprob <= 0 || total_tiles <= 0) return cudaSuccess;
  static const bool uniform_on = [] {
    const char* e = std::getenv("NEGF_ZGEMM_UNIFORM");
    return !(e && e[0] == '0');
  }();
  // every problem has uniform_tiles tiles: the kernels locate their problem by
  // division (signalled by a negative count)
  if (uniform_on && uniform_tiles > 0 && (long long)uniform_tiles * nprob == total_tiles) nprob = -uniform_tiles;
  if (form == 3) {  // small-K 3M kernel; tiles counted by zgemm_tiles_smallk
    pick_smallk(opA, opB, preload)<<<total_tiles, gemm_sk::THREADS, gemm_sk::SMEM_BYTES, stream>>>(
        probs_dev, tile_start_dev, nprob);
    return cudaGetLastError();
  }
  const bool g3m = form == 0 ? use_3m() : form == 2;
  pick_kernel(opA, opB, preload, g3m)<<<total_tiles, g3m ? gemm3m::THREADS : gemm::THREADS, gemm::SMEM_BYTES,
                                        stream>>>(probs_dev, tile_start_dev, nprob);
  return cudaGetLastError();
}

// The four-product kernel without accumulator preload.
cudaError_t launch_zgemm_batched(char opA, char opB, const ZGemmProblem* probs_dev, const int* tile_start_dev,
                                 int nprob, int total_tiles, cudaStream_t stream) {
  if (nprob <= 0 || total_tiles <= 0) return cudaSuccess;
  pick_kernel(opA, opB, false, false)<<<total_tiles, gemm::THREADS, gemm::SMEM_BYTES, stream>>>(
      probs_dev, tile_start_dev, nprob);
  return cudaGetLastError();
}

int zgemm_tiles(int m, int n) {
  if (m <= 0 || n <= 0) return 0;
  return ((m + gemm::BM - 1) / gemm::BM) * ((n + gemm::BN - 1) / gemm::BN);
}

}  // namespace negf
