// Mixed-precision complex GEMM: FP64-accurate products on the INT8 tensor
// cores (tcgen05.mma kind::i8, S32 accumulators in TMEM) by Ozaki-style
// splitting (Ozaki et al., "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication", 2012; the
// integer variant of Ootomo, Ozaki and Yokota, "DGEMM on integer matrix
// multiplication unit", 2024).
//
//   * split: every row r of a real operand Y (R x K) gets a power-of-two scale
//     2^e_r > max_k |Y[r,k]|; Y[r,k] = 2^e_r * sum_{s=1..7} d_s 2^(-7 s) with
//     signed digits |d_s| <= 127 (int8), so seven digits carry 49 bits;
//   * product: sum_k A[r,k] B[c,k] = 2^(eA_r + eB_c) sum_d 2^(-7 d) acc_d with
//     acc_d = sum_{s+t=d} sum_k dA_s dB_t; every acc_d is an exact int32 sum
//     (|acc_d| <= 7 * K * 127^2 < 2^31 for K <= 1024); only pairs with
//     s + t <= 8 are formed (28 of 49), which bounds the error near 2^-49
//     relative to |A||B| (measured ~1e-13 per complex product);
//   * complex: 3M (Gauss) -- P1 = Ar Br, P2 = Ai Bi, P3 = (Ar+Ai)(Br+Bi),
//     Re = P1 - P2, Im = P3 - P1 - P2 -- the three real operands of a side
//     share one scale per row;
//   * the MMA kernel: one CTA per 128 x 64 output tile; 2-stage cp.async
//     staging of the seven digit slices of A and B per 32-byte K chunk into
//     the canonical K-major (no swizzle) UMMA layout; one thread issues the
//     28 MMAs of a chunk into seven TMEM accumulators (one per digit
//     diagonal d = 2..8, 7 x 64 columns) and commits them to an mbarrier;
//     after each real product the eight warps drain the accumulators into FP64
//     registers (warp w reads TMEM lanes 32(w%4).., columns 32(w/4)..).
// All mbarrier waits are bounded: on time-out the kernel records an error
// code, waits (bounded) for its MMAs in flight, releases its TMEM and returns.
#include "negf_common.cuh"

#include <cstdint>

namespace negf {

namespace oz {
constexpr int S = 7;            // digits per operand
constexpr int NP = 3;           // real products (3M)
constexpr int TM = 128, TN = 64, KC = 32;
constexpr int THREADS = 256;
constexpr int A_SLICE = TM * KC;  // bytes of one digit slice of the A tile
constexpr int B_SLICE = TN * KC;
constexpr int STAGE = S * (A_SLICE + B_SLICE);
constexpr int STAGES = 2;
constexpr int TMEM_COLS = 512;  // 7 x 64 used
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 1.9 GHz per wait
}  // namespace oz

// ---------------------------------------------------------------------------
// split

__global__ void __launch_bounds__(256) ozaki_split_kernel(const OzSplitProblem* __restrict__ probs) {
  const OzSplitProblem q = probs[blockIdx.y];
  const int r0 = blockIdx.x * 32;
  if (r0 >= q.rows_pad) return;
  const int rr = threadIdx.x & 31, kg = threadIdx.x >> 5;  // 32 rows x 8 K groups
  const int r = r0 + rr;
  const bool live = r < q.rows;
  __shared__ double red[8][33];
  __shared__ int sh_e[32];
  // pass 1: max over k of |re| + |im| (bounds |re|, |im| and |re + im|)
  double mx = 0.0;
  if (live)
    for (int k = kg; k < q.cols; k += 8) {
      cplx v = q.X[r * q.sr + k * q.sk];
      mx = fmax(mx, fabs(v.x) + fabs(v.y));
    }
  red[kg][rr] = mx;
  __syncthreads();
  if (kg == 0) {
    double m = red[0][rr];
    for (int j = 1; j < 8; ++j) m = fmax(m, red[j][rr]);
    int e = 0;
    if (m > 0.0) frexp(m, &e);  // m < 2^e
    sh_e[rr] = e;
    if (r < q.rows_pad) q.exps[r] = e;
  }
  __syncthreads();
  const int e = sh_e[rr];
  const size_t plane = (size_t)q.rows_pad * q.k_pad;
  // pass 2: digits, 16 consecutive k per store
  for (int kc = kg; kc * 16 < q.k_pad; kc += 8) {
    int8_t dig[3][oz::S][16];
#pragma unroll 1
    for (int j = 0; j < 16; ++j) {
      const int k = kc * 16 + j;
      double comp[3] = {0.0, 0.0, 0.0};
      if (live && k < q.cols) {
        cplx v = q.X[r * q.sr + k * q.sk];
        double re = v.x, im = q.conj ? -v.y : v.y;
        comp[0] = re; comp[1] = im; comp[2] = re + im;
      }
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        double y = ldexp(comp[p], 7 - e);  // |y| < 128
#pragma unroll
        for (int s = 0; s < oz::S; ++s) {
          double d = trunc(y);
          dig[p][s][j] = static_cast<int8_t>(d);
          y = (y - d) * 128.0;
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int s = 0; s < oz::S; ++s) {
        int4 pack;
        int8_t* b = reinterpret_cast<int8_t*>(&pack);
#pragma unroll
        for (int j = 0; j < 16; ++j) b[j] = dig[p][s][j];
        *reinterpret_cast<int4*>(q.slices + (size_t)(p * oz::S + s) * plane + (size_t)r * q.k_pad + kc * 16) = pack;
      }
  }
}

// ---------------------------------------------------------------------------
// MMA

__device__ __forceinline__ uint32_t oz_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, no swizzle
}

__device__ __forceinline__ void oz_cp16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

// bounded wait for completion number `target` (1-based) of an mbarrier whose
// completions we have seen `seen` of; returns false on time-out
__device__ __forceinline__ bool oz_wait(uint32_t mbar, uint32_t& seen, uint32_t target) {
  while (seen < target) {
    uint32_t done = 0;
    const long long t0 = clock64();
    while (!done && clock64() - t0 < oz::WAIT_CYCLES) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
          : "=r"(done)
          : "r"(mbar), "r"(seen & 1u));
    }
    if (!done) return false;
    ++seen;
  }
  return true;
}

__global__ void __launch_bounds__(oz::THREADS, 1)
    ozaki_mma_kernel(const OzMmaProblem* __restrict__ probs, const int* __restrict__ tile_start, int nprob,
                     int* __restrict__ err) {
  using namespace oz;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int eA_sh[TM], eB_sh[TN];

  int bid = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= bid) lo = mid; else hi = mid - 1;
  }
  const OzMmaProblem q = probs[lo];
  const int t = bid - tile_start[lo];
  const int tiles_m = q.m_pad / TM;
  const int m0 = (t % tiles_m) * TM, n0 = (t / tiles_m) * TN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&mbar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  for (int i = tid; i < TM; i += THREADS) eA_sh[i] = q.eA[m0 + i];
  for (int i = tid; i < TN; i += THREADS) eB_sh[i] = q.eB[n0 + i];
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_base_sh;

  const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
  const int kch = q.k_pad / KC;
  const int total = NP * kch;
  const size_t planeA = (size_t)q.m_pad * q.k_pad, planeB = (size_t)q.n_pad * q.k_pad;
  const uint32_t sbase = oz_smem(smem);
  uint32_t seen[STAGES] = {0, 0}, uses[STAGES] = {0, 0};
  bool ok = true;

  // copy the seven A and B digit slices of iteration `it` into stage `st`
  auto load = [&](int it, int st) {
    const int p = it / kch, kc = it % kch;
    const uint32_t sA = sbase + st * STAGE, sB = sA + S * A_SLICE;
    for (int idx = tid; idx < S * TM * 2; idx += THREADS) {  // (slice, row, 16-byte half)
      int s = idx / (TM * 2), rem = idx % (TM * 2), r = rem >> 1, h = rem & 1;
      const int8_t* src = q.SA + (size_t)(p * S + s) * planeA + (size_t)(m0 + r) * q.k_pad + kc * KC + h * 16;
      oz_cp16(sA + s * A_SLICE + h * (TM * 16) + (r >> 3) * 128 + (r & 7) * 16, src);
    }
    for (int idx = tid; idx < S * TN * 2; idx += THREADS) {
      int s = idx / (TN * 2), rem = idx % (TN * 2), r = rem >> 1, h = rem & 1;
      const int8_t* src = q.SB + (size_t)(p * S + s) * planeB + (size_t)(n0 + r) * q.k_pad + kc * KC + h * 16;
      oz_cp16(sB + s * B_SLICE + h * (TN * 16) + (r >> 3) * 128 + (r & 7) * 16, src);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };

  // FP64 accumulators of this thread: tile row 32*(warp%4)+lane, columns 32*(warp/4) + j
  double cr[32], ci[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) { cr[j] = 0.0; ci[j] = 0.0; }
  const int qd = warp & 3, half = warp >> 2;

  if (total > 0) load(0, 0);
  for (int it = 0; it < total && ok; ++it) {
    const int st = it & 1;
    if (it + 1 < total) {
      const int ns = (it + 1) & 1;
      // MMAs of it-1 done (the decision is made CTA-uniform before anyone leaves the loop)
      ok = __syncthreads_and(oz_wait(oz_smem(&mbar[ns]), seen[ns], uses[ns]) ? 1 : 0) != 0;
      if (!ok) break;
      load(it + 1, ns);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::);
    __syncthreads();
    const int p = it / kch, kc = it % kch;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const uint32_t sA = sbase + st * STAGE, sB = sA + S * A_SLICE;
      for (int d = 2; d <= S + 1; ++d) {
        bool first = true;
        for (int s = 1; s <= S; ++s) {
          const int tt = d - s;
          if (tt < 1 || tt > S) continue;
          uint64_t da = oz_desc(sA + (s - 1) * A_SLICE, TM * 16, 128);
          uint64_t db = oz_desc(sB + (tt - 1) * B_SLICE, TN * 16, 128);
          uint32_t acc = (kc == 0 && first) ? 0u : 1u;
          first = false;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                  tmem + (uint32_t)((d - 2) * TN)),
              "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          oz_smem(&mbar[st])));
    }
    uses[st] += 1;
    if (kc == kch - 1) {
      // product p finished: drain the seven accumulators into FP64
      ok = __syncthreads_and(oz_wait(oz_smem(&mbar[st]), seen[st], uses[st]) ? 1 : 0) != 0;
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const double sr = (p == 2) ? 0.0 : (p == 0 ? 1.0 : -1.0);  // P1 -> +Re, P2 -> -Re
      const double si = (p == 2) ? 1.0 : -1.0;                   // P3 -> +Im, P1, P2 -> -Im
#pragma unroll
      for (int c8 = 0; c8 < 4; ++c8) {
        double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < S; ++d) {
          uint32_t x[8];
          uint32_t addr = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(d * TN + half * 32 + c8 * 8);
          asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                       : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]),
                         "=r"(x[7])
                       : "r"(addr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::);
          const double w = ldexp(1.0, -7 * (d + 2));
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = fma((double)(int32_t)x[j], w, v[j]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          cr[c8 * 8 + j] = fma(sr, v[j], cr[c8 * 8 + j]);
          ci[c8 * 8 + j] = fma(si, v[j], ci[c8 * 8 + j]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::);
      __syncthreads();  // accumulators free for the next product
    }
  }

  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // bounded wait for the MMAs this CTA issued, then release TMEM
    for (int s = 0; s < STAGES; ++s) oz_wait(oz_smem(&mbar[s]), seen[s], uses[s]);
  } else {
    // C = alpha * 2^(eA + eB) (Re, Im) + beta * Cin + diag * I
    const int row = qd * 32 + lane;
    const int r = m0 + row;
    const cplx dg = q.diag_ptr ? *q.diag_ptr : q.diag;
    const bool has_cin = q.Cin && (q.beta.x != 0.0 || q.beta.y != 0.0);
    if (r < q.m) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int cl = half * 32 + j;
        const int c = n0 + cl;
        if (c >= q.n) continue;
        const int e = eA_sh[row] + eB_sh[cl];
        const double xr = ldexp(cr[j], e), xi = ldexp(ci[j], e);
        cplx v;
        v.x = q.alpha.x * xr - q.alpha.y * xi;
        v.y = q.alpha.x * xi + q.alpha.y * xr;
        if (has_cin) {
          cplx b = q.Cin[r + (size_t)c * q.ldcin];
          v.x += q.beta.x * b.x - q.beta.y * b.y;
          v.y += q.beta.x * b.y + q.beta.y * b.x;
        }
        if (r == c) { v.x += dg.x; v.y += dg.y; }
        q.C[r + (size_t)c * q.ldc] = v;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// 86 KB of stages; the request is raised to 120 KB so that one CTA (and its
// 512 TMEM columns) owns an SM at a time instead of a second CTA blocking in
// tcgen05.alloc.
size_t ozaki_mma_smem_bytes() {
  size_t need = (size_t)oz::STAGES * oz::STAGE;
  return need < 120 * 1024 ? 120 * 1024 : need;
}

cudaError_t ozaki_prepare() {
  return cudaFuncSetAttribute(ozaki_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ozaki_mma_smem_bytes());
}

cudaError_t launch_ozaki_split(const void* probs, int nprob, int max_rows_pad, cudaStream_t st) {
  if (nprob <= 0) return cudaSuccess;
  dim3 grid((max_rows_pad + 31) / 32, nprob);
  ozaki_split_kernel<<<grid, 256, 0, st>>>(static_cast<const OzSplitProblem*>(probs));
  return cudaGetLastError();
}

cudaError_t launch_ozaki_mma(const void* probs, const int* tile_start, int nprob, int total_tiles, int* err,
                             cudaStream_t st) {
  if (nprob <= 0 || total_tiles <= 0) return cudaSuccess;
  ozaki_mma_kernel<<<total_tiles, oz::THREADS, ozaki_mma_smem_bytes(), st>>>(
      static_cast<const OzMmaProblem*>(probs), tile_start, nprob, err);
  return cudaGetLastError();
}

}  // namespace negf
