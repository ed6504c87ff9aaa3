// Mixed-precision complex GEMM: FP64-accurate products on the INT8 tensor
// cores (tcgen05.mma kind::i8, S32 accumulators in TMEM) by Ozaki-style
// splitting (Ozaki et al., "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication", 2012; the
// integer variant of Ootomo, Ozaki and Yokota, "DGEMM on integer matrix
// multiplication unit", 2024).
//
//   * split: every row r of a real operand Y (R x K) gets a power-of-two scale
//     2^e_r > max_k |Y[r,k]|; x = rint(Y[r,k] 2^(54 - e_r)) is a 54-bit
//     integer, written as seven balanced base-256 digits x = sum_i s_i
//     256^(6 - i) (top digit |s_0| <= 64, lower digits in [-128, 127]); the
//     digits are the bytes of x + C6 (lower ones minus 128), so the split is a
//     rounding (FP64 adds), an add and byte permutes per element
//     (representation error <= 2^(e_r - 55));
//   * product: sum_k A[r,k] B[c,k] = 2^(eA_r + eB_c) sum_D 2^(-12 - 8D) acc_D,
//     acc_D = sum_{i+j=D} sum_k sA_i sB_j; each acc_D is an exact int32 sum
//     (|acc_D| <= 7 * K * 2^14 < 2^31 for K < 18000).  Two accuracy levels:
//     the 34 digit pairs i + j <= 7 (the dropped ones sum to below
//     2^(eA_r + eB_c - 59) K: a product as accurate as an FP64 one), or the 28
//     pairs i + j <= 6 (dropped ones below 2^(eA_r + eB_c - 51.4) K, within 3x
//     of the FP64 rounding bound K u |a| |b|);
//   * complex: 3M (Gauss) -- P1 = Ar Br, P2 = Ai Bi, P3 = (Ar+Ai)(Br+Bi),
//     Re = P1 - P2, Im = P3 - P1 - P2 -- the three real operands of a side
//     share one scale per row and xr + xi is formed exactly in integers;
//   * storage: the split writes, per (real operand, row tile, 32-byte K chunk),
//     one contiguous block of the seven digit slices already in the canonical
//     K-major core-matrix layout of the tensor-core shared-memory descriptors,
//     so that the product kernel moves a whole stage with two bulk copies; the
//     right operand's seven slices form one 448-row matrix, so that one MMA
//     multiplies a left digit slice by several right digit slices at once;
//   * the product kernel (persistent, one CTA per SM, 128 x 64 output tiles,
//     288 threads, warp-specialised): one producer lane streams stages with
//     cp.async.bulk into a 5-deep mbarrier ring, refilling each slot as its
//     MMAs retire; another producer lane issues the
//     12 (or 10) MMAs (N = 64..256) of each stage into eight (seven) TMEM
//     accumulators, one per digit diagonal of 64 columns; after each real
//     product eight warps drain the accumulators into FP64 registers, and at
//     the end of a tile they write C = alpha A B + beta Cin + diag I while the
//     next tile's first product runs on the tensor cores.
// Every mbarrier wait is bounded: a role whose pipeline wait runs past the
// limit (a kernel argument, default ~1 s) records an error code and raises an
// abort flag that ends the other roles' waits; the CTA then waits (bounded by
// the default limit) for its copies and MMAs in flight, releases TMEM and
// returns, and the host reports the error.
#include "negf_common.cuh"

#include <atomic>
#include <cstdint>
#include <vector>

namespace negf {

namespace oz {
constexpr int S = 7;             // base-256 digits per operand
constexpr int NP = 3;            // real products (3M)
constexpr int ND_MAX = 8;        // digit diagonals D = i + j = 0..7 at most (34 digit pairs)
constexpr int TM = 128, TN = 64, KC = 32;
constexpr int A_SLICE = TM * KC;        // 4096 bytes
constexpr int B_SLICE = TN * KC;        // 2048 bytes
constexpr int A_BLOCK = S * A_SLICE;    // 28 KiB: one stage of the left operand
constexpr int B_BLOCK = S * B_SLICE;    // 14 KiB
constexpr int STAGE = A_BLOCK + B_BLOCK;
constexpr int STAGES = 5;
constexpr int DRAIN_WARPS = 8;          // warps 0..7 drain and write the epilogue
// warps 8..11 (one warpgroup) are the producers: lane 0 of warp 8 issues the
// MMAs, lane 0 of warp 9 streams the stages.  Registers are moved from the producer
// warpgroup to the two drain warpgroups after launch (setmaxnreg): launch
// 384 x 168 = 64512 = 256 x 232 (drain) + 128 x 40 (producer).
constexpr int THREADS = 32 * DRAIN_WARPS + 128;
constexpr int REGS_LAUNCH = 168, REGS_DRAIN = 232, REGS_PRODUCER = 40;
static_assert(THREADS * REGS_LAUNCH == 32 * DRAIN_WARPS * REGS_DRAIN + 128 * REGS_PRODUCER, "register split");
constexpr int TMEM_COLS = 512;          // ND_MAX x TN
static_assert(TMEM_COLS == ND_MAX * TN, "one accumulator per digit diagonal");
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 1.9 GHz per wait
constexpr int SPLIT_ROWS = 64;          // rows per split CTA
// offset that turns the six lower bytes of x + C6 into digits + 128:
// C6 = 128 (256^6 - 1) / 255
constexpr long long C6 = 128LL * ((1LL << 48) - 1) / 255;
}  // namespace oz

// weight 2^(-12 - 8D) of digit diagonal D (a compile-time constant)
__host__ __device__ constexpr double oz_diag_weight(int D) {
  double w = 0x1p-12;
  for (int d = 0; d < D; ++d) w *= 0x1p-8;
  return w;
}

// exact int32 -> double on the FP64 pipe: the bits 0x43300000:(x ^ 2^31) are
// 2^52 + 2^31 + x, from which one exact subtraction leaves x
__device__ __forceinline__ double oz_i2d(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 4503601774854144.0;
}

// ---------------------------------------------------------------------------
// split

__device__ __forceinline__ uint32_t oz_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// rint(y) for |y| < 2^54 as an int64, on the FP64 add pipe: with M = 2^52 +
// 2^51, the low word of t + M is rint(t) for |t| < 2^31; y is taken in two
// 27-bit halves (both steps exact but the final rounding of the low half)
__device__ __forceinline__ long long oz_rint54(double y) {
  constexpr double M = 6755399441055744.0;  // 2^52 + 2^51
  const double t = y * 0x1p-27;
  const double th = (t + M) - M;            // rint(t), |th| <= 2^27
  const int hi = __double2loint(t + M);
  const double yl = fma(-th, 0x1p27, y);    // exact, |yl| <= 2^26
  const int lo = __double2loint(yl + M);
  return ((long long)hi << 27) + lo;
}

// gather byte `bb` of four words into one word (element j -> byte j)
__device__ __forceinline__ uint32_t oz_gather(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t bb) {
  const uint32_t sel = bb | ((bb + 4u) << 4);
  return __byte_perm(__byte_perm(w0, w1, sel), __byte_perm(w2, w3, sel), 0x5410);
}

// Digit store of one lane: 4 consecutive k of row `grow` in each K half of
// chunk c (row[16h + j] = element c*32 + 16h + 4kq + j, in shared memory), as
// 3 real operands x 7 byte slices in the product kernel's core-matrix layout.
// A warp whose lanes are (row % 8) * 4 + kq covers one 128-byte core matrix
// per store.
__device__ __forceinline__ void oz_store_digits(const OzSplitProblem& q, int grow, int kq, int c, const cplx* row,
                                                double f1, double fi, double f2) {
  const int TR = q.tile_rows;
  const int t = grow / TR, rt = grow % TR;
  const int kch = q.k_pad / oz::KC;
  // left operand (128-row tiles): slice i at i * 4096, K halves 2048 apart;
  // right operand (64-row tiles): the seven slices form one 448-row K-major
  // matrix (row = 64 i + r), so slice i starts at i * 1024, K halves 7168 apart
  const size_t slice = TR == oz::TM ? (size_t)TR * oz::KC : (size_t)TR * 16;
  const size_t half = TR == oz::TM ? (size_t)TR * 16 : (size_t)oz::S * TR * 16;
  const size_t block = (size_t)oz::S * TR * oz::KC;
  const int ntiles = q.rows_pad / TR;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    // offset fixed-point values x + C6 of re, im and re + im of 4 consecutive
    // k: byte 6 is the top digit, bytes 5..0 are the lower digits + 128
    uint32_t lo[3][4], hi[3][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const cplx v = row[16 * h + j];
      const long long xr = oz_rint54(v.x * f1 * f2);
      const long long xi = oz_rint54(v.y * fi * f2);
      const long long x3[3] = {xr + oz::C6, xi + oz::C6, xr + xi + oz::C6};
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        lo[p][j] = (uint32_t)x3[p];
        hi[p][j] = (uint32_t)((unsigned long long)x3[p] >> 32);
      }
    }
    const size_t inrow = (size_t)h * half + (size_t)(rt >> 3) * 128 + (rt & 7) * 16 + 4 * kq;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      uint8_t* base = reinterpret_cast<uint8_t*>(q.slices) + ((size_t)(p * ntiles + t) * kch + c) * block + inrow;
#pragma unroll
      for (int i = 0; i < oz::S; ++i) {
        const int bi = oz::S - 1 - i;  // byte of digit slice i
        uint32_t w = bi < 4 ? oz_gather(lo[p][0], lo[p][1], lo[p][2], lo[p][3], bi)
                            : oz_gather(hi[p][0], hi[p][1], hi[p][2], hi[p][3], bi - 4);
        if (i > 0) w ^= 0x80808080u;  // lower digits: byte - 128
        *reinterpret_cast<uint32_t*>(base + i * slice) = w;
      }
    }
  }
}

// Scale factors of a row with exponent e: x = rint(v 2^(54 - e)) through two
// exact power-of-two factors (|x| <= 2^54); fi carries the conjugation.
__device__ __forceinline__ void oz_row_factors(int e, int conj, double& f1, double& fi, double& f2) {
  const int sh = 54 - e;
  f1 = ldexp(1.0, sh / 2);
  f2 = ldexp(1.0, sh - sh / 2);
  fi = conj ? -f1 : f1;
}

// Single-read split: the CTA stages R whole rows (all k_pad columns) in shared
// memory once, takes the row maxima there and writes the digits from there,
// so each operand element is read from memory once.  For k_pad <= 512
// (R = 32, 16, 8 rows for k_pad <= 128, 256, 512; <= 66 KB of staging).
template <int R>
__global__ void __launch_bounds__(256, 3) ozaki_split1_kernel(const OzSplitProblem* __restrict__ probs, int ldt) {
  const OzSplitProblem q = probs[blockIdx.y];
  const int r0 = blockIdx.x * R;
  if (r0 >= q.rows_pad) return;
  extern __shared__ __align__(16) unsigned char split_smem[];
  cplx* tile = reinterpret_cast<cplx*>(split_smem);  // R rows x ldt (>= k_pad + 1)
  __shared__ int sh_e[R];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int kp = q.k_pad;
  // stage: zero-filled outside Y; consecutive threads take the contiguous index
  if (q.sr == 1) {
    for (int idx = tid; idx < R * kp; idx += 256) {
      const int r = idx % R, k = idx / R, gr = r0 + r;
      const bool in = gr < q.rows && k < q.cols;
      const void* src = in ? (const void*)(q.X + (long long)gr + (long long)k * q.sk) : (const void*)probs;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(oz_smem(tile + (size_t)r * ldt + k)),
                   "l"(src), "r"(in ? 16 : 0)
                   : "memory");
    }
  } else {
    for (int idx = tid; idx < R * kp; idx += 256) {
      const int k = idx % kp, r = idx / kp, gr = r0 + r;
      const bool in = gr < q.rows && k < q.cols;
      const void* src = in ? (const void*)(q.X + (long long)gr * q.sr + k) : (const void*)probs;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(oz_smem(tile + (size_t)r * ldt + k)),
                   "l"(src), "r"(in ? 16 : 0)
                   : "memory");
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  // row maxima of |re| + |im| (bounds |re|, |im| and |re + im|), a warp per row
  for (int r = warp; r < R; r += 8) {
    double mx = 0.0;
    for (int k = lane; k < kp; k += 32) {
      const cplx v = tile[(size_t)r * ldt + k];
      mx = fmax(mx, fabs(v.x) + fabs(v.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);  // mx < 2^e
      sh_e[r] = e;
      q.exps[r0 + r] = e;
    }
  }
  __syncthreads();
  // digits: work items (group of 8 rows, 32-wide K chunk), a warp each
  const int kch = kp / oz::KC;
  const int kq = lane & 3;
  for (int item = warp; item < (R / 8) * kch; item += 8) {
    const int g = item % (R / 8), c = item / (R / 8);
    const int rl = g * 8 + (lane >> 2);
    double f1, fi, f2;
    oz_row_factors(sh_e[rl], q.conj, f1, fi, f2);
    oz_store_digits(q, r0 + rl, kq, c, tile + (size_t)rl * ldt + c * oz::KC + 4 * kq, f1, fi, f2);
  }
}

__global__ void __launch_bounds__(256, 3) ozaki_split_kernel(const OzSplitProblem* __restrict__ probs) {
  const OzSplitProblem q = probs[blockIdx.y];
  const int r0 = blockIdx.x * oz::SPLIT_ROWS;
  if (r0 >= q.rows_pad) return;
  // two staging buffers of rows r0..r0+63 x one 32-wide K chunk (dynamic)
  extern __shared__ __align__(16) unsigned char split_smem[];
  cplx(*tile)[oz::SPLIT_ROWS][33] = reinterpret_cast<cplx(*)[oz::SPLIT_ROWS][33]>(split_smem);
  __shared__ double red[4][oz::SPLIT_ROWS];
  __shared__ int sh_e[oz::SPLIT_ROWS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool rows_contig = q.sr == 1;
  const int kch = q.k_pad / oz::KC;

  // pass 1: row maxima of |re| + |im| (bounds |re|, |im| and |re + im|),
  // streamed along whichever index is contiguous in memory
  if (rows_contig) {
    const int r = tid & 63, gr = r0 + r;
    double mx = 0.0;
    if (gr < q.rows)
#pragma unroll 4
      for (int k = tid >> 6; k < q.cols; k += 4) {
        const cplx v = q.X[(long long)gr + (long long)k * q.sk];
        mx = fmax(mx, fabs(v.x) + fabs(v.y));
      }
    red[tid >> 6][r] = mx;
    __syncthreads();
    if (tid < oz::SPLIT_ROWS) {
      const double m = fmax(fmax(red[0][tid], red[1][tid]), fmax(red[2][tid], red[3][tid]));
      int e = 0;
      if (m > 0.0) frexp(m, &e);  // m < 2^e
      sh_e[tid] = e;
      q.exps[r0 + tid] = e;
    }
  } else {
    for (int j = 0; j < 8; ++j) {
      const int r = warp + 8 * j, gr = r0 + r;
      double mx = 0.0;
      if (gr < q.rows)
#pragma unroll 4
        for (int k = lane; k < q.cols; k += 32) {
          const cplx v = q.X[(long long)gr * q.sr + k];
          mx = fmax(mx, fabs(v.x) + fabs(v.y));
        }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) {
        int e = 0;
        if (mx > 0.0) frexp(mx, &e);
        sh_e[r] = e;
        q.exps[r0 + r] = e;
      }
    }
  }
  __syncthreads();

  // pass 2: a warp owns 8 rows; lane = (row % 8) * 4 + k quad, so one warp
  // store covers a 128-byte core matrix of one digit slice
  const int rl = warp * 8 + (lane >> 2);
  const int kq = lane & 3;
  double f1, fi, f2;
  oz_row_factors(sh_e[rl], q.conj, f1, fi, f2);
  // asynchronous staging of chunk c into buffer b (zero-filled outside Y)
  auto stage = [&](int c, int b) {
    const int kbase = c * oz::KC;
    if (rows_contig) {
      const int r = tid & 63, gr = r0 + r;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int kk = (tid >> 6) + 4 * j, gk = kbase + kk;
        const bool in = gr < q.rows && gk < q.cols;
        const void* src = in ? (const void*)(q.X + (long long)gr + (long long)gk * q.sk) : (const void*)probs;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(oz_smem(&tile[b][r][kk])), "l"(src),
                     "r"(in ? 16 : 0)
                     : "memory");
      }
    } else {
      const int kk = tid & 31, gk = kbase + kk;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int r = (tid >> 5) + 8 * j, gr = r0 + r;
        const bool in = gr < q.rows && gk < q.cols;
        const void* src = in ? (const void*)(q.X + (long long)gr * q.sr + gk) : (const void*)probs;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(oz_smem(&tile[b][r][kk])), "l"(src),
                     "r"(in ? 16 : 0)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  stage(0, 0);
  for (int c = 0; c < kch; ++c) {
    const int b = c & 1;
    if (c + 1 < kch) {
      stage(c + 1, b ^ 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    oz_store_digits(q, r0 + rl, kq, c, &tile[b][rl][4 * kq], f1, fi, f2);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// product


__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, no swizzle
}

__device__ __forceinline__ bool oz_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the completion of the mbarrier phase of the given parity.
// Returns false when another role raised the abort flag (watch) or after
// `limit` cycles, in which case it raises the flag and records the error.
__device__ __forceinline__ bool oz_wait(uint32_t mbar, uint32_t parity, volatile int* abort_flag, int* err,
                                        bool watch, long long limit = oz::WAIT_CYCLES) {
  if (oz_try(mbar, parity)) return true;
  const long long t0 = clock64();
  while (!oz_try(mbar, parity)) {
    if (watch && *abort_flag) return false;
    if (clock64() - t0 > limit) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// The same wait for a whole warp that has nothing else to do: lane 0 polls
// with a back-off, so that idle warps leave the issue slots to the thread that
// feeds the tensor cores; the result is uniform across the warp.
__device__ __forceinline__ bool oz_wait_warp(uint32_t mbar, uint32_t parity, volatile int* abort_flag, int* err,
                                             long long limit) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) {
    const long long t0 = clock64();
    while (true) {
      if (oz_try(mbar, parity)) {
        ok = 1;
        break;
      }
      if (*abort_flag) break;
      if (clock64() - t0 > limit) {
        *abort_flag = 1;
        atomicExch(err, 1);
        break;
      }
      __nanosleep(256);
    }
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ void oz_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

struct OzTile {
  int prob, mt, nt, tiles_m, tiles_n, kch;
};

// tile t of a batched launch from the host-built map: x = problem, y = m tile
// | n tile << 16, z = K chunks | m tiles << 16, w = n tiles (n fastest, so
// that consecutive tiles share the left operand)
__device__ __forceinline__ OzTile oz_tile(const int4* __restrict__ tile_map, int t) {
  const int4 v = tile_map[t];
  OzTile r;
  r.prob = v.x;
  r.mt = v.y & 0xFFFF;
  r.nt = v.y >> 16;
  r.kch = v.z & 0xFFFF;
  r.tiles_m = v.z >> 16;
  r.tiles_n = v.w;
  return r;
}

// One MMA of a stage: A digit slice I times the contiguous B digit slices
// J0 .. J0 + NJ - 1 (one N = 64 NJ product) into the accumulators of the
// diagonals D = I + J0 .. I + J0 + NJ - 1. INIT marks the MMAs that write
// accumulators first (all of whose columns are first writes); compile-time
// operands keep the issuing thread at one instruction sequence per MMA.
template <int I, int J0, int NJ, int INIT>
__device__ __forceinline__ void oz_mma(uint32_t tmem, uint64_t dA0, uint64_t dB0, bool first_chunk) {
  constexpr uint32_t idesc =
      (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NJ * oz::TN >> 3) << 17) | ((uint32_t)(oz::TM >> 4) << 24);
  // the start-address field of a descriptor is addr >> 4
  const uint64_t da = dA0 + (uint64_t)(I * (oz::A_SLICE >> 4));
  const uint64_t db = dB0 + (uint64_t)(J0 * (oz::TN * 16 >> 4));
  const uint32_t acc = (INIT && first_chunk) ? 0u : 1u;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem + (uint32_t)((I + J0) * oz::TN)),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The digit pairs of a stage: ND = 8 -- the 34 pairs i + j <= 7 as 12 MMAs
// (products as accurate as FP64 ones); ND = 7 -- the 28 pairs i + j <= 6 as
// 10 MMAs.  The order makes every accumulator's first write an INIT one (on
// the first K chunk of a product).
template <int ND>
__device__ __forceinline__ void oz_stage_mmas(uint32_t tmem, uint64_t dA0, uint64_t dB0, bool first_chunk) {
  static_assert(ND == 7 || ND == 8, "digit diagonals");
  oz_mma<0, 0, 4, 1>(tmem, dA0, dB0, first_chunk);
  oz_mma<0, 4, 3, 1>(tmem, dA0, dB0, first_chunk);
  oz_mma<1, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
  if (ND == 8) {
    oz_mma<1, 4, 2, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<1, 6, 1, 1>(tmem, dA0, dB0, first_chunk);
    oz_mma<2, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<2, 4, 2, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<3, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<3, 4, 1, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<4, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<5, 0, 3, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<6, 0, 2, 0>(tmem, dA0, dB0, first_chunk);
  } else {
    oz_mma<1, 4, 2, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<2, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<2, 4, 1, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<3, 0, 4, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<4, 0, 3, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<5, 0, 2, 0>(tmem, dA0, dB0, first_chunk);
    oz_mma<6, 0, 1, 0>(tmem, dA0, dB0, first_chunk);
  }
}

// Persistent: CTA b computes tiles b, b + G, b + 2G, ... (G = gridDim.x).
// Warp-specialised: warps 0..7 drain the accumulators after every real product
// and write each tile's epilogue; warp 8 is the producer -- lane 0 issues the
// MMAs, lane 1 streams the stages into the ring.  Because neither producer
// takes part in the drains or the epilogue, the stage ring keeps streaming and
// the next product's MMAs are issued as soon as the previous product is
// drained, so the first product of a tile runs under the previous tile's
// epilogue.
template <int ND>
__global__ void __launch_bounds__(oz::THREADS, 1)
    ozaki_mma_kernel(const OzMmaProblem* __restrict__ probs, const int4* __restrict__ tile_map, int total_tiles,
                     int* __restrict__ err, long long wait_cycles) {
  using namespace oz;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], accf_bar, acce_bar, done_bar;
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  // per (tile parity, warp): a copy of the tile's problem descriptor, staged
  // at the start of a tile.  The column exponents and scales stay in
  // registers (lane j holds column j's) and reach the other lanes by shuffle:
  // while the tensor cores stream their operands, shared-memory loads wait
  // hundreds of cycles each
  constexpr int PROB_WORDS = (int)(sizeof(OzMmaProblem) / 4);
  static_assert(sizeof(OzMmaProblem) % 16 == 0 && PROB_WORDS <= 40, "epilogue staging layout");
  __shared__ __align__(16) int ep_sh[2][DRAIN_WARPS][40];
  volatile int* abort_flag = &abort_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;
  const int my_tiles = (int)blockIdx.x < total_tiles ? (total_tiles - (int)blockIdx.x + G - 1) / G : 0;
  const int my_products = my_tiles * NP;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tmem_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&full_bar[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&empty_bar[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&accf_bar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&acce_bar)), "r"(DRAIN_WARPS));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&done_bar)));
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_sh;
  const uint32_t sbase = oz_smem(smem);
  const uint32_t full0 = oz_smem(&full_bar[0]), empty0 = oz_smem(&empty_bar[0]);

  if (warp >= DRAIN_WARPS) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REGS_PRODUCER));
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REGS_DRAIN));
  }
  if (warp >= DRAIN_WARPS) {
    if (lane != 0 || warp > DRAIN_WARPS + 1) {
      // the rest of the producer warpgroup has no work
    } else if (warp == DRAIN_WARPS + 1) {
      // ---- loader: every stage of every product of every tile, in order;
      // a slot is refilled once the MMAs of its previous stage retired (its
      // empty barrier); per slot, the parity of its last load is kept for the
      // final wait
      uint32_t loaded = 0, last_ph = 0;
      int ls = 0, use = 0;  // ring slot and how many times the ring wrapped
      bool ok = true;
      for (int q = 0; q < my_tiles && ok; ++q) {
        const OzTile t = oz_tile(tile_map, (int)blockIdx.x + q * G);
        const OzMmaProblem& pq = probs[t.prob];
        for (int p = 0; p < NP && ok; ++p) {
          const int8_t* la = pq.SA + (size_t)(p * t.tiles_m + t.mt) * t.kch * A_BLOCK;
          const int8_t* lb = pq.SB + (size_t)(p * t.tiles_n + t.nt) * t.kch * B_BLOCK;
          for (int c = 0; c < t.kch; ++c) {
            if (use > 0 && !oz_wait(empty0 + ls * 8, (uint32_t)((use - 1) & 1), abort_flag, err, true, wait_cycles)) {
              ok = false;
              break;
            }
            const uint32_t fb = full0 + ls * 8;
            const uint32_t dA = sbase + ls * STAGE, dB = dA + A_BLOCK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(STAGE) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dA),
                "l"(la + (size_t)c * A_BLOCK), "r"(A_BLOCK), "r"(fb)
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dB),
                "l"(lb + (size_t)c * B_BLOCK), "r"(B_BLOCK), "r"(fb)
                : "memory");
            loaded |= 1u << ls;
            last_ph = (last_ph & ~(1u << ls)) | ((uint32_t)(use & 1) << ls);
            if (++ls == STAGES) {
              ls = 0;
              ++use;
            }
          }
        }
      }
      // every issued copy lands before the CTA exits (default limit, also
      // after an abort: issued copies always complete)
      for (int s = 0; s < STAGES; ++s)
        if (loaded & (1u << s)) oz_wait(full0 + s * 8, (last_ph >> s) & 1u, abort_flag, err, false);
    } else {
      // ---- MMA issuer: product P waits for the drain of P - 1 (the
      // accumulators are reused), then issues its stages as they land
      const uint64_t descA0 = oz_desc(sbase, TM * 16, 128), descB0 = oz_desc(sbase + A_BLOCK, S * TN * 16, 128);
      int ms = 0;
      uint32_t mph = 0;
      bool ok = true;
      for (int P = 0; P < my_products && ok; ++P) {
        const int kch = oz_tile(tile_map, (int)blockIdx.x + (P / NP) * G).kch;  // read before the wait
        if (P > 0 && !oz_wait(oz_smem(&acce_bar), (uint32_t)((P - 1) & 1), abort_flag, err, true, wait_cycles))
          break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        for (int c = 0; c < kch; ++c) {
          if (!oz_wait(full0 + ms * 8, mph, abort_flag, err, true, wait_cycles)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::);
          const uint64_t soff = (uint64_t)(ms * (STAGE >> 4));
          oz_stage_mmas<ND>(tmem, descA0 + soff, descB0 + soff, c == 0);
          oz_commit(empty0 + ms * 8);
          if (c == kch - 1) oz_commit(oz_smem(&accf_bar));
          if (++ms == STAGES) {
            ms = 0;
            mph ^= 1u;
          }
        }
      }
      // all MMAs of this CTA complete before TMEM is released (default limit)
      oz_commit(oz_smem(&done_bar));
      oz_wait(oz_smem(&done_bar), 0, abort_flag, err, false);
    }
  } else {
    // ---- warps 0..7: drain each product, then the tile epilogue; warp w
    // reads TMEM lanes 32 (w % 4).. and columns 32 (w / 4)..
    //
    // On this hardware FP64 arithmetic makes no progress while the tensor
    // cores run INT8 MMAs (the two share a datapath), so the drains run
    // between products and the epilogue keeps its FP64 work to two
    // multiplications per output (four more with a Cin term): the column and
    // row scales are combined as exponents in integer arithmetic.
    const int qd = warp & 3, hh = warp >> 2;
    bool ok = true;
    // this tile's inputs: row exponent (per lane), column exponent (lane j
    // holds column j's), alpha; the next tile's are fetched before this
    // tile's epilogue so that their latency is hidden
    int my_eA = 0, my_eB = 0;
    cplx al = make_double2(0.0, 0.0);
    auto fetch = [&](int q, const OzTile& t, int& eA, int& eB, cplx& a) {
      const int* src = reinterpret_cast<const int*>(probs + t.prob);
      int* eps = ep_sh[q & 1][warp];
      for (int w = lane; w < PROB_WORDS; w += 32) eps[w] = src[w];
      const OzMmaProblem* pp = probs + t.prob;
      eB = pp->eB[t.nt * TN + hh * 32 + lane];
      eA = pp->eA[t.mt * TM + qd * 32 + lane];
      a = pp->alpha;
    };
    OzTile tq{};
    if (my_tiles > 0) {
      tq = oz_tile(tile_map, (int)blockIdx.x);
      fetch(0, tq, my_eA, my_eB, al);
      __syncwarp();
    }
    for (int q = 0; q < my_tiles && ok; ++q) {
      double cr[32], ci[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) { cr[j] = 0.0; ci[j] = 0.0; }
      for (int p = 0; p < NP; ++p) {
        const int P = q * NP + p;
        if (!oz_wait_warp(oz_smem(&accf_bar), (uint32_t)(P & 1), abort_flag, err, wait_cycles)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        // product p adds v to Re with sign sr and to Im with sign si (P1: +Re,
        // -Im; P2: -Re, -Im; P3: +Im); alpha is folded in: (kr, ki) = alpha (sr, si)
        const double sr = (p == 2) ? 0.0 : (p == 0 ? 1.0 : -1.0);
        const double si = (p == 2) ? 1.0 : -1.0;
        const double kr = al.x * sr - al.y * si, ki = al.x * si + al.y * sr;
#pragma unroll
        for (int c8 = 0; c8 < 4; ++c8) {
          double v[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = 0.0;
          // all ND diagonals of the column group in one TMEM round trip
          uint32_t x[ND][8];
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const uint32_t addr = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(d * TN + hh * 32 + c8 * 8);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(x[d][0]), "=r"(x[d][1]), "=r"(x[d][2]), "=r"(x[d][3]), "=r"(x[d][4]), "=r"(x[d][5]),
                           "=r"(x[d][6]), "=r"(x[d][7])
                         : "r"(addr));
          }
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const double w = oz_diag_weight(d);
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = fma(oz_i2d(x[d][j]), w, v[j]);
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            cr[c8 * 8 + j] = fma(kr, v[j], cr[c8 * 8 + j]);
            ci[c8 * 8 + j] = fma(ki, v[j], ci[c8 * 8 + j]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::);
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(oz_smem(&acce_bar)) : "memory");
      }
      if (!ok) break;
      // the next tile's inputs (into the other staging slot)
      OzTile tn{};
      int nx_eA = 0, nx_eB = 0;
      cplx nx_al = make_double2(0.0, 0.0);
      if (q + 1 < my_tiles) {
        tn = oz_tile(tile_map, (int)blockIdx.x + (q + 1) * G);
        fetch(q + 1, tn, nx_eA, nx_eB, nx_al);
      }
      // C = alpha 2^(eA + eB) (Re, Im) + beta Cin + diag I (alpha already in
      // cr, ci), from the staged descriptor and the shuffled column exponents
      // (all lanes take part in the shuffles; rows past m skip the memory
      // accesses); Cin is read one group of columns ahead of the stores.  The
      // producer keeps the tensor cores busy with the next tile meanwhile.
      const OzMmaProblem& ps = *reinterpret_cast<const OzMmaProblem*>(ep_sh[q & 1][warp]);
      const int r = tq.mt * TM + qd * 32 + lane;
      const bool row_ok = r < ps.m;
      const int pn = ps.n, ldc = ps.ldc, ldcin = ps.ldcin;
      const cplx beta = ps.beta;
      cplx* const Cout = ps.C;
      const cplx* const Cin = ps.Cin;
      const cplx dg = ps.diag_ptr ? *ps.diag_ptr : ps.diag;
      const bool has_cin = row_ok && Cin && (beta.x != 0.0 || beta.y != 0.0);
      // every exponent of the warp's rows and columns within +-500: the scale
      // 2^(eA + eB) is a normal double built from its exponent bits
      const bool pow2_ok = __all_sync(0xffffffffu, my_eA >= -500 && my_eA <= 500 && my_eB >= -500 && my_eB <= 500);
      const int c0 = tq.nt * TN + hh * 32;
      constexpr int GW = 4;  // columns per group
      cplx cb[GW], cn[GW];
#pragma unroll
      for (int jj = 0; jj < GW; ++jj)
        cn[jj] = (has_cin && c0 + jj < pn) ? Cin[r + (size_t)(c0 + jj) * ldcin] : make_double2(0.0, 0.0);
#pragma unroll
      for (int g8 = 0; g8 < 32 / GW; ++g8) {
#pragma unroll
        for (int jj = 0; jj < GW; ++jj) cb[jj] = cn[jj];
        if (g8 < 32 / GW - 1) {
#pragma unroll
          for (int jj = 0; jj < GW; ++jj) {
            const int c = c0 + (g8 + 1) * GW + jj;
            cn[jj] = (has_cin && c < pn) ? Cin[r + (size_t)c * ldcin] : make_double2(0.0, 0.0);
          }
        }
        int eB[GW];
#pragma unroll
        for (int jj = 0; jj < GW; ++jj) eB[jj] = __shfl_sync(0xffffffffu, my_eB, g8 * GW + jj);
#pragma unroll
        for (int jj = 0; jj < GW; ++jj) {
          const int j = g8 * GW + jj;
          const int c = c0 + j;
          if (!row_ok || c >= pn) continue;
          const int e = my_eA + eB[jj];
          double xr, xi;
          if (pow2_ok) {
            const double sc = __longlong_as_double((long long)(e + 1023) << 52);
            xr = cr[j] * sc;
            xi = ci[j] * sc;
          } else {
            xr = ldexp(cr[j], e);
            xi = ldexp(ci[j], e);
          }
          cplx v;
          if (has_cin) {
            v.x = fma(beta.x, cb[jj].x, fma(-beta.y, cb[jj].y, xr));
            v.y = fma(beta.x, cb[jj].y, fma(beta.y, cb[jj].x, xi));
          } else {
            v.x = xr;
            v.y = xi;
          }
          if (r == c) {
            v.x += dg.x;
            v.y += dg.y;
          }
          Cout[r + (size_t)c * ldc] = v;
        }
      }
      tq = tn;
      my_eA = nx_eA;
      my_eB = nx_eB;
      al = nx_al;
      __syncwarp();
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// measurement: dense INT8 tensor-core throughput of one CTA per SM issuing
// back-to-back 128 x 256 x 32 kind::i8 MMAs on resident shared-memory
// operands (the roofline denominator of the product kernel)

__global__ void __launch_bounds__(128, 1) ozaki_probe_kernel(int rounds, int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tm;
  for (int i = threadIdx.x; i < (4096 + 8192) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sm)[i] = 0u;
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tm)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t t = tm;
  if (threadIdx.x == 0) {
    const uint64_t da = oz_desc(oz_smem(sm), 128 * 16, 128), db = oz_desc(oz_smem(sm) + 4096, 256 * 16, 128);
    constexpr uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    for (int it = 0; it < rounds; ++it) {
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const uint32_t acc = (it > 0 || u >= 2) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                t + (uint32_t)((u & 1) * 256)),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
      }
    }
    oz_commit(oz_smem(&bar));
    int dummy = 0;
    if (!oz_wait(oz_smem(&bar), 0, &dummy, err, false)) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t), "r"(512));
  }
}

cudaError_t ozaki_probe_int8(double* tops) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  constexpr int smem = 16 * 1024, rounds = 625;
  int* err = nullptr;
  if ((e = cudaMalloc(&err, sizeof(int))) != cudaSuccess) return e;
  cudaMemset(err, 0, sizeof(int));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  ozaki_probe_kernel<<<sms, 128, smem>>>(20, err);
  cudaEventRecord(a);
  ozaki_probe_kernel<<<sms, 128, smem>>>(rounds, err);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  int h = 0;
  cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(err);
  if (e != cudaSuccess) return e;
  if (h) return cudaErrorLaunchTimeout;
  if (tops) *tops = 2.0 * 128 * 256 * 32 * 32.0 * rounds * sms / (ms * 1e9);
  return cudaSuccess;
}

// measurement: does FP64 arithmetic progress while the same SM's tensor cores
// run INT8 MMAs?  Thread 0 issues back-to-back 128 x 256 x 32 kind::i8 MMAs
// (when `mma`); warps 1..7 run eight independent DFMA chains per thread (when
// `fp64`).  Per CTA, out[0] = cycles of the MMA thread, out[1] = mean cycles
// of the FP64 warps.  The drain of the product kernel is placed by this
// figure: FP64 work beside the MMAs only waits for them.
__global__ void __launch_bounds__(256, 1) ozaki_overlap_probe_kernel(int mma, int fp64, int rounds, int iters,
                                                                      long long* out, double* sink, int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tm;
  __shared__ long long fp_cycles;
  for (int i = threadIdx.x; i < (4096 + 8192) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sm)[i] = 0x01010101u;
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tm)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    fp_cycles = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(oz_smem(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t t = tm;
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      const long long t0 = clock64();
      if (mma) {
        const uint64_t da = oz_desc(oz_smem(sm), 128 * 16, 128), db = oz_desc(oz_smem(sm) + 4096, 256 * 16, 128);
        constexpr uint32_t idesc =
            (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        for (int it = 0; it < rounds; ++it) {
#pragma unroll
          for (int u = 0; u < 32; ++u) {
            const uint32_t acc = (it > 0 || u >= 2) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                    t + (uint32_t)((u & 1) * 256)),
                "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
          }
        }
      }
      oz_commit(oz_smem(&bar));
      int dummy = 0;
      if (!oz_wait(oz_smem(&bar), 0, &dummy, err, false)) atomicExch(err, 1);
      out[2 * blockIdx.x] = clock64() - t0;
    }
  } else {
    const long long t0 = clock64();
    double d[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) d[k] = 1.0 + threadIdx.x * 1e-3 + k;
    if (fp64) {
      for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) d[k] = fma(d[k], 0.999999, 1e-7);
      }
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += d[k];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
    if ((threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&fp_cycles),
                                           (unsigned long long)(clock64() - t0));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (threadIdx.x == 0) out[2 * blockIdx.x + 1] = fp_cycles / 7;
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t), "r"(512));
  }
}

cudaError_t ozaki_probe_overlap(double* fp64_alone, double* fp64_beside_mma, double* mma_alone) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  constexpr int smem = 160 * 1024;  // one CTA per SM
  constexpr int rounds = 20, iters = 3000;
  e = cudaFuncSetAttribute(ozaki_overlap_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  long long* out = nullptr;
  double* sink = nullptr;
  int* err = nullptr;
  if ((e = cudaMalloc(&out, sizeof(long long) * 2 * sms)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&sink, sizeof(double) * 256 * sms)) != cudaSuccess) { cudaFree(out); return e; }
  if ((e = cudaMalloc(&err, sizeof(int))) != cudaSuccess) { cudaFree(out); cudaFree(sink); return e; }
  cudaMemset(err, 0, sizeof(int));
  std::vector<long long> h(2 * (size_t)sms);
  double res[3][2] = {};
  const int modes[3][2] = {{0, 1}, {1, 1}, {1, 0}};  // (mma, fp64)
  for (int m = 0; m < 3 && e == cudaSuccess; ++m) {
    for (int rep = 0; rep < 2; ++rep)  // the first launch warms up
      ozaki_overlap_probe_kernel<<<sms, 256, smem>>>(modes[m][0], modes[m][1], rounds, iters, out, sink, err);
    e = cudaMemcpy(h.data(), out, sizeof(long long) * h.size(), cudaMemcpyDeviceToHost);
    for (int b = 0; b < sms; ++b) {
      res[m][0] += (double)h[2 * b] / sms;
      res[m][1] += (double)h[2 * b + 1] / sms;
    }
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(out);
  cudaFree(sink);
  cudaFree(err);
  if (e != cudaSuccess) return e;
  if (herr) return cudaErrorLaunchTimeout;
  if (fp64_alone) *fp64_alone = res[0][1];
  if (fp64_beside_mma) *fp64_beside_mma = res[1][1];
  if (mma_alone) *mma_alone = res[2][0];
  return cudaSuccess;
}

size_t ozaki_mma_smem_bytes() { return (size_t)oz::STAGES * oz::STAGE; }

constexpr size_t kSplitSmem = 2 * oz::SPLIT_ROWS * 33 * sizeof(cplx);

// single-read split: rows per CTA for a step whose largest k_pad is kp (0: two-pass kernel)
constexpr int split1_rows(int kp) { return kp <= 128 ? 32 : kp <= 256 ? 16 : kp <= 512 ? 8 : 0; }
constexpr size_t split1_smem(int kp) { return (size_t)split1_rows(kp) * (kp + 1) * sizeof(cplx); }
constexpr size_t kSplit1SmemMax = 32 * 129 * sizeof(cplx);  // the largest of the three cases (66,048 B)
static_assert(split1_smem(128) <= kSplit1SmemMax && split1_smem(256) <= kSplit1SmemMax &&
                  split1_smem(512) <= kSplit1SmemMax,
              "single-read split staging");

cudaError_t ozaki_prepare() {
  // the register split of the product kernel assumes the launch allocates
  // exactly REGS_LAUNCH registers per thread; with fewer, setmaxnreg.inc of
  // the drain warps could never be satisfied, so such a build is refused
  for (const void* f : {(const void*)ozaki_mma_kernel<7>, (const void*)ozaki_mma_kernel<8>}) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
    if (a.numRegs != oz::REGS_LAUNCH) return cudaErrorInvalidKernelImage;
  }
  cudaError_t e = cudaFuncSetAttribute(ozaki_mma_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ozaki_mma_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ozaki_mma_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ozaki_mma_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ozaki_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ozaki_split1_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSplit1SmemMax);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ozaki_split1_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSplit1SmemMax);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ozaki_split1_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSplit1SmemMax);
  return e;
}

cudaError_t launch_ozaki_split(const void* probs, int nprob, int max_rows_pad, int max_k_pad, cudaStream_t st) {
  if (nprob <= 0) return cudaSuccess;
  const OzSplitProblem* p = static_cast<const OzSplitProblem*>(probs);
  const int R = split1_rows(max_k_pad);
  if (R == 0) {
    dim3 grid((max_rows_pad + oz::SPLIT_ROWS - 1) / oz::SPLIT_ROWS, nprob);
    ozaki_split_kernel<<<grid, 256, kSplitSmem, st>>>(p);
    return cudaGetLastError();
  }
  // rows_pad is a multiple of 64, so of R; every problem's k_pad <= max_k_pad
  dim3 grid(max_rows_pad / R, nprob);
  const int ldt = max_k_pad + 1;
  const size_t smem = split1_smem(max_k_pad);
  if (R == 32) ozaki_split1_kernel<32><<<grid, 256, smem, st>>>(p, ldt);
  else if (R == 16) ozaki_split1_kernel<16><<<grid, 256, smem, st>>>(p, ldt);
  else ozaki_split1_kernel<8><<<grid, 256, smem, st>>>(p, ldt);
  return cudaGetLastError();
}

// Pipeline wait limit of the product kernel in clock cycles (process-wide;
// negf_set_tensor_wait_limit).
static std::atomic<long long> g_oz_wait_cycles{oz::WAIT_CYCLES};

void ozaki_set_wait_cycles(long long cycles) { g_oz_wait_cycles.store(cycles > 0 ? cycles : oz::WAIT_CYCLES); }

cudaError_t launch_ozaki_mma(const void* probs, const void* tile_map, int total_tiles, int* err, cudaStream_t st,
                             int pairs) {
  if (total_tiles <= 0) return cudaSuccess;
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
  }
  const int grid = total_tiles < sms ? total_tiles : sms;
  const auto* pr = static_cast<const OzMmaProblem*>(probs);
  const auto* tm = static_cast<const int4*>(tile_map);
  if (pairs == 28)
    ozaki_mma_kernel<7><<<grid, oz::THREADS, ozaki_mma_smem_bytes(), st>>>(pr, tm, total_tiles, err,
                                                                           g_oz_wait_cycles.load());
  else
    ozaki_mma_kernel<8><<<grid, oz::THREADS, ozaki_mma_smem_bytes(), st>>>(pr, tm, total_tiles, err,
                                                                           g_oz_wait_cycles.load());
  return cudaGetLastError();
}

}  // namespace negf
