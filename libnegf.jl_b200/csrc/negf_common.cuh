// Shared device/host definitions of the B200 NEGF block kernels.
//
// Element type: complex128 stored as double2 {re, im}, blocks column-major with
// a leading dimension (the layout of a Julia Matrix{ComplexF64}, which the
// reference's CPU backend hands to LAPACK, src/backend_cpu.jl:7-20).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace negf {

using cplx = double2;

__host__ __device__ inline cplx cmake(double r, double i) { return make_double2(r, i); }
__host__ __device__ inline cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline cplx cneg(cplx a) { return make_double2(-a.x, -a.y); }
// a - b*c
__host__ __device__ inline cplx cfms(cplx a, cplx b, cplx c) {
  return make_double2(a.x - (b.x * c.x - b.y * c.y), a.y - (b.x * c.y + b.y * c.x));
}
// 1/a (Smith's algorithm: scaled to avoid overflow in |a|^2)
__host__ __device__ inline cplx cinv(cplx a) {
  double ar = a.x, ai = a.y;
  if (fabs(ar) >= fabs(ai)) {
    double r = ai / ar, d = ar + ai * r;
    return make_double2(1.0 / d, -r / d);
  } else {
    double r = ar / ai, d = ai + ar * r;
    return make_double2(r / d, -1.0 / d);
  }
}
// |re| + |im|: the pivot magnitude LAPACK's izamax uses (dcabs1)
__host__ __device__ inline double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

// One problem of a batched complex GEMM:
//   C = alpha * op(A) * op(B) + beta * Cin + diag * I
// op(A) is m x k, op(B) is k x n, C and Cin are m x n (Cin may alias C).
// k == 0 turns the problem into C = beta * Cin + diag * I.
struct ZGemmProblem {
  const cplx* A;
  const cplx* B;
  const cplx* Cin;
  cplx* C;
  const cplx* diag_ptr;  // when set, diag is read from device memory (per-energy shift)
  int m, n, k;
  int lda, ldb, ldc, ldcin;
  int pad_;
  cplx alpha, beta, diag;
};

// One matrix of a batched Gauss-Jordan inversion: W (n x n, ld) is inverted in
// place; scratch F (n x nb) and Bbuf (nb x n) hold the rank-nb update of a
// panel; used (n bytes) and piv (n ints) persist across panels; out receives
// the un-permuted inverse (n x n, ldo).
struct ZInvProblem {
  cplx* W;
  cplx* F;
  cplx* Bbuf;
  uint8_t* used;
  int* piv;
  cplx* out;
  int* info;   // set to (global column + 1) on a zero pivot, else left untouched
  int n, ld, ldo, pad_;
};

// One matrix of a batched LU (zlu.cu).
struct ZLuProblem {
  cplx* A;       // n x n, ld
  int* ipiv;     // n (0-based global pivot rows)
  cplx* Linv;    // scratch nb x nb (inverse of the panel's unit-lower block)
  cplx* T;       // scratch nb x n (A12 copy)
  int* info;
  int n, ld;
  int nopiv;     // 1: no row interchanges (the pivot of column c is row c)
  int pad_;
};

// One matrix of a batched triangular inverse (zlu.cu).
struct ZTriProblem {
  const cplx* A;  // packed factors, n x n, lda
  cplx* X;        // output, n x n, ldx
  int n, lda, ldx, pad_;
};

// Digit split of one real-and-imaginary operand view for the Ozaki GEMM
// (zgemm_ozaki.cu): Y[r][k] = X[r*sr + k*sk] (conjugated when conj), R x K.
// The digits are stored pre-tiled for the tensor cores: for every real
// operand p (re, im, re + im), row tile t (tile_rows rows) and 32-wide K chunk
// c one contiguous block of 7 digit slices in the canonical K-major
// core-matrix order (r, k) -> (k / 16) * R * 16 + (r / 8) * 128 + (r % 8) * 16
// + k % 16; blocks ordered [p][t][c]. Left operand (tile_rows 128): each slice
// is its own R = 128 matrix. Right operand (tile_rows 64): the seven slices
// form one R = 448 matrix (row 64 i + r for slice i).
struct OzSplitProblem {
  const cplx* X;
  long long sr, sk;
  int rows, cols, rows_pad, k_pad;
  int conj, tile_rows;  // tile_rows: 128 (left operand) or 64 (right operand)
  int8_t* slices;       // 3 * 7 * rows_pad * k_pad int8 digits
  int* exps;            // [rows_pad] power-of-two row scales
};

// One complex product of the Ozaki GEMM: C = alpha A B + beta Cin + diag I
// from the digit slices of A (m x k) and of B^T (n x k).
struct OzMmaProblem {
  const int8_t* SA;
  const int* eA;
  const int8_t* SB;
  const int* eB;
  cplx* C;
  const cplx* Cin;
  const cplx* diag_ptr;
  int m, n, m_pad, n_pad, k_pad, ldc, ldcin, pad_;
  cplx alpha, beta, diag;
};

// Elementwise block operations (ZBlockOp::kind).
enum ZOpKind : int {
  ZOP_COPY = 0,        // C = A
  ZOP_CTRANSPOSE = 1,  // C = A^H   (A is n x m)
  ZOP_AXPBY = 2,       // C = alpha*A + beta*C
  ZOP_FILL = 3,        // C = alpha (every entry)
  ZOP_IDENTITY = 4,    // C = alpha * I
  ZOP_HERM_PART = 5,   // C = (A + A^H)/2
  ZOP_GAMMA = 6,       // C = i (A - A^H)   (broadening of a self-energy)
  ZOP_CTRANS_AXPBY = 7,  // C = alpha*A^H + beta*C   (A is n x m)
  ZOP_ADD_DIAG = 8,    // C[r, r] += alpha
};

struct ZBlockOp {
  const cplx* A;
  cplx* C;
  const cplx* alpha_ptr;  // when set, alpha is read from device memory
  int m, n, lda, ldc;
  int kind, pad_;
  cplx alpha, beta;
};

}  // namespace negf
