// LU-based backend primitives and the block selected inverse
// (src/selected_inverse.jl:9-206) on the plan engine.
#include "../../include/negf_b200.h"
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

using namespace negf;

namespace {

constexpr cplx ONE{1.0, 0.0};
constexpr cplx MONE{-1.0, 0.0};
constexpr cplx ZERO{0.0, 0.0};

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(NEGF_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

int check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(NEGF_ERR_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
  return NEGF_SUCCESS;
}

ZGemmProblem gp(const cplx* A, int lda, const cplx* B, int ldb, cplx* C, int ldc, int m, int n, int k, cplx alpha,
                const cplx* Cin = nullptr, int ldcin = 1, cplx beta = ZERO) {
  ZGemmProblem p;
  p.A = A; p.B = B; p.Cin = Cin; p.C = C; p.diag_ptr = nullptr;
  p.m = m; p.n = n; p.k = k;
  p.lda = std::max(1, lda); p.ldb = std::max(1, ldb); p.ldc = std::max(1, ldc); p.ldcin = std::max(1, ldcin);
  p.pad_ = 0;
  p.alpha = alpha; p.beta = beta; p.diag = ZERO;
  return p;
}

ZBlockOp copy_op(const cplx* A, int lda, cplx* C, int ldc, int m, int n) {
  ZBlockOp o{};
  o.A = A; o.lda = lda; o.C = C; o.ldc = ldc; o.m = m; o.n = n; o.kind = ZOP_COPY;
  return o;
}

int run_sync(Plan& plan, cudaStream_t st, int* dinfo, int n, const char* what) {
  cudaError_t e = plan.run(st, false);
  if (e != cudaSuccess) return cuda_fail(e, what);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, what);
  if (dinfo) {
    std::vector<int> info(n);
    e = cudaMemcpy(info.data(), dinfo, sizeof(int) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, what);
    for (int s = 0; s < n; ++s)
      if (info[s]) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "%s: matrix %d is singular (zero pivot in column %d)", what, s, info[s]);
        return fail(NEGF_ERR_SINGULAR, buf);
      }
  }
  return NEGF_SUCCESS;
}

// LU request of one block with plan-owned scratch.
LuSpec lu_spec(Plan& plan, cplx* A, int n, int ld, int* info, bool nopiv) {
  const int nb = lu_panel_width(n);
  LuSpec s;
  s.A = A; s.n = n; s.ld = ld;
  s.ipiv = static_cast<int*>(plan.alloc(sizeof(int) * n));
  s.Linv = plan.alloc_c((size_t)nb * nb);
  s.T = plan.alloc_c((size_t)nb * n);
  s.info = info;
  s.nopiv = nopiv;
  return s;
}

TriSpec tri_spec(Plan& plan, const cplx* A, int n, int lda, cplx* X) {
  TriSpec t;
  t.A = A; t.n = n; t.lda = lda; t.X = X; t.ldx = n;
  t.T = plan.alloc_c((size_t)n * kTriNb);
  return t;
}

}  // namespace


namespace negf {

// Block_factorization! then Block_inverse! (src/selected_inverse.jl:9-55,
// :139-206) over systems with one block pattern (that of system 0); every step
// is one batched launch over all systems.
int build_selected_inverse(Plan& plan, std::vector<SelInvSystem>& S, int npl, int b, int mode, bool nopiv) {
  const int ns = static_cast<int>(S.size());
  auto at = [&](int s, int i, int j) -> cplx* { return S[s].A[(size_t)i * npl + j]; };
  for (int s = 0; s < ns; ++s)
    for (int i = 0; i < npl; ++i)
      for (int j = 0; j < npl; ++j)
        if ((at(s, i, j) != nullptr) != (at(0, i, j) != nullptr))
          return fail(NEGF_ERR_INVALID, "the systems of a batched selected inverse must share one block pattern");
  for (int i = 0; i < npl; ++i)
    if (!at(0, i, i)) return fail(NEGF_ERR_INVALID, "every diagonal block must be assigned");
  const size_t bb = (size_t)b * b;
  std::vector<std::vector<cplx*>> Uinv(ns, std::vector<cplx*>(npl)), Linv(ns, std::vector<cplx*>(npl));
  std::vector<cplx*> tmp(ns);
  for (int s = 0; s < ns; ++s) {
    for (int i = 0; i < npl; ++i) { Uinv[s][i] = plan.alloc_c(bb); Linv[s][i] = plan.alloc_c(bb); }
    tmp[s] = plan.alloc_c(bb * (size_t)std::max(2 * npl + 2, 10));
  }
  auto scratch = [&](int s, int k) { return tmp[s] + bb * k; };
  auto inverses = [&](int i) {
    std::vector<TriSpec> up, lo;
    for (int s = 0; s < ns; ++s) {
      up.push_back(tri_spec(plan, at(s, i, i), b, b, Uinv[s][i]));
      lo.push_back(tri_spec(plan, at(s, i, i), b, b, Linv[s][i]));
    }
    plan.trtri(up, true);
    plan.trtri(lo, false);
  };
  if (mode & 1) {
    // Block_factorization! (selected_inverse.jl:9-55).  Fill-in blocks are
    // pre-zeroed, so "assign a zero block, then gemm with beta = 0"
    // (:43-46) is the same as accumulating into them; a fill block that the
    // reference creates at step i is never read or written before step i.
    for (int i = 0; i < npl; ++i) {
      // :18, be_getrf! (backend_cpu.jl:255-265: LAPACK getrf whose pivots the
      // reference discards) or lu(NoPivot()), the factorisation :17 names
      std::vector<LuSpec> lus;
      for (int s = 0; s < ns; ++s) lus.push_back(lu_spec(plan, at(s, i, i), b, b, S[s].info + i, nopiv));
      plan.getrf(lus);
      inverses(i);
      std::vector<ZBlockOp> cp;
      std::vector<ZGemmProblem> g;
      for (int s = 0; s < ns; ++s) {
        int k = 0;
        for (int j = i + 1; j < npl; ++j) {
          if (at(s, j, i)) {                                         // :23  A[j,i] / U_ii
            cp.push_back(copy_op(at(s, j, i), b, scratch(s, k), b, b, b));
            g.push_back(gp(scratch(s, k), b, Uinv[s][i], b, at(s, j, i), b, b, b, b, ONE));
            ++k;
          }
          if (at(s, i, j)) {                                         // :27  L_ii \ A[i,j]
            cp.push_back(copy_op(at(s, i, j), b, scratch(s, k), b, b, b));
            g.push_back(gp(Linv[s][i], b, scratch(s, k), b, at(s, i, j), b, b, b, b, ONE));
            ++k;
          }
        }
      }
      plan.blockops(cp);
      plan.gemm('N', 'N', g);
      std::vector<ZGemmProblem> sch;                                 // :32-51 Schur updates
      for (int s = 0; s < ns; ++s)
        for (int kk = i + 1; kk < npl; ++kk) {
          if (!at(s, i, kk) || !at(s, kk, i)) continue;
          sch.push_back(gp(at(s, kk, i), b, at(s, i, kk), b, at(s, kk, kk), b, b, b, b, MONE, at(s, kk, kk), b, ONE));
          for (int l = kk + 1; l < npl; ++l) {
            if (!at(s, i, l) || !at(s, l, i)) continue;
            if (!at(s, kk, l) || !at(s, l, kk)) return fail(NEGF_ERR_INVALID, "missing fill-in block");
            sch.push_back(gp(at(s, kk, i), b, at(s, i, l), b, at(s, kk, l), b, b, b, b, MONE, at(s, kk, l), b, ONE));
            sch.push_back(gp(at(s, l, i), b, at(s, i, kk), b, at(s, l, kk), b, b, b, b, MONE, at(s, l, kk), b, ONE));
          }
        }
      plan.gemm('N', 'N', sch);
    }
  } else {
    for (int i = 0; i < npl; ++i) inverses(i);
  }
  if (!(mode & 2)) return NEGF_SUCCESS;
  // Block_inverse! (selected_inverse.jl:139-206)
  {
    const int i = npl - 1;                                           // :158 getri(A[N,N])
    std::vector<ZGemmProblem> g;
    for (int s = 0; s < ns; ++s) g.push_back(gp(Uinv[s][i], b, Linv[s][i], b, at(s, i, i), b, b, b, b, ONE));
    plan.gemm('N', 'N', g);
  }
  for (int i = npl - 2; i >= 0; --i) {
    std::vector<int> js;
    for (int j = i + 1; j < npl; ++j)
      if (at(0, i, j)) js.push_back(j);
    if (js.size() > 2) return fail(NEGF_ERR_INVALID, "Block_inverse! supports at most two upper neighbours per block row");
    for (int j : js)
      if (!at(0, j, i)) return fail(NEGF_ERR_INVALID, "Block_inverse! needs a symmetric block pattern");
    // Uij = sum_k A[i,k] A[k,j];  Lji = sum_k A[j,k] A[k,i]   (:161-169)
    std::vector<std::vector<int>> ks(js.size());
    size_t rounds = 0;
    for (size_t v = 0; v < js.size(); ++v) {
      for (int k = i + 1; k < npl; ++k)
        if (at(0, i, k) && at(0, k, js[v])) ks[v].push_back(k);
      rounds = std::max(rounds, ks[v].size());
    }
    auto U = [&](int s, size_t v) { return scratch(s, (int)v); };
    auto L = [&](int s, size_t v) { return scratch(s, 2 + (int)v); };
    auto T = [&](int s, size_t v) { return scratch(s, 4 + (int)v); };
    auto Aii = [&](int s) { return scratch(s, 6); };
    for (size_t r = 0; r < rounds; ++r) {
      std::vector<ZGemmProblem> g;
      for (int s = 0; s < ns; ++s)
        for (size_t v = 0; v < js.size(); ++v) {
          if (r >= ks[v].size()) continue;
          const int j = js[v], k = ks[v][r];
          g.push_back(gp(at(s, i, k), b, at(s, k, j), b, U(s, v), b, b, b, b, ONE, r ? U(s, v) : nullptr, b,
                         r ? ONE : ZERO));
          g.push_back(gp(at(s, j, k), b, at(s, k, i), b, L(s, v), b, b, b, b, ONE, r ? L(s, v) : nullptr, b,
                         r ? ONE : ZERO));
        }
      plan.gemm('N', 'N', g);
    }
    // Uij = -U_ii^{-1} Uij ;  Lji = -Lji L_ii^{-1}   (:172, :174)
    {
      std::vector<ZGemmProblem> g1, g2;
      for (int s = 0; s < ns; ++s)
        for (size_t v = 0; v < js.size(); ++v) {
          g1.push_back(gp(Uinv[s][i], b, U(s, v), b, T(s, v), b, b, b, b, MONE));
          g2.push_back(gp(L(s, v), b, Linv[s][i], b, scratch(s, 7 + (int)v), b, b, b, b, MONE));
        }
      plan.gemm('N', 'N', g1);
      plan.gemm('N', 'N', g2);
    }
    // Aii = sum_j Uij A[j,i]  (:183), then A[j,i] = Lji, A[i,j] = Uij (:185-187)
    for (size_t v = 0; v < js.size(); ++v) {
      std::vector<ZGemmProblem> g;
      for (int s = 0; s < ns; ++s)
        g.push_back(gp(T(s, v), b, at(s, js[v], i), b, Aii(s), b, b, b, b, ONE, v ? Aii(s) : nullptr, b,
                       v ? ONE : ZERO));
      plan.gemm('N', 'N', g);
    }
    std::vector<ZBlockOp> cp;
    for (int s = 0; s < ns; ++s) {
      if (js.empty()) {
        ZBlockOp z{};
        z.C = Aii(s); z.ldc = b; z.m = z.n = b; z.kind = ZOP_FILL;
        cp.push_back(z);
      }
      for (size_t v = 0; v < js.size(); ++v) {
        cp.push_back(copy_op(scratch(s, 7 + (int)v), b, at(s, js[v], i), b, b, b));
        cp.push_back(copy_op(T(s, v), b, at(s, i, js[v]), b, b, b));
      }
    }
    plan.blockops(cp);
    // A[i,i] = getri(A[i,i]) - Aii L_ii^{-1}   (:195-199)
    std::vector<ZGemmProblem> g1, g2;
    for (int s = 0; s < ns; ++s) {
      g1.push_back(gp(Aii(s), b, Linv[s][i], b, scratch(s, 9), b, b, b, b, ONE));
      g2.push_back(gp(Uinv[s][i], b, Linv[s][i], b, at(s, i, i), b, b, b, b, ONE, scratch(s, 9), b, MONE));
    }
    plan.gemm('N', 'N', g1);
    plan.gemm('N', 'N', g2);
  }
  return NEGF_SUCCESS;
}

}  // namespace negf

extern "C" {

int negf_zgetrf_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* const* ipiv,
                        int32_t* info, void* stream) {
  if (int r = check_device()) return r;
  if (nprob < 0 || (nprob > 0 && (!n || !A || !lda))) return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * std::max(1, nprob)));
    std::vector<LuSpec> specs;
    std::vector<int*> piv0(nprob, nullptr);
    for (int i = 0; i < nprob; ++i) {
      if (n[i] < 0 || n[i] > kMaxBlock) return fail(NEGF_ERR_INVALID, "n must be in [0, 1024]");
      if (n[i] == 0) continue;
      int nb = lu_panel_width(n[i]);
      LuSpec s;
      s.A = static_cast<cplx*>(A[i]); s.n = n[i]; s.ld = lda[i];
      s.ipiv = static_cast<int*>(plan.alloc(sizeof(int) * n[i]));
      s.Linv = plan.alloc_c((size_t)nb * nb);
      s.T = plan.alloc_c((size_t)nb * n[i]);
      s.info = dinfo + i;
      piv0[i] = s.ipiv;
      specs.push_back(s);
    }
    plan.getrf(specs);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = run_sync(plan, st, nullptr, 0, "negf_zgetrf_batched");
    if (rc) return rc;
    std::vector<int> h(std::max(1, nprob));
    if (cudaMemcpy(h.data(), dinfo, sizeof(int) * std::max(1, nprob), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(NEGF_ERR_CUDA, "negf_zgetrf_batched: info copy failed");
    for (int i = 0; i < nprob; ++i) {
      if (info) info[i] = h[i];
      if (ipiv && ipiv[i] && piv0[i]) {
        std::vector<int> p(n[i]);
        if (cudaMemcpy(p.data(), piv0[i], sizeof(int) * n[i], cudaMemcpyDeviceToHost) != cudaSuccess)
          return fail(NEGF_ERR_CUDA, "negf_zgetrf_batched: pivot copy failed");
        for (int& x : p) x += 1;  // LAPACK 1-based
        if (cudaMemcpy(ipiv[i], p.data(), sizeof(int) * n[i], cudaMemcpyHostToDevice) != cudaSuccess)
          return fail(NEGF_ERR_CUDA, "negf_zgetrf_batched: pivot copy failed");
      }
    }
    for (int i = 0; i < nprob; ++i)
      if (h[i] && !info) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "negf_zgetrf_batched: matrix %d is singular (U(%d,%d) = 0)", i, h[i], h[i]);
        return fail(NEGF_ERR_SINGULAR, buf);
      }
    return NEGF_SUCCESS;
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_ztrsm_batched(char side, char uplo, char trans, char diag, const double* alpha, int32_t nprob,
                       const int32_t* m, const int32_t* n, void* const* A, const int32_t* lda, void* const* B,
                       const int32_t* ldb, void* stream) {
  if (int r = check_device()) return r;
  if (trans != 'N') return fail(NEGF_ERR_INVALID, "only trans = 'N' is supported");
  if (!((uplo == 'U' && diag == 'N') || (uplo == 'L' && diag == 'U')))
    return fail(NEGF_ERR_INVALID, "supported triangles: upper non-unit, lower unit (the factors of getrf)");
  if ((side != 'L' && side != 'R') || !alpha || nprob < 0 || (nprob > 0 && (!m || !n || !A || !lda || !B || !ldb)))
    return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    const cplx al = make_double2(alpha[0], alpha[1]);
    std::vector<TriSpec> tri;
    std::vector<ZBlockOp> cp;
    std::vector<ZGemmProblem> g;
    for (int i = 0; i < nprob; ++i) {
      if (m[i] <= 0 || n[i] <= 0) continue;
      int t = side == 'L' ? m[i] : n[i];  // order of the triangle
      cplx* X = plan.alloc_c((size_t)t * t);
      tri.push_back(tri_spec(plan, static_cast<const cplx*>(A[i]), t, lda[i], X));
      cplx* Bc = plan.alloc_c((size_t)m[i] * n[i]);
      cp.push_back(copy_op(static_cast<const cplx*>(B[i]), ldb[i], Bc, m[i], m[i], n[i]));
      if (side == 'L')
        g.push_back(gp(X, t, Bc, m[i], static_cast<cplx*>(B[i]), ldb[i], m[i], n[i], t, al));
      else
        g.push_back(gp(Bc, m[i], X, t, static_cast<cplx*>(B[i]), ldb[i], m[i], n[i], t, al));
    }
    plan.trtri(tri, uplo == 'U');
    plan.blockops(cp);
    plan.gemm('N', 'N', g);
    return run_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_ztrsm_batched");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_zgetri_nopiv_batched(int32_t nprob, const int32_t* n, void* const* A, const int32_t* lda, void* stream) {
  if (int r = check_device()) return r;
  if (nprob < 0 || (nprob > 0 && (!n || !A || !lda))) return fail(NEGF_ERR_INVALID, "bad arguments");
  try {
    Plan plan;
    std::vector<TriSpec> up, lo;
    std::vector<ZGemmProblem> g;
    for (int i = 0; i < nprob; ++i) {
      if (n[i] <= 0) continue;
      cplx* X = plan.alloc_c((size_t)n[i] * n[i]);
      cplx* Y = plan.alloc_c((size_t)n[i] * n[i]);
      up.push_back(tri_spec(plan, static_cast<const cplx*>(A[i]), n[i], lda[i], X));
      lo.push_back(tri_spec(plan, static_cast<const cplx*>(A[i]), n[i], lda[i], Y));
      g.push_back(gp(X, n[i], Y, n[i], static_cast<cplx*>(A[i]), lda[i], n[i], n[i], n[i], ONE));
    }
    plan.trtri(up, true);
    plan.trtri(lo, false);
    plan.gemm('N', 'N', g);
    return run_sync(plan, static_cast<cudaStream_t>(stream), nullptr, 0, "negf_zgetri_nopiv_batched");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_selected_inverse(int32_t npl, int32_t b, void* const* Ab, const uint8_t* fill, int32_t mode, void* stream) {
  return negf_selected_inverse_batched(1, npl, b, Ab, fill, mode, 1, NEGF_PREC_FP64, stream);
}

int negf_selected_inverse_batched(int32_t nsys, int32_t npl, int32_t b, void* const* Ab, const uint8_t* fill,
                                  int32_t mode, int32_t pivoting, int32_t precision, void* stream) {
  if (int r = check_device()) return r;
  if (nsys <= 0 || npl <= 0 || b <= 0 || b > kMaxBlock || !Ab || mode < 1 || mode > 3 ||
      (precision != NEGF_PREC_FP64 && precision != NEGF_PREC_MIXED))
    return fail(NEGF_ERR_INVALID, "bad arguments");
  (void)fill;  // fill-in blocks arrive pre-zeroed; they act as assigned from the start (see the builder)
  try {
    Plan plan;
    plan.set_mixed(precision == NEGF_PREC_MIXED);
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * (size_t)nsys * npl));
    std::vector<SelInvSystem> sys(nsys);
    for (int s = 0; s < nsys; ++s) {
      sys[s].A.resize((size_t)npl * npl);
      for (size_t k = 0; k < (size_t)npl * npl; ++k) sys[s].A[k] = static_cast<cplx*>(Ab[(size_t)s * npl * npl + k]);
      sys[s].info = dinfo + (size_t)s * npl;
    }
    if (int r = build_selected_inverse(plan, sys, npl, b, mode, pivoting == 0)) return r;
    return run_sync(plan, static_cast<cudaStream_t>(stream), dinfo, nsys * npl, "negf_selected_inverse");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

}  // extern "C"
