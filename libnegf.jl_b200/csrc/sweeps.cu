// Band-w RGF, multi-level DDRGF and the reference's run_bndiag_wrapper C entry
// point, all expressed as batched launches of the plan engine.
#include "../../include/negf_b200.h"
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

using namespace negf;

namespace {

constexpr cplx ONE{1.0, 0.0};
constexpr cplx MONE{-1.0, 0.0};
constexpr cplx ZERO{0.0, 0.0};
constexpr int kMaxDdrgfLevels = NEGF_DDRGF_MAX_LEVELS;

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

int run_sync(Plan& plan, cudaStream_t st, int* dinfo, int nsys, const char* what) {
  cudaError_t e = plan.run(st, false);
  if (e != cudaSuccess) return cuda_fail(e, what);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, what);
  if (dinfo) {
    std::vector<int> info(nsys);
    e = cudaMemcpy(info.data(), dinfo, sizeof(int) * nsys, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, what);
    for (int s = 0; s < nsys; ++s)
      if (info[s]) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "%s: zero pivot in system %d (column %d of a diagonal block)", what, s, info[s]);
        return fail(NEGF_ERR_SINGULAR, buf);
      }
  }
  return NEGF_SUCCESS;
}

// ---------------------------------------------------------------------------
// DDRGF partition (src/matinvertndiag_ddrgf_utils.jl:278-312, :478-575)

void get_nr_tasks(int npl, int d1, int& nr, int& last) {
  int per = d1 + 1;
  int n = npl / per + 1;
  int left = npl - (n - 1) * per;
  int d1left = left - 1;
  if (left == 0) { nr = n - 1; last = 0; return; }
  if (d1left == 0) { nr = -1; last = 0; return; }
  nr = n; last = d1left;
}

struct Partition {
  std::vector<int> seps;
  std::vector<std::vector<int>> doms;
};

bool make_partition(int npl, int d1, Partition& P) {
  int nr, last;
  get_nr_tasks(npl, d1, nr, last);
  if (nr < 1) return false;
  int x = 0;
  for (int t = 0; t < nr; ++t) {
    P.seps.push_back(x);
    int size = (t == nr - 1 && last != 0) ? last : d1;
    std::vector<int> d;
    for (int i = 0; i < size; ++i) d.push_back(x + 1 + i);
    P.doms.push_back(d);
    x += 1 + size;
  }
  return true;
}

// Cost model of the GPU DDRGF, in seconds, for nsys systems of npl layers of
// size b.  One b^3 complex GEMM takes gemm_s at ~30 TFLOP/s; one batched
// launch step costs at least step_s (launch + tail latency).  Per level with
// interior size D1 and T tasks:
//   work   ~ nsys * T * ((4 + D1) D1 + 8 D1 + 20) GEMMs (domain RGF + full
//            inverse, Schur complement, 12/21/11 parts; all tasks share the
//            same launches),
//   serial ~ (2 D1 + 6) steps;
// the level costs max(work, serial) + 0.1 min(work, serial).  The Schur
// complement (T layers) is solved by the next level or by sequential RGF,
// 7 steps per layer.  Levels are chosen by a memoised search over layer counts
// (interior sizes up to 256, at most max_levels levels).
struct GpuCost {
  double gemm_s, step_s;
  int nsys;
  GpuCost(int b, int nsys_) : nsys(nsys_) {
    gemm_s = 8.0 * b * (double)b * b / 30e12;
    step_s = std::max(8e-6, gemm_s / std::max(1.0, 148.0 * 2.0 / std::max(1.0, (b / 64.0) * (b / 64.0))));
  }
  double seq(int n) const { return 7.0 * n * std::max(step_s, nsys * gemm_s / 148.0); }
  double level(int d1, int nr) const {
    double work = nsys * (double)nr * ((4.0 + d1) * d1 + 8.0 * d1 + 20.0) * gemm_s;
    double serial = (2.0 * d1 + 6.0) * step_s;
    return std::max(work, serial) + 0.1 * std::min(work, serial);
  }
};

}  // namespace

namespace negf {

std::vector<int> choose_levels(int npl, int b, int nsys, int max_levels) {
  GpuCost c(b, nsys);
  // best[lev][n]: (time, first interior size or 0 for sequential RGF)
  std::vector<std::map<int, std::pair<double, int>>> memo(max_levels + 1);
  std::function<std::pair<double, int>(int, int)> best = [&](int n, int lev) -> std::pair<double, int> {
    auto it = memo[lev].find(n);
    if (it != memo[lev].end()) return it->second;
    std::pair<double, int> r{c.seq(n), 0};
    if (lev < max_levels)
      for (int d1 = 1; d1 < n && d1 <= 256; ++d1) {
        int nr, last;
        get_nr_tasks(n, d1, nr, last);
        if (nr < 2) continue;
        double t = c.level(d1, nr) + best(nr, lev + 1).first;
        if (t < r.first) r = {t, d1};
      }
    memo[lev][n] = r;
    return r;
  };
  std::vector<int> d1s;
  int n = npl;
  for (int lev = 0; lev < max_levels; ++lev) {
    int d1 = best(n, lev).second;
    if (d1 == 0) break;
    d1s.push_back(d1);
    int nr, last;
    get_nr_tasks(n, d1, nr, last);
    n = nr;
  }
  return d1s;
}

}  // namespace negf

namespace {

// One level: the interior size, or npl (sequential RGF) when DDRGF does not pay.
int choose_d1(int npl, int b, int nsys) {
  std::vector<int> d1s = choose_levels(npl, b, nsys, 1);
  return d1s.empty() ? npl : d1s[0];
}

// The reference's partition search, restated (src/matinvertndiag_ddrgf_utils.jl):
// cost_rgf :221-247, cost_ddrgf :249-276, check_nr_threads :455-465 and
// opt_params :357-453 (CPU cost in units of one GEMM; levels <= 6, D1 <= 4).
double ref_cost_rgf(int L, double rLU, double rMLDIV, bool full) {
  if (full && L > 4) return HUGE_VAL;
  int nfull = 0;
  if (full && L == 3) nfull = 3;
  if (full && L == 4) nfull = 9;
  const int ngemm = 4 * (L - 1) + nfull, nmldiv = 3 * (L - 1) + 1;
  return ngemm + rLU * L + rMLDIV * nmldiv;
}

double ref_cost_ddrgf(double rLU, double rMLDIV, int nr, int thr, int d1) {
  const double f = 1.0 / thr;
  double c = f * nr * ref_cost_rgf(d1, rLU, rMLDIV, true);
  c += 4.0 * f * nr * d1;            // r22(12) and r22(21)
  c += 4.0 * f * nr;                 // r22S
  c += 4.0 * f * nr * d1;            // r12
  c += 4.0 * f * nr;                 // r21
  c += f * nr * (4.0 * (d1 - 1) + 2.0 * d1);  // r11
  return c;
}

int ref_check_nr_threads(int thr, int nr) {
  for (;;) {
    const int per = (nr + thr - 1) / thr;
    if (nr - (thr - 1) * per > 0) return thr;
    --thr;
  }
}

struct RefOpt {
  int levels = 0;
  int tasks[kMaxDdrgfLevels] = {0};
  int d1[kMaxDdrgfLevels] = {0};
  double cost = HUGE_VAL;
};

RefOpt ref_opt_params(int npl, int threads, double rLU, double rMLDIV, double damp) {
  constexpr int kD1Max = 4;
  RefOpt best;
  for (int levels = 1; levels <= kMaxDdrgfLevels; ++levels) {
    int arr[kMaxDdrgfLevels];
    for (int k = 0; k < levels; ++k) arr[k] = kD1Max;
    for (;;) {
      int prev = npl, tasks[kMaxDdrgfLevels], d1l[kMaxDdrgfLevels];
      double cost = 0.0, coarse = 0.0;
      for (int lev = 0; lev < levels; ++lev) {
        const int d1 = arr[lev];
        // once a finite cost is known, only the largest size is tried at level 1
        if (best.cost != HUGE_VAL && lev == 0 && d1 < kD1Max) break;
        cost -= coarse;
        int nr, last;
        get_nr_tasks(prev, d1, nr, last);
        if (nr == -1) break;
        prev = nr;
        cost += ref_cost_ddrgf(rLU, rMLDIV, nr, ref_check_nr_threads(threads, nr), d1);
        coarse = damp * ref_cost_rgf(nr, rLU, rMLDIV, false);
        cost += coarse;
        tasks[lev] = nr;
        d1l[lev] = d1;
        if (cost < best.cost) {
          best.cost = cost;
          best.levels = lev + 1;
          for (int k = 0; k <= lev; ++k) { best.tasks[k] = tasks[k]; best.d1[k] = d1l[k]; }
        }
      }
      // next combination, the first level fastest (Julia's Iterators.product)
      int k = 0;
      for (; k < levels; ++k) {
        if (arr[k] > 1) { --arr[k]; break; }
        arr[k] = kD1Max;
      }
      if (k == levels) break;
    }
  }
  return best;
}

// Sequential RGF of a batch of systems into out (src/matinvertndiag_rgf.jl:114-182).
void build_seq_rgf(Plan& plan, const std::vector<TriSystem>& sys, std::vector<TriOut>& out) {
  std::vector<RgfWork> w(sys.size());
  for (size_t k = 0; k < sys.size(); ++k) alloc_rgf_work(plan, sys[k], w[k]);
  build_rgf_upward(plan, sys, w);
  build_rgf_downward(plan, sys, w, out);
}

}  // namespace

namespace negf {

// One DDRGF level over systems with the same layer count (block sizes may
// differ per system), writing the tridiagonal of every system's inverse into
// out.  d1s[level] is this level's interior size; the separator Schur
// complement recurses into level + 1, and past the last level (or when the
// partition has a single task) sequential RGF runs, as
// bndiag_of_inv_ddrgf! does (src/matinvertndiag_ddrgf_core.jl:719-758,
// :656-680, :726-729).  All domains / separators of all systems share each
// batched launch.
int build_ddrgf_level(Plan& plan, const std::vector<TriSystem>& sys, std::vector<TriOut>& out,
                      const std::vector<int>& d1s, size_t level) {
  const int nsys = static_cast<int>(sys.size());
  const int npl = sys[0].npl();
  const int d1 = level < d1s.size() ? d1s[level] : npl;
  Partition P;
  if (d1 < npl && !make_partition(npl, d1, P))
    return fail(NEGF_ERR_INVALID, "DDRGF partition impossible at level " + std::to_string(level + 1) + " (" +
                                      std::to_string(npl) + " layers, interior size " + std::to_string(d1) + ")");
  if (d1 >= npl || P.seps.size() < 2) {
    build_seq_rgf(plan, sys, out);
    return NEGF_SUCCESS;
  }
  const int T = static_cast<int>(P.seps.size());
  // input blocks of system s: M(i,i), M(i,i+1), M(i+1,i) and their leading dimensions
  auto Dm = [&](int s, int i) { return sys[s].D[i]; };
  auto Um = [&](int s, int i) { return sys[s].U[i]; };
  auto Lm = [&](int s, int i) { return sys[s].Lw[i]; };
  auto ldD = [&](int s, int i) { return sys[s].ldD[i]; };
  auto ldU = [&](int s, int i) { return sys[s].ldU[i]; };
  auto ldL = [&](int s, int i) { return sys[s].ldL[i]; };
  auto bsz = [&](int s, int i) { return sys[s].b[i]; };

  // 1. domain systems and their full inverses (_inv_of_T11!, core.jl:437-498)
  std::vector<TriSystem> dsys;
  for (int s = 0; s < nsys; ++s)
    for (int t = 0; t < T; ++t) {
      const auto& d = P.doms[t];
      TriSystem ts;
      for (int a = 0; a < (int)d.size(); ++a) {
        const int i = d[a];
        ts.b.push_back(bsz(s, i));
        ts.D.push_back(Dm(s, i)); ts.ldD.push_back(ldD(s, i));
        if (a + 1 < (int)d.size()) {
          ts.U.push_back(Um(s, i)); ts.ldU.push_back(ldU(s, i));
          ts.Lw.push_back(Lm(s, i)); ts.ldL.push_back(ldL(s, i));
        }
      }
      ts.info = sys[s].info;
      dsys.push_back(ts);
    }
  std::vector<RgfWork> dwork(dsys.size());
  std::vector<std::vector<cplx*>> dfull(dsys.size());
  std::vector<TriOut> dout(dsys.size());
  for (size_t k = 0; k < dsys.size(); ++k) {
    const TriSystem& ts = dsys[k];
    const int nd = ts.npl();
    alloc_rgf_work(plan, ts, dwork[k]);
    dfull[k].assign((size_t)nd * nd, nullptr);
    for (int i = 0; i < nd; ++i)
      for (int j = 0; j < nd; ++j) dfull[k][(size_t)i * nd + j] = plan.alloc_c((size_t)ts.b[i] * ts.b[j]);
    TriOut& o = dout[k];
    for (int i = 0; i < nd; ++i) { o.d.push_back(dfull[k][(size_t)i * nd + i]); o.ldd.push_back(ts.b[i]); }
    for (int i = 0; i + 1 < nd; ++i) {
      o.u.push_back(dfull[k][(size_t)i * nd + i + 1]); o.ldu.push_back(ts.b[i]);
      o.l.push_back(dfull[k][(size_t)(i + 1) * nd + i]); o.ldl.push_back(ts.b[i + 1]);
    }
  }
  build_rgf_upward(plan, dsys, dwork);
  build_rgf_downward(plan, dsys, dwork, dout);
  build_rgf_full_inverse(plan, dsys, dwork, dfull);
  auto Tinv = [&](int s, int t, int i, int j) -> cplx* {
    const size_t k = (size_t)s * T + t;
    const int nd = (int)P.doms[t].size();
    return dfull[k][(size_t)i * nd + j];
  };

  // 2. separator Schur complement (core.jl:48-114, :203-266, :500-654)
  std::vector<TriSystem> ssys(nsys);
  {
    std::vector<ZGemmProblem> l1, l2, l3;
    for (int s = 0; s < nsys; ++s) {
      TriSystem& ts = ssys[s];
      ts.info = sys[s].info;
      std::vector<cplx*> Sd(T), Su(T - 1), Sl(T - 1);
      for (int t = 0; t < T; ++t) {
        const int bs = bsz(s, P.seps[t]);
        ts.b.push_back(bs);
        Sd[t] = plan.alloc_c((size_t)bs * bs);
      }
      for (int t = 0; t + 1 < T; ++t) {
        Su[t] = plan.alloc_c((size_t)ts.b[t] * ts.b[t + 1]);
        Sl[t] = plan.alloc_c((size_t)ts.b[t] * ts.b[t + 1]);
      }
      for (int t = 0; t < T; ++t) {
        const int sp = P.seps[t], bs = bsz(s, sp);
        const int fl = P.doms[t].front(), ll = P.doms[t].back(), nd = (int)P.doms[t].size();
        const int bfl = bsz(s, fl), bll = bsz(s, ll);
        // X1 = M[s, fl] Tinv[0,0];  S_tt = M[s, s] - X1 M[fl, s]
        cplx* X1 = plan.alloc_c((size_t)bs * bfl);
        l1.push_back(gp(Um(s, sp), ldU(s, sp), Tinv(s, t, 0, 0), bfl, X1, bs, bs, bfl, bfl, ONE));
        l2.push_back(gp(X1, bs, Lm(s, sp), ldL(s, sp), Sd[t], bs, bs, bs, bfl, MONE, Dm(s, sp), ldD(s, sp), ONE));
        if (t > 0) {
          const int pl = P.doms[t - 1].back(), pnd = (int)P.doms[t - 1].size(), bpl = bsz(s, pl);
          // X2 = M[s, ll_{t-1}] Tinv_{t-1}[last,last];  S_tt -= X2 M[ll_{t-1}, s]
          cplx* X2 = plan.alloc_c((size_t)bs * bpl);
          l1.push_back(gp(Lm(s, sp - 1), ldL(s, sp - 1), Tinv(s, t - 1, pnd - 1, pnd - 1), bpl, X2, bs, bs, bpl,
                          bpl, ONE));
          l3.push_back(gp(X2, bs, Um(s, sp - 1), ldU(s, sp - 1), Sd[t], bs, bs, bs, bpl, MONE, Sd[t], bs, ONE));
        }
        if (t + 1 < T) {
          const int sn = P.seps[t + 1], bn = bsz(s, sn);
          // S_{t,t+1} = -M[s, fl] Tinv[0,last] M[ll, sn];  S_{t+1,t} = -M[sn, ll] Tinv[last,0] M[fl, s]
          cplx* Y = plan.alloc_c((size_t)bs * bll);
          cplx* Z = plan.alloc_c((size_t)bn * bfl);
          l1.push_back(gp(Um(s, sp), ldU(s, sp), Tinv(s, t, 0, nd - 1), bfl, Y, bs, bs, bll, bfl, ONE));
          l1.push_back(gp(Lm(s, sn - 1), ldL(s, sn - 1), Tinv(s, t, nd - 1, 0), bll, Z, bn, bn, bfl, bll, ONE));
          l2.push_back(gp(Y, bs, Um(s, sn - 1), ldU(s, sn - 1), Su[t], bs, bs, bn, bll, MONE));
          l2.push_back(gp(Z, bn, Lm(s, sp), ldL(s, sp), Sl[t], bn, bn, bs, bfl, MONE));
        }
      }
      for (int t = 0; t < T; ++t) { ts.D.push_back(Sd[t]); ts.ldD.push_back(ts.b[t]); }
      for (int t = 0; t + 1 < T; ++t) {
        ts.U.push_back(Su[t]); ts.ldU.push_back(ts.b[t]);
        ts.Lw.push_back(Sl[t]); ts.ldL.push_back(ts.b[t + 1]);
      }
    }
    plan.gemm('N', 'N', l1);
    plan.gemm('N', 'N', l2);
    plan.gemm('N', 'N', l3);
  }

  // 3. the Schur complement's tridiagonal inverse: its diagonal goes straight
  //    to the separator output blocks (core.jl:656-680)
  std::vector<TriOut> sout(nsys);
  for (int s = 0; s < nsys; ++s) {
    TriOut& o = sout[s];
    for (int t = 0; t < T; ++t) {
      o.d.push_back(out[s].d[P.seps[t]]);
      o.ldd.push_back(out[s].ldd[P.seps[t]]);
    }
    for (int t = 0; t + 1 < T; ++t) {
      o.u.push_back(plan.alloc_c((size_t)ssys[s].b[t] * ssys[s].b[t + 1])); o.ldu.push_back(ssys[s].b[t]);
      o.l.push_back(plan.alloc_c((size_t)ssys[s].b[t] * ssys[s].b[t + 1])); o.ldl.push_back(ssys[s].b[t + 1]);
    }
  }
  if (int r = build_ddrgf_level(plan, ssys, sout, d1s, level + 1)) return r;

  // 4. the 12, 21 and 11 parts (core.jl:116-201, :268-344, :346-435)
  std::vector<ZGemmProblem> L1, L2, L3, L5, L6;
  for (int s = 0; s < nsys; ++s) {
    TriOut& G = out[s];
    const TriOut& GS = sout[s];
    for (int t = 0; t < T; ++t) {
      const auto& d = P.doms[t];
      const int nd = (int)d.size();
      const int sp = P.seps[t], bs = bsz(s, sp);
      const bool nx = t + 1 < T;
      const int sn = nx ? P.seps[t + 1] : -1, bn = nx ? bsz(s, sn) : 0;
      const int fl = d.front(), ll = d.back(), bfl = bsz(s, fl), bll = bsz(s, ll);
      std::vector<cplx*> a1(nd), a2(nd), B12(nd), B12n(nd), C21(nd), C21n(nd);
      std::vector<int> ld12(nd), ld12n(nd);
      for (int i = 0; i < nd; ++i) {
        const int bi = bsz(s, d[i]);
        a1[i] = plan.alloc_c((size_t)bi * bs);
        C21[i] = plan.alloc_c((size_t)bs * bi);
        // B12[0] is the output block G[fl, sep_t]; B12n[last] is G[ll, sep_{t+1}]
        if (i == 0) { B12[i] = G.l[sp]; ld12[i] = G.ldl[sp]; }
        else { B12[i] = plan.alloc_c((size_t)bi * bs); ld12[i] = bi; }
        L1.push_back(gp(Tinv(s, t, i, 0), bi, Lm(s, sp), ldL(s, sp), a1[i], bi, bi, bs, bfl, ONE));
        L1.push_back(gp(Um(s, sp), ldU(s, sp), Tinv(s, t, 0, i), bfl, C21[i], bs, bs, bi, bfl, ONE));
        L2.push_back(gp(a1[i], bi, GS.d[t], GS.ldd[t], B12[i], ld12[i], bi, bs, bs, MONE));
        if (nx) {
          a2[i] = plan.alloc_c((size_t)bi * bn);
          C21n[i] = plan.alloc_c((size_t)bn * bi);
          if (i == nd - 1) { B12n[i] = G.u[sn - 1]; ld12n[i] = G.ldu[sn - 1]; }
          else { B12n[i] = plan.alloc_c((size_t)bi * bn); ld12n[i] = bi; }
          L1.push_back(gp(Tinv(s, t, i, nd - 1), bi, Um(s, sn - 1), ldU(s, sn - 1), a2[i], bi, bi, bn, bll, ONE));
          L1.push_back(gp(Lm(s, sn - 1), ldL(s, sn - 1), Tinv(s, t, nd - 1, i), bll, C21n[i], bn, bn, bi, bll, ONE));
          L2.push_back(gp(a1[i], bi, GS.u[t], GS.ldu[t], B12n[i], ld12n[i], bi, bn, bs, MONE));
          L3.push_back(gp(a2[i], bi, GS.l[t], GS.ldl[t], B12[i], ld12[i], bi, bs, bn, MONE, B12[i], ld12[i], ONE));
          L3.push_back(gp(a2[i], bi, GS.d[t + 1], GS.ldd[t + 1], B12n[i], ld12n[i], bi, bn, bn, MONE, B12n[i],
                          ld12n[i], ONE));
        }
      }
      // G[sep_t, fl] and G[sep_{t+1}, ll]
      L2.push_back(gp(GS.d[t], GS.ldd[t], C21[0], bs, G.u[sp], G.ldu[sp], bs, bfl, bs, MONE));
      if (nx) {
        L3.push_back(gp(GS.u[t], GS.ldu[t], C21n[0], bn, G.u[sp], G.ldu[sp], bs, bfl, bn, MONE, G.u[sp], G.ldu[sp],
                        ONE));
        L2.push_back(gp(GS.l[t], GS.ldl[t], C21[nd - 1], bs, G.l[sn - 1], G.ldl[sn - 1], bn, bll, bs, MONE));
        L3.push_back(gp(GS.d[t + 1], GS.ldd[t + 1], C21n[nd - 1], bn, G.l[sn - 1], G.ldl[sn - 1], bn, bll, bn, MONE,
                        G.l[sn - 1], G.ldl[sn - 1], ONE));
      }
      // interior tridiagonal: G = Tinv - B12 C21 - B12n C21n
      for (int i = 0; i < nd; ++i)
        for (int j = std::max(0, i - 1); j <= std::min(nd - 1, i + 1); ++j) {
          cplx* o;
          int ldo;
          if (j == i) { o = G.d[d[i]]; ldo = G.ldd[d[i]]; }
          else if (j == i + 1) { o = G.u[d[i]]; ldo = G.ldu[d[i]]; }
          else { o = G.l[d[j]]; ldo = G.ldl[d[j]]; }
          const int bi = bsz(s, d[i]), bj = bsz(s, d[j]);
          L5.push_back(gp(B12[i], ld12[i], C21[j], bs, o, ldo, bi, bj, bs, MONE, Tinv(s, t, i, j), bi, ONE));
          if (nx) L6.push_back(gp(B12n[i], ld12n[i], C21n[j], bn, o, ldo, bi, bj, bn, MONE, o, ldo, ONE));
        }
    }
  }
  plan.gemm('N', 'N', L1);
  plan.gemm('N', 'N', L2);
  plan.gemm('N', 'N', L3);
  plan.gemm('N', 'N', L5);
  plan.gemm('N', 'N', L6);
  return NEGF_SUCCESS;
}

}  // namespace negf

extern "C" {

int negf_ddrgf_get_nr_tasks(int32_t npl, int32_t block_size_d1, int32_t* nr_tasks, int32_t* last_d1) {
  if (npl <= 0 || block_size_d1 <= 0 || !nr_tasks || !last_d1) return fail(NEGF_ERR_INVALID, "bad arguments");
  int nr, last;
  get_nr_tasks(npl, block_size_d1, nr, last);
  *nr_tasks = nr;
  *last_d1 = last;
  return NEGF_SUCCESS;
}

int negf_ddrgf_choose_d1(int32_t npl, int32_t b, int32_t nsys, int32_t* block_size_d1) {
  if (npl <= 0 || b <= 0 || !block_size_d1) return fail(NEGF_ERR_INVALID, "bad arguments");
  *block_size_d1 = choose_d1(npl, b, std::max(1, nsys));
  return NEGF_SUCCESS;
}

// ---------------------------------------------------------------------------
// band-w RGF (src/matinvertndiag_general_rgf.jl:31-146)

int negf_general_rgf(int32_t nsys, int32_t npl, int32_t ndiag, const int32_t* block_sizes, void* const* Mb,
                     void* const* Gb, void* stream) {
  if (int r = check_device()) return r;
  if (nsys <= 0 || npl <= 0 || ndiag < 1 || (ndiag % 2) == 0 || !block_sizes || !Mb || !Gb)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  const int w = (ndiag - 1) / 2;
  try {
    Plan plan;
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * nsys));
    struct Sys {
      std::vector<int> b;
      std::map<std::pair<int, int>, cplx*> A, R, L, G;
      std::vector<cplx*> g;
      cplx *W, *F, *Bbuf;
      uint8_t* used;
      int* piv;
    };
    std::vector<Sys> S(nsys);
    std::vector<ZBlockOp> copies;
    for (int s = 0; s < nsys; ++s) {
      Sys& y = S[s];
      y.b.assign(block_sizes + (size_t)s * npl, block_sizes + (size_t)(s + 1) * npl);
      int mb = 0;
      for (int x : y.b) {
        if (x <= 0 || x > kMaxBlock) return fail(NEGF_ERR_INVALID, "block sizes must be in [1, 1024]");
        mb = std::max(mb, x);
      }
      for (int i = 0; i < npl; ++i)
        for (int j = std::max(0, i - w); j <= std::min(npl - 1, i + w); ++j) {
          const cplx* src = static_cast<const cplx*>(Mb[(size_t)s * npl * npl + (size_t)i * npl + j]);
          cplx* dst = static_cast<cplx*>(Gb[(size_t)s * npl * npl + (size_t)i * npl + j]);
          if (!src || !dst) return fail(NEGF_ERR_INVALID, "missing band block");
          cplx* a = plan.alloc_c((size_t)y.b[i] * y.b[j]);
          copies.push_back(copy_op(src, y.b[i], a, y.b[i], y.b[i], y.b[j]));
          y.A[{i, j}] = a;
          y.G[{i, j}] = dst;
        }
      y.g.resize(npl);
      for (int i = 0; i < npl; ++i) y.g[i] = plan.alloc_c((size_t)y.b[i] * y.b[i]);
      int nb = gj_panel_width(mb);
      y.W = plan.alloc_c((size_t)mb * mb);
      y.F = plan.alloc_c((size_t)mb * nb);
      y.Bbuf = plan.alloc_c((size_t)mb * nb);
      y.used = static_cast<uint8_t*>(plan.alloc(mb));
      y.piv = static_cast<int*>(plan.alloc(sizeof(int) * mb));
    }
    plan.blockops(copies);
    auto spec = [&](int s, int i) {
      Sys& y = S[s];
      InvSpec sp;
      sp.W = y.W; sp.n = y.b[i]; sp.ld = y.b[i]; sp.out = y.g[i]; sp.ldo = y.b[i];
      sp.F = y.F; sp.Bbuf = y.Bbuf; sp.used = y.used; sp.piv = y.piv; sp.info = dinfo + s;
      return sp;
    };
    // bottom element (:49)
    {
      std::vector<ZBlockOp> c;
      std::vector<InvSpec> iv;
      for (int s = 0; s < nsys; ++s) {
        Sys& y = S[s];
        int i = npl - 1;
        c.push_back(copy_op(y.A[{i, i}], y.b[i], y.W, y.b[i], y.b[i], y.b[i]));
        iv.push_back(spec(s, i));
      }
      plan.blockops(c);
      plan.inv(iv);
    }
    for (int ix = npl - 2; ix >= 0; --ix) {
      const int kmax = std::min(w, ix + 1);
      // multipliers (:56-67)
      std::vector<ZGemmProblem> mp;
      for (int s = 0; s < nsys; ++s) {
        Sys& y = S[s];
        for (int k = 1; k <= kmax; ++k) {
          int t = ix - k + 1, j = ix + 1;
          cplx* R = plan.alloc_c((size_t)y.b[t] * y.b[j]);
          cplx* L = plan.alloc_c((size_t)y.b[t] * y.b[j]);
          y.R[{t, j}] = R;
          y.L[{j, t}] = L;
          mp.push_back(gp(y.A[{t, j}], y.b[t], y.g[j], y.b[j], R, y.b[t], y.b[t], y.b[j], y.b[j], ONE));
          mp.push_back(gp(y.g[j], y.b[j], y.A[{j, t}], y.b[j], L, y.b[j], y.b[j], y.b[t], y.b[j], ONE));
        }
      }
      plan.gemm('N', 'N', mp);
      // Schur updates on the kmax x kmax grid (:70-86)
      std::vector<ZGemmProblem> up;
      std::vector<InvSpec> iv;
      for (int s = 0; s < nsys; ++s) {
        Sys& y = S[s];
        int j = ix + 1;
        for (int i1 = 1; i1 <= kmax; ++i1)
          for (int j1 = 1; j1 <= kmax; ++j1) {
            int r = ix - i1 + 1, c = ix - j1 + 1;
            cplx* dst = (r == ix && c == ix) ? y.W : y.A[{r, c}];
            up.push_back(gp(y.A[{r, j}], y.b[r], y.L[{j, c}], y.b[j], dst, y.b[r], y.b[r], y.b[c], y.b[j], MONE,
                            y.A[{r, c}], y.b[r], ONE));
          }
        iv.push_back(spec(s, ix));
      }
      plan.gemm('N', 'N', up);
      plan.inv(iv);
    }
    // downward pass (:95-127)
    {
      std::vector<ZBlockOp> c;
      for (int s = 0; s < nsys; ++s) c.push_back(copy_op(S[s].g[0], S[s].b[0], S[s].G[{0, 0}], S[s].b[0], S[s].b[0], S[s].b[0]));
      plan.blockops(c);
    }
    for (int ix = 1; ix < npl; ++ix) {
      const int kmax = std::min(w, ix);
      for (int k2 = 1; k2 <= kmax; ++k2) {
        std::vector<ZGemmProblem> pr;
        for (int s = 0; s < nsys; ++s) {
          Sys& y = S[s];
          int m = ix - k2;
          for (int k = 1; k <= kmax; ++k) {
            int tp = ix - k;
            const cplx* cin = k2 == 1 ? nullptr : y.G[{tp, ix}];
            pr.push_back(gp(y.G[{tp, m}], y.b[tp], y.R[{m, ix}], y.b[m], y.G[{tp, ix}], y.b[tp], y.b[tp], y.b[ix],
                            y.b[m], MONE, cin, y.b[tp], k2 == 1 ? ZERO : ONE));
            const cplx* cin2 = k2 == 1 ? nullptr : y.G[{ix, tp}];
            pr.push_back(gp(y.L[{ix, m}], y.b[ix], y.G[{m, tp}], y.b[m], y.G[{ix, tp}], y.b[ix], y.b[ix], y.b[tp],
                            y.b[m], MONE, cin2, y.b[ix], k2 == 1 ? ZERO : ONE));
          }
        }
        plan.gemm('N', 'N', pr);
      }
      for (int k2 = 1; k2 <= kmax; ++k2) {
        std::vector<ZGemmProblem> pr;
        for (int s = 0; s < nsys; ++s) {
          Sys& y = S[s];
          int m = ix - k2;
          const cplx* cin = k2 == 1 ? y.g[ix] : y.G[{ix, ix}];
          pr.push_back(gp(y.L[{ix, m}], y.b[ix], y.G[{m, ix}], y.b[m], y.G[{ix, ix}], y.b[ix], y.b[ix], y.b[ix],
                          y.b[m], MONE, cin, y.b[ix], ONE));
        }
        plan.gemm('N', 'N', pr);
      }
    }
    if (npl == 1) {
      // nothing beyond G[0,0]
    }
    return run_sync(plan, static_cast<cudaStream_t>(stream), dinfo, nsys, "negf_general_rgf");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

// ---------------------------------------------------------------------------
// DDRGF, any number of levels (src/matinvertndiag_ddrgf_core.jl:719-758; the
// Schur complement recursion at :656-680)

int negf_ddrgf_levels(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                      void* const* Ml, int32_t nlevels, const int32_t* block_size_d1, void* const* Gd,
                      void* const* Gu, void* const* Gl, void* stream) {
  return negf_ddrgf_levels_ex(nsys, npl, block_sizes, Md, Mu, Ml, nlevels, block_size_d1, Gd, Gu, Gl,
                              NEGF_PREC_FP64, stream);
}

int negf_ddrgf_levels_ex(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
                         void* const* Ml, int32_t nlevels, const int32_t* block_size_d1, void* const* Gd,
                         void* const* Gu, void* const* Gl, int32_t precision, void* stream) {
  if (int r = check_device()) return r;
  if (nsys <= 0 || npl <= 0 || !block_sizes || !Md || !Gd || (npl > 1 && (!Mu || !Ml)) || nlevels < 0 ||
      nlevels > kMaxDdrgfLevels || (nlevels > 0 && !block_size_d1) ||
      (precision != NEGF_PREC_FP64 && precision != NEGF_PREC_MIXED))
    return fail(NEGF_ERR_INVALID, "bad arguments");
  std::vector<int> d1s;
  if (nlevels == 0) {
    int mb = 0;
    for (int i = 0; i < nsys * npl; ++i) mb = std::max(mb, block_sizes[i]);
    d1s = choose_levels(npl, mb, nsys, kMaxDdrgfLevels);
  } else {
    d1s.assign(block_size_d1, block_size_d1 + nlevels);
    for (int d : d1s)
      if (d <= 0) return fail(NEGF_ERR_INVALID, "interior sizes must be positive");
  }
  for (int i = 0; i < nsys * npl; ++i)
    if (block_sizes[i] <= 0 || block_sizes[i] > kMaxBlock)
      return fail(NEGF_ERR_INVALID, "block sizes must be in [1, 1024]");
  try {
    Plan plan;
    plan.set_mixed(precision == NEGF_PREC_MIXED);
    int* dinfo = static_cast<int*>(plan.alloc(sizeof(int) * nsys));
    std::vector<TriSystem> sys(nsys);
    std::vector<TriOut> out(nsys);
    for (int s = 0; s < nsys; ++s) {
      const int32_t* b = block_sizes + (size_t)s * npl;
      TriSystem& ts = sys[s];
      TriOut& o = out[s];
      ts.info = dinfo + s;
      for (int i = 0; i < npl; ++i) {
        ts.b.push_back(b[i]);
        ts.D.push_back(static_cast<const cplx*>(Md[(size_t)s * npl + i]));
        ts.ldD.push_back(b[i]);
        o.d.push_back(static_cast<cplx*>(Gd[(size_t)s * npl + i]));
        o.ldd.push_back(b[i]);
      }
      for (int i = 0; i + 1 < npl; ++i) {
        const size_t k = (size_t)s * (npl - 1) + i;
        ts.U.push_back(static_cast<const cplx*>(Mu[k])); ts.ldU.push_back(b[i]);
        ts.Lw.push_back(static_cast<const cplx*>(Ml[k])); ts.ldL.push_back(b[i + 1]);
        // outputs the caller does not want go to scratch (the recursion needs them)
        o.u.push_back(Gu ? static_cast<cplx*>(Gu[k]) : plan.alloc_c((size_t)b[i] * b[i + 1]));
        o.ldu.push_back(b[i]);
        o.l.push_back(Gl ? static_cast<cplx*>(Gl[k]) : plan.alloc_c((size_t)b[i] * b[i + 1]));
        o.ldl.push_back(b[i + 1]);
      }
    }
    if (int r = build_ddrgf_level(plan, sys, out, d1s, 0)) return r;
    return run_sync(plan, static_cast<cudaStream_t>(stream), dinfo, nsys, "negf_ddrgf");
  } catch (const std::bad_alloc&) {
    return fail(NEGF_ERR_NOMEM, "device allocation failed");
  }
}

int negf_ddrgf(int32_t nsys, int32_t npl, const int32_t* block_sizes, void* const* Md, void* const* Mu,
               void* const* Ml, int32_t block_size_d1, void* const* Gd, void* const* Gu, void* const* Gl,
               void* stream) {
  if (block_size_d1 > 0) return negf_ddrgf_levels(nsys, npl, block_sizes, Md, Mu, Ml, 1, &block_size_d1, Gd, Gu, Gl,
                                                  stream);
  if (nsys <= 0 || npl <= 0 || !block_sizes) return fail(NEGF_ERR_INVALID, "bad arguments");
  int mb = 0;
  for (int i = 0; i < nsys * npl; ++i) mb = std::max(mb, block_sizes[i]);
  const int32_t d1 = choose_d1(npl, mb, nsys);
  return negf_ddrgf_levels(nsys, npl, block_sizes, Md, Mu, Ml, 1, &d1, Gd, Gu, Gl, stream);
}

int negf_ddrgf_choose_levels(int32_t npl, int32_t b, int32_t nsys, int32_t max_levels, int32_t* nlevels,
                             int32_t* block_size_d1) {
  if (npl <= 0 || b <= 0 || max_levels < 1 || max_levels > kMaxDdrgfLevels || !nlevels || !block_size_d1)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  std::vector<int> d1s = choose_levels(npl, b, std::max(1, nsys), max_levels);
  *nlevels = static_cast<int32_t>(d1s.size());
  for (size_t k = 0; k < d1s.size(); ++k) block_size_d1[k] = d1s[k];
  return NEGF_SUCCESS;
}

int negf_ddrgf_cost_rgf(int32_t L, double r_lu, double r_mldiv, int32_t do_full, double* cost) {
  if (L <= 0 || !cost) return fail(NEGF_ERR_INVALID, "bad arguments");
  if (do_full && L > 4) return fail(NEGF_ERR_INVALID, "cost_rgf: a full inverse by RGF is modelled for L <= 4 only");
  *cost = ref_cost_rgf(L, r_lu, r_mldiv, do_full != 0);
  return NEGF_SUCCESS;
}

int negf_ddrgf_cost_ddrgf(double r_lu, double r_mldiv, int32_t nr_tasks, int32_t nr_threads, int32_t block_size_d1,
                          double* cost) {
  if (nr_tasks <= 0 || nr_threads <= 0 || block_size_d1 <= 0 || block_size_d1 > 4 || !cost)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  *cost = ref_cost_ddrgf(r_lu, r_mldiv, nr_tasks, nr_threads, block_size_d1);
  return NEGF_SUCCESS;
}

int negf_ddrgf_check_nr_threads(int32_t nr_threads, int32_t nr_tasks, int32_t* threads, int32_t* max_per_thread,
                                int32_t* last_per_thread) {
  if (nr_threads <= 0 || nr_tasks <= 0 || !threads || !max_per_thread || !last_per_thread)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  const int thr = ref_check_nr_threads(nr_threads, nr_tasks);
  const int per = (nr_tasks + thr - 1) / thr;
  *threads = thr;
  *max_per_thread = per;
  *last_per_thread = nr_tasks - (thr - 1) * per;
  return NEGF_SUCCESS;
}

int negf_ddrgf_opt_params(int32_t npl, int32_t nr_threads, double r_lu, double r_mldiv, double damp_rgf,
                          int32_t* nr_levels, int32_t* nr_tasks, int32_t* block_size_d1, double* cost) {
  if (npl <= 0 || nr_threads <= 0 || !nr_levels || !nr_tasks || !block_size_d1)
    return fail(NEGF_ERR_INVALID, "bad arguments");
  RefOpt o = ref_opt_params(npl, nr_threads, r_lu, r_mldiv, damp_rgf);
  *nr_levels = o.levels;
  for (int k = 0; k < o.levels; ++k) {
    nr_tasks[k] = o.tasks[k];
    block_size_d1[k] = o.d1[k];
  }
  if (cost) *cost = o.cost;
  return NEGF_SUCCESS;
}

// ---------------------------------------------------------------------------
// src/c_interface/libnegf_c_interface.jl:85-142

CCscMatrix run_bndiag_wrapper(int32_t m, int32_t n, int32_t nnz_in, int32_t* colptr_in, int32_t* rowval_in,
                              void* nzval_in, int32_t n_blocks, int32_t* block_sizes_in, int32_t n_dict,
                              const char** dict_keys_in, int32_t* dict_vals_in, int32_t is_hermitian) {
  CCscMatrix bad{0, 0, 0, nullptr, nullptr, nullptr};
  if (m != n || m <= 0 || n_blocks <= 0 || !colptr_in || !rowval_in || !nzval_in || !block_sizes_in) {
    fail(NEGF_ERR_INVALID, "run_bndiag_wrapper: bad arguments");
    return bad;
  }
  int nd_in = 3, nd_out = 3;
  for (int i = 0; i < n_dict; ++i) {
    if (!dict_keys_in || !dict_keys_in[i]) continue;
    if (std::strcmp(dict_keys_in[i], "in") == 0) nd_in = dict_vals_in[i];
    if (std::strcmp(dict_keys_in[i], "out") == 0) nd_out = dict_vals_in[i];
  }
  if (nd_in != 3) {
    fail(NEGF_ERR_INVALID, "run_bndiag_wrapper: DDRGF needs a block tridiagonal input (ndiag in = 3)");
    return bad;
  }
  const int npl = n_blocks;
  std::vector<int> b(block_sizes_in, block_sizes_in + npl), off(npl + 1, 0);
  for (int i = 0; i < npl; ++i) off[i + 1] = off[i] + b[i];
  if (off[npl] != n) {
    fail(NEGF_ERR_INVALID, "run_bndiag_wrapper: block sizes do not add up to the matrix size");
    return bad;
  }
  std::vector<int> blk_of(n);
  for (int i = 0; i < npl; ++i)
    for (int r = off[i]; r < off[i + 1]; ++r) blk_of[r] = i;
  // device buffers: the CSC input, index tables, one arena for the input and
  // result band blocks (the conversions run on the device; the reference
  // converts on the host, src/blockmatrix.jl:34-127)
  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* p : owned) cudaFree(p);
  };
  auto dalloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return p;
  };
  auto oom = [&]() {
    cleanup();
    fail(NEGF_ERR_NOMEM, "run_bndiag_wrapper: device allocation failed");
    return bad;
  };
  auto cerr = [&](cudaError_t e) {
    cleanup();
    cuda_fail(e, "run_bndiag_wrapper");
    return bad;
  };
  size_t band = 0;
  for (int i = 0; i < npl; ++i) band += (size_t)b[i] * b[i];
  for (int i = 0; i + 1 < npl; ++i) band += 2 * (size_t)b[i] * b[i + 1];
  int* d_colptr = static_cast<int*>(dalloc(sizeof(int) * (n + 1)));
  int* d_rowval = static_cast<int*>(dalloc(sizeof(int) * (size_t)std::max(1, nnz_in)));
  cplx* d_nz = static_cast<cplx*>(dalloc(sizeof(cplx) * (size_t)std::max(1, nnz_in)));
  int* d_blk = static_cast<int*>(dalloc(sizeof(int) * n));
  int* d_off = static_cast<int*>(dalloc(sizeof(int) * (npl + 1)));
  int* d_b = static_cast<int*>(dalloc(sizeof(int) * npl));
  cplx* arena = static_cast<cplx*>(dalloc(2 * band * sizeof(cplx)));  // input band | result band
  cplx** d_tab = static_cast<cplx**>(dalloc(sizeof(cplx*) * 6 * npl));
  int* d_counts = static_cast<int*>(dalloc(sizeof(int) * n));
  int* d_colptr_out = static_cast<int*>(dalloc(sizeof(int) * (n + 1)));
  if (!d_colptr || !d_rowval || !d_nz || !d_blk || !d_off || !d_b || !arena || !d_tab || !d_counts || !d_colptr_out)
    return oom();
  std::vector<void*> Md(npl), Mu(std::max(1, npl - 1)), Ml(std::max(1, npl - 1)), Gd(npl),
      Gu(std::max(1, npl - 1)), Gl(std::max(1, npl - 1));
  std::vector<cplx*> tin(3 * npl, nullptr), tres(3 * npl, nullptr);  // slot 3i + (j - i + 1)
  {
    size_t o = 0;
    auto take = [&](size_t cnt) { cplx* p = arena + o; o += cnt; return p; };
    for (int i = 0; i < npl; ++i) {
      tin[3 * i + 1] = static_cast<cplx*>(Md[i] = take((size_t)b[i] * b[i]));
      tres[3 * i + 1] = static_cast<cplx*>(Gd[i] = take((size_t)b[i] * b[i]));
    }
    for (int i = 0; i + 1 < npl; ++i) {
      const size_t cnt = (size_t)b[i] * b[i + 1];
      tin[3 * i + 2] = static_cast<cplx*>(Mu[i] = take(cnt));
      tin[3 * (i + 1) + 0] = static_cast<cplx*>(Ml[i] = take(cnt));
      tres[3 * i + 2] = static_cast<cplx*>(Gu[i] = take(cnt));
      tres[3 * (i + 1) + 0] = static_cast<cplx*>(Gl[i] = take(cnt));
    }
  }
  cudaError_t e;
  if ((e = cudaMemset(arena, 0, 2 * band * sizeof(cplx))) != cudaSuccess) return cerr(e);
  if ((e = cudaMemcpy(d_colptr, colptr_in, sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
  if (nnz_in > 0) {
    if ((e = cudaMemcpy(d_rowval, rowval_in, sizeof(int) * nnz_in, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cerr(e);
    if ((e = cudaMemcpy(d_nz, nzval_in, sizeof(cplx) * nnz_in, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cerr(e);
  }
  if ((e = cudaMemcpy(d_blk, blk_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
  if ((e = cudaMemcpy(d_off, off.data(), sizeof(int) * (npl + 1), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  if ((e = cudaMemcpy(d_b, b.data(), sizeof(int) * npl, cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
  std::vector<cplx*> tabs(tin);
  tabs.insert(tabs.end(), tres.begin(), tres.end());
  if ((e = cudaMemcpy(d_tab, tabs.data(), sizeof(cplx*) * 6 * npl, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  if ((e = launch_csc_scatter(n, d_colptr, d_rowval, d_nz, std::max(0, nnz_in), d_blk, d_off, d_b, d_tab,
                              is_hermitian ? 1 : 0, 0)) != cudaSuccess)
    return cerr(e);
  if (is_hermitian && npl > 1) {
    // lower band blocks are the conjugate transposes of the upper ones
    std::vector<int32_t> mm(npl - 1), nn(npl - 1), la(npl - 1), lc(npl - 1);
    for (int i = 0; i + 1 < npl; ++i) { mm[i] = b[i + 1]; nn[i] = b[i]; la[i] = b[i]; lc[i] = b[i + 1]; }
    if (negf_zcopy_batched('C', npl - 1, mm.data(), nn.data(), Mu.data(), la.data(), Ml.data(), lc.data(), nullptr) !=
        NEGF_SUCCESS) {
      cleanup();
      return bad;
    }
  }
  // levels from the GPU cost model, as the reference's wrapper takes them
  // from allocate_aux_data_DDRGF (libnegf_c_interface.jl:119)
  int rc = negf_ddrgf_levels(1, npl, b.data(), Md.data(), Mu.data(), Ml.data(), 0, nullptr, Gd.data(), Gu.data(),
                             Gl.data(), nullptr);
  if (rc != NEGF_SUCCESS) { cleanup(); return bad; }
  // output: the input's "out" band; DDRGF fills the tridiagonal, wider bands keep
  // the input blocks as the reference's bm_copy(MbmIN) + bm_copy!(MbmOUT,
  // buffMout) does (rows sorted within a column, as in Julia's SparseMatrixCSC)
  const int wout = std::max(1, (nd_out - 1) / 2);
  if ((e = launch_csc_band_out(0, n, npl, wout, d_blk, d_off, d_b, d_tab + 3 * npl, d_colptr, d_rowval, d_nz,
                               std::max(0, nnz_in), d_counts, nullptr, nullptr, nullptr, 0)) != cudaSuccess)
    return cerr(e);
  std::vector<int> counts(n), colptr(n + 1, 0);
  if ((e = cudaMemcpy(counts.data(), d_counts, sizeof(int) * n, cudaMemcpyDeviceToHost)) != cudaSuccess) return cerr(e);
  for (int c = 0; c < n; ++c) colptr[c + 1] = colptr[c] + counts[c];
  const int nnz_out = colptr[n];
  int* d_rows = static_cast<int*>(dalloc(sizeof(int) * (size_t)std::max(1, nnz_out)));
  cplx* d_vals = static_cast<cplx*>(dalloc(sizeof(cplx) * (size_t)std::max(1, nnz_out)));
  if (!d_rows || !d_vals) return oom();
  if ((e = cudaMemcpy(d_colptr_out, colptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  if ((e = launch_csc_band_out(1, n, npl, wout, d_blk, d_off, d_b, d_tab + 3 * npl, d_colptr, d_rowval, d_nz,
                               std::max(0, nnz_in), nullptr, d_colptr_out, d_rows, d_vals, 0)) != cudaSuccess)
    return cerr(e);
  CCscMatrix out;
  out.m = m;
  out.n = n;
  out.nnz = nnz_out;
  out.colptr = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (n + 1)));
  out.rowval = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max(1, nnz_out)));
  out.nzval = std::malloc(sizeof(cplx) * std::max(1, nnz_out));
  if (!out.colptr || !out.rowval || !out.nzval) {
    std::free(out.colptr); std::free(out.rowval); std::free(out.nzval);
    cleanup();
    fail(NEGF_ERR_NOMEM, "run_bndiag_wrapper: host allocation failed");
    return bad;
  }
  std::memcpy(out.colptr, colptr.data(), sizeof(int32_t) * (n + 1));
  if (nnz_out > 0) {
    e = cudaMemcpy(out.rowval, d_rows, sizeof(int32_t) * nnz_out, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out.nzval, d_vals, sizeof(cplx) * nnz_out, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      std::free(out.colptr); std::free(out.rowval); std::free(out.nzval);
      return cerr(e);
    }
  }
  cleanup();
  return out;
}

// ---------------------------------------------------------------------------
// Dense debug path: bndiag_of_inv_direct / bndiag_of_inv_direct!
// (src/matinvertndiag_direct.jl:17-61, :78-85)

int negf_bndiag_of_inv_direct(int32_t n, int32_t nnz, const int32_t* colptr, const int32_t* rowval,
                              const void* nzval, int32_t n_blocks, const int32_t* block_sizes, int32_t ndiag_out,
                              CCscMatrix* result) {
  if (int r = check_device()) return r;
  if (!result || n <= 0 || nnz < 0 || !colptr || (nnz > 0 && (!rowval || !nzval)) || n_blocks <= 0 ||
      !block_sizes || ndiag_out < 1 || (ndiag_out % 2) == 0)
    return fail(NEGF_ERR_INVALID, "negf_bndiag_of_inv_direct: bad arguments");
  *result = CCscMatrix{0, 0, 0, nullptr, nullptr, nullptr};
  const int npl = n_blocks;
  std::vector<int> b(block_sizes, block_sizes + npl), off(npl + 1, 0);
  for (int i = 0; i < npl; ++i) {
    if (b[i] <= 0) return fail(NEGF_ERR_INVALID, "negf_bndiag_of_inv_direct: block sizes must be positive");
    off[i + 1] = off[i] + b[i];
  }
  if (off[npl] != n) return fail(NEGF_ERR_INVALID, "negf_bndiag_of_inv_direct: block sizes do not add up to n");
  // the inversion's partition: the whole matrix as one block (Gauss-Jordan
  // with partial pivoting over all rows, as LAPACK's inverse) up to 1024,
  // else block elimination over the reference's layers (full band)
  std::vector<int> ib = n <= kMaxBlock ? std::vector<int>{n} : b;
  const int nb = static_cast<int>(ib.size());
  for (int x : ib)
    if (x > kMaxBlock)
      return fail(NEGF_ERR_INVALID, "negf_bndiag_of_inv_direct: above n = 1024 every block must be <= 1024");
  std::vector<int> ioff(nb + 1, 0);
  for (int i = 0; i < nb; ++i) ioff[i + 1] = ioff[i] + ib[i];
  std::vector<int> blk_of(n), iblk_of(n);
  for (int i = 0; i < npl; ++i)
    for (int r = off[i]; r < off[i + 1]; ++r) blk_of[r] = i;
  for (int i = 0; i < nb; ++i)
    for (int r = ioff[i]; r < ioff[i + 1]; ++r) iblk_of[r] = i;

  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* p : owned) cudaFree(p);
  };
  auto dalloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return p;
  };
  auto cerr = [&](cudaError_t e) {
    cleanup();
    return cuda_fail(e, "negf_bndiag_of_inv_direct");
  };
  const size_t nn = (size_t)n * n;
  int* d_colptr = static_cast<int*>(dalloc(sizeof(int) * (n + 1)));
  int* d_rowval = static_cast<int*>(dalloc(sizeof(int) * (size_t)std::max(1, nnz)));
  cplx* d_nz = static_cast<cplx*>(dalloc(sizeof(cplx) * (size_t)std::max(1, nnz)));
  int* d_idx = static_cast<int*>(dalloc(sizeof(int) * (2 * (size_t)n + (npl + 1) + (nb + 1) + nb)));
  cplx* arena = static_cast<cplx*>(dalloc(2 * nn * sizeof(cplx)));  // input blocks | inverse blocks
  cplx** d_tab = static_cast<cplx**>(dalloc(sizeof(cplx*) * 2 * (size_t)nb * nb));
  int* d_counts = static_cast<int*>(dalloc(sizeof(int) * n));
  int* d_colptr_out = static_cast<int*>(dalloc(sizeof(int) * (n + 1)));
  if (!d_colptr || !d_rowval || !d_nz || !d_idx || !arena || !d_tab || !d_counts || !d_colptr_out) {
    cleanup();
    return fail(NEGF_ERR_NOMEM, "negf_bndiag_of_inv_direct: device allocation failed");
  }
  int* d_blk = d_idx;
  int* d_iblk = d_blk + n;
  int* d_off = d_iblk + n;
  int* d_ioff = d_off + (npl + 1);
  int* d_ib = d_ioff + (nb + 1);
  std::vector<void*> Mb((size_t)nb * nb), Gb((size_t)nb * nb);
  {
    size_t o = 0;
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) {
        const size_t cnt = (size_t)ib[i] * ib[j];
        Mb[(size_t)i * nb + j] = arena + o;
        Gb[(size_t)i * nb + j] = arena + nn + o;
        o += cnt;
      }
  }
  std::vector<int> idx;
  idx.insert(idx.end(), blk_of.begin(), blk_of.end());
  idx.insert(idx.end(), iblk_of.begin(), iblk_of.end());
  idx.insert(idx.end(), off.begin(), off.end());
  idx.insert(idx.end(), ioff.begin(), ioff.end());
  idx.insert(idx.end(), ib.begin(), ib.end());
  std::vector<void*> tabs(Mb);
  tabs.insert(tabs.end(), Gb.begin(), Gb.end());
  cudaError_t e;
  if ((e = cudaMemset(arena, 0, nn * sizeof(cplx))) != cudaSuccess) return cerr(e);
  if ((e = cudaMemcpy(d_colptr, colptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
  if (nnz > 0) {
    if ((e = cudaMemcpy(d_rowval, rowval, sizeof(int) * nnz, cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
    if ((e = cudaMemcpy(d_nz, nzval, sizeof(cplx) * nnz, cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e);
  }
  if ((e = cudaMemcpy(d_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  if ((e = cudaMemcpy(d_tab, tabs.data(), sizeof(void*) * tabs.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  // Mdense = Array(M), scattered into the inversion's blocks (direct.jl:21)
  if ((e = launch_csc_full_scatter(n, d_colptr, d_rowval, d_nz, nnz, d_iblk, d_ioff, d_ib, d_tab, nb, 0)) !=
      cudaSuccess)
    return cerr(e);
  // MdenseInv = be_inv(Mdense) (direct.jl:26-28): the full band of the block
  // inverse; one block = the batched Gauss-Jordan inverse
  int rc = negf_general_rgf(1, nb, 2 * nb - 1, ib.data(), Mb.data(), Gb.data(), nullptr);
  if (rc != NEGF_SUCCESS) {
    cleanup();
    return rc;
  }
  // the reference writes the out band of the inverse into M (direct.jl:32-58)
  const int wout = (ndiag_out - 1) / 2;
  cplx* const* d_res = d_tab + (size_t)nb * nb;
  if ((e = launch_csc_direct_out(0, n, npl, wout, d_blk, d_off, d_iblk, d_ioff, d_ib, nb, d_res, d_colptr, d_rowval,
                                 d_nz, nnz, d_counts, nullptr, nullptr, nullptr, 0)) != cudaSuccess)
    return cerr(e);
  std::vector<int> counts(n), cp(n + 1, 0);
  if ((e = cudaMemcpy(counts.data(), d_counts, sizeof(int) * n, cudaMemcpyDeviceToHost)) != cudaSuccess) return cerr(e);
  for (int c = 0; c < n; ++c) cp[c + 1] = cp[c] + counts[c];
  const int nnz_out = cp[n];
  int* d_rows = static_cast<int*>(dalloc(sizeof(int) * (size_t)std::max(1, nnz_out)));
  cplx* d_vals = static_cast<cplx*>(dalloc(sizeof(cplx) * (size_t)std::max(1, nnz_out)));
  if (!d_rows || !d_vals) {
    cleanup();
    return fail(NEGF_ERR_NOMEM, "negf_bndiag_of_inv_direct: device allocation failed");
  }
  if ((e = cudaMemcpy(d_colptr_out, cp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cerr(e);
  if ((e = launch_csc_direct_out(1, n, npl, wout, d_blk, d_off, d_iblk, d_ioff, d_ib, nb, d_res, d_colptr, d_rowval,
                                 d_nz, nnz, nullptr, d_colptr_out, d_rows, d_vals, 0)) != cudaSuccess)
    return cerr(e);
  CCscMatrix out{n, n, nnz_out, nullptr, nullptr, nullptr};
  out.colptr = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (n + 1)));
  out.rowval = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max(1, nnz_out)));
  out.nzval = std::malloc(sizeof(cplx) * std::max(1, nnz_out));
  auto free_out = [&]() {
    std::free(out.colptr); std::free(out.rowval); std::free(out.nzval);
  };
  if (!out.colptr || !out.rowval || !out.nzval) {
    free_out();
    cleanup();
    return fail(NEGF_ERR_NOMEM, "negf_bndiag_of_inv_direct: host allocation failed");
  }
  std::memcpy(out.colptr, cp.data(), sizeof(int32_t) * (n + 1));
  if (nnz_out > 0) {
    e = cudaMemcpy(out.rowval, d_rows, sizeof(int32_t) * nnz_out, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out.nzval, d_vals, sizeof(cplx) * nnz_out, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      free_out();
      return cerr(e);
    }
  }
  cleanup();
  *result = out;
  return NEGF_SUCCESS;
}

}  // extern "C"
