// Sweep planner: turns the reference's per-block call sequences into batched
// launches (one launch per recursion step over all systems).
#include "engine.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

namespace negf {

cudaError_t zgj_prepare(size_t smem);

namespace {
thread_local std::string g_last_error;

inline ZGemmProblem gp(const cplx* A, int lda, const cplx* B, int ldb, cplx* C, int ldc, int m, int n, int k,
                       cplx alpha, const cplx* Cin = nullptr, int ldcin = 1, cplx beta = {0.0, 0.0},
                       cplx diag = {0.0, 0.0}) {
  ZGemmProblem p;
  p.A = A; p.B = B; p.Cin = Cin; p.C = C; p.diag_ptr = nullptr;
  p.m = m; p.n = n; p.k = k;
  p.lda = lda > 0 ? lda : 1; p.ldb = ldb > 0 ? ldb : 1; p.ldc = ldc; p.ldcin = ldcin > 0 ? ldcin : 1;
  p.pad_ = 0;
  p.alpha = alpha; p.beta = beta; p.diag = diag;
  return p;
}
constexpr cplx ONE{1.0, 0.0};
constexpr cplx MONE{-1.0, 0.0};
constexpr cplx ZERO{0.0, 0.0};
inline cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
}  // namespace

std::string& last_error() { return g_last_error; }
void set_error(const std::string& msg) { g_last_error = msg; }

int gj_panel_width(int max_n) {
  if (max_n <= 112) return max_n;
  if (max_n <= 400) return 32;
  if (max_n <= 800) return 16;
  return 8;
}

int Plan::panel_width(int max_n) const {
  if (gj_nb_ > 0 && max_n > 112) return gj_nb_;
  return gj_panel_width(max_n);
}

int TriSystem::maxb() const {
  int m = 0;
  for (int x : b) m = std::max(m, x);
  return m;
}

// ---------------------------------------------------------------------------
// Plan

namespace {
// Per-device cache of freed plan chunks, keyed by size.  It holds at most half
// of the device's memory; a chunk that does not fit is freed.
struct ChunkCache {
  std::mutex mu;
  std::map<int, std::multimap<size_t, void*>> free_by_dev;
  std::map<int, size_t> bytes;
  std::map<int, size_t> total;  // device memory, read once per device
};
ChunkCache& chunk_cache() {
  static ChunkCache* c = new ChunkCache();  // kept until exit: chunks may be returned during teardown
  return *c;
}
int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}
// a non-blocking stream per device for zeroing new chunks (no legacy-stream work)
cudaStream_t zero_stream() {
  static std::mutex mu;
  static std::map<int, cudaStream_t> streams;
  std::lock_guard<std::mutex> lk(mu);
  const int d = current_device();
  auto it = streams.find(d);
  if (it != streams.end()) return it->second;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
  streams[d] = s;
  return s;
}
// a cached chunk of at least `bytes` and at most 5/4 of it, or null
void* cache_take(size_t bytes, size_t* got) {
  ChunkCache& c = chunk_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  const int d = current_device();
  auto& m = c.free_by_dev[d];
  auto it = m.lower_bound(bytes);
  if (it == m.end() || it->first > bytes + bytes / 4) return nullptr;
  void* p = it->second;
  *got = it->first;
  c.bytes[d] -= it->first;
  m.erase(it);
  return p;
}
void cache_put(void* p, size_t bytes) {
  ChunkCache& c = chunk_cache();
  const int d = current_device();
  {
    std::lock_guard<std::mutex> lk(c.mu);
    size_t& tot = c.total[d];
    if (tot == 0) {
      size_t fr = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) tot = 0;
    }
    if (c.bytes[d] + bytes <= tot / 2) {
      c.free_by_dev[d].emplace(bytes, p);
      c.bytes[d] += bytes;
      return;
    }
  }
  cudaFree(p);
}
void cache_flush(int d) {
  ChunkCache& c = chunk_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  for (auto& kv : c.free_by_dev[d]) cudaFree(kv.second);
  c.free_by_dev[d].clear();
  c.bytes[d] = 0;
}
}  // namespace

size_t cached_bytes(int device) {
  ChunkCache& c = chunk_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.bytes.find(device);
  return it == c.bytes.end() ? 0 : it->second;
}

void release_cached_memory() {
  int n = 0, cur = 0;
  cudaGetDevice(&cur);
  if (cudaGetDeviceCount(&n) != cudaSuccess) return;
  for (int d = 0; d < n; ++d) {
    if (cached_bytes(d) == 0) continue;
    cudaSetDevice(d);
    cache_flush(d);
  }
  cudaSetDevice(cur);
}

Plan::~Plan() {
  if (gexec_) cudaGraphExecDestroy(gexec_);
  if (graph_) cudaGraphDestroy(graph_);
  // The chunks go back to the cache once the last recorded use on every
  // stream is complete.  Only those uses are waited for: a device-wide
  // synchronisation would invalidate CUDA-graph captures that other threads
  // have in progress.  A plan without recorded uses, or whose wait fails,
  // frees its chunks (cudaFree waits for the device itself).
  bool idle = !fences_.empty();
  for (auto& f : fences_) {
    if (cudaEventSynchronize(f.second) != cudaSuccess) idle = false;
    cudaEventDestroy(f.second);
  }
  if (!idle) cudaGetLastError();
  if (dblob_) cudaFree(dblob_);
  for (auto& c : owned_) {
    if (idle) cache_put(c.first, c.second);
    else cudaFree(c.first);
  }
}

void Plan::fence(cudaStream_t s) {
  cudaEvent_t ev = nullptr;
  for (auto& f : fences_)
    if (f.first == s) ev = f.second;
  if (!ev) {
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return;
    fences_.push_back({s, ev});
  }
  cudaEventRecord(ev, s);
}

// Workspace comes from a bump arena of zeroed chunks: the first is 1 MiB and
// each next one doubles up to 64 MiB, so a plan of thousands of small blocks
// costs a handful of cudaMalloc calls instead of one per block; a request of
// 32 MiB or more gets a chunk of its own.  Every piece is 256-byte aligned.
void* Plan::raw_alloc(size_t bytes) {
  size_t got = bytes;
  void* p = cache_take(bytes, &got);
  if (!p) {
    got = bytes;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();  // clear the allocation error, then retry without the cache
      cache_flush(current_device());
      if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw std::bad_alloc();
      }
    }
  }
  // zeroed before the chunk is handed out: callers write plan memory from
  // their own streams before the plan is finalised
  cudaStream_t zs = zero_stream();
  if (!zs || cudaMemsetAsync(p, 0, bytes, zs) != cudaSuccess || cudaStreamSynchronize(zs) != cudaSuccess) {
    cudaFree(p);
    throw std::bad_alloc();
  }
  owned_.push_back({p, got});
  owned_bytes_ += got;
  return p;
}

void* Plan::alloc(size_t bytes) {
  constexpr size_t kFirst = size_t(1) << 20, kCap = size_t(64) << 20;
  bytes = (std::max<size_t>(bytes, 16) + 255) & ~size_t(255);
  if (bytes >= kCap / 2) return raw_alloc(bytes);
  if (chunk_left_ < bytes) {
    chunk_size_ = chunk_size_ ? std::min(kCap, 2 * chunk_size_) : kFirst;
    while (chunk_size_ < bytes) chunk_size_ *= 2;
    chunk_ = static_cast<unsigned char*>(raw_alloc(chunk_size_));
    chunk_left_ = chunk_size_;
  }
  void* p = chunk_;
  chunk_ += bytes;
  chunk_left_ -= bytes;
  return p;
}

size_t Plan::push_bytes(const void* p, size_t n) {
  size_t off = (blob_.size() + 255) & ~size_t(255);
  blob_.resize(off + n);
  if (n) std::memcpy(blob_.data() + off, p, n);
  return off;
}

void Plan::gemm(char opA, char opB, const std::vector<ZGemmProblem>& probs) {
  if (!mixed_) {
    gemm_fp64(opA, opB, probs);
    return;
  }
  std::vector<ZGemmProblem> dbl, mix;
  for (const auto& p : probs) (p.k > 0 ? mix : dbl).push_back(p);
  gemm_fp64(opA, opB, dbl);
  gemm_mixed(opA, opB, mix);
}

namespace {
// views of the operands as R x K real-and-imaginary matrices (K = contraction)
struct OzKey {
  const cplx* X;
  long long sr, sk;
  int rows, cols, conj, side;
  bool operator<(const OzKey& o) const {
    return std::tie(X, sr, sk, rows, cols, conj, side) < std::tie(o.X, o.sr, o.sk, o.rows, o.cols, o.conj, o.side);
  }
};
inline int round_up(int x, int m) { return (x + m - 1) / m * m; }
}  // namespace

void Plan::gemm_mixed(char opA, char opB, const std::vector<ZGemmProblem>& probs, int pairs) {
  if (probs.empty()) return;
  if (!err_) err_ = static_cast<int*>(alloc(sizeof(int)));
  std::map<OzKey, int> index;
  std::vector<OzKey> keys;
  std::vector<std::pair<int, int>> which(probs.size());
  auto key_of = [&](const ZGemmProblem& p, bool A) {
    OzKey k;
    if (A) {  // Y = op(A): m x k
      k.X = p.A; k.rows = p.m; k.cols = p.k; k.side = 0;
      if (opA == 'N') { k.sr = 1; k.sk = p.lda; k.conj = 0; }
      else { k.sr = p.lda; k.sk = 1; k.conj = opA == 'C'; }
    } else {  // Y = op(B)^T: n x k
      k.X = p.B; k.rows = p.n; k.cols = p.k; k.side = 1;
      if (opB == 'N') { k.sr = p.ldb; k.sk = 1; k.conj = 0; }
      else { k.sr = 1; k.sk = p.ldb; k.conj = opB == 'C'; }
    }
    return k;
  };
  auto get = [&](const OzKey& k) {
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    int id = (int)keys.size();
    index[k] = id;
    keys.push_back(k);
    return id;
  };
  for (size_t i = 0; i < probs.size(); ++i) which[i] = {get(key_of(probs[i], true)), get(key_of(probs[i], false))};
  // Digits the previous mixed step made are used again when no other step
  // came in between, the operand view is the same (pointer, strides, shape,
  // conjugation, side) and none of that step's products wrote into it.
  if (steps.size() != oz_prev_steps_) {
    oz_prev_.clear();
    oz_prev_out_.clear();
    oz_prev_end_ = 0;
  }
  auto view_key = [](const OzKey& k) {
    return std::vector<long long>{(long long)(uintptr_t)k.X, k.sr, k.sk, k.rows, k.cols, k.conj, k.side};
  };
  auto written_before = [&](const OzKey& k) {
    const char* lo = reinterpret_cast<const char*>(k.X);
    const char* hi = lo + sizeof(cplx) * ((size_t)(k.rows - 1) * k.sr + (size_t)(k.cols - 1) * k.sk + 1);
    for (const auto& r : oz_prev_out_)
      if (lo < r.second && r.first < hi) return true;
    return false;
  };
  const size_t nk = keys.size();
  std::vector<int> rpad(nk), kpad(nk);
  std::vector<int8_t*> slc(nk, nullptr);
  std::vector<int*> exs(nk, nullptr);
  bool any_reuse = false;
  for (size_t i = 0; i < nk; ++i) {
    rpad[i] = round_up(std::max(keys[i].rows, 1), keys[i].side == 0 ? 128 : 64);
    kpad[i] = round_up(std::max(keys[i].cols, 1), 32);
    auto it = oz_prev_.find(view_key(keys[i]));
    if (it != oz_prev_.end() && it->second.rpad == rpad[i] && it->second.kpad == kpad[i] && !written_before(keys[i])) {
      slc[i] = it->second.slices;
      exs[i] = it->second.exps;
      any_reuse = true;
    }
  }
  // new digits: 3 real operands x 7 digit slices, then a scale per row; they go
  // after the reused ones when those are in the pool and there is room, else
  // the pool is laid out afresh (and grown as needed) without reuse
  std::vector<size_t> off_s(nk, 0), off_e(nk, 0);
  auto layout = [&](size_t base) {
    size_t need = base;
    for (size_t i = 0; i < nk; ++i) {
      if (slc[i]) continue;
      off_s[i] = need;
      need += (size_t)21 * rpad[i] * kpad[i];
      need = (need + 255) & ~size_t(255);
      off_e[i] = need;
      need += sizeof(int) * (size_t)rpad[i];
      need = (need + 255) & ~size_t(255);
    }
    return need;
  };
  size_t base = 0, need = 0;
  if (any_reuse && oz_prev_pool_ == oz_pool_ && layout(oz_prev_end_) <= oz_pool_bytes_) {
    base = oz_prev_end_;
  } else if (any_reuse) {
    any_reuse = false;
    for (size_t i = 0; i < nk; ++i) {
      slc[i] = nullptr;
      exs[i] = nullptr;
    }
  }
  need = layout(base);
  if (need > oz_pool_bytes_) {
    oz_pool_ = static_cast<unsigned char*>(alloc(need));
    oz_pool_bytes_ = need;
  }
  std::vector<OzSplitProblem> sp;
  int max_rows = 0, max_kpad = 0;
  double split_bytes = 0.0;
  for (size_t i = 0; i < nk; ++i) {
    if (slc[i]) continue;
    slc[i] = reinterpret_cast<int8_t*>(oz_pool_ + off_s[i]);
    exs[i] = reinterpret_cast<int*>(oz_pool_ + off_e[i]);
    OzSplitProblem q;
    q.X = keys[i].X; q.sr = keys[i].sr; q.sk = keys[i].sk;
    q.rows = keys[i].rows; q.cols = keys[i].cols; q.rows_pad = rpad[i]; q.k_pad = kpad[i];
    q.conj = keys[i].conj; q.tile_rows = keys[i].side == 0 ? 128 : 64;
    q.slices = slc[i];
    q.exps = exs[i];
    sp.push_back(q);
    max_rows = std::max(max_rows, rpad[i]);
    max_kpad = std::max(max_kpad, kpad[i]);
    split_bytes += 16.0 * keys[i].rows * keys[i].cols + 21.0 * rpad[i] * kpad[i] + 4.0 * rpad[i];
  }
  if (!sp.empty()) {
    Step s1;
    s1.kind = Step::OZ_SPLIT;
    s1.off = push_bytes(sp.data(), sp.size() * sizeof(OzSplitProblem));
    s1.count = (int)sp.size();
    s1.max_m = max_rows;
    s1.max_n = max_kpad;
    s1.bytes = split_bytes;
    steps.push_back(s1);
  }
  std::vector<OzMmaProblem> mp;
  std::vector<int> tmap;  // 4 ints per output tile, see launch_ozaki_mma
  int total = 0;
  double fl = 0.0;
  for (size_t i = 0; i < probs.size(); ++i) {
    const ZGemmProblem& p = probs[i];
    const int a = which[i].first, b = which[i].second;
    OzMmaProblem q;
    q.SA = slc[a]; q.eA = exs[a]; q.SB = slc[b]; q.eB = exs[b];
    q.C = p.C; q.Cin = p.Cin; q.diag_ptr = p.diag_ptr;
    q.m = p.m; q.n = p.n; q.m_pad = rpad[a]; q.n_pad = rpad[b]; q.k_pad = kpad[a];
    q.ldc = p.ldc; q.ldcin = p.ldcin; q.pad_ = 0;
    q.alpha = p.alpha; q.beta = p.beta; q.diag = p.diag;
    const int tm = q.m_pad / 128, tn = q.n_pad / 64, kc = q.k_pad / 32;
    for (int t = 0; t < tm * tn; ++t) {
      tmap.push_back((int)i);
      tmap.push_back((t / tn) | ((t % tn) << 16));
      tmap.push_back(kc | (tm << 16));
      tmap.push_back(tn);
    }
    total += tm * tn;
    fl += 8.0 * p.m * (double)p.n * p.k;
    mp.push_back(q);
  }
  Step s2;
  s2.kind = Step::OZ_MMA;
  s2.off = push_bytes(mp.data(), mp.size() * sizeof(OzMmaProblem));
  s2.tiles_off = push_bytes(tmap.data(), tmap.size() * sizeof(int));
  s2.count = (int)mp.size();
  s2.total_tiles = total;
  s2.flops = fl;
  s2.form = pairs == 28 || pairs == 34 ? pairs : oz_pairs_;
  steps.push_back(s2);
  // what the next mixed step may use again
  oz_prev_.clear();
  for (size_t i = 0; i < nk; ++i) oz_prev_[view_key(keys[i])] = OzSplitDone{slc[i], exs[i], rpad[i], kpad[i]};
  oz_prev_out_.clear();
  for (const auto& p : probs) {
    if (p.m <= 0 || p.n <= 0) continue;
    const char* lo = reinterpret_cast<const char*>(p.C);
    oz_prev_out_.push_back({lo, lo + sizeof(cplx) * ((size_t)(p.n - 1) * p.ldc + p.m)});
  }
  oz_prev_end_ = need;
  oz_prev_pool_ = oz_pool_;
  oz_prev_steps_ = steps.size();
}

void Plan::gemm_fp64(char opA, char opB, const std::vector<ZGemmProblem>& probs) {
  std::vector<ZGemmProblem> v;
  std::vector<int> starts;
  int total = 0;
  double fl = 0.0;
  bool pre = true;
  int max_k = 0;
  for (const auto& p : probs)
    if (zgemm_tiles(p.m, p.n) > 0) max_k = std::max(max_k, p.k);
  const bool small = zgemm_smallk_ok(gemm_form_, max_k);
  for (const auto& p : probs) {
    int t = small ? zgemm_tiles_smallk(p.m, p.n) : zgemm_tiles(p.m, p.n);
    if (t == 0) continue;
    v.push_back(p);
    starts.push_back(total);
    total += t;
    fl += 8.0 * p.m * (double)p.n * p.k;
    pre = pre && zgemm_preload_ok(p);
  }
  if (v.empty()) return;
  Step s;
  s.kind = Step::GEMM;
  s.opA = opA;
  s.opB = opB;
  s.preload = pre;
  s.form = small ? 3 : gemm_form_;
  s.uniform_tiles = total / (int)v.size();
  if ((long long)s.uniform_tiles * (long long)v.size() != total) s.uniform_tiles = 0;
  for (size_t i = 1; i < starts.size() && s.uniform_tiles; ++i)
    if (starts[i] - starts[i - 1] != s.uniform_tiles) s.uniform_tiles = 0;
  s.off = push_bytes(v.data(), v.size() * sizeof(ZGemmProblem));
  s.tiles_off = push_bytes(starts.data(), starts.size() * sizeof(int));
  s.count = static_cast<int>(v.size());
  s.total_tiles = total;
  s.flops = fl;
  steps.push_back(s);
}

void Plan::inv(const std::vector<InvSpec>& specs) {
  std::vector<ZInvProblem> v;
  int max_n = 0;
  for (const auto& sp : specs) {
    if (sp.n <= 0) continue;
    ZInvProblem p;
    p.W = sp.W; p.F = sp.F; p.Bbuf = sp.Bbuf; p.used = sp.used; p.piv = sp.piv; p.out = sp.out;
    p.info = sp.info; p.n = sp.n; p.ld = sp.ld; p.ldo = sp.ldo; p.pad_ = 0;
    v.push_back(p);
    max_n = std::max(max_n, sp.n);
  }
  if (v.empty()) return;
  int nb = panel_width(max_n);
  bool blocked = nb < max_n;
  size_t off = push_bytes(v.data(), v.size() * sizeof(ZInvProblem));
  double gj_flops = 0.0;
  for (const auto& p : v) gj_flops += 8.0 * p.n * (double)p.n * p.n;
  if (!blocked) {
    Step s;
    s.kind = Step::GJ_PANEL;
    s.off = off; s.count = (int)v.size(); s.k0 = 0; s.nb = nb; s.blocked = 0;
    s.smem = zgj_panel_smem_bytes(max_n, nb);
    s.max_n = max_n;
    s.flops = gj_flops;
    steps.push_back(s);
    return;
  }
  for (int k0 = 0; k0 < max_n; k0 += nb) {
    Step s;
    s.kind = Step::GJ_PANEL;
    s.off = off; s.count = (int)v.size(); s.k0 = k0; s.nb = nb; s.blocked = 1;
    s.smem = zgj_panel_smem_bytes(max_n, nb);
    s.max_n = max_n;
    steps.push_back(s);
    std::vector<ZGemmProblem> g;
    for (const auto& p : v) {
      if (p.n <= k0) continue;
      int w = std::min(nb, p.n - k0);
      g.push_back(gp(p.F, p.n, p.Bbuf, w, p.W, p.ld, p.n, p.n, w, ONE, p.W, p.ld, ONE));
    }
    // W += F Bbuf: INT8 digit products at FP64 accuracy in a mixed plan (the
    // panels stay in FP64), else DMMA
    if (gj_update_int8())
      gemm_mixed('N', 'N', g, 34);
    else
      gemm_fp64('N', 'N', g);
  }
  // the GEMM updates carry their own flop count; the panel work is the rest
  Step u;
  u.kind = Step::GJ_UNPERMUTE;
  u.off = off; u.count = (int)v.size(); u.max_n = max_n;
  steps.push_back(u);
}

int lu_panel_width(int max_n) {
  if (max_n <= 96) return max_n;
  if (max_n <= 400) return 32;
  if (max_n <= 800) return 16;
  return 8;
}

void Plan::getrf(const std::vector<LuSpec>& specs) {
  std::vector<ZLuProblem> v;
  int max_n = 0;
  for (const auto& s : specs) {
    if (s.n <= 0) continue;
    ZLuProblem p;
    p.A = s.A; p.ipiv = s.ipiv; p.Linv = s.Linv; p.T = s.T; p.info = s.info;
    p.n = s.n; p.ld = s.ld; p.nopiv = s.nopiv ? 1 : 0; p.pad_ = 0;
    v.push_back(p);
    max_n = std::max(max_n, s.n);
  }
  if (v.empty()) return;
  const int nb = lu_panel_width(max_n);
  size_t off = push_bytes(v.data(), v.size() * sizeof(ZLuProblem));
  for (int k0 = 0; k0 < max_n; k0 += nb) {
    Step s;
    s.kind = Step::LU_PANEL;
    s.off = off; s.count = (int)v.size(); s.k0 = k0; s.nb = nb; s.max_n = max_n;
    s.smem = zgetrf_panel_smem_bytes(max_n - k0, nb);
    steps.push_back(s);
    if (nb >= max_n) break;
    Step w = s;
    w.kind = Step::LU_SWAP;
    w.smem = 0;
    steps.push_back(w);
    // A12 = L11^{-1} T ;  A22 -= A21 A12
    std::vector<ZGemmProblem> g1, g2;
    for (const auto& p : v) {
      if (p.n <= k0 + nb) continue;
      int wd = std::min(nb, p.n - k0);
      int rest = p.n - k0 - wd;
      cplx* A12 = p.A + k0 + (size_t)(k0 + wd) * p.ld;
      g1.push_back(gp(p.Linv, wd, p.T, wd, A12, p.ld, wd, rest, wd, ONE));
      const cplx* A21 = p.A + (k0 + wd) + (size_t)k0 * p.ld;
      cplx* A22 = p.A + (k0 + wd) + (size_t)(k0 + wd) * p.ld;
      g2.push_back(gp(A21, p.ld, A12, p.ld, A22, p.ld, rest, rest, wd, MONE, A22, p.ld, ONE));
    }
    gemm_fp64('N', 'N', g1);  // factorisations stay in FP64
    gemm_fp64('N', 'N', g2);
  }
}

void Plan::trtri(const std::vector<TriSpec>& specs, bool upper) {
  std::vector<ZTriProblem> v;
  int max_n = 0;
  std::vector<ZBlockOp> zero;
  for (const auto& s : specs) {
    if (s.n <= 0) continue;
    ZTriProblem p;
    p.A = s.A; p.X = s.X; p.n = s.n; p.lda = s.lda; p.ldx = s.ldx; p.pad_ = 0;
    v.push_back(p);
    max_n = std::max(max_n, s.n);
    ZBlockOp z{};
    z.C = s.X; z.ldc = s.ldx; z.m = z.n = s.n; z.kind = ZOP_FILL;
    zero.push_back(z);
  }
  if (v.empty()) return;
  blockops(zero);
  const int nb = kTriNb;
  Step s;
  s.kind = Step::TRI_DIAG;
  s.off = push_bytes(v.data(), v.size() * sizeof(ZTriProblem));
  s.count = (int)v.size(); s.nb = nb; s.blocked = upper ? 1 : 0; s.max_n = max_n;
  s.smem = ztrtri_smem_bytes(nb);
  steps.push_back(s);
  const int q = (max_n + nb - 1) / nb;
  for (int j = 1; j < q; ++j) {
    std::vector<ZGemmProblem> g1, g2;
    for (size_t t = 0; t < v.size(); ++t) {
      const ZTriProblem& p = v[t];
      const TriSpec& sp = specs[t];
      int j0 = j * nb;
      if (j0 >= p.n) continue;
      int wj = std::min(nb, p.n - j0);
      if (upper) {
        // T = X[0:j0, 0:j0] U[0:j0, j-block];  X[0:j0, j-block] = -T X[j-block, j-block]
        g1.push_back(gp(p.X, p.ldx, p.A + (size_t)j0 * p.lda, p.lda, sp.T, p.n, j0, wj, j0, ONE));
        g2.push_back(gp(sp.T, p.n, p.X + j0 + (size_t)j0 * p.ldx, p.ldx, p.X + (size_t)j0 * p.ldx, p.ldx, j0, wj,
                        wj, MONE));
      } else {
        // T = L[j-block, 0:j0] Y[0:j0, 0:j0];  Y[j-block, 0:j0] = -Y[j-block, j-block] T
        g1.push_back(gp(p.A + j0, p.lda, p.X, p.ldx, sp.T, nb, wj, j0, j0, ONE));
        g2.push_back(gp(p.X + j0 + (size_t)j0 * p.ldx, p.ldx, sp.T, nb, p.X + j0, p.ldx, wj, j0, wj, MONE));
      }
    }
    gemm_fp64('N', 'N', g1);
    gemm_fp64('N', 'N', g2);
  }
}

void Plan::blockops(const std::vector<ZBlockOp>& ops) {
  if (ops.empty()) return;
  Step s;
  s.kind = Step::BLOCKOP;
  s.off = push_bytes(ops.data(), ops.size() * sizeof(ZBlockOp));
  s.count = (int)ops.size();
  for (const auto& o : ops) { s.max_m = std::max(s.max_m, o.m); s.max_n = std::max(s.max_n, o.n); }
  steps.push_back(s);
}

void Plan::trace(const std::vector<ZTraceProblemHost>& probs) {
  if (probs.empty()) return;
  Step s;
  s.kind = Step::TRACE;
  s.off = push_bytes(probs.data(), probs.size() * sizeof(ZTraceProblemHost));
  s.count = (int)probs.size();
  steps.push_back(s);
}

cudaError_t Plan::finalize() {
  if (finalized_) return cudaSuccess;
  if (!blob_.empty()) {
    cudaError_t e = cudaMalloc(&dblob_, blob_.size());
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(dblob_, blob_.data(), blob_.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
  }
  std::set<std::pair<char, char>> ops;
  size_t max_smem = 0, lu_smem = 0, tri_smem = 0;
  for (const auto& s : steps) {
    if (s.kind == Step::GEMM) ops.insert({s.opA, s.opB});
    if (s.kind == Step::GJ_PANEL) max_smem = std::max(max_smem, s.smem);
    if (s.kind == Step::LU_PANEL) lu_smem = std::max(lu_smem, s.smem);
    if (s.kind == Step::TRI_DIAG) tri_smem = std::max(tri_smem, s.smem);
  }
  if (lu_smem || tri_smem) {
    cudaError_t e = zlu_prepare(lu_smem, tri_smem);
    if (e != cudaSuccess) return e;
  }
  for (const auto& s : steps)
    if (s.kind == Step::OZ_MMA) {
      cudaError_t e = ozaki_prepare();
      if (e != cudaSuccess) return e;
      break;
    }
  for (auto& o : ops) {
    cudaError_t e = zgemm_prepare(o.first, o.second);
    if (e != cudaSuccess) return e;
  }
  if (max_smem) {
    cudaError_t e = zgj_prepare(max_smem);
    if (e != cudaSuccess) return e;
  }
  finalized_ = true;
  return cudaSuccess;
}

double Plan::flops() const {
  double f = 0.0;
  for (const auto& s : steps) f += s.flops;
  return f;
}

size_t Plan::num_launches() const { return steps.size(); }

cudaError_t Plan::run_events(cudaStream_t stream, const std::vector<cudaEvent_t>& events) {
  if (events.size() < steps.size() + 1) return cudaErrorInvalidValue;
  cudaError_t e = finalize();
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(events[0], stream);
  if (e != cudaSuccess) return e;
  const unsigned char* base = static_cast<const unsigned char*>(dblob_);
  for (size_t i = 0; i < steps.size(); ++i) {
    e = launch_step(steps[i], base, stream);
    if (e == cudaSuccess) e = cudaEventRecord(events[i + 1], stream);
    if (e != cudaSuccess) break;
  }
  fence(stream);
  return e;
}

cudaError_t Plan::run_marked(cudaStream_t stream, const std::function<cudaError_t(int)>& at_mark) {
  cudaError_t e = finalize();
  if (e != cudaSuccess) return e;
  const unsigned char* base = static_cast<const unsigned char*>(dblob_);
  size_t m = 0;
  for (size_t i = 0; i <= steps.size() && e == cudaSuccess; ++i) {
    for (; m < marks_.size() && marks_[m].first == i && e == cudaSuccess; ++m) e = at_mark(marks_[m].second);
    if (i == steps.size() || e != cudaSuccess) break;
    e = launch_step(steps[i], base, stream);
  }
  fence(stream);
  return e;
}

cudaError_t Plan::run(cudaStream_t stream, bool use_graph) {
  cudaError_t e = finalize();
  if (e != cudaSuccess) return e;
  if (use_graph && gexec_ && graph_stream_ == stream) {
    e = cudaGraphLaunch(gexec_, stream);
    fence(stream);
    return e;
  }
  if (use_graph) {
    e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
  }
  const unsigned char* base = static_cast<const unsigned char*>(dblob_);
  for (const auto& s : steps) {
    e = launch_step(s, base, stream);
    if (e != cudaSuccess) break;
  }
  if (use_graph) {
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(stream, &g);
    if (e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return e;
    }
    if (e2 != cudaSuccess) return e2;
    if (gexec_) cudaGraphExecDestroy(gexec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_ = g;
    e = cudaGraphInstantiate(&gexec_, graph_, 0);
    if (e != cudaSuccess) return e;
    graph_stream_ = stream;
    e = cudaGraphLaunch(gexec_, stream);
    fence(stream);
    return e;
  }
  fence(stream);
  return e;
}

cudaError_t Plan::launch_step(const Step& s, const unsigned char* base, cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  {
    switch (s.kind) {
      case Step::GEMM:
        e = launch_zgemm_batched_ex(s.opA, s.opB, s.preload, reinterpret_cast<const ZGemmProblem*>(base + s.off),
                                    reinterpret_cast<const int*>(base + s.tiles_off), s.count, s.total_tiles, stream, s.form,
                                    s.uniform_tiles);
        break;
      case Step::GJ_PANEL:
        e = launch_zgj_panel(reinterpret_cast<const ZInvProblem*>(base + s.off), s.count, s.k0, s.nb, s.blocked,
                             s.smem, stream, s.max_n);
        break;
      case Step::GJ_UNPERMUTE:
        e = launch_zgj_unpermute(reinterpret_cast<const ZInvProblem*>(base + s.off), s.count, s.max_n, stream);
        break;
      case Step::BLOCKOP:
        e = launch_zblockops(reinterpret_cast<const ZBlockOp*>(base + s.off), s.count, s.max_m, s.max_n, stream);
        break;
      case Step::TRACE:
        e = launch_ztrace_prod(base + s.off, s.count, stream);
        break;
      case Step::LU_PANEL:
        e = launch_zgetrf_panel(base + s.off, s.count, s.k0, s.nb, s.smem, stream);
        break;
      case Step::LU_SWAP:
        e = launch_zlaswp_copy(base + s.off, s.count, s.k0, s.nb, s.max_n, stream);
        break;
      case Step::TRI_DIAG:
        e = launch_ztrtri_diag(base + s.off, s.count, s.nb, s.blocked, s.max_n, s.smem, stream);
        break;
      case Step::OZ_SPLIT:
        e = launch_ozaki_split(base + s.off, s.count, s.max_m, s.max_n, stream);
        break;
      case Step::OZ_MMA:
        e = launch_ozaki_mma(base + s.off, base + s.tiles_off, s.total_tiles, err_, stream, s.form);
        break;
    }
  }
  return e;
}

// ---------------------------------------------------------------------------
// RGF

void alloc_rgf_work(Plan& plan, const TriSystem& s, RgfWork& w) {
  int n = s.npl();
  int mb = s.maxb();
  int nb = std::max(plan.panel_width(mb), mb > 112 ? 32 : 0);  // room for any tuned width
  w.g.assign(n, nullptr);
  w.R.assign(n > 0 ? n - 1 : 0, nullptr);
  w.L.assign(n > 0 ? n - 1 : 0, nullptr);
  size_t total = 0;
  for (int i = 0; i < n; ++i) total += (size_t)s.b[i] * s.b[i];
  for (int i = 0; i + 1 < n; ++i) total += 2 * (size_t)s.b[i] * s.b[i + 1];
  total += (size_t)mb * mb;              // W
  total += 2 * (size_t)mb * nb;          // F, Bbuf
  cplx* arena = plan.alloc_c(total);
  size_t o = 0;
  for (int i = 0; i < n; ++i) { w.g[i] = arena + o; o += (size_t)s.b[i] * s.b[i]; }
  for (int i = 0; i + 1 < n; ++i) {
    w.R[i] = arena + o; o += (size_t)s.b[i] * s.b[i + 1];
    w.L[i] = arena + o; o += (size_t)s.b[i] * s.b[i + 1];
  }
  w.W = arena + o; o += (size_t)mb * mb;
  w.F = arena + o; o += (size_t)mb * nb;
  w.Bbuf = arena + o; o += (size_t)mb * nb;
  w.used = static_cast<uint8_t*>(plan.alloc(mb));
  w.piv = static_cast<int*>(plan.alloc(sizeof(int) * mb));
}

static InvSpec inv_spec(const TriSystem& s, RgfWork& w, int i) {
  InvSpec sp;
  sp.W = w.W; sp.n = s.b[i]; sp.ld = s.b[i];
  sp.out = w.g[i]; sp.ldo = s.b[i];
  sp.F = w.F; sp.Bbuf = w.Bbuf; sp.used = w.used; sp.piv = w.piv; sp.info = s.info;
  return sp;
}

void build_rgf_upward(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work) {
  int maxN = 0;
  for (const auto& s : sys) maxN = std::max(maxN, s.npl());
  // bottom layer: X_{N-1} = M[N-1,N-1]  (rgf.jl:144)
  {
    std::vector<ZGemmProblem> pr;
    std::vector<InvSpec> iv;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      int i = s.npl() - 1;
      if (i < 0) continue;
      pr.push_back(gp(nullptr, 1, nullptr, 1, work[k].W, s.b[i], s.b[i], s.b[i], 0, ZERO, s.D[i], s.ldD[i],
                      s.dscale, s.shift));
      pr.back().diag_ptr = s.shift_ptr;
      iv.push_back(inv_spec(s, work[k], i));
    }
    plan.gemm('N', 'N', pr);
    plan.inv(iv);
  }
  for (int j = 1; j < maxN; ++j) {
    // R_i = M[i,i+1] g_{i+1}  (rgf.jl:152-154) and L_{i+1} = g_{i+1} M[i+1,i]  (rgf.jl:157)
    std::vector<ZGemmProblem> rN, lN, lC;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      int i = s.npl() - 1 - j;
      if (i < 0) continue;
      RgfWork& w = work[k];
      rN.push_back(gp(s.U[i], s.ldU[i], w.g[i + 1], s.b[i + 1], w.R[i], s.b[i], s.b[i], s.b[i + 1], s.b[i + 1],
                      s.uscale));
      auto p = gp(w.g[i + 1], s.b[i + 1], s.Lw[i], s.ldL[i], w.L[i], s.b[i + 1], s.b[i + 1], s.b[i], s.b[i + 1],
                  s.lscale);
      (s.lop == 'N' ? lN : lC).push_back(p);
    }
    std::vector<ZGemmProblem> nn = rN;
    nn.insert(nn.end(), lN.begin(), lN.end());
    plan.gemm('N', 'N', nn);
    plan.gemm('N', 'C', lC);
    // X_i = M[i,i] - M[i,i+1] L_{i+1}  (rgf.jl:159-160), then its inverse (rgf.jl:161)
    std::vector<ZGemmProblem> xp;
    std::vector<InvSpec> iv;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      int i = s.npl() - 1 - j;
      if (i < 0) continue;
      RgfWork& w = work[k];
      xp.push_back(gp(s.U[i], s.ldU[i], w.L[i], s.b[i + 1], w.W, s.b[i], s.b[i], s.b[i], s.b[i + 1],
                      cscale(s.uscale, -1.0), s.D[i], s.ldD[i], s.dscale, s.shift));
      xp.back().diag_ptr = s.shift_ptr;
      iv.push_back(inv_spec(s, w, i));
    }
    plan.gemm('N', 'N', xp);
    plan.inv(iv);
  }
}

void build_rgf_downward(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
                        std::vector<TriOut>& out, const std::function<void(int)>& on_final) {
  int maxN = 0;
  for (const auto& s : sys) maxN = std::max(maxN, s.npl());
  // G_11 = X_1^{-1}  (rgf.jl:169)
  {
    std::vector<ZBlockOp> ops;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (s.npl() == 0) continue;
      ZBlockOp o{};
      o.A = work[k].g[0]; o.lda = s.b[0]; o.C = out[k].d[0]; o.ldc = out[k].ldd[0];
      o.m = o.n = s.b[0]; o.kind = ZOP_COPY;
      ops.push_back(o);
    }
    plan.blockops(ops);
  }
  if (on_final && maxN > 0) on_final(0);
  for (int i = 1; i < maxN; ++i) {
    // G[i-1,i] = -G[i-1,i-1] R_{i-1};  G[i,i-1] = -L_i G[i-1,i-1]  (rgf.jl:174,177)
    std::vector<ZGemmProblem> pr;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (i >= s.npl()) continue;
      RgfWork& w = work[k];
      TriOut& o = out[k];
      pr.push_back(gp(o.d[i - 1], o.ldd[i - 1], w.R[i - 1], s.b[i - 1], o.u[i - 1], o.ldu[i - 1], s.b[i - 1], s.b[i],
                      s.b[i - 1], MONE));
      pr.push_back(gp(w.L[i - 1], s.b[i], o.d[i - 1], o.ldd[i - 1], o.l[i - 1], o.ldl[i - 1], s.b[i], s.b[i - 1],
                      s.b[i - 1], MONE));
    }
    plan.gemm('N', 'N', pr);
    // G[i,i] = X_i^{-1} - L_i G[i-1,i]  (rgf.jl:180-181)
    std::vector<ZGemmProblem> dp;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (i >= s.npl()) continue;
      RgfWork& w = work[k];
      TriOut& o = out[k];
      dp.push_back(gp(w.L[i - 1], s.b[i], o.u[i - 1], o.ldu[i - 1], o.d[i], o.ldd[i], s.b[i], s.b[i], s.b[i - 1],
                      MONE, w.g[i], s.b[i], ONE));
    }
    plan.gemm('N', 'N', dp);
    if (on_final) on_final(i);
  }
}

void build_rgf_full_inverse(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
                            std::vector<std::vector<cplx*>>& full) {
  // G[i,j] = -G[i,j-1] R_{j-1};  G[j,i] = -L_j G[j-1,i]  for j >= i+2  (rgf.jl:185-199)
  int maxN = 0;
  for (const auto& s : sys) maxN = std::max(maxN, s.npl());
  for (int d = 2; d < maxN; ++d) {
    std::vector<ZGemmProblem> pr;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      int n = s.npl();
      auto& F = full[k];
      RgfWork& w = work[k];
      for (int i = 0; i + d < n; ++i) {
        int j = i + d;
        if (F[i * n + j] && F[i * n + j - 1])
          pr.push_back(gp(F[i * n + j - 1], s.b[i], w.R[j - 1], s.b[j - 1], F[i * n + j], s.b[i], s.b[i], s.b[j],
                          s.b[j - 1], MONE));
        if (F[j * n + i] && F[(j - 1) * n + i])
          pr.push_back(gp(w.L[j - 1], s.b[j], F[(j - 1) * n + i], s.b[j - 1], F[j * n + i], s.b[j], s.b[j], s.b[i],
                          s.b[j - 1], MONE));
      }
    }
    plan.gemm('N', 'N', pr);
  }
}

// ---------------------------------------------------------------------------
// RKD (recursive Keldysh), src/keldyshndiag.jl:221-317, with every
// be_mldivide!('N', ., ., LU(X_i)) applied as a product with g_i = X_i^{-1}.

void build_rkd(Plan& plan, const std::vector<TriSystem>& sys, std::vector<RgfWork>& work,
               std::vector<HermBlocks>& S, const std::function<void(int)>& on_final) {
  int maxN = 0;
  for (const auto& s : sys) maxN = std::max(maxN, s.npl());
  // workspace: xb diagonal chain (npl blocks), m2/t temporaries (npl blocks each)
  std::vector<std::vector<cplx*>> xb(sys.size()), t1(sys.size()), t2(sys.size());
  for (size_t k = 0; k < sys.size(); ++k) {
    const auto& s = sys[k];
    int n = s.npl();
    size_t tot = 0;
    for (int i = 0; i < n; ++i) tot += 3 * (size_t)s.maxb() * s.maxb();
    cplx* a = plan.alloc_c(tot);
    size_t o = 0;
    size_t bb = (size_t)s.maxb() * s.maxb();
    for (int i = 0; i < n; ++i) {
      xb[k].push_back(a + o); o += bb;
      t1[k].push_back(a + o); o += bb;
      t2[k].push_back(a + o); o += bb;
    }
  }
  // upward RKD pass (keldyshndiag.jl:230-234), ix = N-2 .. 0
  for (int j = 1; j < maxN; ++j) {
    std::vector<ZGemmProblem> p1, p2, p3;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      int i = s.npl() - 1 - j;
      if (i < 0) continue;
      RgfWork& w = work[k];
      HermBlocks& h = S[k];
      // S[i,i] -= R_i S[i,i+1]^H
      p1.push_back(gp(w.R[i], s.b[i], h.u[i], h.ldu[i], h.d[i], h.ldd[i], s.b[i], s.b[i], s.b[i + 1], MONE, h.d[i],
                      h.ldd[i], ONE));
      // S[i,i+1] -= R_i S[i+1,i+1]
      p2.push_back(gp(w.R[i], s.b[i], h.d[i + 1], h.ldd[i + 1], h.u[i], h.ldu[i], s.b[i], s.b[i + 1], s.b[i + 1],
                      MONE, h.u[i], h.ldu[i], ONE));
      // S[i,i] -= S[i,i+1] R_i^H
      p3.push_back(gp(h.u[i], h.ldu[i], w.R[i], s.b[i], h.d[i], h.ldd[i], s.b[i], s.b[i], s.b[i + 1], MONE, h.d[i],
                      h.ldd[i], ONE));
    }
    plan.gemm('N', 'C', p1);
    plan.gemm('N', 'N', p2);
    plan.gemm('N', 'C', p3);
  }
  // central pass, phase A: the X chain (keldyshndiag.jl:270-283)
  //   xb[0] = I;  xb[i] = I + M[i,i-1] g_{i-1} xb[i-1] R_{i-1}
  {
    std::vector<ZBlockOp> ops;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (s.npl() < 2) continue;
      ZBlockOp o{};
      o.C = xb[k][0]; o.ldc = s.b[0]; o.m = o.n = s.b[0]; o.kind = ZOP_IDENTITY; o.alpha = ONE;
      ops.push_back(o);
    }
    plan.blockops(ops);
  }
  for (int i = 1; i + 1 < maxN; ++i) {
    std::vector<ZGemmProblem> a1, a2, a3N, a3C;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (i + 1 >= s.npl()) continue;
      RgfWork& w = work[k];
      // m2[i-1,i] = xb[i-1] R_{i-1}  (:273)
      a1.push_back(gp(xb[k][i - 1], s.b[i - 1], w.R[i - 1], s.b[i - 1], t1[k][i], s.b[i - 1], s.b[i - 1], s.b[i],
                      s.b[i - 1], ONE));
      // xbo[i-1,i] = g_{i-1} m2[i-1,i]  (:274)
      a2.push_back(gp(w.g[i - 1], s.b[i - 1], t1[k][i], s.b[i - 1], t2[k][i], s.b[i - 1], s.b[i - 1], s.b[i],
                      s.b[i - 1], ONE));
      // xb[i] = M[i,i-1] xbo[i-1,i] + I  (:275, :280-283)
      auto p = gp(s.Lw[i - 1], s.ldL[i - 1], t2[k][i], s.b[i - 1], xb[k][i], s.b[i], s.b[i], s.b[i], s.b[i - 1],
                  s.lscale, nullptr, 1, ZERO, ONE);
      (s.lop == 'N' ? a3N : a3C).push_back(p);
    }
    plan.gemm('N', 'N', a1);
    plan.gemm('N', 'N', a2);
    plan.gemm('N', 'N', a3N);
    plan.gemm('C', 'N', a3C);
  }
  // central pass, phase B (all layers at once), keldyshndiag.jl:257-260 and :285-291:
  //   m2[i,i] = g_i xb[i];  m2[i,i+1] = m2[i,i] S[i,i+1];  S[i,i+1] = m2[i,i+1] g_{i+1}^H
  {
    std::vector<ZGemmProblem> b1, b2, b3;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      RgfWork& w = work[k];
      HermBlocks& h = S[k];
      for (int i = 0; i + 1 < s.npl(); ++i) {
        b1.push_back(gp(w.g[i], s.b[i], xb[k][i], s.b[i], t1[k][i], s.b[i], s.b[i], s.b[i], s.b[i], ONE));
        b2.push_back(gp(t1[k][i], s.b[i], h.u[i], h.ldu[i], t2[k][i], s.b[i], s.b[i], s.b[i + 1], s.b[i], ONE));
        b3.push_back(gp(t2[k][i], s.b[i], w.g[i + 1], s.b[i + 1], h.u[i], h.ldu[i], s.b[i], s.b[i + 1], s.b[i + 1],
                        ONE));
      }
    }
    plan.gemm('N', 'N', b1);
    plan.gemm('N', 'N', b2);
    plan.gemm('N', 'C', b3);
  }
  // diagonal rescale (keldyshndiag.jl:296-301): S[i,i] = g_i S[i,i] g_i^H
  {
    std::vector<ZGemmProblem> c1, c2;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      RgfWork& w = work[k];
      HermBlocks& h = S[k];
      for (int i = 0; i < s.npl(); ++i) {
        c1.push_back(gp(w.g[i], s.b[i], h.d[i], h.ldd[i], t1[k][i], s.b[i], s.b[i], s.b[i], s.b[i], ONE));
        c2.push_back(gp(t1[k][i], s.b[i], w.g[i], s.b[i], h.d[i], h.ldd[i], s.b[i], s.b[i], s.b[i], ONE));
      }
    }
    plan.gemm('N', 'N', c1);
    plan.gemm('N', 'C', c2);
  }
  // downward RKD pass (keldyshndiag.jl:313-317), ix = 0 .. N-2
  for (int i = 0; i + 1 < maxN; ++i) {
    std::vector<ZGemmProblem> d1, d2, d3;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (i + 1 >= s.npl()) continue;
      RgfWork& w = work[k];
      HermBlocks& h = S[k];
      // S[i+1,i+1] -= S[i,i+1]^H L_{i+1}^H
      d1.push_back(gp(h.u[i], h.ldu[i], w.L[i], s.b[i + 1], h.d[i + 1], h.ldd[i + 1], s.b[i + 1], s.b[i + 1], s.b[i],
                      MONE, h.d[i + 1], h.ldd[i + 1], ONE));
      // S[i,i+1] -= S[i,i] L_{i+1}^H
      d2.push_back(gp(h.d[i], h.ldd[i], w.L[i], s.b[i + 1], h.u[i], h.ldu[i], s.b[i], s.b[i + 1], s.b[i], MONE,
                      h.u[i], h.ldu[i], ONE));
    }
    plan.gemm('C', 'C', d1);
    plan.gemm('N', 'C', d2);
    std::vector<ZGemmProblem> d3v;
    for (size_t k = 0; k < sys.size(); ++k) {
      const auto& s = sys[k];
      if (i + 1 >= s.npl()) continue;
      RgfWork& w = work[k];
      HermBlocks& h = S[k];
      // S[i+1,i+1] -= L_{i+1} S[i,i+1]
      d3v.push_back(gp(w.L[i], s.b[i + 1], h.u[i], h.ldu[i], h.d[i + 1], h.ldd[i + 1], s.b[i + 1], s.b[i + 1], s.b[i],
                       MONE, h.d[i + 1], h.ldd[i + 1], ONE));
    }
    plan.gemm('N', 'N', d3v);
    // iteration i last reads S[i,i] (d2)
    if (on_final) on_final(i);
  }
  if (on_final && maxN > 0) on_final(maxN - 1);
}

}  // namespace negf
