// Native request server: NEGF solves of different devices submitted from any
// host language (C, Julia through ccall), batched continuously on one GPU.
//
// The reference has no request loop: it solves one system and one energy per
// call (src/matinvertndiag_rgf.jl:114-200, src/keldyshndiag.jl:120-317).  A
// request here is one device (H blocks, Sigma_L, Sigma_R) with a list of
// energies and host output buffers.  submit() stamps the arrival, uploads the
// device and queues the request.  Several lanes -- worker threads, each with
// its own non-blocking CUDA stream -- admit work continuously: whenever the
// HBM budget has room (the library's own estimate, negf_batch_bytes, of every
// group in flight is counted against it), a free lane takes the queued
// requests first in, first out, as many as fit the room left, and solves them
// as one batch plan (negf_solver_create_batch: one launch per recursion step
// over every (device, energy) pair) on its stream.  So a request that arrives
// while other groups are on the GPU starts as soon as memory allows, and its
// launches overlap theirs on the device.  Each lane copies its requests'
// G^R / G^< diagonal blocks and T(E) into the callers' buffers on its own
// stream and marks them done with their latency (arrival to completion).  A
// group that fails to allocate is halved; a single request larger than the
// budget runs alone through negf_solve, which splits its energies.
#include "../../include/negf_b200.h"
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t ticket = 0;
  int64_t bytes = 0;  // negf_batch_bytes estimate of the request alone
  negf_device_t dev = nullptr;
  std::vector<int32_t> sizes;
  std::vector<double> energies;
  void* gr = nullptr;
  void* gl = nullptr;
  double* t = nullptr;
  Clock::time_point arrival;
};

struct Outcome {
  bool done = false;
  int status = NEGF_SUCCESS;
  double latency_s = 0.0;
  std::string message;  // the lane's error text of a failed request
};

size_t per_energy(const std::vector<int32_t>& sizes) {
  size_t p = 0;
  for (int32_t b : sizes) p += (size_t)b * b;
  return p;
}

}  // namespace

struct negf_server_s {
  negf_solve_opts opts{};
  double budget_gb = 0.0;
  double budget = 0.0;        // bytes every group in flight shares
  int device = 0;
  int lanes = 2;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Request>> queue;
  std::map<int64_t, Outcome> outcomes;
  std::vector<double> latencies;
  int64_t next_ticket = 1;
  int64_t groups = 0;
  double inflight_bytes = 0.0;  // estimates of the groups being solved
  int inflight_groups = 0;
  int peak_inflight = 0;        // most groups ever solved at once
  bool stop = false;
  std::vector<std::thread> workers;
};

namespace {

// Greedy first-in-first-out grouping: group sizes (requests per group) such
// that each group's byte estimate fits the budget; a request alone above the
// budget forms a group of one.
std::vector<int> group_sizes(const std::vector<int64_t>& bytes, double budget) {
  std::vector<int> out;
  size_t i = 0;
  while (i < bytes.size()) {
    double used = 0.0;
    int n = 0;
    while (i + n < bytes.size() && (n == 0 || used + (double)bytes[i + n] <= budget)) {
      used += (double)bytes[i + n];
      ++n;
    }
    out.push_back(n);
    i += n;
  }
  return out;
}

// Copy request outputs out of a finished batch solver (device-major layout)
// on the lane's stream, then wait for them.
int deliver(negf_solver_t s, const std::vector<Request*>& group, cudaStream_t st) {
  void *gr = nullptr, *gl = nullptr;
  double* t2 = nullptr;
  if (int r = negf_solver_outputs(s, &gr, &gl, &t2)) return r;
  size_t off = 0, e0 = 0, nt = 0;
  for (Request* q : group) nt += q->energies.size();
  std::vector<double> tt(2 * nt);
  if (t2 && cudaMemcpyAsync(tt.data(), t2, 2 * nt * sizeof(double), cudaMemcpyDeviceToHost, st))
    return NEGF_ERR_CUDA;
  for (Request* q : group) {
    const size_t n = q->energies.size(), per = per_energy(q->sizes), bytes = n * per * sizeof(negf::cplx);
    if (q->gr && gr &&
        cudaMemcpyAsync(q->gr, static_cast<negf::cplx*>(gr) + off, bytes, cudaMemcpyDeviceToHost, st))
      return NEGF_ERR_CUDA;
    if (q->gl && gl &&
        cudaMemcpyAsync(q->gl, static_cast<negf::cplx*>(gl) + off, bytes, cudaMemcpyDeviceToHost, st))
      return NEGF_ERR_CUDA;
    off += n * per;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return NEGF_ERR_CUDA;
  for (Request* q : group) {
    const size_t n = q->energies.size();
    if (q->t && t2)
      for (size_t e = 0; e < n; ++e) q->t[e] = tt[2 * (e0 + e)];
    e0 += n;
  }
  return NEGF_SUCCESS;
}

// Solve a group as one batch plan on stream st; NEGF_ERR_NOMEM is returned to
// the caller (which halves the group) only for groups of two or more requests.
int solve_group(negf_server_s& S, const std::vector<Request*>& group, cudaStream_t st) {
  negf_solve_opts o = S.opts;
  o.want_gr = o.want_gl = o.want_t = 0;
  for (Request* q : group) {
    o.want_gr |= q->gr != nullptr;
    o.want_gl |= q->gl != nullptr;
    o.want_t |= q->t != nullptr;
  }
  if (group.size() == 1) {
    // negf_solve splits the energies of a request that does not fit at once
    Request* q = group[0];
    o.hbm_budget_gb = S.budget / 1e9;
    return negf_solve(q->dev, (int32_t)q->energies.size(), q->energies.data(), &o, q->gr, q->gl, q->t, 0, st);
  }
  std::vector<negf_device_t> devs;
  std::vector<int32_t> counts;
  std::vector<double> E;
  for (Request* q : group) {
    devs.push_back(q->dev);
    counts.push_back((int32_t)q->energies.size());
    E.insert(E.end(), q->energies.begin(), q->energies.end());
  }
  negf_solver_t s = nullptr;
  if (int r = negf_solver_create_batch((int32_t)devs.size(), devs.data(), counts.data(), &o, &s)) return r;
  int r = negf_solver_set_energies(s, E.data(), st);
  // launches replayed directly on the lane's stream (no graph for a one-off plan)
  if (r == NEGF_SUCCESS) r = negf::solver_run_direct(s, st);
  if (r == NEGF_SUCCESS && cudaStreamSynchronize(st) != cudaSuccess) r = NEGF_ERR_CUDA;
  if (r == NEGF_SUCCESS) r = negf_solver_check(s);
  if (r == NEGF_SUCCESS) r = deliver(s, group, st);
  negf_solver_destroy(s);
  return r;
}

void finish(negf_server_s& S, std::vector<std::unique_ptr<Request>>& reqs, int status) {
  const auto now = Clock::now();
  const std::string msg = status == NEGF_SUCCESS ? std::string() : negf::last_error();
  for (auto& q : reqs) negf_device_destroy(q->dev);
  std::lock_guard<std::mutex> lk(S.mu);
  for (auto& q : reqs) {
    Outcome& oc = S.outcomes[q->ticket];
    oc.done = true;
    oc.status = status;
    oc.message = msg;
    oc.latency_s = std::chrono::duration<double>(now - q->arrival).count();
    if (status == NEGF_SUCCESS) S.latencies.push_back(oc.latency_s);
  }
  S.cv_done.notify_all();
}

// One lane: admit the queue's head group whenever the budget has room for it
// next to the groups already in flight (or nothing runs), solve it on this
// lane's stream, release its share of the budget.
void lane_loop(negf_server_s* S) {
  cudaSetDevice(S->device);
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) st = nullptr;
  for (;;) {
    std::vector<std::unique_ptr<Request>> taken;
    double taken_bytes = 0.0;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] {
        if (S->queue.empty()) return S->stop;
        return S->inflight_groups == 0 || S->inflight_bytes + (double)S->queue.front()->bytes <= S->budget;
      });
      if (S->queue.empty()) break;  // stopping with nothing left
      const double room = S->budget - S->inflight_bytes;
      do {
        taken_bytes += (double)S->queue.front()->bytes;
        taken.push_back(std::move(S->queue.front()));
        S->queue.pop_front();
      } while (!S->queue.empty() && taken_bytes + (double)S->queue.front()->bytes <= room);
      S->inflight_bytes += taken_bytes;
      S->peak_inflight = std::max(S->peak_inflight, ++S->inflight_groups);
    }
    // halve a group whose allocation fails; the second half goes back to the queue front
    for (;;) {
      std::vector<Request*> g;
      for (auto& q : taken) g.push_back(q.get());
      const int r = solve_group(*S, g, st);
      if (r == NEGF_ERR_NOMEM && taken.size() > 1) {
        const size_t half = taken.size() / 2;
        std::lock_guard<std::mutex> lk(S->mu);
        for (size_t k = taken.size(); k-- > half;) S->queue.push_front(std::move(taken[k]));
        taken.resize(half);
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->groups;
      }
      if (r != NEGF_SUCCESS && taken.size() > 1) {
        // one request's failure (a singular block, an unsupported shape) does not fail the others
        for (auto& q : taken) {
          std::vector<Request*> one{q.get()};
          const int ri = solve_group(*S, one, st);
          std::vector<std::unique_ptr<Request>> v;
          v.push_back(std::move(q));
          finish(*S, v, ri);
        }
        break;
      }
      finish(*S, taken, r);
      break;
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->inflight_bytes -= taken_bytes;
      --S->inflight_groups;
    }
    S->cv_work.notify_all();
  }
  if (st) cudaStreamDestroy(st);
  S->cv_work.notify_all();
}

}  // namespace

extern "C" {

int negf_server_group_sizes(int32_t nreq, const int64_t* bytes, double budget, int32_t* sizes, int32_t* ngroups) {
  if (nreq < 0 || (nreq > 0 && (!bytes || !sizes)) || !ngroups) {
    negf::set_error("negf_server_group_sizes: bad arguments");
    return NEGF_ERR_INVALID;
  }
  std::vector<int> g = group_sizes(std::vector<int64_t>(bytes, bytes + nreq), budget);
  for (size_t k = 0; k < g.size(); ++k) sizes[k] = g[k];
  *ngroups = (int32_t)g.size();
  return NEGF_SUCCESS;
}

int negf_server_create(const negf_solve_opts* opts, double budget_gb, negf_server_t* out) {
  return negf_server_create_ex(opts, budget_gb, 2, out);
}

int negf_server_create_ex(const negf_solve_opts* opts, double budget_gb, int32_t lanes, negf_server_t* out) {
  if (!opts || !out || lanes < 1 || lanes > 16) {
    negf::set_error("negf_server_create: bad arguments");
    return NEGF_ERR_INVALID;
  }
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    negf::set_error("negf_server_create: no usable CUDA device");
    return NEGF_ERR_CUDA;
  }
  if (opts->sigma_per_energy) {
    negf::set_error("negf_server_create: requests carry constant self-energies (sigma_per_energy = 0)");
    return NEGF_ERR_INVALID;
  }
  auto* S = new negf_server_s();
  S->opts = *opts;
  S->budget_gb = budget_gb;
  S->lanes = lanes;
  cudaGetDevice(&S->device);
  if (budget_gb > 0.0) {
    S->budget = budget_gb * 1e9;
  } else {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
      int d = 0;
      cudaGetDevice(&d);
      S->budget = 0.8 * (double)(fr + negf::cached_bytes(d));  // cached plan chunks are free to the library
    } else {
      S->budget = 0.0;
    }
  }
  for (int k = 0; k < lanes; ++k) S->workers.emplace_back(lane_loop, S);
  *out = S;
  return NEGF_SUCCESS;
}

int negf_server_submit(negf_server_t S, int32_t npl, const int32_t* block_sizes, const void* const* Hd,
                       const void* const* Hu, const void* sigL, const void* sigR, int32_t nE, const double* energies,
                       void* gr_out, void* gl_out, double* t_out, int64_t* ticket) {
  if (!S || npl <= 0 || !block_sizes || !Hd || (npl > 1 && !Hu) || !sigL || !sigR || nE <= 0 || !energies ||
      !ticket) {
    negf::set_error("negf_server_submit: bad arguments");
    return NEGF_ERR_INVALID;
  }
  const auto arrival = Clock::now();  // latency includes the upload below
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != S->device) {
    negf::set_error("negf_server_submit: call with the server's device current (the device is uploaded there)");
    return NEGF_ERR_INVALID;
  }
  auto q = std::make_unique<Request>();
  if (int r = negf_device_create(npl, block_sizes, Hd, Hu, sigL, sigR, &q->dev)) return r;
  q->sizes.assign(block_sizes, block_sizes + npl);
  q->energies.assign(energies, energies + nE);
  q->gr = gr_out;
  q->gl = gl_out;
  q->t = t_out;
  q->arrival = arrival;
  {
    negf_solve_opts o = S->opts;
    o.want_gr = gr_out != nullptr;
    o.want_gl = gl_out != nullptr;
    o.want_t = t_out != nullptr;
    if (negf_batch_bytes(1, &q->dev, &nE, &o, &q->bytes) != NEGF_SUCCESS) q->bytes = 0;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) {
    negf_device_destroy(q->dev);
    negf::set_error("negf_server_submit: the server is shutting down");
    return NEGF_ERR_INVALID;
  }
  q->ticket = S->next_ticket++;
  *ticket = q->ticket;
  S->outcomes[q->ticket] = Outcome{};
  S->queue.push_back(std::move(q));
  S->cv_work.notify_one();
  return NEGF_SUCCESS;
}

int negf_server_poll(negf_server_t S, int64_t ticket, int32_t* done) {
  if (!S || !done) {
    negf::set_error("negf_server_poll: bad arguments");
    return NEGF_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->outcomes.find(ticket);
  if (it == S->outcomes.end()) {
    negf::set_error("negf_server_poll: unknown ticket");
    return NEGF_ERR_INVALID;
  }
  *done = it->second.done ? 1 : 0;
  if (it->second.done && it->second.status != NEGF_SUCCESS)
    negf::set_error("negf_server_poll: the request failed: " + it->second.message);
  return it->second.done ? it->second.status : NEGF_SUCCESS;
}

int negf_server_wait(negf_server_t S, int64_t ticket, double timeout_s, double* latency_s) {
  if (!S) {
    negf::set_error("negf_server_wait: bad arguments");
    return NEGF_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->outcomes.find(ticket);
  if (it == S->outcomes.end()) {
    negf::set_error("negf_server_wait: unknown ticket");
    return NEGF_ERR_INVALID;
  }
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(std::max(0.0, timeout_s)));
  if (!S->cv_done.wait_until(lk, deadline, [&] { return S->outcomes[ticket].done; })) {
    negf::set_error("negf_server_wait: timed out");
    return NEGF_ERR_TIMEOUT;
  }
  const Outcome oc = S->outcomes[ticket];
  if (latency_s) *latency_s = oc.latency_s;
  if (oc.status != NEGF_SUCCESS) negf::set_error("negf_server_wait: the request failed: " + oc.message);
  return oc.status;
}

int negf_server_stats(negf_server_t S, int64_t* completed, int64_t* groups, double* p50_s, double* p99_s) {
  if (!S) {
    negf::set_error("negf_server_stats: bad arguments");
    return NEGF_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  std::vector<double> l = S->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double p) {
    if (l.empty()) return 0.0;
    const double x = p / 100.0 * (double)(l.size() - 1);  // linear interpolation between order statistics
    const size_t i = (size_t)x;
    const double f = x - (double)i;
    return i + 1 < l.size() ? l[i] + f * (l[i + 1] - l[i]) : l[i];
  };
  if (completed) *completed = (int64_t)l.size();
  if (groups) *groups = S->groups;
  if (p50_s) *p50_s = pct(50.0);
  if (p99_s) *p99_s = pct(99.0);
  return NEGF_SUCCESS;
}

int negf_server_destroy(negf_server_t S) {
  if (!S) return NEGF_SUCCESS;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto& w : S->workers)
    if (w.joinable()) w.join();  // the lanes finish the queued requests first
  delete S;
  return NEGF_SUCCESS;
}

int negf_server_stats_ex(negf_server_t S, int64_t* queued, int32_t* inflight_groups, int32_t* peak_inflight_groups,
                         double* inflight_gb) {
  if (!S) {
    negf::set_error("negf_server_stats_ex: bad arguments");
    return NEGF_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  if (queued) *queued = (int64_t)S->queue.size();
  if (inflight_groups) *inflight_groups = S->inflight_groups;
  if (peak_inflight_groups) *peak_inflight_groups = S->peak_inflight;
  if (inflight_gb) *inflight_gb = S->inflight_bytes / 1e9;
  return NEGF_SUCCESS;
}

}  // extern "C"
