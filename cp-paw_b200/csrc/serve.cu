// Serving runtime: a request loop with continuous batching over wave-function
// sets kept on the GPU (host code only; the device work is the engine's).
//
// A request carries the complete input set of one system (what the Fortran host
// would load into a WVSET) and either a single-point solve (energy and forces,
// nsteps = 0) or nsteps CP steps.  Requests queue in arrival order and are
// admitted while the estimated device memory of all admitted systems stays
// within the HBM budget.  Worker threads each take one unit of work at a time
// from the admitted systems in round-robin order (set-up, one CP step, or the
// single point), each system on its own CUDA stream, so the steps of different
// systems overlap on the device and a request that arrives while others run
// starts as soon as memory allows.  The wave functions stay on the device from
// admission to completion; the handle is released when the request finishes.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuwaves.h"

namespace cuw {
int handle_recycle(cuw_handle* h);  // capi.cu
}

namespace {

using Clock = std::chrono::steady_clock;

// Input arrays of one request: either views of the caller's arrays
// (CUW_REQ_BORROW) or of the copies the job owns.
struct Inputs {
  const int *isp = nullptr, *igvec = nullptr, *minusg = nullptr;
  const double *gbas = nullptr, *gvec = nullptr, *g2 = nullptr, *pro = nullptr, *ylm = nullptr, *mpsi = nullptr,
               *v = nullptr, *dh = nullptr, *dover = nullptr, *r0 = nullptr, *occ = nullptr, *psi = nullptr,
               *mass = nullptr;
};

struct Job {
  long long id = 0;
  cuw_dims dims{};
  Inputs in;
  std::vector<int> own_i;     // owned copies (isp, igvec, minusg)
  std::vector<double> own_d;  // owned copies of the double arrays
  double gweight = 0.0, delt = 0.0, annee = 0.0;
  int lmnxx = 0, lnxx = 0, nsteps = 0, done_steps = 0;
  cuw_handle* h = nullptr;
  bool reused = false;        // h came from the pool: same G set, set-up without cuwaves_set_gset
  bool ready = false;         // set-up done
  uint64_t gkey = 0;          // identity of the G set and sizes (pool key)
  size_t bytes = 0;
  bool busy = false, finished = false;
  int status = CUW_OK;
  std::string err;
  double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<double> force;
  Clock::time_point t_submit, t_done;
};

// 64-bit hash of byte arrays, word by word (a key for pooled handles whose
// G set and sizes equal a new request's)
struct Hash64 {
  uint64_t h = 0x9E3779B97F4A7C15ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
      uint64_t w;
      std::memcpy(&w, b + i, 8);
      mix(w);
    }
    uint64_t w = 0;
    std::memcpy(&w, b + i, n - i);
    mix(w ^ ((uint64_t)n << 56));
  }
  void mix(uint64_t w) {
    h ^= w + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
  }
};

// projectors of the set (sum over atoms of 2l+1 per radial function)
int count_projectors(const cuw_dims& d, const int* isp) {
  int n = 0;
  for (int a = 0; a < d.nat; ++a) {
    const int s = isp[a] - 1;
    for (int ln = 0; ln < d.lnx[s]; ++ln) n += 2 * d.lox[s][ln] + 1;
  }
  return n;
}

// Upper estimate of the device memory of one handle (the allocations of
// cuwaves_create and the FFT set-up, plus the split-K scratch).
size_t estimate_bytes(const cuw_dims& d, const int* isp) {
  const size_t ldg = (size_t)((d.ngl + 31) / 32) * 32, nbh = d.nbh, nb = d.nb, ngl = d.ngl;
  const size_t npro = count_projectors(d, isp);
  size_t nbare = 0;
  for (int s = 0; s < d.nsp; ++s) nbare += d.lnx[s];
  const size_t nr = (size_t)d.nr1 * d.nr2 * d.nr3;
  size_t b = 4 * ldg * nbh * 16;                       // psi0, psim, hpsi, opsi
  b += 4 * nbh * npro * 16;                            // proj, oproj, hproj, pbuf
  b += 2 * nb * nb * 16 + 24 * nb * nb * 8;            // Lagrange and solve matrices
  b += ngl * (3 * 4 + 7 * 8) + ngl * (nbare + d.lmx) * 8;  // G set and tables
  b += ngl * (size_t)d.nat * 16;                       // EIGR
  b += nr * 8;                                         // V(r)
  b += std::min(nbh * nr * 16, ((size_t)48 << 20) + nr * 16);  // FFT work grid
  b += (size_t)20 << 20;                               // split-K partials and small tables
  if (d.precision == CUW_PREC_MIXED) b += ldg * npro * 8;  // fp32 projector table
  else b += ldg * npro * 16;                               // fp64 projector table
  return b;
}

}  // namespace

// requests with at least this many CP steps replay their steps as CUDA graphs
constexpr int kGraphSteps = 64;
constexpr double kLongWork = 1e8;  // bands x plane waves x steps of a long request

struct cuw_server {
  size_t budget = 0;
  int max_active = 0;         // admitted sets at most (sets beyond wait in the queue)
  std::mutex mu;
  std::condition_variable cv;
  std::map<long long, std::unique_ptr<Job>> jobs;
  std::deque<Job*> queue;    // submitted, not admitted
  std::vector<Job*> active;  // admitted, unfinished
  size_t rr = 0;             // round-robin position in active
  size_t in_use = 0, peak = 0;
  long long next_id = 1, completed = 0, failed = 0;
  std::vector<double> latencies_ms;
  Clock::time_point t_first, t_last;
  bool have_first = false, stop = false;
  double busy_integral = 0.0;  // time-weighted number of admitted systems
  Clock::time_point t_mark;
  std::vector<std::thread> workers;
  // handles of finished requests, kept for requests of the same G set and
  // sizes (no device allocation at their set-up); their bytes stay in in_use
  std::multimap<uint64_t, std::pair<cuw_handle*, size_t>> pool;
  std::deque<std::pair<uint64_t, cuw_handle*>> pool_order;  // oldest first
  long long reused = 0;

  void pool_drop(cuw_handle* h) {
    for (auto it = pool_order.begin(); it != pool_order.end(); ++it)
      if (it->second == h) {
        pool_order.erase(it);
        break;
      }
  }
  // destroys the oldest pooled handle (false when the pool is empty)
  bool evict_one() {
    if (pool_order.empty()) return false;
    const auto [key, h] = pool_order.front();
    pool_order.pop_front();
    auto r = pool.equal_range(key);
    for (auto it = r.first; it != r.second; ++it)
      if (it->second.first == h) {
        in_use -= it->second.second;
        pool.erase(it);
        break;
      }
    cuwaves_destroy(h);
    return true;
  }

  void account(Clock::time_point now) {
    busy_integral += std::chrono::duration<double>(now - t_mark).count() * (double)active.size();
    t_mark = now;
  }

  // admission in arrival order while the budget allows
  void admit() {
    while (!queue.empty()) {
      Job* j = queue.front();
      if ((int)active.size() >= max_active) break;
      auto hit = pool.find(j->gkey);
      if (hit != pool.end()) {
        // a pooled handle of the same G set: its memory is already counted
        j->h = hit->second.first;
        j->bytes = hit->second.second;
        j->reused = true;
        pool_drop(j->h);
        pool.erase(hit);
        ++reused;
      } else {
        while (in_use + j->bytes > budget && evict_one()) {
        }
        if (in_use + j->bytes > budget) break;
        in_use += j->bytes;
      }
      queue.pop_front();
      account(Clock::now());
      peak = std::max(peak, in_use);
      active.push_back(j);
    }
  }

  Job* pick() {
    const size_t n = active.size();
    for (size_t k = 0; k < n; ++k) {
      Job* j = active[(rr + k) % n];
      if (!j->busy) {
        rr = (rr + k + 1) % n;
        return j;
      }
    }
    return nullptr;
  }

  static void fail(Job* j, int rc, const char* what) {
    j->status = rc;
    char buf[256] = {0};
    if (j->h) cuwaves_last_error(j->h, buf, sizeof(buf));
    j->err = std::string(what) + ": " + buf;
  }

  // one unit of work of job j, outside the lock
  static bool run_unit(Job* j) {
    int rc;
    if (!j->ready) {
      const Inputs& in = j->in;
      j->ready = true;
      if (j->h) {
        // a pooled handle of the same G set: back to the state of a fresh one
        if ((rc = cuw::handle_recycle(j->h)) != CUW_OK) {
          fail(j, rc, "recycle");
          return true;
        }
      } else {
        j->dims.isp = in.isp;
        if ((rc = cuwaves_create(&j->dims, &j->h)) != CUW_OK) {
          j->h = nullptr;
          fail(j, rc, "create");
          return true;
        }
        if ((rc = cuwaves_set_gset(j->h, in.igvec, in.minusg, in.gbas, in.gvec, in.g2, in.pro, in.ylm, in.mpsi,
                                   nullptr, j->gweight)) != CUW_OK) {
          fail(j, rc, "set-up");
          return true;
        }
      }
      // Step graphs pay for their capture and instantiation (two per set)
      // only over long runs; on the serving mix of 20-step requests they
      // nearly halved the measured capacity (8.3 against 15-17 solves/s).
      cuwaves_set_option(j->h, CUW_OPT_GRAPHS, j->nsteps < kGraphSteps ? 0.0 : 1.0);
      // the longest requests (bands x plane waves x steps at least kLongWork)
      // set the latency tail: their kernels go first when SMs free up
      const double work = (double)j->dims.nb * j->dims.ngl * std::max(1, j->nsteps);
      cuwaves_set_option(j->h, CUW_OPT_STREAM_PRIORITY, work >= kLongWork ? 1.0 : 0.0);
      // PSIM starts equal to PSI0 (from rest): its Gram-Schmidt would repeat
      // PSI0's bit for bit, so WAVES$STOP copies it instead
      if ((rc = cuwaves_set_potential(j->h, in.v)) || (rc = cuwaves_set_dh(j->h, j->lmnxx, in.dh)) ||
          (rc = cuwaves_set_do(j->h, j->lnxx, in.dover)) || (rc = cuwaves_reset_atoms(j->h, in.r0)) ||
          (rc = cuwaves_set_occ(j->h, in.occ)) || (rc = cuwaves_set_dynamics(j->h, j->delt, j->annee)) ||
          (rc = cuwaves_upload_psi(j->h, CUW_PSI0, in.psi)) || (rc = cuwaves_gramschmidt(j->h, CUW_PSI0, in.r0)) ||
          (rc = cuwaves_stop(j->h)) || (rc = cuwaves_projections(j->h))) {
        fail(j, rc, "set-up");
        return true;
      }
      return false;
    }
    j->force.assign(3 * (size_t)j->dims.nat, 0.0);
    if (j->nsteps == 0) {
      if ((rc = cuwaves_etot(j->h, j->out, j->force.data())) != CUW_OK) fail(j, rc, "single point");
      return true;
    }
    const bool move = j->in.mass != nullptr;
    if ((rc = cuwaves_cp_step(j->h, move ? 1 : 0, j->in.mass, 200, 1e-8, j->out,
                              j->force.data())) != CUW_OK) {
      fail(j, rc, "CP step");
      return true;
    }
    return ++j->done_steps >= j->nsteps;
  }

  void worker() {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
      admit();
      Job* j = pick();
      if (!j) {
        cv.wait(lk);
        continue;
      }
      j->busy = true;
      lk.unlock();
      const bool done = run_unit(j);
      if (done && j->h && j->status != CUW_OK) {
        cuwaves_destroy(j->h);
        j->h = nullptr;
      }
      lk.lock();
      j->busy = false;
      if (done) {
        const Clock::time_point now = Clock::now();
        account(now);
        j->finished = true;
        j->t_done = now;
        t_last = now;
        active.erase(std::find(active.begin(), active.end(), j));
        if (rr > 0 && rr >= active.size()) rr = 0;
        if (j->h) {
          // into the pool; its bytes stay counted until it is evicted or reused
          pool.emplace(j->gkey, std::make_pair(j->h, j->bytes));
          pool_order.emplace_back(j->gkey, j->h);
          j->h = nullptr;
        } else {
          in_use -= j->bytes;
        }
        if (j->status == CUW_OK) {
          ++completed;
          latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - j->t_submit).count());
        } else {
          ++failed;
        }
      }
      cv.notify_all();
    }
  }
};

namespace {

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" int cuwaves_server_create(size_t hbm_budget, int nworkers, cuw_server** out) {
  if (!out || nworkers < 1 || nworkers > 64 || hbm_budget == 0) return CUW_ERR_ARG;
  cuw_server* s = new (std::nothrow) cuw_server;
  if (!s) return CUW_ERR_NOMEM;
  s->budget = hbm_budget;
  s->max_active = 4 * nworkers;
  s->t_mark = Clock::now();
  for (int w = 0; w < nworkers; ++w) s->workers.emplace_back([s] { s->worker(); });
  *out = s;
  return CUW_OK;
}

extern "C" int cuwaves_server_set_max_active(cuw_server* s, int max_active) {
  if (!s || max_active < 1) return CUW_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_active = max_active;
  s->cv.notify_all();
  return CUW_OK;
}

extern "C" int cuwaves_server_submit(cuw_server* s, const cuw_request* r, long long* id) {
  if (!s || !r || !id) return CUW_ERR_ARG;
  const cuw_dims& d = r->dims;
  if (d.ngl <= 0 || d.nb <= 0 || d.nbh <= 0 || d.nat <= 0 || d.nsp <= 0 || d.nsp > CUW_MAXSP || d.lmx <= 0 ||
      d.nr1 <= 0 || d.nr2 <= 0 || d.nr3 <= 0 || !d.isp || r->nsteps < 0 || r->lmnxx <= 0 || r->lnxx <= 0)
    return CUW_ERR_ARG;
  for (int a = 0; a < d.nat; ++a)
    if (d.isp[a] < 1 || d.isp[a] > d.nsp) return CUW_ERR_ARG;
  for (int sp = 0; sp < d.nsp; ++sp)
    if (d.lnx[sp] < 0 || d.lnx[sp] > CUW_MAXLN) return CUW_ERR_ARG;
  std::unique_ptr<Job> j(new (std::nothrow) Job);
  if (!j) return CUW_ERR_NOMEM;
  j->dims = d;
  const size_t ngl = d.ngl, nat = d.nat, nr = (size_t)d.nr1 * d.nr2 * d.nr3;
  size_t nbare = 0;
  for (int sp = 0; sp < d.nsp; ++sp) nbare += d.lnx[sp];
  // (source, element count) of every array, in the order of Inputs
  const int* isrc[3] = {d.isp, r->igvec, r->minusg};
  const size_t icnt[3] = {nat, 3 * ngl, ngl};
  const double* dsrc[13] = {r->gbas, r->gvec, r->g2, r->pro, r->ylm, r->mpsi, r->v,
                            r->dh, r->dover, r->r0, r->occ, r->psi, r->mass};
  const size_t dcnt[13] = {9, 3 * ngl, ngl, ngl * nbare, ngl * (size_t)d.lmx, ngl, nr,
                           2 * (size_t)r->lmnxx * r->lmnxx * nat, (size_t)r->lnxx * r->lnxx * d.nsp, 3 * nat,
                           (size_t)d.nb, 2 * ngl * (size_t)d.nbh, nat};
  for (int k = 0; k < 3; ++k)
    if (!isrc[k]) return CUW_ERR_ARG;
  for (int k = 0; k < 12; ++k)  // mass (the last) is optional
    if (!dsrc[k]) return CUW_ERR_ARG;
  const int* ip[3];
  const double* dp[13];
  if (r->flags & CUW_REQ_BORROW) {
    for (int k = 0; k < 3; ++k) ip[k] = isrc[k];
    for (int k = 0; k < 13; ++k) dp[k] = dsrc[k];
  } else {
    size_t ni = 0, nd = 0;
    for (int k = 0; k < 3; ++k) ni += icnt[k];
    for (int k = 0; k < 13; ++k) nd += dsrc[k] ? dcnt[k] : 0;
    try {
      j->own_i.resize(ni);
      j->own_d.resize(nd);
    } catch (const std::bad_alloc&) {
      return CUW_ERR_NOMEM;
    }
    size_t oi = 0, od = 0;
    for (int k = 0; k < 3; ++k) {
      std::memcpy(j->own_i.data() + oi, isrc[k], sizeof(int) * icnt[k]);
      ip[k] = j->own_i.data() + oi;
      oi += icnt[k];
    }
    for (int k = 0; k < 13; ++k) {
      dp[k] = nullptr;
      if (!dsrc[k]) continue;
      std::memcpy(j->own_d.data() + od, dsrc[k], sizeof(double) * dcnt[k]);
      dp[k] = j->own_d.data() + od;
      od += dcnt[k];
    }
  }
  Inputs& in = j->in;
  in.isp = ip[0], in.igvec = ip[1], in.minusg = ip[2];
  in.gbas = dp[0], in.gvec = dp[1], in.g2 = dp[2], in.pro = dp[3], in.ylm = dp[4], in.mpsi = dp[5], in.v = dp[6];
  in.dh = dp[7], in.dover = dp[8], in.r0 = dp[9], in.occ = dp[10], in.psi = dp[11], in.mass = dp[12];
  j->dims.isp = nullptr;
  j->gweight = r->gweight;
  j->delt = r->delt;
  j->annee = r->annee;
  j->lmnxx = r->lmnxx;
  j->lnxx = r->lnxx;
  j->nsteps = r->nsteps;
  j->bytes = estimate_bytes(d, in.isp);
  if (j->bytes > s->budget) return CUW_ERR_NOMEM;  // could never be admitted
  {
    // sizes and G set: a pooled handle with the same key serves this request
    Hash64 hk;
    cuw_dims dk = d;
    dk.isp = nullptr;
    hk.add(&dk, sizeof(dk));
    hk.add(in.isp, sizeof(int) * nat);
    hk.add(in.igvec, sizeof(int) * 3 * ngl);
    hk.add(in.minusg, sizeof(int) * ngl);
    hk.add(in.gbas, sizeof(double) * 9);
    hk.add(in.gvec, sizeof(double) * 3 * ngl);
    hk.add(in.g2, sizeof(double) * ngl);
    hk.add(in.pro, sizeof(double) * ngl * nbare);
    hk.add(in.ylm, sizeof(double) * ngl * (size_t)d.lmx);
    hk.add(in.mpsi, sizeof(double) * ngl);
    const double gw = r->gweight;
    const int lx[2] = {r->lmnxx, r->lnxx};
    hk.add(&gw, sizeof(gw));
    hk.add(lx, sizeof(lx));
    j->gkey = hk.h;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return CUW_ERR_STATE;
  j->id = s->next_id++;
  j->t_submit = Clock::now();
  if (!s->have_first) {
    s->have_first = true;
    s->t_first = j->t_submit;
  }
  *id = j->id;
  s->queue.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  s->cv.notify_all();
  return CUW_OK;
}

extern "C" int cuwaves_server_poll(cuw_server* s, long long id, int* done, int* status, double* out,
                                   double* force, double* latency_ms) {
  if (!s || !done) return CUW_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return CUW_ERR_ARG;
  Job* j = it->second.get();
  *done = j->finished ? 1 : 0;
  if (!j->finished) return CUW_OK;
  if (status) *status = j->status;
  if (out) std::memcpy(out, j->out, sizeof(j->out));
  if (force && !j->force.empty()) std::memcpy(force, j->force.data(), sizeof(double) * j->force.size());
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
  return CUW_OK;
}

extern "C" int cuwaves_server_error(cuw_server* s, long long id, char* buf, int len) {
  if (!s || !buf || len <= 0) return CUW_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return CUW_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", it->second->err.c_str());
  return CUW_OK;
}

extern "C" int cuwaves_server_release(cuw_server* s, long long id) {
  if (!s) return CUW_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end() || !it->second->finished) return CUW_ERR_ARG;
  s->jobs.erase(it);
  return CUW_OK;
}

extern "C" int cuwaves_server_wait_all(cuw_server* s) {
  if (!s) return CUW_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv.wait(lk, [s] { return s->queue.empty() && s->active.empty(); });
  return s->failed ? CUW_ERR_STATE : CUW_OK;
}

extern "C" int cuwaves_server_stats(cuw_server* s, double* out, int n) {
  if (!s || !out || n < 0) return CUW_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->account(Clock::now());
  const double span = s->have_first ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
  const double v[10] = {(double)s->completed,
                        (double)s->failed,
                        percentile(s->latencies_ms, 0.50),
                        percentile(s->latencies_ms, 0.99),
                        span > 0 ? (double)s->completed / span : 0.0,
                        (double)s->peak,
                        (double)s->in_use,
                        (double)(s->queue.size() + s->active.size()),
                        span > 0 ? s->busy_integral / span : 0.0,
                        s->latencies_ms.empty() ? 0.0 : *std::max_element(s->latencies_ms.begin(), s->latencies_ms.end())};
  for (int i = 0; i < n && i < 10; ++i) out[i] = v[i];
  return CUW_OK;
}

extern "C" int cuwaves_server_destroy(cuw_server* s) {
  if (!s) return CUW_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;  // workers finish the unit they hold, then leave
    s->cv.notify_all();
  }
  for (auto& t : s->workers) t.join();
  for (Job* j : s->active)
    if (j->h) cuwaves_destroy(j->h);
  for (auto& kv : s->pool) cuwaves_destroy(kv.second.first);
  delete s;
  return CUW_OK;
}
