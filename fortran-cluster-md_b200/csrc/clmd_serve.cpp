// clmd_serve.cpp -- the served mode: a continuous-batching request loop over
// a clmd_ensemble.  Requests are admitted at window boundaries as they arrive
// and as pool atoms free up, run resident on the device alongside everything
// else, and are retired when chk_nucleation fires or their budget is spent.
#include <math.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/clmd.h"

namespace {

struct Prepared {
  std::vector<double> x, y, z, vx, vy, vz;
  double box = 0.0;
  int status = -1;  // -1 pending, CLMD_OK ready, else the generator's error
};

// host worker pool: start states in arrival order, at most kAhead requests
// ahead of admission (a long trace's states are not all held in memory)
class Generator {
 public:
  Generator(const clmd_request* reqs, int n, int threads) : reqs_(reqs), n_(n), prep_(n) {
    for (int t = 0; t < threads; t++) pool_.emplace_back([this] { run(); });
  }
  ~Generator() {
    stop_ = true;
    for (auto& t : pool_) t.join();
  }
  bool ready(int k) {
    std::lock_guard<std::mutex> lock(mu_);
    return prep_[k].status != -1;
  }
  Prepared& get(int k) { return prep_[k]; }
  // requests before k have been admitted or dropped
  void consumed(int k) { consumed_ = k; }
  void release(int k) {
    std::lock_guard<std::mutex> lock(mu_);
    Prepared& p = prep_[k];
    std::vector<double>().swap(p.x);
    std::vector<double>().swap(p.y);
    std::vector<double>().swap(p.z);
    std::vector<double>().swap(p.vx);
    std::vector<double>().swap(p.vy);
    std::vector<double>().swap(p.vz);
  }

 private:
  void run() {
    for (;;) {
      if (stop_) return;
      int k = next_.fetch_add(1);
      if (k >= n_) return;
      while (k >= consumed_.load() + kAhead) {
        if (stop_) return;
        std::this_thread::sleep_for(std::chrono::microseconds(500));
      }
      const clmd_request& r = reqs_[k];
      Prepared p;
      const int n = r.natom;
      p.box = cbrt((double)n / r.rho);
      p.x.resize(n); p.y.resize(n); p.z.resize(n);
      p.vx.resize(n); p.vy.resize(n); p.vz.resize(n);
      int st = clmd_init_random(n, p.box, p.box, p.box, 0.9, r.temp, r.seed, p.x.data(),
                                p.y.data(), p.z.data(), p.vx.data(), p.vy.data(),
                                p.vz.data());
      std::lock_guard<std::mutex> lock(mu_);
      prep_[k] = std::move(p);
      prep_[k].status = st;
    }
  }
  const clmd_request* reqs_;
  int n_;
  std::vector<Prepared> prep_;
  std::vector<std::thread> pool_;
  static constexpr int kAhead = 256;
  std::atomic<int> next_{0};
  std::atomic<int> consumed_{0};
  std::atomic<bool> stop_{false};
  std::mutex mu_;
};

// device time of one round: every resident replica advances about this long
// between two admission points; much shorter rounds spend a noticeable share
// on launches and the per-round host work
constexpr float kMinRoundMs = 25.0f;

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" int clmd_serve(clmd_ensemble* e, const clmd_request* reqs, int32_t nreq,
                          double max_seconds, clmd_request_result* out,
                          clmd_serve_stats* stats) {
  if (!e || !reqs || nreq < 0 || !out) return CLMD_ERR_ARG;
  for (int k = 0; k < nreq; k++) {
    out[k].arrival = reqs[k].arrival;
    out[k].admitted = -1.0;
    out[k].finished = -1.0;
    out[k].natom = reqs[k].natom;
    out[k].steps = 0;
    out[k].done = 0;
    out[k].clbrkt = 0;
    out[k].status = CLMD_OK;
    out[k].pad = 0;
  }
  clmd_serve_stats S;
  memset(&S, 0, sizeof(S));
  unsigned hw = std::thread::hardware_concurrency();
  int threads = hw > 2 ? (int)hw - 1 : 1;
  if (threads > 16) threads = 16;
  Generator gen(reqs, nreq, threads);
  std::vector<int> slot_of(nreq, -1);
  std::vector<int> req_of;  // slot -> request
  std::vector<clmd_replica_result> res(1024);
  const auto t0 = std::chrono::steady_clock::now();
  int next = 0, resident = 0;
  long long resident_atoms = 0;
  int st = CLMD_OK;
  for (;;) {
    double t = now_s(t0);
    if (t > max_seconds) break;
    // admit arrived requests in order while they fit
    while (next < nreq && reqs[next].arrival <= t && gen.ready(next)) {
      Prepared& p = gen.get(next);
      if (p.status != CLMD_OK) {  // the generator could not pack this request
        out[next].done = 0;
        out[next].status = p.status;
        gen.release(next);
        next++;
        gen.consumed(next);
        continue;
      }
      clmd_replica_spec sp;
      memset(&sp, 0, sizeof(sp));
      sp.natom = reqs[next].natom;
      sp.box = p.box;
      sp.temp = reqs[next].temp;
      sp.csover = reqs[next].csover;
      sp.clwait = 0;
      sp.budget = reqs[next].budget;
      sp.ethst = 'N';
      int32_t slot = -1;
      int a = clmd_ens_add(e, &sp, p.x.data(), p.y.data(), p.z.data(), p.vx.data(),
                           p.vy.data(), p.vz.data(), &slot);
      if (a == CLMD_ERR_NOMEM) break;  // wait for space (arrival order)
      if (a != CLMD_OK) {
        st = a;
        break;
      }
      gen.release(next);
      if ((int)req_of.size() <= slot) req_of.resize(slot + 1, -1);
      req_of[slot] = next;
      slot_of[next] = slot;
      out[next].admitted = now_s(t0);
      resident++;
      resident_atoms += sp.natom;
      S.admitted++;
      next++;
      gen.consumed(next);
    }
    if (st) break;
    if (resident > S.peak_resident) S.peak_resident = resident;
    if (resident_atoms > S.peak_atoms) S.peak_atoms = resident_atoms;
    if (resident == 0) {
      if (next >= nreq) break;
      std::this_thread::sleep_for(std::chrono::microseconds(200));
      continue;
    }
    st = clmd_ens_step_timed(e, kMinRoundMs);
    if (st) break;
    S.windows++;
    int32_t n = 0;
    st = clmd_ens_poll(e, res.data(), (int32_t)res.size(), &n);
    if (st) break;
    if (n > (int32_t)res.size()) {
      res.resize(n);
      st = clmd_ens_poll(e, res.data(), n, &n);
      if (st) break;
    }
    double tw = now_s(t0);
    for (int k = 0; k < n; k++) {
      const clmd_replica_result& r = res[k];
      if (r.slot < 0 || r.slot >= (int)req_of.size()) continue;
      int q = req_of[r.slot];
      if (q < 0) continue;
      S.atom_steps += (double)r.natom * (r.step - out[q].steps);
      out[q].steps = r.step;
      if (r.done == 1 || r.done == 2 || r.status) {
        out[q].done = r.status ? 0 : r.done;
        out[q].status = r.status;
        out[q].clbrkt = r.clbrkt;
        out[q].finished = tw;
        S.completed++;
        resident--;
        resident_atoms -= r.natom;
        req_of[r.slot] = -1;
        clmd_ens_remove(e, r.slot);
      }
    }
    if (next >= nreq && resident == 0) break;
  }
  S.wall = now_s(t0);
  if (stats) *stats = S;
  return st;
}
