// lcs_serve.cpp -- the batching and serving forms (no reference counterpart),
// written against the public C ABI of include/lcs_b200.h only: a batch or a
// server drives ordinary handles the way any host program could.
//
// Batch: every member's steps are enqueued (graph replays on the member's own
// stream, lcs_step_begin) before any is waited for, so the members' kernels
// run concurrently on the GPU; a member's arithmetic is exactly its solo run.
//
// Server: a scheduler thread owns every device call.  It admits queued
// requests oldest first while a slot is free and the admitted runs' predicted
// device bytes (lcs_footprint, the pool each handle allocates) fit the budget,
// then keeps a slice of steps in flight for every admitted run and retires
// finished runs (final state downloaded, handle destroyed, bytes returned).
// User threads only touch host-side queues and results, under a mutex.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lcs_b200.h"

namespace {

thread_local std::string t_err;

int serve_fail(int rc, const std::string& msg) {
  t_err = msg;
  return rc;
}

std::string handle_error(const lcs_handle* h) {
  const char* m = lcs_last_error(h);
  return m ? std::string(m) : std::string();
}

using Clock = std::chrono::steady_clock;

}  // namespace

// ------------------------------------------------------------------ batch
struct MemberTuning {
  int32_t rw_rows = 0, zchunk = 0;
  double share = 1.0, probe_ms = 0.0;
};

struct lcs_batch {
  std::vector<lcs_handle*> members;
  std::vector<lcs_config> cfgs;
  std::vector<MemberTuning> tuning;
  std::vector<lcs_group*> groups;          // members stepped as one graph (lcs_group_*)
  std::vector<std::vector<int32_t>> group_members;
  std::vector<int32_t> group_of;           // member -> index in groups, or -1
};

namespace {

bool grouping_enabled() {
  const char* g = std::getenv("LCS_BATCH_GROUP");
  return !(g && std::string(g) == "0");
}

// Steps one batch of handles once (a group when there is one) and waits.
bool probe_step(const std::vector<lcs_handle*>& probes, lcs_group* pg) {
  bool ok = true;
  size_t begun = 0;
  if (pg) {
    ok = lcs_group_step_begin(pg, 1) == LCS_OK;
    begun = ok ? probes.size() : 0;
  } else {
    for (; begun < probes.size() && ok; begun++) ok = lcs_step_begin(probes[begun], 1) == LCS_OK;
  }
  for (size_t q = 0; q < begun; q++) ok = lcs_step_finish(probes[q], nullptr) == LCS_OK && ok;
  return ok;
}

// The batch's autotuner.  Members that share a shape (dims and precision) get
// the same launch shapes: for every candidate (tile rows of the sweep x z
// chunk x the part of the GPU a launch is sized for) it steps probe handles of
// that shape, one per member, together (as one group when grouping is on;
// zero fields, exactly 20 sweeps per couple, no particles) and times one
// step; the fastest candidate is applied to the members.  Probes never touch
// a member's state, and no result depends on the launch shapes.
int autotune(lcs_batch* b) {
  const size_t m = b->members.size();
  double total_cells = 0.0;
  for (const auto& c : b->cfgs) total_cells += (double)c.dims[0] * c.dims[1] * c.dims[2];
  std::vector<bool> done(m, false);
  for (size_t i = 0; i < m; i++) {
    if (done[i]) continue;
    const lcs_config& ci = b->cfgs[i];
    std::vector<size_t> group;
    for (size_t q = i; q < m; q++) {
      const lcs_config& cq = b->cfgs[q];
      if (cq.dims[0] == ci.dims[0] && cq.dims[1] == ci.dims[1] && cq.dims[2] == ci.dims[2] &&
          cq.precision == ci.precision) {
        group.push_back(q);
        done[q] = true;
      }
    }
    const double cells = (double)ci.dims[0] * ci.dims[1] * ci.dims[2];
    const double share = std::min(1.0, std::max(1e-3, cells / total_cells));
    lcs_config pc = ci;  // the probe: flow only, unforced (zero fields), a fixed sweep count
    pc.mode = LCS_MODE_FLOW;
    pc.n_species = 0;
    pc.forcing = LCS_FORCING_NO;
    pc.itrmin = pc.itrmax = 20;
    pc.use_graphs = 1;
    std::vector<lcs_handle*> probes;
    const int64_t n3 = (int64_t)ci.dims[0] * ci.dims[1] * ci.dims[2];
    std::vector<double> zero((size_t)n3, 0.0);
    for (size_t q = 0; q < group.size(); q++) {
      lcs_handle* h = nullptr;
      if (lcs_create(&pc, &h) != LCS_OK) break;
      if (lcs_upload_flow(h, zero.data(), zero.data(), zero.data(), zero.data()) != LCS_OK) {
        lcs_destroy(h);
        break;
      }
      probes.push_back(h);
    }
    lcs_group* pg = nullptr;
    if (grouping_enabled() && probes.size() >= 2 && probes.size() <= 64 &&
        lcs_group_create(probes.data(), (int32_t)probes.size(), &pg) != LCS_OK)
      pg = nullptr;
    MemberTuning best;
    best.share = share;
    best.probe_ms = 1e300;
    const int nz = ci.dims[2];
    // tile rows: FP32 also has 29-row tiles (two rows a warp)
    std::vector<int32_t> rows_c = {13, 8, 5};
    if (ci.precision == LCS_PRECISION_FP32_MIXED) rows_c.insert(rows_c.begin(), 29);
    std::vector<int32_t> zc_c = {0};
    for (int d : {1, 2, 4})
      if (nz / d >= 8) zc_c.push_back((nz + 2) / d + 2);
    // candidates: tile rows x (the cost model sized for the member's share or
    // for the whole GPU, or a fixed chunk)
    struct Cand { int32_t rows, zc; double share; };
    std::vector<Cand> cands;
    // a grouped launch covers every member of the shape: each member's share of it
    const double share_m = std::max(1e-3, share / (double)std::max<size_t>(1, group.size()));
    for (int32_t rows : rows_c) {
      cands.push_back({rows, 0, share});
      cands.push_back({rows, 0, 1.0});
      if (pg) cands.push_back({rows, 0, share_m});
      for (int32_t zc : zc_c)
        if (zc > 0) cands.push_back({rows, zc, pg ? share_m : share});
    }
    for (const Cand& cd : cands) {
      bool ok = !probes.empty();
      for (lcs_handle* h : probes) ok = ok && lcs_set_tuning(h, cd.rows, cd.zc, cd.share) == LCS_OK;
      for (int rep = 0; ok && rep < 2; rep++) {  // rep 0 captures the graphs; rep 1 is timed
        const auto t0 = Clock::now();
        ok = probe_step(probes, pg);
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        if (ok && rep == 1 && ms < best.probe_ms) {
          best.rw_rows = cd.rows;
          best.zchunk = cd.zc;
          best.share = cd.share;
          best.probe_ms = ms;
        }
      }
    }
    if (pg) lcs_group_destroy(pg);
    for (lcs_handle* h : probes) lcs_destroy(h);
    if (best.probe_ms >= 1e300) {  // no probe could run: the built-in shapes
      best.rw_rows = 0;
      best.zchunk = 0;
      best.share = 1.0;
      best.probe_ms = 0.0;
    }
    for (size_t q : group) {
      const int rc = lcs_set_tuning(b->members[q], best.rw_rows, best.zchunk, best.share);
      if (rc != LCS_OK) return serve_fail(rc, "batch member " + std::to_string(q) + ": " + handle_error(b->members[q]));
      b->tuning[q] = best;
    }
  }
  return LCS_OK;
}

// Members and served runs step on their own streams.  CUDA maps streams onto
// CUDA_DEVICE_MAX_CONNECTIONS hardware work queues (8 unless set); streams
// beyond that share queues and serialise behind each other's launches.  The
// variable is read when the process creates its CUDA context, so this widens
// the queues to the maximum (32) only when no context exists yet and the user
// has not chosen a value.
void widen_work_queues() { setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0); }

// Members with the same dims, precision and launch shapes step as groups of
// up to 64 (lcs_group_create checks the rest: halo and HSMAC settings); a
// member no group accepts steps alone.
void make_groups(lcs_batch* b) {
  const size_t m = b->members.size();
  b->group_of.assign(m, -1);
  if (!grouping_enabled()) return;
  std::vector<bool> done(m, false);
  for (size_t i = 0; i < m; i++) {
    if (done[i]) continue;
    std::vector<int32_t> same;
    for (size_t q = i; q < m; q++) {
      const lcs_config &a = b->cfgs[i], &c = b->cfgs[q];
      const MemberTuning &ta = b->tuning[i], &tc = b->tuning[q];
      if (!done[q] && a.dims[0] == c.dims[0] && a.dims[1] == c.dims[1] && a.dims[2] == c.dims[2] &&
          a.precision == c.precision && ta.rw_rows == tc.rw_rows && ta.zchunk == tc.zchunk && ta.share == tc.share) {
        same.push_back((int32_t)q);
        done[q] = true;
      }
    }
    for (size_t c0 = 0; c0 + 1 < same.size(); c0 += 64) {
      const size_t cn = std::min<size_t>(64, same.size() - c0);
      if (cn < 2) break;
      std::vector<lcs_handle*> hs;
      for (size_t q = 0; q < cn; q++) hs.push_back(b->members[same[c0 + q]]);
      lcs_group* g = nullptr;
      if (lcs_group_create(hs.data(), (int32_t)cn, &g) != LCS_OK) continue;
      const int32_t gi = (int32_t)b->groups.size();
      b->groups.push_back(g);
      b->group_members.emplace_back(same.begin() + c0, same.begin() + c0 + cn);
      for (size_t q = 0; q < cn; q++) b->group_of[same[c0 + q]] = gi;
    }
  }
}

}  // namespace

extern "C" {

const char* lcs_serve_last_error(void) { return t_err.c_str(); }

int lcs_batch_create(const lcs_config* members, int32_t m, lcs_batch** out) {
  if (!out) return serve_fail(LCS_EINVAL, "null output");
  *out = nullptr;
  if (!members || m < 1) return serve_fail(LCS_EINVAL, "a batch needs at least one member config");
  widen_work_queues();
  std::unique_ptr<lcs_batch> b(new lcs_batch);
  for (int32_t i = 0; i < m; i++) {
    lcs_config c = members[i];
    c.use_graphs = 1;  // members run their steps as graph replays
    lcs_handle* h = nullptr;
    const int rc = lcs_create(&c, &h);
    if (rc != LCS_OK) {
      const std::string why = handle_error(nullptr);
      for (lcs_handle* q : b->members) lcs_destroy(q);
      return serve_fail(rc, "batch member " + std::to_string(i) + ": " + why);
    }
    b->members.push_back(h);
    b->cfgs.push_back(c);
  }
  b->tuning.resize(b->members.size());
  const char* tune = std::getenv("LCS_BATCH_TUNE");
  if (!(tune && std::string(tune) == "0")) {
    const int rc = autotune(b.get());
    if (rc != LCS_OK) {
      for (lcs_handle* q : b->members) lcs_destroy(q);
      return rc;
    }
  }  // else: the built-in shapes of a solo run
  make_groups(b.get());
  *out = b.release();
  return LCS_OK;
}

int lcs_batch_tuning(const lcs_batch* b, int32_t i, int32_t* rw_rows, int32_t* zchunk, double* share,
                     double* probe_ms) {
  if (!b) return serve_fail(LCS_EINVAL, "null batch");
  if (i < 0 || i >= (int32_t)b->members.size()) return serve_fail(LCS_EINVAL, "member index out of range");
  const MemberTuning& t = b->tuning[i];
  if (rw_rows) *rw_rows = t.rw_rows;
  if (zchunk) *zchunk = t.zchunk;
  if (share) *share = t.share;
  if (probe_ms) *probe_ms = t.probe_ms;
  return LCS_OK;
}

int lcs_batch_size(const lcs_batch* b, int32_t* m) {
  if (!b || !m) return serve_fail(LCS_EINVAL, "null argument");
  *m = (int32_t)b->members.size();
  return LCS_OK;
}

int lcs_batch_member(lcs_batch* b, int32_t i, lcs_handle** h) {
  if (!b || !h) return serve_fail(LCS_EINVAL, "null argument");
  if (i < 0 || i >= (int32_t)b->members.size()) return serve_fail(LCS_EINVAL, "member index out of range");
  *h = b->members[i];
  return LCS_OK;
}

int lcs_batch_step(lcs_batch* b, int32_t nsteps, lcs_log* logs) {
  if (!b) return serve_fail(LCS_EINVAL, "null batch");
  if (nsteps < 0) return serve_fail(LCS_EINVAL, "nsteps < 0");
  const int32_t m = (int32_t)b->members.size();
  int32_t done = 0;
  while (done < nsteps) {
    const int32_t chunk = std::min<int32_t>(nsteps - done, LCS_MAX_ASYNC_STEPS);
    int first_rc = LCS_OK;
    std::string first_err;
    std::vector<char> begun(m, 0);
    for (size_t gi = 0; gi < b->groups.size() && first_rc == LCS_OK; gi++) {  // enqueue everything first
      const int rc = lcs_group_step_begin(b->groups[gi], chunk);
      if (rc != LCS_OK) {
        first_rc = rc;
        first_err = "batch group " + std::to_string(gi) + ": " + handle_error(nullptr);
        for (int32_t q : b->group_members[gi]) {  // members whose steps were enqueued before the failure
          int32_t d = 0;
          if (lcs_step_poll(b->members[q], &d) == LCS_OK) begun[q] = 1;
        }
      } else {
        for (int32_t q : b->group_members[gi]) begun[q] = 1;
      }
    }
    for (int32_t i = 0; i < m && first_rc == LCS_OK; i++) {
      if (b->group_of[i] >= 0) continue;
      const int rc = lcs_step_begin(b->members[i], chunk);
      if (rc != LCS_OK) {
        first_rc = rc;
        first_err = "batch member " + std::to_string(i) + ": " + handle_error(b->members[i]);
      } else {
        begun[i] = 1;
      }
    }
    for (int32_t i = 0; i < m; i++) {
      if (!begun[i]) continue;
      const int rc = lcs_step_finish(b->members[i], logs ? logs + (size_t)i * nsteps + done : nullptr);
      if (rc != LCS_OK && first_rc == LCS_OK) {
        first_rc = rc;
        first_err = "batch member " + std::to_string(i) + ": " + handle_error(b->members[i]);
      }
    }
    if (first_rc != LCS_OK) return serve_fail(first_rc, first_err);
    done += chunk;
  }
  return LCS_OK;
}

void lcs_batch_destroy(lcs_batch* b) {
  if (!b) return;
  for (lcs_group* g : b->groups) lcs_group_destroy(g);
  for (lcs_handle* h : b->members) lcs_destroy(h);
  delete b;
}

}  // extern "C"

// ----------------------------------------------------------------- server
namespace {

struct SpeciesData {
  std::vector<int64_t> ids;
  std::vector<double> diam, x, y, z, u, v, w;
};

struct Request {
  int64_t ticket = 0;
  lcs_config cfg{};
  // inputs (released once the run is on the device)
  std::vector<double> U, V, W, P;
  std::vector<SpeciesData> sp;
  int interp = 0;
  int64_t nsteps = 0, steps_done = 0;
  int64_t bytes = 0;
  // scheduler-thread state
  lcs_handle* h = nullptr;
  int32_t in_flight = 0;
  // outcome
  int state = LCS_REQ_QUEUED;
  int rc = LCS_OK;
  std::string err;
  std::vector<double> rU, rV, rW, rP;
  std::vector<SpeciesData> rsp;
  lcs_log last{};
  Clock::time_point t_submit, t_done;
};

int64_t interior_cells(const lcs_config& c) { return (int64_t)c.dims[0] * c.dims[1] * c.dims[2]; }

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);  // linear interpolation between order statistics
  const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

struct lcs_server {
  lcs_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv;  // wakes the scheduler (submissions, stop) and drain (completions)
  std::deque<Request*> queue;
  std::map<int64_t, std::unique_ptr<Request>> all;
  std::vector<double> latencies;
  int64_t next_ticket = 1, submitted = 0, completed = 0, failed = 0, active_count = 0;
  int64_t bytes_in_use = 0, peak_bytes = 0;
  double busy_s = 0.0;
  bool stop = false;
  std::thread th;
  std::vector<Request*> active;  // scheduler thread only

  // Create the run's handle and put its initial state on the device.
  int start(Request* r) {
    lcs_handle* h = nullptr;
    int rc = lcs_create(&r->cfg, &h);
    if (rc != LCS_OK) {
      r->err = handle_error(nullptr);
      return rc;
    }
    r->h = h;
    rc = lcs_upload_flow(h, r->U.data(), r->V.data(), r->W.data(), r->P.data());
    for (int s = 0; rc == LCS_OK && s < (int)r->sp.size(); s++) {
      SpeciesData& d = r->sp[s];
      rc = lcs_upload_particles(h, s, (int64_t)d.x.size(), d.ids.empty() ? nullptr : d.ids.data(), d.diam.data(),
                                d.x.data(), d.y.data(), d.z.data(), d.u.data(), d.v.data(), d.w.data());
      if (rc == LCS_OK && r->interp) rc = lcs_init_particle_velocity(h, s);
    }
    if (rc != LCS_OK) r->err = handle_error(h);
    // the inputs are on the device now
    std::vector<double>().swap(r->U);
    std::vector<double>().swap(r->V);
    std::vector<double>().swap(r->W);
    std::vector<double>().swap(r->P);
    std::vector<SpeciesData>().swap(r->sp);
    return rc;
  }

  // Download the final state of a finished run and free its handle.
  int finish(Request* r) {
    const int64_t n3 = interior_cells(r->cfg);
    r->rU.resize(n3);
    r->rV.resize(n3);
    r->rW.resize(n3);
    r->rP.resize(n3);
    int rc = lcs_download_flow(r->h, r->rU.data(), r->rV.data(), r->rW.data(), r->rP.data());
    const int ns = r->cfg.mode == LCS_MODE_FLOW_PARTICLE ? r->cfg.n_species : 0;
    r->rsp.resize(ns);
    for (int s = 0; rc == LCS_OK && s < ns; s++) {
      SpeciesData& d = r->rsp[s];
      const size_t n = (size_t)r->cfg.species[s].nvalid;
      d.ids.resize(n);
      for (auto* a : {&d.diam, &d.x, &d.y, &d.z, &d.u, &d.v, &d.w}) a->resize(n);
      rc = lcs_download_particles(r->h, s, d.ids.data(), d.diam.data(), d.x.data(), d.y.data(), d.z.data(),
                                  d.u.data(), d.v.data(), d.w.data());
    }
    if (rc != LCS_OK) r->err = handle_error(r->h);
    lcs_destroy(r->h);
    r->h = nullptr;
    return rc;
  }

  void retire(Request* r, int rc) {
    std::lock_guard<std::mutex> lk(mu);
    r->t_done = Clock::now();
    bytes_in_use -= r->bytes;
    active_count--;
    if (rc == LCS_OK) {
      r->state = LCS_REQ_DONE;
      completed++;
      latencies.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
    } else {
      r->state = LCS_REQ_FAILED;
      r->rc = rc;
      failed++;
    }
    cv.notify_all();
  }

  void run() {
    std::vector<lcs_log> logs;
    auto t_busy = Clock::now();
    while (true) {
      bool progressed = false;
      // 1. admission: oldest first, while a slot is free and the budget holds
      while (true) {
        Request* r = nullptr;
        {
          std::unique_lock<std::mutex> lk(mu);
          if (stop) return;
          if (queue.empty() || (int)active.size() >= cfg.max_active) break;
          Request* q = queue.front();
          if (bytes_in_use + q->bytes > cfg.hbm_budget_bytes) {
            if (active.empty()) {  // it would not fit even alone
              queue.pop_front();
              q->state = LCS_REQ_FAILED;
              q->rc = LCS_ENOMEM;
              q->err = "request needs " + std::to_string(q->bytes) + " device bytes, over the server budget";
              q->t_done = Clock::now();
              failed++;
              cv.notify_all();
              continue;
            }
            break;
          }
          queue.pop_front();
          bytes_in_use += q->bytes;
          peak_bytes = std::max(peak_bytes, bytes_in_use);
          if (active_count == 0) t_busy = Clock::now();
          active_count++;
          q->state = LCS_REQ_RUNNING;
          r = q;
        }
        const int rc = start(r);
        progressed = true;
        if (rc != LCS_OK) {
          if (r->h) lcs_destroy(r->h);
          r->h = nullptr;
          retire(r, rc);
          continue;
        }
        active.push_back(r);
      }
      // 2. keep a slice of steps in flight for every admitted run
      for (Request* r : active) {
        if (r->in_flight || r->steps_done >= r->nsteps) continue;
        const int32_t n = (int32_t)std::min<int64_t>(cfg.steps_per_slice, r->nsteps - r->steps_done);
        const int rc = lcs_step_begin(r->h, n);
        if (rc != LCS_OK) {
          r->err = handle_error(r->h);
          r->rc = rc;
          r->steps_done = r->nsteps + 1;  // marks the failure for step 3
          continue;
        }
        r->in_flight = n;
      }
      // 3. collect finished slices; retire finished runs
      for (size_t i = 0; i < active.size();) {
        Request* r = active[i];
        bool finished = r->steps_done > r->nsteps;  // a failed begin
        int rc = finished ? r->rc : LCS_OK;
        if (!finished && r->in_flight) {
          int32_t done = 0;
          rc = lcs_step_poll(r->h, &done);
          if (rc == LCS_OK && done) {
            logs.resize(r->in_flight);
            rc = lcs_step_finish(r->h, logs.data());
            if (rc == LCS_OK) {
              r->steps_done += r->in_flight;
              r->last = logs.back();
            }
            r->in_flight = 0;
            progressed = true;
          }
          if (rc != LCS_OK) {
            r->err = handle_error(r->h);
            finished = true;
          }
        }
        if (!finished && r->steps_done >= r->nsteps && !r->in_flight) {
          finished = true;
          rc = finish(r);
        }
        if (finished) {
          if (r->h) {
            lcs_destroy(r->h);
            r->h = nullptr;
          }
          {
            std::lock_guard<std::mutex> lk(mu);
            if (active_count == 1) busy_s += std::chrono::duration<double>(Clock::now() - t_busy).count();
          }
          retire(r, rc);
          active.erase(active.begin() + (long)i);
          progressed = true;
          continue;
        }
        i++;
      }
      if (!progressed) {
        std::unique_lock<std::mutex> lk(mu);
        if (stop) return;
        if (active.empty() && queue.empty()) {
          cv.wait_for(lk, std::chrono::milliseconds(50));
        } else {
          lk.unlock();
          std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
      }
    }
  }
};

extern "C" {

int lcs_server_create(const lcs_server_config* c, lcs_server** out) {
  if (!out) return serve_fail(LCS_EINVAL, "null output");
  *out = nullptr;
  if (!c) return serve_fail(LCS_EINVAL, "null server config");
  if (c->max_active < 1) return serve_fail(LCS_EINVAL, "max_active must be >= 1");
  if (c->steps_per_slice < 1 || c->steps_per_slice > LCS_MAX_ASYNC_STEPS)
    return serve_fail(LCS_EINVAL, "steps_per_slice out of range");
  if (c->hbm_budget_bytes <= 0) return serve_fail(LCS_EINVAL, "hbm_budget_bytes must be positive");
  widen_work_queues();
  std::unique_ptr<lcs_server> s(new lcs_server);
  s->cfg = *c;
  s->th = std::thread([p = s.get()] { p->run(); });
  *out = s.release();
  return LCS_OK;
}

int lcs_server_submit(lcs_server* s, const lcs_request* r, int64_t* ticket) {
  if (!s || !r || !ticket) return serve_fail(LCS_EINVAL, "null argument");
  if (!r->U || !r->V || !r->W || !r->P) return serve_fail(LCS_EINVAL, "null initial field");
  if (r->nsteps < 0) return serve_fail(LCS_EINVAL, "nsteps < 0");
  std::unique_ptr<Request> q(new Request);
  q->cfg = r->config;
  q->cfg.use_graphs = 1;
  q->cfg.device = s->cfg.device;
  int64_t bytes = 0;
  const int rc = lcs_footprint(&q->cfg, &bytes);  // validates the config too
  if (rc != LCS_OK) return serve_fail(rc, handle_error(nullptr));
  q->bytes = bytes;
  const int64_t n3 = interior_cells(q->cfg);
  q->U.assign(r->U, r->U + n3);
  q->V.assign(r->V, r->V + n3);
  q->W.assign(r->W, r->W + n3);
  q->P.assign(r->P, r->P + n3);
  const int ns = q->cfg.mode == LCS_MODE_FLOW_PARTICLE ? q->cfg.n_species : 0;
  q->sp.resize(ns);
  for (int sp = 0; sp < ns; sp++) {
    const lcs_species_state& in = r->species[sp];
    const size_t n = (size_t)q->cfg.species[sp].nvalid;
    if (!in.diam || !in.x || !in.y || !in.z || !in.u || !in.v || !in.w)
      return serve_fail(LCS_EINVAL, "null particle array in species " + std::to_string(sp));
    SpeciesData& d = q->sp[sp];
    if (in.ids) d.ids.assign(in.ids, in.ids + n);
    d.diam.assign(in.diam, in.diam + n);
    d.x.assign(in.x, in.x + n);
    d.y.assign(in.y, in.y + n);
    d.z.assign(in.z, in.z + n);
    d.u.assign(in.u, in.u + n);
    d.v.assign(in.v, in.v + n);
    d.w.assign(in.w, in.w + n);
  }
  q->interp = r->interp_velocity;
  q->nsteps = r->nsteps;
  q->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  q->ticket = s->next_ticket++;
  *ticket = q->ticket;
  s->queue.push_back(q.get());
  s->all[q->ticket] = std::move(q);
  s->submitted++;
  s->cv.notify_all();
  return LCS_OK;
}

int lcs_server_poll(lcs_server* s, int64_t ticket, int32_t* state, int64_t* steps_done) {
  if (!s || !state) return serve_fail(LCS_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return serve_fail(LCS_EINVAL, "unknown ticket");
  *state = it->second->state;
  if (steps_done) *steps_done = std::min(it->second->steps_done, it->second->nsteps);
  return LCS_OK;
}

int lcs_server_result(lcs_server* s, int64_t ticket, double* U, double* V, double* W, double* P,
                      lcs_species_out* species, lcs_log* last_log, double* latency_s) {
  if (!s) return serve_fail(LCS_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return serve_fail(LCS_EINVAL, "unknown ticket");
  Request* r = it->second.get();
  if (r->state == LCS_REQ_FAILED) return serve_fail(r->rc, r->err);
  if (r->state != LCS_REQ_DONE) return serve_fail(LCS_ESTATE, "the request has not finished");
  auto put = [](double* dst, const std::vector<double>& src) {
    if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(double));
  };
  put(U, r->rU);
  put(V, r->rV);
  put(W, r->rW);
  put(P, r->rP);
  if (species)
    for (size_t sp = 0; sp < r->rsp.size(); sp++) {
      const SpeciesData& d = r->rsp[sp];
      put(species[sp].x, d.x);
      put(species[sp].y, d.y);
      put(species[sp].z, d.z);
      put(species[sp].u, d.u);
      put(species[sp].v, d.v);
      put(species[sp].w, d.w);
    }
  if (last_log) *last_log = r->last;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  return LCS_OK;
}

int lcs_server_release(lcs_server* s, int64_t ticket) {
  if (!s) return serve_fail(LCS_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return serve_fail(LCS_EINVAL, "unknown ticket");
  const int st = it->second->state;
  if (st != LCS_REQ_DONE && st != LCS_REQ_FAILED) return serve_fail(LCS_ESTATE, "the request has not finished");
  s->all.erase(it);
  return LCS_OK;
}

int lcs_server_stats_get(lcs_server* s, lcs_server_stats* out) {
  if (!s || !out) return serve_fail(LCS_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->queued = (int64_t)s->queue.size();
  out->active = s->active_count;
  out->bytes_in_use = s->bytes_in_use;
  out->peak_bytes_in_use = s->peak_bytes;
  out->p50_latency_s = percentile(s->latencies, 0.50);
  out->p99_latency_s = percentile(s->latencies, 0.99);
  double m = 0.0;
  for (double v : s->latencies) m += v;
  out->mean_latency_s = s->latencies.empty() ? 0.0 : m / (double)s->latencies.size();
  out->busy_s = s->busy_s;
  return LCS_OK;
}

int lcs_server_drain(lcs_server* s, double timeout_s) {
  if (!s) return serve_fail(LCS_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
  while (s->completed + s->failed < s->submitted) {
    if (s->cv.wait_until(lk, until) == std::cv_status::timeout && s->completed + s->failed < s->submitted)
      return serve_fail(LCS_ETIMEDOUT, "requests still running after the drain timeout");
  }
  return LCS_OK;
}

void lcs_server_destroy(lcs_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  for (Request* r : s->active) {
    if (r->h) {
      if (r->in_flight) lcs_step_finish(r->h, nullptr);  // let in-flight work end before freeing its memory
      lcs_destroy(r->h);
    }
  }
  delete s;
}

}  // extern "C"
