// Serving on top of the batch engine: requests (each one job) are admitted
// while their device footprint fits a byte budget, join the running batch
// at the next step boundary, step with everything else that is running
// (continuous batching), and on completion have their final point state
// copied to host memory and their device memory released, so that queued
// requests can take its place.
//
// Collection never stalls the device: the round in which a request runs
// its last step is followed, in stream order, by copies of its point
// arrays into pinned host memory and by the release of its device memory;
// the host converts those copies during the next advance, while the device
// runs the next round. A request is reported finished once its copies are
// converted (at most one round after its last step).
//
// The caller owns the queue and the clock of arrivals: submit() either
// admits a request at once or answers that it does not fit now (the caller
// keeps it and retries after the next advance()).
#pragma once

#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "engine.cuh"

namespace mpmb200 {

class Server {
 public:
  struct Result {
    int64_t n = 0;
    std::vector<double> x, u, x_t, T, v, active;  // reference layout (3, 3, 3, 9, 1, 1 per point)
  };
  struct Request {
    int job = -1;
    int state = 0;  // 1 running, 4 copying out, 2 done, 3 released, 5 cancelled
    int64_t footprint = 0;
    int64_t points = 0;
    int64_t steps = 0;
    double t_admit = 0.0, t_done = 0.0;
    std::vector<Result> bodies;
  };

  Server(std::unique_ptr<BatchBase> b, int mode, bool keep_debug, int64_t budget)
      : batch_(std::move(b)), mode_(mode), keep_debug_(keep_debug), budget_(budget),
        t0_(std::chrono::steady_clock::now()) {}

  ~Server() {
    batch_->synchronize();
    for (auto& p : pending_) cudaEventDestroy(p.ev);
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    for (auto& kv : pinned_) cudaFreeHost(kv.second);
    for (auto& kv : pinned_size_) cudaFreeHost(kv.first);
  }

  std::string last_error;
  mpmgpu_status fail(mpmgpu_status s, const std::string& m) {
    last_error = m;
    return s;
  }

  int mode() const { return mode_; }

  double clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

  mpmgpu_status footprint(const mpmgpu_job_desc& d, int64_t* bytes) const {
    if (!d.grid || d.nbodies < 1 || !d.bodies || d.nbodies > kMaxBodies) return MPMGPU_ERR_ARG;
    mpmgpu_config cfg = *d.grid;
    cfg.dim = batch_->dim();
    *bytes = job_footprint(cfg, mode(), keep_debug_, d.bodies, d.nbodies, d.ncontacts);
    return MPMGPU_OK;
  }

  // Admits the request if its footprint fits the budget left now.
  // MPMGPU_ERR_STATE: does not fit now, retry later. MPMGPU_ERR_NOMEM: the
  // footprint exceeds the whole budget, so the request can never run.
  mpmgpu_status submit(const mpmgpu_job_desc& d, int* id) {
    if (!d.grid || d.nbodies < 1 || !d.bodies || d.nbodies > kMaxBodies || d.ncontacts < 0 ||
        (d.ncontacts > 0 && !d.contacts))
      return fail(MPMGPU_ERR_ARG, "invalid job description");
    int64_t pts = 0;
    for (int b = 0; b < d.nbodies; b++) pts += d.bodies[b].n;
    mpmgpu_config cfg = *d.grid;
    cfg.dim = batch_->dim();
    const int64_t fp = job_footprint(cfg, mode(), keep_debug_, d.bodies, d.nbodies, d.ncontacts);
    if (fp > budget_)
      return fail(MPMGPU_ERR_NOMEM, "request footprint of " + std::to_string(fp) + " bytes exceeds the whole budget of " +
                                        std::to_string(budget_) + " bytes");
    if (reserved_ + fp > budget_) return fail(MPMGPU_ERR_STATE, "request does not fit the memory budget now");
    int job = -1;
    mpmgpu_status st = batch_->new_job(cfg, d.steps, &job);
    for (int b = 0; b < d.nbodies && st == MPMGPU_OK; b++) st = batch_->add_body(job, d.bodies[b], nullptr);
    for (int c = 0; c < d.ncontacts && st == MPMGPU_OK; c++)
      st = batch_->add_contact(job, d.contacts[c].body1, d.contacts[c].body2, d.contacts[c].mu, nullptr,
                               d.contacts[c].reflected);
    if (st == MPMGPU_OK) st = batch_->set_gravity(job, d.gravity_vector, d.gravity);
    if (st == MPMGPU_OK) st = batch_->admit(job);
    if (st != MPMGPU_OK) {
      const std::string m = batch_->last_error;
      if (job >= 0) batch_->remove_job(job);
      return fail(st, m);
    }
    Request r;
    r.job = job;
    r.state = 1;
    r.footprint = fp;
    r.points = pts;
    r.steps = d.steps;
    r.t_admit = clock();
    reqs_.push_back(std::move(r));
    running_++;
    reserved_ += fp;
    *id = (int)reqs_.size() - 1;
    return MPMGPU_OK;
  }

  // `steps` steps of every running request. Requests that run their last
  // step in this call are copied out and released in stream order; those
  // copied out by earlier calls are converted to host results and reported
  // (they were queued before this call's steps, so their copies complete
  // while the device runs them).
  mpmgpu_status advance(int steps) {
    if (steps < 0) return fail(MPMGPU_ERR_ARG, "negative step count");
    std::vector<Pending> earlier;
    earlier.swap(pending_);
    mpmgpu_status st = batch_->step(steps);
    if (st != MPMGPU_OK) return fail(st, batch_->last_error);
    for (int id = 0; id < (int)reqs_.size(); id++) {
      Request& r = reqs_[(size_t)id];
      if (r.state != 1) continue;
      int64_t done = 0, left = 0;
      batch_->job_state(r.job, &done, &left);
      if (left != 0) continue;
      st = copy_out(id);
      if (st != MPMGPU_OK) return st;
    }
    for (auto& p : earlier) {
      st = finish(p);
      if (st != MPMGPU_OK) return st;
    }
    return MPMGPU_OK;
  }

  int poll(int* ids, int max) {
    int k = 0;
    while (!finished_.empty() && k < max) {
      ids[k++] = finished_.front();
      finished_.pop_front();
    }
    return k;
  }

  mpmgpu_status request(int id, int* state, double* t_admit, double* t_done, int64_t* points, int64_t* steps) const {
    if (id < 0 || id >= (int)reqs_.size()) return MPMGPU_ERR_ARG;
    const Request& r = reqs_[(size_t)id];
    if (state) *state = r.state;
    if (t_admit) *t_admit = r.t_admit;
    if (t_done) *t_done = r.t_done;
    if (points) *points = r.points;
    if (steps) *steps = r.steps;
    return MPMGPU_OK;
  }

  mpmgpu_status result(int id, int body, int field, double* out) {
    if (id < 0 || id >= (int)reqs_.size() || !out) return fail(MPMGPU_ERR_ARG, "no such request");
    const Request& r = reqs_[(size_t)id];
    if (r.state != 2) return fail(MPMGPU_ERR_STATE, "request not finished (or released)");
    if (body < 0 || body >= (int)r.bodies.size()) return fail(MPMGPU_ERR_ARG, "no such body");
    const Result& b = r.bodies[(size_t)body];
    const std::vector<double>* src = nullptr;
    switch (field) {
      case MPMGPU_P_X: src = &b.x; break;
      case MPMGPU_P_U: src = &b.u; break;
      case MPMGPU_P_X_T: src = &b.x_t; break;
      case MPMGPU_P_T: src = &b.T; break;
      case MPMGPU_P_V: src = &b.v; break;
      case MPMGPU_P_ACTIVE: src = &b.active; break;
      default: return fail(MPMGPU_ERR_UNSUPPORTED, "the server keeps x, u, x_t, T, v and active");
    }
    std::copy(src->begin(), src->end(), out);
    return MPMGPU_OK;
  }

  // Cancels a running request between advances: its job leaves the batch at
  // the next step boundary (the steps already queued finish with it, in
  // stream order), its device memory returns to the pool and its footprint
  // to the budget. The other requests' results do not change: every job
  // steps on its own nodes and points.
  mpmgpu_status cancel(int id) {
    if (id < 0 || id >= (int)reqs_.size()) return fail(MPMGPU_ERR_ARG, "no such request");
    Request& r = reqs_[(size_t)id];
    if (r.state != 1) return fail(MPMGPU_ERR_STATE, "request is not running");
    mpmgpu_status st = batch_->remove_job(r.job);
    if (st != MPMGPU_OK) return fail(st, batch_->last_error);
    r.state = 5;
    r.t_done = clock();
    running_--;
    reserved_ -= r.footprint;
    return MPMGPU_OK;
  }

  mpmgpu_status release(int id) {
    if (id < 0 || id >= (int)reqs_.size()) return fail(MPMGPU_ERR_ARG, "no such request");
    Request& r = reqs_[(size_t)id];
    if (r.state != 2) return fail(MPMGPU_ERR_STATE, "request not finished");
    r.bodies.clear();
    r.bodies.shrink_to_fit();
    r.state = 3;
    return MPMGPU_OK;
  }

  void stats(int* running, int64_t* reserved, int64_t* live_points, int64_t* particle_steps_done) const {
    if (running) *running = running_;
    if (reserved) *reserved = reserved_;
    if (live_points) {
      int lj = 0;
      batch_->counts(&lj, live_points);
    }
    if (particle_steps_done) *particle_steps_done = points_done_;
  }

  BatchBase* batch() { return batch_.get(); }

 private:
  struct Pending {
    int id = -1;
    cudaEvent_t ev = nullptr;
    std::vector<std::pair<void*, int64_t>> bodies;  // pinned snapshot, points
  };

  // Pinned host buffers for the snapshots, reused by size.
  mpmgpu_status pinned_get(size_t bytes, void** out) {
    auto it = pinned_.lower_bound(bytes);
    if (it != pinned_.end()) {
      *out = it->second;
      pinned_size_[it->second] = it->first;
      pinned_.erase(it);
      return MPMGPU_OK;
    }
    const size_t cap = std::max<size_t>(bytes, (size_t)1 << 20);
    void* h = nullptr;
    cudaError_t e = cudaHostAlloc(&h, cap, cudaHostAllocDefault);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
    pinned_size_[h] = cap;
    *out = h;
    return MPMGPU_OK;
  }
  void pinned_put(void* h) {
    auto it = pinned_size_.find(h);
    pinned_.emplace(it->second, h);
    pinned_size_.erase(it);
  }

  // Queues the copies of a finished request's bodies and its release; the
  // request leaves the budget now (its memory returns to the pool after
  // the copies, in stream order).
  mpmgpu_status copy_out(int id) {
    Request& r = reqs_[(size_t)id];
    Pending p;
    p.id = id;
    int64_t npts = 0;
    for (int b = 0;; b++) {
      if (batch_->sizes(r.job, b, &npts, nullptr) != MPMGPU_OK) break;
      void* h = nullptr;
      mpmgpu_status st = pinned_get(std::max<size_t>(batch_->snapshot_bytes(npts), 1), &h);
      if (st == MPMGPU_OK) st = batch_->snapshot_body(r.job, b, h);
      if (st != MPMGPU_OK) {
        if (h) pinned_put(h);
        for (auto& hb : p.bodies) pinned_put(hb.first);
        return fail(st, batch_->last_error);
      }
      p.bodies.emplace_back(h, npts);
    }
    if (events_.empty()) {
      cudaEvent_t e = nullptr;
      cudaError_t ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (ce != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(ce));
      events_.push_back(e);
    }
    p.ev = events_.back();
    events_.pop_back();
    cudaError_t ce = cudaEventRecord(p.ev, batch_->stream());
    if (ce != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(ce));
    batch_->remove_job(r.job);
    r.state = 4;
    running_--;
    reserved_ -= r.footprint;
    points_done_ += r.points * r.steps;
    pending_.push_back(std::move(p));
    return MPMGPU_OK;
  }

  // Waits for a request's copies, converts them and reports it finished.
  mpmgpu_status finish(Pending& p) {
    cudaError_t ce = cudaEventSynchronize(p.ev);
    events_.push_back(p.ev);
    if (ce != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("snapshot copy: ") + cudaGetErrorString(ce));
    Request& r = reqs_[(size_t)p.id];
    for (auto& hb : p.bodies) {
      Result res;
      const int64_t n = hb.second;
      res.n = n;
      res.x.assign((size_t)(3 * n), 0.0);
      res.u.assign((size_t)(3 * n), 0.0);
      res.x_t.assign((size_t)(3 * n), 0.0);
      res.T.assign((size_t)(9 * n), 0.0);
      res.v.assign((size_t)n, 0.0);
      res.active.assign((size_t)n, 0.0);
      if (n > 0)
        batch_->snapshot_fields(hb.first, n, res.x.data(), res.u.data(), res.x_t.data(), res.T.data(), res.v.data(),
                                res.active.data());
      pinned_put(hb.first);
      r.bodies.push_back(std::move(res));
    }
    r.state = 2;
    r.t_done = clock();
    finished_.push_back(p.id);
    return MPMGPU_OK;
  }

  std::unique_ptr<BatchBase> batch_;
  int mode_;
  bool keep_debug_;
  int64_t budget_;
  std::chrono::steady_clock::time_point t0_;
  std::vector<Request> reqs_;
  std::deque<int> finished_;
  int running_ = 0;
  int64_t reserved_ = 0;
  int64_t points_done_ = 0;
  std::vector<Pending> pending_;
  std::vector<cudaEvent_t> events_;
  std::multimap<size_t, void*> pinned_;        // free pinned buffers by size
  std::map<void*, size_t> pinned_size_;        // pinned buffers in use
};

}  // namespace mpmb200
