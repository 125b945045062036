// Serving on top of the batch engine: requests (each one job) are admitted
// while their device footprint fits a byte budget, join the running batch
// at the next step boundary, step with everything else that is running
// (continuous batching), and on completion have their final point state
// copied to host memory and their device memory released, so that queued
// requests can take its place.
//
// The caller owns the queue and the clock of arrivals: submit() either
// admits a request at once or answers that it does not fit now (the caller
// keeps it and retries after the next advance()).
#pragma once

#include <chrono>
#include <deque>
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
    int state = 0;  // 1 running, 2 done, 3 released
    int64_t footprint = 0;
    int64_t points = 0;
    int64_t steps = 0;
    double t_admit = 0.0, t_done = 0.0;
    std::vector<Result> bodies;
  };

  Server(std::unique_ptr<BatchBase> b, bool mixed, bool keep_debug, int64_t budget)
      : batch_(std::move(b)), mixed_(mixed), keep_debug_(keep_debug), budget_(budget),
        t0_(std::chrono::steady_clock::now()) {}

  std::string last_error;
  mpmgpu_status fail(mpmgpu_status s, const std::string& m) {
    last_error = m;
    return s;
  }

  double clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

  mpmgpu_status footprint(const mpmgpu_job_desc& d, int64_t* bytes) const {
    if (!d.grid || d.nbodies < 1 || !d.bodies || d.nbodies > kMaxBodies) return MPMGPU_ERR_ARG;
    std::vector<int64_t> n((size_t)d.nbodies);
    for (int b = 0; b < d.nbodies; b++) n[(size_t)b] = d.bodies[b].n;
    mpmgpu_config cfg = *d.grid;
    cfg.dim = batch_->dim();
    *bytes = job_footprint(cfg, mixed_, keep_debug_, d.nbodies, n.data(), d.ncontacts);
    return MPMGPU_OK;
  }

  // Admits the request if its footprint fits the budget now (or nothing is
  // running, so that a request larger than the budget still runs alone).
  // MPMGPU_ERR_STATE: does not fit now, retry later.
  mpmgpu_status submit(const mpmgpu_job_desc& d, int* id) {
    if (!d.grid || d.nbodies < 1 || !d.bodies || d.nbodies > kMaxBodies || d.ncontacts < 0 ||
        (d.ncontacts > 0 && !d.contacts))
      return fail(MPMGPU_ERR_ARG, "invalid job description");
    std::vector<int64_t> n((size_t)d.nbodies);
    int64_t pts = 0;
    for (int b = 0; b < d.nbodies; b++) pts += (n[(size_t)b] = d.bodies[b].n);
    mpmgpu_config cfg = *d.grid;
    cfg.dim = batch_->dim();
    const int64_t fp = job_footprint(cfg, mixed_, keep_debug_, d.nbodies, n.data(), d.ncontacts);
    if (running_ > 0 && reserved_ + fp > budget_) return fail(MPMGPU_ERR_STATE, "request does not fit the memory budget now");
    int job = -1;
    mpmgpu_status st = batch_->new_job(cfg, d.steps, &job);
    for (int b = 0; b < d.nbodies && st == MPMGPU_OK; b++) st = batch_->add_body(job, d.bodies[b], nullptr);
    for (int c = 0; c < d.ncontacts && st == MPMGPU_OK; c++)
      st = batch_->add_contact(job, d.contacts[c].body1, d.contacts[c].body2, d.contacts[c].mu, nullptr);
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

  // `steps` steps of every running request, then collection of the ones
  // that have run all their steps (results to host memory, device memory
  // released).
  mpmgpu_status advance(int steps) {
    if (steps < 0) return fail(MPMGPU_ERR_ARG, "negative step count");
    mpmgpu_status st = batch_->step(steps);
    if (st != MPMGPU_OK) return fail(st, batch_->last_error);
    bool any = false;
    for (auto& r : reqs_) {
      if (r.state != 1) continue;
      int64_t done = 0, left = 0;
      batch_->job_state(r.job, &done, &left);
      if (left == 0) any = true;
    }
    if (!any) return MPMGPU_OK;
    st = batch_->synchronize();
    if (st != MPMGPU_OK) return fail(st, batch_->last_error);
    const double now = clock();
    for (int id = 0; id < (int)reqs_.size(); id++) {
      Request& r = reqs_[(size_t)id];
      if (r.state != 1) continue;
      int64_t done = 0, left = 0;
      batch_->job_state(r.job, &done, &left);
      if (left != 0) continue;
      st = collect(r);
      if (st != MPMGPU_OK) return st;
      batch_->remove_job(r.job);
      r.state = 2;
      r.t_done = now;
      running_--;
      reserved_ -= r.footprint;
      points_done_ += r.points * r.steps;
      finished_.push_back(id);
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
  mpmgpu_status collect(Request& r) {
    int64_t npts = 0;
    for (int b = 0;; b++) {
      if (batch_->sizes(r.job, b, &npts, nullptr) != MPMGPU_OK) break;
      Result res;
      res.n = npts;
      res.x.resize((size_t)(3 * npts));
      res.u.resize((size_t)(3 * npts));
      res.x_t.resize((size_t)(3 * npts));
      res.T.resize((size_t)(9 * npts));
      res.v.resize((size_t)npts);
      res.active.resize((size_t)npts);
      mpmgpu_status st = MPMGPU_OK;
      if (npts > 0) {
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_X, res.x.data());
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_U, res.u.data());
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_X_T, res.x_t.data());
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_T, res.T.data());
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_V, res.v.data());
        if (st == MPMGPU_OK) st = batch_->download_points(r.job, b, MPMGPU_P_ACTIVE, res.active.data());
      }
      if (st != MPMGPU_OK) return fail(st, batch_->last_error);
      r.bodies.push_back(std::move(res));
    }
    return MPMGPU_OK;
  }

  std::unique_ptr<BatchBase> batch_;
  bool mixed_;
  bool keep_debug_;
  int64_t budget_;
  std::chrono::steady_clock::time_point t0_;
  std::vector<Request> reqs_;
  std::deque<int> finished_;
  int running_ = 0;
  int64_t reserved_ = 0;
  int64_t points_done_ = 0;
};

}  // namespace mpmb200
