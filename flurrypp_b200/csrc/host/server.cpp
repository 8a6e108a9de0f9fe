// Solve server: a request loop over the case C ABI (include/fr_b200.h).
//
// Requests (a deck, optionally a mesh, an initial condition, a residual-drop
// target) arrive at any time; a scheduler thread admits them while the
// device-memory budget and the slot count allow, keeps every admitted case's
// state on the device, advances all cases in flight together (each on its
// own stream, each step a CUDA-graph replay, so their kernels overlap on the
// GPU), checks convergence from the reference's residual norm
// (writeResidual, src/output.cpp:1011-1090), retires converged cases and
// admits waiting ones in their place.  No reference counterpart: the
// reference solves one case per process.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/fr_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  long long id = 0;
  std::string deck;
  bool hasMesh = false;
  fr_mesh mesh{};
  std::vector<double> xv;
  std::vector<int> c2v, bfv, bfb;
  int icKind = 0;
  std::vector<double> icPrm;
  double tol = 1e-8;
  int maxSteps = 100000;
  Clock::time_point arrival;
  // in flight
  fr_case *c = nullptr;
  size_t bytes = 0;
  int steps = 0;
  int pending = 0;  // steps issued and not yet seen complete
  int nFields = 0;
  std::vector<double> res0;
  // FR_PREC_MIXED_REFINE: in the precision form until the residual stops
  // falling, then in FP64
  bool refine = false, fp32 = false;
  int form = FR_PREC_FP64;
  double best = 0.0;
  int sinceBest = 0, stepsFp32 = 0;
  // result
  int status = 0;  // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
  int code = FR_OK;
  std::string error;
  double latency = 0.0, finalRatio = 0.0;
  std::vector<double> state;
};

}  // namespace

struct fr_server {
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  size_t budget = 0, inflightBytes = 0;
  int maxInflight = 8, checkEvery = 10, device = 0;
  int precision = FR_PREC_FP64;  // form of the cases admitted from now on
  long long nextId = 1;
  std::deque<long long> queue;
  std::map<long long, std::unique_ptr<Request>> reqs;
  std::vector<long long> inflight;
  std::string err;

  // device bytes of a case, from its sizes (setup allocations; P-multigrid
  // levels add their share)
  static size_t case_bytes(fr_case *c) {
    fr_info inf;
    if (fr_get_info(c, &inf) != FR_OK) return 0;
    size_t nU = (size_t)inf.nSpts * inf.nEles * inf.nFields, nUf = (size_t)inf.nFpts * inf.nEles * inf.nFields;
    size_t words = nU * (3 + inf.nRKSteps + 3) + nUf * 2 + (size_t)inf.nDims * inf.nDims * inf.nSpts * inf.nEles +
                   (size_t)inf.nFpts * inf.nEles * (inf.nDims + 2) + (size_t)inf.nFacePts * (inf.nDims + 4);
    return words * sizeof(double) * 2;  // coarse P levels and tables: at most as much again
  }

  static fr_case *create(Request &r, int device, int prec, int &st) {
    fr_setup_opts o;
    fr_setup_opts_default(&o);
    o.device = device;
    o.precision = prec;
    fr_case *c = nullptr;
    st = r.hasMesh ? fr_create_with_mesh(r.deck.c_str(), &r.mesh, &o, &c)
                   : fr_create_from_deck(r.deck.c_str(), &o, &c);
    return c;
  }

  // The precision form's residual stops falling at its FP32 floor (about
  // 1e-7 of the flux terms, scaled by the operators): a request of the
  // refining form goes on from its state in FP64.  The case is set up again
  // in FP64 (same deck and mesh) and given the state; its coarse P-multigrid
  // levels start as at any setup.  The request keeps its steps and its
  // residual normalisation.
  static constexpr int kStallChecks = 20;     // checks without a new best
  static constexpr double kStallGain = 0.8;   // a new best is 20% below the last
  bool to_fp64(Request &r) {
    fr_info inf;
    if (fr_get_info(r.c, &inf) != FR_OK) return false;
    std::vector<double> U((size_t)inf.nSpts * inf.nEles * inf.nFields);
    if (fr_get_state(r.c, U.data(), U.size()) != FR_OK) return false;
    int st = FR_OK;
    fr_case *c = create(r, device, FR_PREC_FP64, st);
    if (st != FR_OK || fr_set_state(c, U.data(), U.size()) != FR_OK) {
      fr_destroy(c);
      return false;
    }
    fr_destroy(r.c);
    r.c = c;
    const size_t b = case_bytes(c);
    {
      std::lock_guard<std::mutex> lk(mu);
      inflightBytes += b;
      inflightBytes -= r.bytes;
    }
    r.bytes = b;
    r.fp32 = false;
    r.form = FR_PREC_FP64;
    r.stepsFp32 = r.steps;
    return true;
  }

  bool admit_one() {
    // caller holds mu; setup runs without it
    long long id = queue.front();
    Request &r = *reqs[id];
    r.refine = precision == FR_PREC_MIXED_REFINE;
    r.form = r.refine ? FR_PREC_MIXED : precision;
    r.fp32 = r.form == FR_PREC_MIXED;
    int st = FR_OK;
    fr_case *c = create(r, device, r.form, st);
    if (st == FR_OK) st = fr_init_solution(c, r.icKind, r.icPrm.empty() ? nullptr : r.icPrm.data(), (int)r.icPrm.size());
    if (st != FR_OK) {
      r.status = 3;
      r.code = st;
      r.error = c ? fr_last_error(c) : "create failed";
      fr_destroy(c);
      queue.pop_front();
      return true;
    }
    size_t b = case_bytes(c);
    if (!inflight.empty() && inflightBytes + b > budget) {
      fr_destroy(c);  // no room yet: wait for a retirement
      return false;
    }
    if (inflight.empty() && b > budget) {
      r.status = 3;
      r.code = FR_ERR_BUDGET;
      r.error = "case exceeds the device-memory budget";
      fr_destroy(c);
      queue.pop_front();
      return true;
    }
    r.c = c;
    r.bytes = b;
    r.status = 1;
    fr_info inf;
    fr_get_info(c, &inf);
    r.nFields = inf.nFields;
    inflightBytes += b;
    inflight.push_back(id);
    queue.pop_front();
    return true;
  }

  void retire(Request &r, int status, int code, const std::string &e) {
    r.latency = std::chrono::duration<double>(Clock::now() - r.arrival).count();
    if (status == 2) {
      fr_info inf;
      fr_get_info(r.c, &inf);
      r.state.resize((size_t)inf.nSpts * inf.nEles * inf.nFields);
      fr_get_state(r.c, r.state.data(), r.state.size());
    }
    r.status = status;
    r.code = code;
    r.error = e;
    fr_destroy(r.c);
    r.c = nullptr;
    inflightBytes -= r.bytes;
  }

  void loop() {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
      // admission while memory and slots allow
      while (!queue.empty() && (int)inflight.size() < maxInflight)
        if (!admit_one()) break;
      if (inflight.empty()) {
        cv.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
      std::vector<long long> ids = inflight;
      lk.unlock();
      // every case advances on its own stream at its own pace: a case whose
      // last chunk of steps has completed is checked and given its next
      // chunk at once, so small cases do not wait for large ones and the
      // kernels of all cases overlap on the device
      bool progressed = false;
      for (long long id : ids) {
        Request &r = *reqs[id];
        if (r.pending == 0) {
          int n = std::min(checkEvery, r.maxSteps - r.steps);
          if (n > 0 && fr_run(r.c, n) == FR_OK) r.pending = n;
          progressed = true;
        }
      }
      std::vector<std::pair<long long, int>> done;  // id, status
      for (long long id : ids) {
        Request &r = *reqs[id];
        if (r.pending == 0 || fr_stream_idle(r.c) != 1) continue;
        progressed = true;
        r.steps += r.pending;
        r.pending = 0;
        std::vector<double> res(r.nFields);
        int st = fr_residual_norm(r.c, 2, res.data(), r.nFields);
        if (st != FR_OK) {
          done.push_back({id, 3});
          continue;
        }
        if (r.res0.empty()) r.res0 = res;
        double ratio = 0.0;
        for (int k = 0; k < r.nFields; k++)
          ratio = std::max(ratio, r.res0[k] > 0 ? res[k] / r.res0[k] : 0.0);
        r.finalRatio = ratio;
        if (ratio <= r.tol) {
          done.push_back({id, 2});
        } else if (r.steps >= r.maxSteps) {
          done.push_back({id, 2});
        } else if (r.refine && r.fp32) {
          if (r.best == 0.0 || ratio < kStallGain * r.best) {
            r.best = ratio;
            r.sinceBest = 0;
          } else if (++r.sinceBest >= kStallChecks && !to_fp64(r)) {
            done.push_back({id, 3});
          }
        }
      }
      if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
      lk.lock();
      for (auto &d : done) {
        Request &r = *reqs[d.first];
        if (r.status != 1) continue;
        retire(r, d.second, d.second == 2 ? FR_OK : FR_ERR_NONFINITE, d.second == 2 ? "" : fr_last_error(r.c));
        inflight.erase(std::find(inflight.begin(), inflight.end(), d.first));
      }
      // cancelled requests in flight
      for (size_t i = 0; i < inflight.size();) {
        Request &r = *reqs[inflight[i]];
        if (r.status == 4) {
          fr_synchronize(r.c);
          fr_destroy(r.c);
          r.c = nullptr;
          inflightBytes -= r.bytes;
          inflight.erase(inflight.begin() + i);
        } else {
          i++;
        }
      }
      cv.notify_all();
    }
  }
};

extern "C" {

int fr_server_create(size_t budget_bytes, int max_inflight, int check_every, int device, fr_server **out) {
  if (!out || budget_bytes == 0 || max_inflight <= 0 || check_every <= 0) return FR_ERR_ARG;
  fr_server *s = new fr_server();
  s->budget = budget_bytes;
  s->maxInflight = max_inflight;
  s->checkEvery = check_every;
  s->device = device;
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return FR_OK;
}

int fr_server_set_precision(fr_server *s, int precision) {
  if (!s || (precision != FR_PREC_FP64 && precision != FR_PREC_MIXED && precision != FR_PREC_MIXED_REFINE))
    return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->precision = precision;
  return FR_OK;
}

int fr_server_submit(fr_server *s, const char *deck, const fr_mesh *mesh, int ic_kind, const double *ic_prm,
                     int n_prm, double tol, int max_steps, long long *id) {
  if (!s || !deck || !id || tol <= 0 || max_steps <= 0) return FR_ERR_ARG;
  std::unique_ptr<Request> r(new Request());
  r->deck = deck;
  if (mesh) {
    r->hasMesh = true;
    r->mesh = *mesh;
    r->xv.assign(mesh->xv, mesh->xv + (size_t)mesh->nVerts * mesh->nDims);
    r->c2v.assign(mesh->c2v, mesh->c2v + (size_t)mesh->nEles * mesh->nNodes);
    r->bfv.assign(mesh->bndFaceVerts, mesh->bndFaceVerts + (size_t)mesh->nBndFaces * 4);
    r->bfb.assign(mesh->bndFaceBc, mesh->bndFaceBc + mesh->nBndFaces);
    r->mesh.xv = r->xv.data();
    r->mesh.c2v = r->c2v.data();
    r->mesh.bndFaceVerts = r->bfv.data();
    r->mesh.bndFaceBc = r->bfb.data();
  }
  r->icKind = ic_kind;
  if (ic_prm && n_prm > 0) r->icPrm.assign(ic_prm, ic_prm + n_prm);
  r->tol = tol;
  r->maxSteps = max_steps;
  r->arrival = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->nextId++;
  *id = r->id;
  s->queue.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  s->cv.notify_all();
  return FR_OK;
}

int fr_server_poll(fr_server *s, long long id, int *status, double *latency_s, int *steps, double *res_ratio) {
  if (!s) return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return FR_ERR_ARG;
  Request &r = *it->second;
  if (status) *status = r.status;
  if (latency_s) *latency_s = r.latency;
  if (steps) *steps = r.steps;
  if (res_ratio) *res_ratio = r.finalRatio;
  return r.status == 3 ? r.code : FR_OK;
}

int fr_server_poll_form(fr_server *s, long long id, int *precision, int *steps_fp32) {
  if (!s) return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return FR_ERR_ARG;
  Request &r = *it->second;
  if (precision) *precision = r.form;
  if (steps_fp32) *steps_fp32 = r.fp32 ? r.steps : r.stepsFp32;
  return FR_OK;
}

int fr_server_wait(fr_server *s, long long id, double timeout_s) {
  if (!s) return FR_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return FR_ERR_ARG;
  Request &r = *it->second;
  bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r.status >= 2; });
  if (!ok) return FR_ERR_TIMEOUT;
  return r.status == 3 ? r.code : FR_OK;
}

int fr_server_result(fr_server *s, long long id, double *U, size_t count) {
  if (!s || !U) return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->status != 2) return FR_ERR_STATE;
  if (count != it->second->state.size()) return FR_ERR_ARG;
  std::memcpy(U, it->second->state.data(), count * sizeof(double));
  return FR_OK;
}

int fr_server_cancel(fr_server *s, long long id) {
  if (!s) return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return FR_ERR_ARG;
  Request &r = *it->second;
  if (r.status == 0) {
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), id));
    r.status = 4;
  } else if (r.status == 1) {
    r.status = 4;  // released by the scheduler at its next pass
  }
  return FR_OK;
}

int fr_server_stats(fr_server *s, int *queued, int *inflight, size_t *inflight_bytes) {
  if (!s) return FR_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (queued) *queued = (int)s->queue.size();
  if (inflight) *inflight = (int)s->inflight.size();
  if (inflight_bytes) *inflight_bytes = s->inflightBytes;
  return FR_OK;
}

void fr_server_destroy(fr_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (long long id : s->inflight) fr_destroy(s->reqs[id]->c);
  delete s;
}

}  // extern "C"
