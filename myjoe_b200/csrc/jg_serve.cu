// jg_serve.cu -- the serving engine: a request loop that keeps many cases
// resident on one GPU (host code only; the device work is the cases' own
// captured steps).
//
// Each admitted case gets its own handle (device layout, non-blocking stream,
// captured step) created with stream-ordered allocation, so that admitting or
// retiring a case never waits on the other cases' work.  jg_serve_poll walks
// the resident cases: a case whose last batch of steps has finished (its event
// is complete) has its residuals checked from pinned host memory and is then
// retired, restarted or given its next batch of steps; queued cases are then
// admitted in arrival order while the memory budget and the resident limit
// allow.  Cases never share device data, so a case's result does not depend
// on what else is resident.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "jg_internal.h"

namespace {

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return jg::serve_set_err(code, buf);
}

#define SCK(x)                                                                                          \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) return fail(JG_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define SRC(x)                        \
  do {                                \
    int rc_ = (x);                    \
    if (rc_ != JG_OK) return rc_;     \
  } while (0)

// a deep copy of a jg_mesh (the caller's arrays may go away after submit)
struct MeshCopy {
  std::vector<int> cvofa, faocv_i, faocv_v, nbocv_i, nbocv_v;
  std::vector<double> x_cv, x_fa, fa_normal, vol, lsq, blsq;
  std::vector<jg_zone> zones;
  jg_mesh m;

  void copy(const jg_mesh& src) {
    const size_t N = src.ncv, F = src.nfa, FB = src.nfa_b, S = src.nbocv_s;
    cvofa.assign(src.cvofa, src.cvofa + 2 * F);
    faocv_i.assign(src.faocv_i, src.faocv_i + N + 1);
    faocv_v.assign(src.faocv_v, src.faocv_v + src.faocv_i[N]);
    nbocv_i.assign(src.nbocv_i, src.nbocv_i + N + 1);
    nbocv_v.assign(src.nbocv_v, src.nbocv_v + S);
    x_cv.assign(src.x_cv, src.x_cv + 3 * N);
    x_fa.assign(src.x_fa, src.x_fa + 3 * F);
    fa_normal.assign(src.fa_normal, src.fa_normal + 3 * F);
    vol.assign(src.cv_volume, src.cv_volume + N);
    lsq.assign(src.nbocv_lsg_coeff, src.nbocv_lsg_coeff + 3 * S);
    blsq.assign(src.boundary_fa_lsg_coeff, src.boundary_fa_lsg_coeff + 3 * FB);
    zones.assign(src.zones, src.zones + src.nzones);
    m = src;
    m.cvofa = cvofa.data();
    m.faocv_i = faocv_i.data();
    m.faocv_v = faocv_v.data();
    m.nbocv_i = nbocv_i.data();
    m.nbocv_v = nbocv_v.data();
    m.x_cv = x_cv.data();
    m.x_fa = x_fa.data();
    m.fa_normal = fa_normal.data();
    m.cv_volume = vol.data();
    m.nbocv_lsg_coeff = lsq.data();
    m.boundary_fa_lsg_coeff = blsq.data();
    m.zones = zones.data();
  }
};

struct Request {
  long long id = 0;
  MeshCopy mesh;
  jg_params params{};
  std::vector<double> rho, rhou, rhoE;  // initial state (kept for restarts)
  double t_arrival = 0.0, t_admit = -1.0;
  double footprint = 0.0;
  int restarts = 0;
  int steps_total = 0;
  // while resident
  jg_case* h = nullptr;
  int slot = -1;
  bool inflight = false;
  int steps = 0;      // steps of the current attempt that have finished
  int launched = 0;   // steps of the batch in flight
  double r0 = 0.0;    // first-step energy residual of the current attempt
  int conv_step = -1;
  double drop = NAN;
  double best = INFINITY;         // smallest drop of the current attempt
  double window_best = INFINITY;  // ... at the last stall check
  int next_check = 0;             // step of the next stall check
  int flags = 0;
  size_t bytes = 0;
};

struct SlotBuf {
  double* ring = nullptr;  // pinned [ring][5] residual history
  int* err = nullptr;      // pinned error flags (handle, case)
  cudaEvent_t ev = nullptr;
  bool used = false;
};

struct Finished {
  jg_serve_result res{};
  std::vector<double> rho, rhou, rhoE;
};

enum Outcome { RUNNING, CONVERGED, MAX_STEPS, FAILED, STALLED };

}  // namespace

struct jg_server {
  jg_serve_config cfg{};
  std::chrono::steady_clock::time_point t0;
  std::deque<std::unique_ptr<Request>> queue;
  std::vector<std::unique_ptr<Request>> resident;
  std::vector<SlotBuf> slots;
  std::map<long long, Finished> done;
  std::deque<long long> unreported;
  long long next_id = 1;
  double bytes_resident = 0.0;
  double budget = 0.0;
  int ring = 64;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

static int release_case(jg_server* s, Request* r) {
  if (r->h) {
    s->bytes_resident -= (double)r->bytes;
    jg_destroy(r->h);
    r->h = nullptr;
  }
  if (r->slot >= 0) {
    s->slots[r->slot].used = false;
    r->slot = -1;
  }
  r->inflight = false;
  return JG_OK;
}

// (re)create the case's handle, upload its initial state and launch its first steps
static int start_case(jg_server* s, Request* r) {
  int slot = -1;
  for (size_t k = 0; k < s->slots.size(); k++)
    if (!s->slots[k].used) {
      slot = (int)k;
      break;
    }
  if (slot < 0) return fail(JG_ERR_STATE, "no free slot");
  SRC(jg::serve_case_create(&r->mesh.m, &r->params, &r->h));
  r->bytes = jg::serve_case_bytes(r->h);
  s->bytes_resident += (double)r->bytes;
  s->slots[slot].used = true;
  r->slot = slot;
  r->steps = 0;
  r->r0 = 0.0;
  r->conv_step = -1;
  r->drop = NAN;
  r->best = r->window_best = INFINITY;
  r->next_check = s->cfg.stall_steps;
  r->flags = 0;
  SRC(jg::serve_case_start(r->h, r->rho.data(), r->rhou.data(), r->rhoE.data()));
  return JG_OK;
}

static int launch_batch(jg_server* s, Request* r) {
  int n = std::min(s->cfg.steps_per_poll, s->cfg.max_steps - r->steps);
  n = std::max(n, 1);
  SlotBuf& b = s->slots[r->slot];
  SRC(jg::serve_case_launch(r->h, n, b.ring, b.err, b.ev));
  r->launched = n;
  r->inflight = true;
  return JG_OK;
}

// residuals of the batch that just finished
static Outcome check_batch(jg_server* s, Request* r) {
  const SlotBuf& b = s->slots[r->slot];
  int flags = b.err[0] | b.err[1];
  const int ring = jg::serve_case_ring(r->h);
  for (int k = 0; k < r->launched; k++) {
    const int step = r->steps + k + 1;
    const double e = b.ring[5 * ((step - 1) % ring) + 4];
    if (!std::isfinite(e)) flags |= 4;
    if (step == 1) r->r0 = e;
    const double drop = r->r0 > 0.0 ? e / r->r0 : 0.0;
    r->drop = drop;
    r->best = std::min(r->best, drop);
    if (r->conv_step < 0 && drop <= s->cfg.resid_drop) r->conv_step = step;
  }
  r->steps += r->launched;
  r->steps_total += r->launched;
  r->inflight = false;
  r->flags = flags;
  if (flags) return FAILED;
  if (r->conv_step > 0) return CONVERGED;
  if (r->steps >= s->cfg.max_steps) return MAX_STEPS;
  if (s->cfg.stall_steps > 0 && r->steps >= r->next_check) {
    if (!(r->best <= 0.5 * r->window_best)) return STALLED;
    r->window_best = r->best;
    r->next_check += s->cfg.stall_steps;
  }
  return RUNNING;
}

static int finish(jg_server* s, Request* r, int status) {
  Finished f;
  const int N = r->mesh.m.ncv;
  f.rho.resize(N);
  f.rhou.resize(3 * (size_t)N);
  f.rhoE.resize(N);
  if (r->h) {
    SRC(jg_get_state(r->h, f.rho.data(), f.rhou.data(), f.rhoE.data()));
  } else {  // never started: its initial state
    f.rho = r->rho;
    f.rhou = r->rhou;
    f.rhoE = r->rhoE;
  }
  jg_serve_result& o = f.res;
  o.id = r->id;
  o.status = status;
  o.steps = r->steps;
  o.steps_total = r->steps_total;
  o.restarts = r->restarts;
  o.ncv = N;
  o.conv_step = r->conv_step;
  o.drop = r->drop;
  o.t_arrival = r->t_arrival;
  o.t_admit = r->t_admit;
  o.bytes = (double)r->bytes;
  release_case(s, r);
  o.t_done = s->now();
  s->done.emplace(r->id, std::move(f));
  s->unreported.push_back(r->id);
  return JG_OK;
}

extern "C" {

int jg_serve_create(const jg_serve_config* cfg, jg_server_t** out) {
  if (!cfg || !out) return fail(JG_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->max_resident < 1 || cfg->steps_per_poll < 1 || cfg->steps_per_poll > 64 || cfg->max_steps < 1 ||
      !(cfg->resid_drop > 0.0) || cfg->max_restarts < 0 ||
      !(cfg->restart_cfl_factor > 0.0 && cfg->restart_cfl_factor <= 1.0) || cfg->stall_steps < 0 ||
      (cfg->admission != JG_ADMIT_FIFO && cfg->admission != JG_ADMIT_SMALLEST))
    return fail(JG_ERR_ARG, "bad serve config (max_resident >= 1, steps_per_poll 1..64, resid_drop > 0, "
                            "0 < restart_cfl_factor <= 1)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(JG_ERR_NODEVICE, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(JG_ERR_ARG, "device %d of %d", cfg->device, ndev);
  SCK(cudaSetDevice(cfg->device));
  // keep freed case memory in the stream-ordered pool for the next admission
  cudaMemPool_t pool;
  SCK(cudaDeviceGetDefaultMemPool(&pool, cfg->device));
  uint64_t keep = UINT64_MAX;
  SCK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  std::unique_ptr<jg_server> s(new jg_server());
  s->cfg = *cfg;
  size_t free_b = 0, total_b = 0;
  SCK(cudaMemGetInfo(&free_b, &total_b));
  s->budget = cfg->hbm_budget > 0.0 ? cfg->hbm_budget : 0.9 * (double)free_b;
  s->slots.resize(cfg->max_resident);
  for (SlotBuf& b : s->slots) {
    SCK(cudaHostAlloc((void**)&b.ring, 5 * (size_t)s->ring * sizeof(double), cudaHostAllocDefault));
    SCK(cudaHostAlloc((void**)&b.err, 2 * sizeof(int), cudaHostAllocDefault));
    SCK(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
  }
  s->t0 = std::chrono::steady_clock::now();
  *out = s.release();
  return JG_OK;
}

int jg_serve_now(jg_server_t* s, double* t) {
  if (!s || !t) return fail(JG_ERR_ARG, "null argument");
  *t = s->now();
  return JG_OK;
}

int jg_serve_submit(jg_server_t* s, const jg_mesh* mesh, const jg_params* params, const double* rho,
                    const double* rhou, const double* rhoE, double t_arrival, long long* id) {
  if (!s || !mesh || !params || !rho || !rhou || !rhoE) return fail(JG_ERR_ARG, "null argument");
  if (params->lin_solver == JG_LS_BCGSTAB || params->lin_solver == JG_LS_BCGSTAB_LINELET ||
      params->lin_solver == JG_LS_LINE)
    return fail(JG_ERR_ARG, "served cases relax with JACOBI, SGS or LUSGS (captured steps)");
  double fp = 0.0;
  SRC(jg_case_footprint(mesh, params, &fp));
  std::unique_ptr<Request> r(new Request());
  r->id = s->next_id++;
  r->mesh.copy(*mesh);
  r->params = *params;
  const size_t N = mesh->ncv;
  r->rho.assign(rho, rho + N);
  r->rhou.assign(rhou, rhou + 3 * N);
  r->rhoE.assign(rhoE, rhoE + N);
  r->t_arrival = t_arrival >= 0.0 ? t_arrival : s->now();
  r->footprint = fp;
  if (id) *id = r->id;
  s->queue.push_back(std::move(r));
  return JG_OK;
}

int jg_serve_poll(jg_server_t* s, double max_wait_s, jg_serve_result* out, int cap, int* n) {
  if (!s || !n || (cap > 0 && !out)) return fail(JG_ERR_ARG, "null argument");
  *n = 0;
  SCK(cudaSetDevice(s->cfg.device));
  const double t_end = s->now() + std::max(0.0, max_wait_s);
  for (;;) {
    bool progressed = false;
    // resident cases whose steps have finished
    for (size_t i = 0; i < s->resident.size();) {
      Request* r = s->resident[i].get();
      if (r->inflight) {
        cudaError_t e = cudaEventQuery(s->slots[r->slot].ev);
        if (e == cudaErrorNotReady) {
          i++;
          continue;
        }
        SCK(e);
        progressed = true;
        Outcome oc = check_batch(s, r);
        if (oc == FAILED && r->restarts < s->cfg.max_restarts) {
          // restart from the initial state with a smaller CFL
          release_case(s, r);
          r->restarts++;
          r->params.cfl_max *= s->cfg.restart_cfl_factor;
          r->params.cfl = std::min(r->params.cfl, r->params.cfl_max);
          SRC(start_case(s, r));
          SRC(launch_batch(s, r));
          i++;
          continue;
        }
        if (oc != RUNNING) {
          const int status = oc == CONVERGED ? JG_SERVE_CONVERGED
                             : oc == MAX_STEPS ? JG_SERVE_MAX_STEPS
                             : oc == STALLED ? JG_SERVE_STALLED
                                             : JG_SERVE_FAILED;
          SRC(finish(s, r, status));
          s->resident.erase(s->resident.begin() + i);
          continue;
        }
      }
      if (!r->inflight) SRC(launch_batch(s, r));
      i++;
    }
    // admissions, in arrival order, into the memory and slots that are free
    while (!s->queue.empty() && (int)s->resident.size() < s->cfg.max_resident) {
      size_t pick = 0;
      if (s->cfg.admission == JG_ADMIT_SMALLEST)
        for (size_t k = 1; k < s->queue.size(); k++)
          if (s->queue[k]->footprint < s->queue[pick]->footprint) pick = k;
      Request* r = s->queue[pick].get();
      if (!s->resident.empty() && s->bytes_resident + r->footprint > s->budget) break;
      std::unique_ptr<Request> own = std::move(s->queue[pick]);
      s->queue.erase(s->queue.begin() + pick);
      // a case that cannot fit even an empty device (its footprint above the budget, or its
      // allocation failing with nothing else resident) is retired as failed, so that poll
      // reports it, and the server goes on with the others
      int rc = r->footprint > s->budget ? JG_ERR_NOMEM : start_case(s, r);
      if (rc == JG_ERR_NOMEM && !s->resident.empty()) {
        // the pool is fuller than the estimate says: wait for a retirement
        release_case(s, r);
        s->queue.insert(s->queue.begin() + pick, std::move(own));
        break;
      }
      if (rc == JG_ERR_NOMEM || rc == JG_ERR_ARG) {
        release_case(s, r);
        SRC(finish(s, r, JG_SERVE_FAILED));
        progressed = true;
        continue;
      }
      if (rc != JG_OK) {
        // a CUDA error: the request goes back to the queue (not lost) and the error to the caller
        release_case(s, r);
        s->queue.insert(s->queue.begin() + pick, std::move(own));
        return rc;
      }
      r->t_admit = r->t_admit < 0.0 ? s->now() : r->t_admit;
      SRC(launch_batch(s, r));
      s->resident.push_back(std::move(own));
      progressed = true;
    }
    while (!s->unreported.empty() && *n < cap) {
      out[(*n)++] = s->done[s->unreported.front()].res;
      s->unreported.pop_front();
    }
    if (*n > 0 || (s->resident.empty() && s->queue.empty()) || s->now() >= t_end) return JG_OK;
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

int jg_serve_fetch(jg_server_t* s, long long id, double* rho, double* rhou, double* rhoE) {
  if (!s) return fail(JG_ERR_ARG, "null argument");
  auto it = s->done.find(id);
  if (it == s->done.end()) return fail(JG_ERR_ARG, "case %lld is not retired (or was fetched)", id);
  const Finished& f = it->second;
  if (rho) std::copy(f.rho.begin(), f.rho.end(), rho);
  if (rhou) std::copy(f.rhou.begin(), f.rhou.end(), rhou);
  if (rhoE) std::copy(f.rhoE.begin(), f.rhoE.end(), rhoE);
  s->done.erase(it);
  return JG_OK;
}

int jg_serve_stats(jg_server_t* s, int* resident, int* queued, int* finished_unfetched, double* bytes_resident) {
  if (!s) return fail(JG_ERR_ARG, "null argument");
  if (resident) *resident = (int)s->resident.size();
  if (queued) *queued = (int)s->queue.size();
  if (finished_unfetched) *finished_unfetched = (int)s->done.size();
  if (bytes_resident) *bytes_resident = s->bytes_resident;
  return JG_OK;
}

int jg_serve_destroy(jg_server_t* s) {
  if (!s) return JG_OK;
  cudaSetDevice(s->cfg.device);
  for (auto& r : s->resident) {
    if (r->inflight) cudaEventSynchronize(s->slots[r->slot].ev);
    release_case(s, r.get());
  }
  cudaDeviceSynchronize();
  for (SlotBuf& b : s->slots) {
    if (b.ring) cudaFreeHost(b.ring);
    if (b.err) cudaFreeHost(b.err);
    if (b.ev) cudaEventDestroy(b.ev);
  }
  delete s;
  return JG_OK;
}

}  // extern "C"
