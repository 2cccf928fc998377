// server.cu -- continuous batching of scenario solves on one device (the
// reference has no serving layer; this is the request loop behind the
// hydist_server_* entry points).
//
// A request is a scenario (its host inputs are copied at submit) with a
// horizon in steps. Each round:
//   1. queued requests are admitted in arrival order while their device
//      footprint (hydist_scenario_bytes) fits in the budget left by the
//      active ones; a request is created on the device when admitted;
//   2. every active request is advanced by up to steps_per_round steps.
//      Active requests of one mesh size and form that advance the same
//      number of steps are stepped as one ensemble (hydist_ensemble_*): each
//      kernel of a step is one launch over all of them while they are in the
//      same sediment phase (their sweeps batched together). The ensemble of
//      a group is kept while the group's membership stays the same (its step
//      graphs are reused) and released when it changes. A request alone in
//      its group steps through its own replayed step graph. Groups and lone
//      requests run on their own streams, so their kernels overlap;
//   3. the round waits for the device, and requests that reached their
//      horizon are retired: their state stays on the device (and counts
//      against the budget) until released, so results can be downloaded.
// Requests arriving between rounds join at the next round (continuous
// batching). A request stepped alone gives bit for bit what its scenario
// gives alone; one stepped in a batch gives it to rounding (the batched
// kernels are separately compiled variants of the same arithmetic).
#include <cuda_runtime.h>

#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace hyd {
void set_last_error(const char* m);
}

namespace {

int sfail(int code, const char* m) {
  hyd::set_last_error(m);
  return code;
}

// host copy of a scenario's inputs (submit copies, create reads later)
struct ScenarioCopy {
  HydistScenario sc{};
  std::vector<double> h, hsnham, visco, Fw, bc[4], CC[4], FS0, z0;
  std::vector<int32_t> btype;

  explicit ScenarioCopy(const HydistScenario& in) : sc(in) {
    const size_t n = (size_t)(in.M + 3) * (in.N + 3);
    auto cp = [](std::vector<double>& v, const double* p, size_t k) {
      if (p) v.assign(p, p + k);
    };
    cp(h, in.h, n);
    cp(hsnham, in.hsnham, n);
    cp(visco, in.visco, n);
    cp(Fw, in.Fw, n);
    const double* bcs[4] = {in.bc_up, in.bc_down, in.bc_left, in.bc_right};
    const double* ccs[4] = {in.CC_up, in.CC_down, in.CC_left, in.CC_right};
    for (int k = 0; k < 4; ++k) {
      cp(bc[k], bcs[k], (size_t)in.total_time);
      cp(CC[k], ccs[k], (size_t)in.total_time);
    }
    cp(FS0, in.FS0, n);
    cp(z0, in.z0, n);
    btype.assign(in.boundary_type, in.boundary_type + in.n_boundary_type);
    sc.h = h.data();
    sc.hsnham = hsnham.data();
    sc.visco = visco.data();
    sc.Fw = Fw.data();
    double const** bdst[4] = {&sc.bc_up, &sc.bc_down, &sc.bc_left, &sc.bc_right};
    double const** cdst[4] = {&sc.CC_up, &sc.CC_down, &sc.CC_left, &sc.CC_right};
    for (int k = 0; k < 4; ++k) {
      *bdst[k] = bc[k].empty() ? nullptr : bc[k].data();
      *cdst[k] = CC[k].empty() ? nullptr : CC[k].data();
    }
    sc.FS0 = FS0.empty() ? nullptr : FS0.data();
    sc.z0 = z0.empty() ? nullptr : z0.data();
    sc.boundary_type = btype.data();
  }
};

enum ReqState { RQ_QUEUED = 0, RQ_ACTIVE = 1, RQ_DONE = 2 };

struct Request {
  int64_t id = 0;
  ScenarioCopy input;
  HydistParams p{};
  HydistOptions o{};
  int32_t nsteps = 0, done_steps = 0;
  uint64_t bytes = 0;
  HydistHandle* h = nullptr;
  int state = RQ_QUEUED;
  Request(int64_t i, const HydistScenario& sc, const HydistParams& pp, const HydistOptions& oo,
          int32_t n, uint64_t b)
      : id(i), input(sc), p(pp), o(oo), nsteps(n), bytes(b) {}
};

}  // namespace

struct HydistServer {
  int device = 0;
  uint64_t budget = 0, held = 0;
  int32_t steps_per_round = 0;
  int64_t next_id = 1;
  std::deque<Request*> queue;        // arrival order
  std::map<int64_t, Request*> reqs;  // every request not yet released
  // the ensembles of the current groups, by their members' ids
  std::map<std::vector<int64_t>, HydistEnsemble*> groups;
};

namespace {

// requests that can share launches: mesh size, form and the options that
// shape the launches (the ensemble checks the rest), and the round's steps
struct GroupKey {
  int32_t M, N, precision, kenhhepd, kenhhepng, reset_horizontal, bed_feedback, steps;
  bool operator<(const GroupKey& o) const {
    return std::memcmp(this, &o, sizeof(GroupKey)) < 0;
  }
};

}  // namespace

extern "C" {

int64_t hydist_scenario_bytes(int32_t M, int32_t N) {
  if (M < 1 || N < 1) return 0;
  // the allocations of hydist_create (engine.cu), each rounded up to the
  // 2 MiB granule of large device allocations
  const uint64_t W = (uint64_t)M + 3, H = (uint64_t)N + 3, n = W * H;
  auto r = [](uint64_t b) { return (b + (2u << 20) - 1) / (2u << 20) * (2u << 20); };
  uint64_t t = 0;
  t += 29 * r(n * 8 + 64);  // 4 inputs, 6 derived, 17 state, 2 smoothing buffers
  t += r(n * 4 + 64);       // mask
  t += r(4 * n * 8 + 64);   // the concentration sweep's rows (StateT::pre)
  int nsm = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t U = 2 * (uint64_t)(M > N ? M : N);
  t += r((uint64_t)2 * nsm * 3 * U * 4 * 8 + 64);  // line-solver scratch
  t += 24 * r(4096);                              // series, tables, flags, clock, ...
  return (int64_t)t;
}

int hydist_server_create(int device, uint64_t budget_bytes, int32_t steps_per_round,
                         HydistServer** out) {
  if (!out || budget_bytes == 0 || steps_per_round < 1)
    return sfail(HYDIST_ERR_ARG, "null output, zero budget or steps_per_round < 1");
  auto* s = new HydistServer();
  if (device < 0) cudaGetDevice(&device);
  s->device = device;
  s->budget = budget_bytes;
  s->steps_per_round = steps_per_round;
  *out = s;
  return HYDIST_OK;
}

int hydist_server_destroy(HydistServer* s) {
  if (!s) return HYDIST_OK;
  for (auto& g : s->groups) hydist_ensemble_destroy(g.second);
  for (auto& kv : s->reqs) {
    if (kv.second->h) hydist_destroy(kv.second->h);
    delete kv.second;
  }
  delete s;
  return HYDIST_OK;
}

int hydist_server_submit(HydistServer* s, const HydistScenario* sc, const HydistParams* p,
                         const HydistOptions* o, int32_t nsteps, int64_t* id) {
  if (!s || !sc || !p || !o || !id) return sfail(HYDIST_ERR_ARG, "null argument");
  if (nsteps < 0) return sfail(HYDIST_ERR_ARG, "negative horizon");
  if (!sc->h || !sc->hsnham || !sc->visco || !sc->Fw || !sc->boundary_type || sc->M < 4 ||
      sc->N < 4 || sc->total_time < 2 || sc->n_boundary_type < 4 * HYDIST_SEGMENT_LIMIT)
    return sfail(HYDIST_ERR_ARG, "incomplete scenario");
  const uint64_t b = (uint64_t)hydist_scenario_bytes(sc->M, sc->N);
  if (b > s->budget) return sfail(HYDIST_ERR_BUDGET, "the scenario does not fit the server's budget");
  auto* r = new Request(s->next_id++, *sc, *p, *o, nsteps, b);
  s->reqs[r->id] = r;
  s->queue.push_back(r);
  *id = r->id;
  return HYDIST_OK;
}

int hydist_server_round(HydistServer* s, int64_t* done, int32_t cap, int32_t* ndone) {
  if (!s || !ndone || (cap > 0 && !done)) return sfail(HYDIST_ERR_ARG, "null argument");
  *ndone = 0;
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(HYDIST_ERR_CUDA, "cudaSetDevice failed");
  // 1. admission in arrival order while the footprint fits
  while (!s->queue.empty() && s->held + s->queue.front()->bytes <= s->budget) {
    Request* r = s->queue.front();
    s->queue.pop_front();
    const int rc = hydist_create(&r->input.sc, &r->p, &r->o, s->device, &r->h);
    if (rc != HYDIST_OK) {
      // leaves the request out; the caller sees the error and may release it
      r->state = RQ_DONE;
      r->nsteps = r->done_steps;
      return rc;
    }
    r->state = RQ_ACTIVE;
    s->held += r->bytes;
  }
  // 2. the active requests advance: grouped by mesh size, form and steps
  std::map<GroupKey, std::vector<Request*>> byKey;
  for (auto& kv : s->reqs) {
    Request* r = kv.second;
    if (r->state != RQ_ACTIVE) continue;
    const int k = std::min(s->steps_per_round, r->nsteps - r->done_steps);
    if (k <= 0) continue;
    GroupKey g;
    std::memset(&g, 0, sizeof(g));
    g.M = r->input.sc.M;
    g.N = r->input.sc.N;
    g.precision = r->o.precision;
    g.kenhhepd = r->o.kenhhepd;
    g.kenhhepng = r->o.kenhhepng;
    g.reset_horizontal = r->o.reset_horizontal;
    g.bed_feedback = r->o.bed_change && r->o.bed_feedback;
    g.steps = k;
    byKey[g].push_back(r);
  }
  std::map<std::vector<int64_t>, HydistEnsemble*> keep;
  for (auto& kv : byKey) {
    std::vector<Request*>& rs = kv.second;
    const int k = kv.first.steps;
    int rc = HYDIST_OK;
    if (rs.size() == 1) {
      rc = hydist_step_graph(rs[0]->h, k);
    } else {
      std::vector<int64_t> ids;
      std::vector<HydistHandle*> hs;
      for (Request* r : rs) {
        ids.push_back(r->id);
        hs.push_back(r->h);
      }
      HydistEnsemble* e = nullptr;
      auto it = s->groups.find(ids);
      if (it != s->groups.end()) {
        e = it->second;
        s->groups.erase(it);
      } else {
        rc = hydist_ensemble_create(hs.data(), (int32_t)hs.size(), &e);
      }
      if (rc == HYDIST_OK) {
        keep[ids] = e;
        rc = hydist_ensemble_step(e, k);
      }
    }
    if (rc != HYDIST_OK) {
      for (auto& g : keep) s->groups[g.first] = g.second;
      return rc;
    }
    for (Request* r : rs) r->done_steps += k;
  }
  // the ensembles of groups that no longer exist (their work is ordered
  // before any later work of their members)
  for (auto& g : s->groups) hydist_ensemble_destroy(g.second);
  s->groups.swap(keep);
  // 3. wait, then retire the requests that reached their horizon
  for (auto& kv : s->reqs) {
    Request* r = kv.second;
    if (r->state != RQ_ACTIVE) continue;
    const int rc = hydist_sync(r->h);
    if (rc != HYDIST_OK) return rc;
    if (r->done_steps >= r->nsteps) {
      r->state = RQ_DONE;
      if (*ndone < cap) done[*ndone] = r->id;
      ++*ndone;
    }
  }
  return HYDIST_OK;
}

int hydist_server_status(HydistServer* s, int64_t id, int32_t* state, int32_t* steps_done) {
  if (!s || !state) return sfail(HYDIST_ERR_ARG, "null argument");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(HYDIST_ERR_ARG, "unknown request");
  *state = it->second->state;
  if (steps_done) *steps_done = it->second->done_steps;
  return HYDIST_OK;
}

int hydist_server_counts(HydistServer* s, int32_t* queued, int32_t* active, uint64_t* held_bytes) {
  if (!s) return sfail(HYDIST_ERR_ARG, "null server");
  int q = 0, a = 0;
  for (auto& kv : s->reqs) {
    q += kv.second->state == RQ_QUEUED;
    a += kv.second->state == RQ_ACTIVE;
  }
  if (queued) *queued = q;
  if (active) *active = a;
  if (held_bytes) *held_bytes = s->held;
  return HYDIST_OK;
}

HydistHandle* hydist_server_handle(HydistServer* s, int64_t id) {
  if (!s) return nullptr;
  auto it = s->reqs.find(id);
  return (it == s->reqs.end() || it->second->state != RQ_DONE) ? nullptr : it->second->h;
}

int hydist_server_release(HydistServer* s, int64_t id) {
  if (!s) return sfail(HYDIST_ERR_ARG, "null server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(HYDIST_ERR_ARG, "unknown request");
  Request* r = it->second;
  if (r->state == RQ_ACTIVE) return sfail(HYDIST_ERR_STATE, "the request is still running");
  // an ensemble holding the request goes first
  for (auto g = s->groups.begin(); g != s->groups.end();) {
    bool has = false;
    for (int64_t x : g->first) has |= x == id;
    if (has) {
      hydist_ensemble_destroy(g->second);
      g = s->groups.erase(g);
    } else {
      ++g;
    }
  }
  if (r->state == RQ_QUEUED) {
    for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
      if (*q == r) {
        s->queue.erase(q);
        break;
      }
  }
  if (r->h) {
    hydist_destroy(r->h);
    s->held -= r->bytes;
  }
  s->reqs.erase(it);
  delete r;
  return HYDIST_OK;
}

}  // extern "C"
