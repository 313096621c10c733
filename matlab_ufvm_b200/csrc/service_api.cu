// service_api.cu -- extern "C" entry points of the batched steady-case service.
//
// Admission policy: first come, first served, while the estimated HBM footprint of the resident
// cases stays within the memory budget (and the sum of resident cells within max_resident_cells);
// a case that alone exceeds the budget is admitted when the service is empty. Each
// ufvm_service_step advances every resident case by one SIMPLE iteration (fast.cu), then retires
// finished cases and admits queued ones, so requests that arrive while others run join the batch
// as soon as memory frees up (continuous batching).
//
// A finished case keeps its slot in the batch, frozen, until the slots are next rebuilt: its
// result (U, p, mdot at the finishing iteration) is copied to a snapshot on the device, and the
// case may run more iterations that nobody reads. Rebuilding the slot tables re-captures the
// tick's CUDA graph, so departures are gathered: the frozen slots are dropped when queued cases
// are admitted, when the device time spent on them since they froze (their share of each tick, by
// cells) reaches the host time the last drop and rebuild took, when one has waited
// kMaxFrozenSteps steps, or when no active case is left. A departed case's device memory is
// freed later, when admission finds too little free memory or the service ends. The service's
// arrays are stream-ordered allocations (common.cuh), so a free no longer waits for the device,
// but a departed case's hundreds of frees still stay out of the steps that run the batch.
#include <deque>
#include <map>
#include <memory>

#include <atomic>
#include <chrono>
#include <thread>

#include "fast.cuh"
#include "linsolve.cuh"

namespace ufvm {

constexpr int kMaxFrozenSteps = 256;  // a finished case leaves the batch at the latest after this

struct Pending {
  long long ticket;
  int max_iter;
  double nu;
  std::vector<double> points, bvu, bvp;
  std::vector<int32_t> fs, fn, own, nei, ptype, pstart, pn, bcu, bcp;
  double t_submit;  // service clock (ms) at submission
  long long cells = 0, est_raw = 0;
};

// Result of a finished case, copied on the device when it finished.
struct Snapshot {
  double *U = nullptr, *p = nullptr, *mdot = nullptr;
  size_t nU = 0, np = 0, nm = 0;
  long long bytes() const { return (long long)((nU + np + nm) * sizeof(double)); }
};

struct Record {
  int state = 0;  // 0 queued, 1 resident, 2 converged, 3 stopped
  int status = UFVM_OK;
  int iterations = 0, max_iter = 0;
  double res[16] = {0};
  double t_submit = 0, t_admit = 0, t_done = 0;
  Case* c = nullptr;  // the case while it holds a slot; after that only if it has no snapshot
  Snapshot snap;
  long long cells = 0, est_raw = 0;
  bool released = false;  // released while its slot was still frozen in the batch
  std::string err;        // why admission or a step failed
};

struct ServiceImpl {
  Service svc;
  long long max_cells = 0, resident_cells = 0, next_ticket = 1, finished = 0;
  // HBM budget of the resident cases (their measured allocations, or the estimate of a case whose
  // hierarchy is not built yet) and of the snapshots of finished, unreleased results
  long long max_bytes = 0, snap_bytes = 0;
  double est_scale = 1.0;  // largest measured footprint / estimate seen so far (>= 1)
  long long n_deferred_mem = 0, n_oom_requeue = 0, n_drops = 0;
  std::deque<Pending> queue;
  std::map<long long, Record> rec;
  std::vector<char> frozen;     // per slot of svc.cases: finished, result in its snapshot
  std::vector<int> frozen_age;  // steps since the slot froze
  bool force_drop = false;
  // departures are gathered while the work spent on frozen slots (their share of each tick's
  // device time) stays below what dropping them costs on the host (the last rebuild of the slot
  // tables with its graph capture, plus freeing the departed cases)
  double waste_ms = 0.0, last_drop_ms = 0.0, host_drop_ms = 0.0;
  double host_admit_ms = 0.0;  // host time in admissions
  // Cases that left the batch are not freed at once: freeing a case's device arrays (hundreds
  // of them) costs more host time than the rest of a departure. They wait here until admission
  // finds too little memory, or the service ends.
  std::vector<Case*> graveyard;
  void bury() {
    if (graveyard.empty()) return;
    for (Case* c : graveyard) delete c;
    graveyard.clear();
    // the cases' arrays went back to the device's memory pool (stream-ordered frees on the
    // service stream): once those frees have run, hand the pool's idle memory back to the device
    if (cudaStreamSynchronize(svc.stream) == cudaSuccess) {
      int dev = 0;
      cudaMemPool_t pool = nullptr;
      if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
          cudaMemPoolTrimTo(pool, 0) != cudaSuccess)
        cudaGetLastError();
    } else {
      cudaGetLastError();
    }
  }
  std::map<long long, int> inject_oom;  // fault injection: admissions of a ticket that fail as OOM
  double clock_ms = 0;  // accumulated device time of all steps
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // admission runs at most every admit_interval steps unless the resident cells fall to half
  // the budget: a newly admitted case's first iteration builds its AMG hierarchy, a step that
  // cannot be replayed from the captured graph, so admissions are gathered into few steps
  int admit_interval = 8;
  long long steps_since_admit = 1 << 30;
  // schedule autotuner: times the candidate CTA thresholds of the V-cycle on the live batch
  // (graph-replayed steps only; the first step after each switch, which re-captures the graph,
  // is not timed) over two rounds, the second in reverse order so that a batch whose ticks get
  // shorter as cases finish favours no candidate, and switches to the fastest only if it beats
  // the threshold in use by kTuneMargin. The threshold does not change any result, only which
  // launches run the small levels. Re-tunes every tune_every steps.
  bool tune_on = true;
  long long tune_every = 2000, next_tune = 24, steps = 0;
  std::vector<int> tune_cand = {2048, 4096, 8192, 16384, 65536};
  int tune_pos = -1, tune_in_cand = 0;  // position in the candidate sequence; steps at it
  int tune_prev = 0;                    // the threshold in use when the tuning started
  std::vector<double> tune_ms;
  std::vector<int> tune_n;
  std::vector<long long> finished_unpolled;  // tickets finished since the last poll
  ~ServiceImpl() {
    bury();
    for (auto& kv : rec) {
      // ufvm_service_destroy has cleared the cases that hold slots (the Service frees those)
      if (kv.second.c) delete kv.second.c;
      kv.second.c = nullptr;
      free_snapshot(kv.second.snap);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
  static void free_snapshot(Snapshot& s) {
    for (double** q : {&s.U, &s.p, &s.mdot})
      if (*q) { cudaFree(*q); *q = nullptr; }
    s.nU = s.np = s.nm = 0;
  }
  long long active_cells() const { return resident_cells; }
  long long slot_bytes() const {
    long long b = 0;
    for (size_t q = 0; q < svc.cases.size(); ++q) {
      const Record& r = rec.at(svc.tickets[q]);
      // before its first iteration a case holds no hierarchy yet: count the estimate
      b += std::max<long long>(svc.cases[q]->dev_bytes, r.iterations == 0 ? estimate(r.est_raw) : 0);
    }
    return b;
  }
  long long estimate(long long raw) const { return (long long)(1.05 * est_scale * (double)raw); }
};

// Device bytes of a case before its hierarchy, from its sizes: the mesh geometry (23 face and
// cell arrays), the fields over cells and boundary rows (U, its gradient, p, the p and PP
// gradients, DU: 23 rows of doubles), the per-face momentum terms and fluxes, the level-0 matrix,
// its schedules and colour-major copies, and the agglomeration hierarchy with its FP32 and ELL
// copies (about as much again as the level-0 matrix). The service scales it by the largest
// ratio of measured to estimated bytes it has seen.
// Device memory a new case can take: the driver's free bytes plus what the device's default
// memory pool holds without an allocation in it (the service allocates from that pool, and the
// pool keeps what departed cases gave back).
static bool device_room(size_t* room) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int dev = 0;
  cudaMemPool_t pool = nullptr;
  unsigned long long reserved = 0, used = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess) {
    if (reserved > used) fr += (size_t)(reserved - used);
  } else {
    cudaGetLastError();
  }
  *room = fr;
  return true;
}

static long long estimate_raw(long long Nc, long long F, long long Fi, long long nodes) {
  const long long Fb = F - Fi, R = Nc + Fb, nnz = 2 * Fi;
  // per face: 19 geometry arrays, mdot, two Rhie-Chow coefficients and 3 x 7 staged momentum terms
  const long long dbl = 19 * F + 4 * Nc + 23 * R + 24 * F + 8 * Nc + 2 * (nnz + 8 * Nc) + 4 * nnz;
  const long long ints = 3 * F + 4 * Fi + 6 * Nc + 3 * nnz + nodes / 4;
  return 8 * dbl + 4 * ints;
}

static void fill_desc(const Pending& p, ufvm_mesh_desc& d) {
  d.n_points = (int32_t)(p.points.size() / 3); d.points = p.points.data();
  d.n_faces = (int32_t)p.own.size(); d.face_start = p.fs.data(); d.face_nodes = p.fn.data();
  d.n_interior = (int32_t)p.nei.size(); d.owner = p.own.data(); d.neighbour = p.nei.data();
  d.n_patches = (int32_t)p.ptype.size(); d.patch_type = p.ptype.data(); d.patch_start = p.pstart.data();
  d.patch_n = p.pn.data();
}

static void drop_frozen_(ServiceImpl& S);

// Finished slots leave the batch: each case's memory is freed (its result lives in its
// snapshot) and the slot tables are rebuilt at the next iteration.
static void drop_frozen(ServiceImpl& S) {
  const auto t0 = std::chrono::steady_clock::now();
  drop_frozen_(S);
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  S.host_drop_ms += ms;
  S.last_drop_ms = ms;
}

static void drop_frozen_(ServiceImpl& S) {
  Service& V = S.svc;
  std::vector<Case*> keep;
  std::vector<long long> keept;
  std::vector<char> kf;
  std::vector<int> ka;
  bool any = false;
  for (size_t q = 0; q < V.cases.size(); ++q) {
    if (!S.frozen[q]) {
      keep.push_back(V.cases[q]); keept.push_back(V.tickets[q]); kf.push_back(0); ka.push_back(S.frozen_age[q]);
      continue;
    }
    any = true;
    auto it = S.rec.find(V.tickets[q]);
    Record& r = it->second;
    if (r.released) {  // nobody will read it: the case goes to be freed, the ticket is forgotten
      S.graveyard.push_back(V.cases[q]);
      S.rec.erase(it);
    } else if (r.snap.U) {  // the snapshot holds the result: the case goes to be freed
      S.graveyard.push_back(V.cases[q]);
      r.c = nullptr;
    }  // else the record keeps the case (its fields are the result)
  }
  if (!any) return;
  V.cases = keep; V.tickets = keept; S.frozen = kf; S.frozen_age = ka;
  V.tables_dirty = true;
  ++S.n_drops;
  S.force_drop = false;
  S.waste_ms = 0.0;
}

static bool admission_due(const ServiceImpl& S) {
  if (S.queue.empty()) return false;
  return S.resident_cells == 0 || S.steps_since_admit >= S.admit_interval || 2 * S.resident_cells <= S.max_cells;
}

// A case created ahead of the admission loop (by precreate below).
struct Precreated {
  Case* c = nullptr;
  int status = UFVM_OK;
  long long bytes = 0;
  std::string err;
};

static void case_settings(const ServiceImpl& S, const Pending& p, ufvm_settings& cs) {
  cs = S.svc.S;
  cs.nu = p.nu;
  // the pressure reference cell is per case, as in cfdReadSystem.m:238-252: a case whose
  // boundaries are all walls, empty or symmetry planes pins p at the settings' pRefCell
  // (cell 0 when the shared settings carry none); any other case has no reference cell
  bool closed = true;
  for (int32_t t : p.ptype)
    if (t != UFVM_PATCH_WALL && t != UFVM_PATCH_EMPTY && t != UFVM_PATCH_SYMMETRY) closed = false;
  cs.fixed_element = closed ? std::max(0, S.svc.S.fixed_element) : -1;
}

// Creating a case (mesh connectivity on the host, uploads, geometry kernels, a wait for them) is
// independent from case to case, so when several queued cases are about to be admitted they are
// created ahead on up to kBuildThreads host threads, each on its own stream, and the admission
// loop below takes them in queue order. The queue prefix is the one the loop would admit by the
// same checks (estimated bytes and cells); a case the loop does not take is freed again. A
// created case then runs on the service stream like any other.
static std::map<long long, Precreated> precreate(ServiceImpl& S) {
  std::map<long long, Precreated> out;
  std::vector<Pending*> pick;
  long long cells = S.resident_cells, bytes = S.slot_bytes() + S.snap_bytes, est_sum = 0;
  bool empty = S.svc.cases.empty();
  size_t fr = 0;
  if (!device_room(&fr)) return out;
  for (Pending& p : S.queue) {
    const long long est = S.estimate(p.est_raw);
    if (!empty && (cells + p.cells > S.max_cells || bytes + est > S.max_bytes)) break;
    if (est_sum + est + (est >> 3) > (long long)fr) break;
    cells += p.cells;
    bytes += est;
    est_sum += est;
    empty = false;
    pick.push_back(&p);
  }
  if (pick.size() < 4) return out;  // a few cases: the loop creates them itself
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return out;
  }
  const int nt = (int)std::min<size_t>(pick.size(), kBuildThreads);
  std::vector<Precreated> res(pick.size());
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    cudaStream_t st = nullptr;
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return;  // the cases this thread would have made are created by the loop instead
    }
    AllocStreamScope scope(st);  // this thread's allocations are ordered on its stream
    for (size_t k = next++; k < pick.size(); k = next++) {
      const Pending& p = *pick[k];
      ufvm_mesh_desc d;
      fill_desc(p, d);
      ufvm_settings cs;
      case_settings(S, p, cs);
      Case* c = new Case();
      const long long b0 = t_dev_bytes;
      int rc = create_case_into(*c, &d, cs, p.bcu.data(), p.bcp.data(), p.bvu.data(), p.bvp.data(), nullptr,
                                nullptr, nullptr, st);
      // the level-0 system and its colouring depend on the mesh only: made here too, in parallel,
      // instead of one case after another in the first step
      if (rc == UFVM_OK) rc = c->fresh_level0();
      if (rc == UFVM_OK) rc = build_coloring(c->lin, c->lev[0]);
      if (cudaStreamSynchronize(st) != cudaSuccess) cudaGetLastError();
      res[k].bytes = t_dev_bytes - b0;
      res[k].status = rc;
      if (rc != UFVM_OK) res[k].err = get_error();
      c->stream = S.svc.stream;  // from here on the case runs on the service stream
      c->lin.stream = S.svc.stream;
      res[k].c = c;
    }
    cudaStreamDestroy(st);
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nt; ++w) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
  for (size_t k = 0; k < pick.size(); ++k)
    if (res[k].c) out[pick[k]->ticket] = res[k];
  return out;
}

static int admit_(ServiceImpl& S);
// Admission with its host time accounted (mesh uploads and processing of the admitted cases).
static int admit(ServiceImpl& S) {
  if (!admission_due(S)) return UFVM_OK;
  const double t0 = host_ms_now();
  const int rc = admit_(S);
  S.host_admit_ms += host_ms_now() - t0;
  return rc;
}

static int admit_(ServiceImpl& S) {
  drop_frozen(S);  // departures are gathered into the admission's table rebuild
  const size_t before = S.svc.cases.size();
  std::map<long long, Precreated> pre = precreate(S);
  auto take_pre = [&](long long ticket, Precreated& out) -> bool {
    auto it = pre.find(ticket);
    if (it == pre.end()) return false;
    out = it->second;
    pre.erase(it);
    return true;
  };
  while (!S.queue.empty()) {
    Pending& p = S.queue.front();
    const long long est = S.estimate(p.est_raw);
    if (!S.svc.cases.empty()) {
      if (S.resident_cells + p.cells > S.max_cells) break;
      if (S.slot_bytes() + S.snap_bytes + est > S.max_bytes) { ++S.n_deferred_mem; break; }
      size_t fr = 0;
      if (device_room(&fr) && (long long)fr < est + (est >> 3)) {
        if (!S.graveyard.empty()) {  // free the departed cases, then look again
          S.bury();
          continue;
        }
        ++S.n_deferred_mem;
        break;
      }
    }
    ufvm_mesh_desc d;
    fill_desc(p, d);
    ufvm_settings cs;
    case_settings(S, p, cs);
    Case* c = nullptr;
    int st;
    bool injected = false;
    Precreated made;
    const bool premade = take_pre(p.ticket, made);
    auto inj = S.inject_oom.find(p.ticket);
    if (inj != S.inject_oom.end() && inj->second > 0) {  // a failed device allocation, injected
      --inj->second;
      if (premade) delete made.c;
      c = new Case();
      set_error("cudaMalloc: out of memory (injected)");
      st = UFVM_E_OOM;
      injected = true;
    } else if (premade) {
      c = made.c;
      st = made.status;
      c->dev_bytes = made.bytes;
      if (st != UFVM_OK) set_error(made.err);
    } else {
      c = new Case();
      const long long b0 = t_dev_bytes;
      st = create_case_into(*c, &d, cs, p.bcu.data(), p.bcp.data(), p.bvu.data(), p.bvp.data(), nullptr, nullptr,
                            nullptr, S.svc.stream);
      c->dev_bytes = t_dev_bytes - b0;
    }
    Record& r = S.rec[p.ticket];
    if (st == UFVM_E_OOM && !injected && !S.graveyard.empty()) {  // room held by departed cases: free it, retry
      delete c;
      cudaGetLastError();
      S.bury();
      continue;
    }
    if (st == UFVM_E_OOM && !S.svc.cases.empty()) {
      // the device is full after all: the request waits at the head of the queue for memory
      delete c;
      cudaGetLastError();
      ++S.n_oom_requeue;
      break;
    }
    r.t_admit = S.clock_ms;
    if (st != UFVM_OK) {
      r.err = get_error();
      delete c;
      r.state = 3;
      r.status = st;
      r.t_done = S.clock_ms;
      ++S.finished;
      S.finished_unpolled.push_back(p.ticket);
      S.queue.pop_front();
      continue;
    }
    r.state = 1;
    r.c = c;
    r.cells = p.cells;
    r.est_raw = p.est_raw;
    S.resident_cells += p.cells;
    S.svc.cases.push_back(c);
    S.svc.tickets.push_back(p.ticket);
    S.frozen.push_back(0);
    S.frozen_age.push_back(0);
    S.svc.tables_dirty = true;
    S.queue.pop_front();
  }
  for (auto& kv : pre) delete kv.second.c;  // created ahead but not admitted this time
  if (S.svc.cases.size() != before) S.steps_since_admit = 0;
  return UFVM_OK;
}

// Copies a finishing case's result to a device snapshot (stream-ordered allocations, no device
// synchronisation). Returns false when there is no memory for it: the slot then leaves the batch
// at once and the record keeps the case itself.
static bool snapshot(ServiceImpl& S, Record& r, Case& C) {
  Snapshot& s = r.snap;
  const size_t R = C.M.Nc + C.M.Fb;
  s.nU = 3 * (size_t)C.rowsU; s.np = R; s.nm = (size_t)C.M.F;
  cudaStream_t st = S.svc.stream;
  if (cudaMallocAsync((void**)&s.U, s.nU * sizeof(double), st) != cudaSuccess ||
      cudaMallocAsync((void**)&s.p, s.np * sizeof(double), st) != cudaSuccess ||
      cudaMallocAsync((void**)&s.mdot, s.nm * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    for (double** q : {&s.U, &s.p, &s.mdot})
      if (*q) { cudaFreeAsync(*q, st); *q = nullptr; }
    s.nU = s.np = s.nm = 0;
    return false;
  }
  bool ok = true;
  for (int c = 0; c < 3; ++c)
    ok = ok && cudaMemcpyAsync(s.U + (size_t)c * C.rowsU, C.U[c].p, (size_t)C.rowsU * sizeof(double),
                               cudaMemcpyDeviceToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(s.p, C.p.p, R * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(s.mdot, C.mdot.p, (size_t)C.M.F * sizeof(double), cudaMemcpyDeviceToDevice, st) ==
                 cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    for (double** q : {&s.U, &s.p, &s.mdot})
      if (*q) { cudaFreeAsync(*q, st); *q = nullptr; }
    s.nU = s.np = s.nm = 0;
    return false;
  }
  S.snap_bytes += s.bytes();
  return true;
}

// One step of the schedule autotuner (called after every timed step).
constexpr double kTuneMargin = 0.02;
static void tune_step(ServiceImpl& S, double ms, bool graph_step) {
  if (!S.tune_on) return;
  const int nc = (int)S.tune_cand.size();
  // candidate at sequence position q: forward in the first round, backward in the second
  auto cand_at = [nc](int q) { return q < nc ? q : 2 * nc - 1 - q; };
  if (S.tune_pos < 0) {
    if (S.steps < S.next_tune || S.svc.cases.size() < 2) return;
    S.tune_ms.assign(nc, 0.0);
    S.tune_n.assign(nc, 0);
    S.tune_pos = 0;
    S.tune_in_cand = 0;
    S.tune_prev = S.svc.cta_rows;
    S.svc.cta_rows = S.tune_cand[cand_at(0)];
    S.svc.tables_dirty = true;
    return;
  }
  const int cand = cand_at(S.tune_pos);
  // step 0 at a candidate re-captures the graph; steps 1-2 are timed
  if (S.tune_in_cand >= 1 && graph_step) {
    S.tune_ms[cand] += ms;
    S.tune_n[cand] += 1;
  }
  if (++S.tune_in_cand < 3) return;
  S.tune_in_cand = 0;
  if (++S.tune_pos < 2 * nc) {
    S.svc.cta_rows = S.tune_cand[cand_at(S.tune_pos)];
    S.svc.tables_dirty = true;
    return;
  }
  int best = -1, prev = -1;
  double best_ms = 0;
  for (int k = 0; k < nc; ++k) {
    if (S.tune_n[k] == 0) continue;
    if (S.tune_cand[k] == S.tune_prev) prev = k;
    if (best < 0 || S.tune_ms[k] / S.tune_n[k] < best_ms) {
      best = k;
      best_ms = S.tune_ms[k] / S.tune_n[k];
    }
  }
  // keep the threshold in use unless the fastest candidate is clearly faster
  if (prev >= 0 && best_ms >= (1.0 - kTuneMargin) * (S.tune_ms[prev] / S.tune_n[prev])) best = prev;
  if (best >= 0) S.svc.cta_rows = S.tune_cand[best];
  S.svc.tables_dirty = true;
  S.tune_pos = -1;
  S.next_tune = S.steps + S.tune_every;
  ++S.svc.n_tunes;
}

}  // namespace ufvm

using namespace ufvm;

struct ufvm_service {
  ServiceImpl impl;
};

extern "C" {

int ufvm_service_create(const ufvm_settings* settings, int64_t max_resident_cells, ufvm_service** out) {
  if (!settings || !out || max_resident_cells <= 0) { set_error("bad argument"); return UFVM_E_INVALID; }
  if (settings->precision != UFVM_PREC_FP32_AMG || !settings->p_amg) {
    set_error("the service solves p with FP32 AMG inside FP64 refinement: set precision = UFVM_PREC_FP32_AMG");
    return UFVM_E_INVALID;
  }
  ufvm_service* h = new ufvm_service();
  ServiceImpl& S = h->impl;
  S.svc.S = *settings;
  S.svc.use_graph = settings->service_eager ? 0 : 1;
  S.max_cells = max_resident_cells;
  if (cudaStreamCreateWithFlags(&S.svc.stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&S.e0) != cudaSuccess || cudaEventCreate(&S.e1) != cudaSuccess) {
    set_error("CUDA initialisation failed (no device?)");
    delete h;
    return UFVM_E_CUDA;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&S.svc.nsm, cudaDevAttrMultiProcessorCount, dev);
  S.svc.lin.stream = S.svc.stream;
  // Result snapshots come from the device's default memory pool (stream-ordered, no device
  // synchronisation); the pool keeps what released results give back for the next ones instead
  // of returning it to the driver at every synchronisation, which would unmap and map memory
  // between steps.
  {
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long keep = ~0ull;
      if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) cudaGetLastError();
    } else {
      cudaGetLastError();
    }
  }
  // default HBM budget: 90% of the device memory free when the service starts
  size_t fr = 0;
  if (!device_room(&fr)) fr = 0;
  S.max_bytes = (long long)(0.9 * (double)fr);
  *out = h;
  return UFVM_OK;
}

int ufvm_service_submit(ufvm_service* h, const ufvm_mesh_desc* m, double nu, const int32_t* bc_type_u,
                        const int32_t* bc_type_p, const double* bc_val_u, const double* bc_val_p, int32_t max_iter,
                        int64_t* ticket) {
  if (!h || !m || !bc_type_u || !bc_type_p || !bc_val_u || !bc_val_p || !ticket) {
    set_error("null argument");
    return UFVM_E_INVALID;
  }
  ServiceImpl& S = h->impl;
  Pending p;
  p.ticket = S.next_ticket++;
  p.max_iter = max_iter;
  p.nu = nu;
  const int F = m->n_faces, Fb = m->n_faces - m->n_interior;
  p.points.assign(m->points, m->points + 3 * (size_t)m->n_points);
  p.fs.assign(m->face_start, m->face_start + F + 1);
  p.fn.assign(m->face_nodes, m->face_nodes + m->face_start[F]);
  p.own.assign(m->owner, m->owner + F);
  p.nei.assign(m->neighbour, m->neighbour + m->n_interior);
  p.ptype.assign(m->patch_type, m->patch_type + m->n_patches);
  p.pstart.assign(m->patch_start, m->patch_start + m->n_patches);
  p.pn.assign(m->patch_n, m->patch_n + m->n_patches);
  p.bcu.assign(bc_type_u, bc_type_u + m->n_patches);
  p.bcp.assign(bc_type_p, bc_type_p + m->n_patches);
  p.bvu.assign(bc_val_u, bc_val_u + 3 * (size_t)Fb);
  p.bvp.assign(bc_val_p, bc_val_p + Fb);
  p.t_submit = S.clock_ms;
  for (int32_t o : p.own) p.cells = std::max<long long>(p.cells, (long long)o + 1);
  for (int32_t o : p.nei) p.cells = std::max<long long>(p.cells, (long long)o + 1);
  p.est_raw = estimate_raw(p.cells, F, m->n_interior, (long long)p.fn.size());
  Record& r = S.rec[p.ticket];
  r.state = 0;
  r.max_iter = max_iter;
  r.t_submit = S.clock_ms;
  *ticket = p.ticket;
  S.queue.push_back(std::move(p));
  return UFVM_OK;
}

int ufvm_service_step(ufvm_service* h, int32_t* n_resident, int32_t* n_queued, int64_t* n_finished_total) {
  if (!h) return UFVM_E_INVALID;
  AllocStreamScope alloc_scope(h->impl.svc.stream);  // the service allocates on its stream
  ServiceImpl& S = h->impl;
  Service& V = S.svc;
  {
    // gather departures: drop the frozen slots once the device time they have taken since they
    // froze reaches the host cost of dropping them, when one has waited kMaxFrozenSteps steps,
    // when no active case is left, or after a failure (admission drops them too)
    int oldest = 0;
    bool anyf = false;
    for (size_t q = 0; q < V.cases.size(); ++q)
      if (S.frozen[q]) {
        anyf = true;
        oldest = std::max(oldest, S.frozen_age[q]);
      }
    if (anyf && (S.force_drop || S.waste_ms >= V.last_rebuild_ms + S.last_drop_ms || oldest >= kMaxFrozenSteps ||
                 S.resident_cells == 0))
      drop_frozen(S);
  }
  UFVM_CHECK(admit(S));
  ++S.steps;
  if (!V.cases.empty()) {
    const long long graph_before = V.n_graph_ticks;
    UFVM_CUDA(cudaEventRecord(S.e0, V.stream));
    std::vector<double> res;
    std::vector<int> conv;
    const int st = V.iterate(res, conv);
    if (st != UFVM_OK) return st;
    UFVM_CUDA(cudaEventRecord(S.e1, V.stream));
    UFVM_CUDA(cudaEventSynchronize(S.e1));
    float ms = 0;
    UFVM_CUDA(cudaEventElapsedTime(&ms, S.e0, S.e1));
    S.clock_ms += ms;
    tune_step(S, ms, V.n_graph_ticks != graph_before);
    {  // the share of this tick spent on frozen slots (work in proportion to cells)
      long long fcells = 0;
      for (size_t q = 0; q < V.cases.size(); ++q)
        if (S.frozen[q]) fcells += S.rec[V.tickets[q]].cells;
      if (fcells > 0) S.waste_ms += ms * (double)fcells / (double)(fcells + S.resident_cells);
    }
    for (size_t q = 0; q < V.cases.size(); ++q) {
      if (S.frozen[q]) { ++S.frozen_age[q]; continue; }
      Record& r = S.rec[V.tickets[q]];
      r.iterations += 1;
      if (r.iterations == 1 && r.est_raw > 0)  // hierarchy built: learn the footprint estimate's error
        S.est_scale = std::max(S.est_scale, (double)V.cases[q]->dev_bytes / (double)r.est_raw);
      std::copy(&res[q * 16], &res[q * 16] + 16, r.res);
      bool done = false;
      if (conv[q] == 1) { r.state = 2; r.status = UFVM_OK; done = true; }
      else if (conv[q] < 0) { r.state = 3; r.status = -conv[q]; done = true; S.force_drop = true; }
      else if (r.max_iter > 0 && r.iterations >= r.max_iter) { r.state = 3; r.status = UFVM_E_NOT_CONVERGED; done = true; }
      if (done) {
        r.t_done = S.clock_ms;
        S.resident_cells -= r.cells;
        ++S.finished;
        S.finished_unpolled.push_back(V.tickets[q]);
        S.frozen[q] = 1;
        S.frozen_age[q] = 0;
        if (!snapshot(S, r, *V.cases[q])) S.force_drop = true;  // no room: the case leaves at once
      }
    }
  }
  ++S.steps_since_admit;
  UFVM_CHECK(admit(S));
  int active = 0;
  for (char f : S.frozen) active += f ? 0 : 1;
  if (n_resident) *n_resident = active;
  if (n_queued) *n_queued = (int32_t)S.queue.size();
  if (n_finished_total) *n_finished_total = S.finished;
  return UFVM_OK;
}

int ufvm_service_status(ufvm_service* h, int64_t ticket, int32_t* state, int32_t* status, int32_t* iterations,
                        double* res16, double* latency_ms, double* queue_ms) {
  if (!h) return UFVM_E_INVALID;
  auto it = h->impl.rec.find(ticket);
  if (it == h->impl.rec.end() || it->second.released) { set_error("unknown ticket"); return UFVM_E_INVALID; }
  const Record& r = it->second;
  if (state) *state = r.state;
  if (status) *status = r.status;
  if (iterations) *iterations = r.iterations;
  if (res16) std::copy(r.res, r.res + 16, res16);
  const double now = h->impl.clock_ms;
  if (latency_ms) *latency_ms = r.state >= 2 ? r.t_done - r.t_admit : (r.state == 1 ? now - r.t_admit : 0.0);
  if (queue_ms) *queue_ms = r.state >= 1 ? r.t_admit - r.t_submit : now - r.t_submit;
  return UFVM_OK;
}

int ufvm_service_get_field(ufvm_service* h, int64_t ticket, const char* name, double* host, int64_t n,
                           int64_t* written) {
  if (!h) return UFVM_E_INVALID;
  auto it = h->impl.rec.find(ticket);
  if (it == h->impl.rec.end() || it->second.released) { set_error("unknown ticket"); return UFVM_E_INVALID; }
  const Record& rc = it->second;
  if (!rc.c && !rc.snap.U) {
    set_error("ticket has no resident or finished case" +
              (rc.err.empty() ? std::string() : " (admission failed: " + rc.err + ")"));
    return UFVM_E_INVALID;
  }
  std::string s(name ? name : "");
  std::vector<std::pair<const double*, size_t>> src;
  cudaStream_t stream = h->impl.svc.stream;
  if (rc.snap.U) {  // a finished case: its result as of the iteration it finished
    if (s == "U") src.push_back({rc.snap.U, rc.snap.nU});
    else if (s == "p") src.push_back({rc.snap.p, rc.snap.np});
    else if (s == "mdot") src.push_back({rc.snap.mdot, rc.snap.nm});
    else { set_error("unknown field " + s); return UFVM_E_INVALID; }
  } else {
    Case& C = *rc.c;
    const size_t R = C.M.Nc + C.M.Fb;
    if (s == "U") { for (int c = 0; c < 3; ++c) src.push_back({C.U[c].p, (size_t)C.rowsU}); }
    else if (s == "p") src.push_back({C.p.p, R});
    else if (s == "mdot") src.push_back({C.mdot.p, (size_t)C.M.F});
    else { set_error("unknown field " + s); return UFVM_E_INVALID; }
  }
  size_t tot = 0;
  for (auto& x : src) tot += x.second;
  if (written) *written = (int64_t)tot;
  if (!host) return UFVM_OK;
  if ((int64_t)tot > n) { set_error("host buffer too small"); return UFVM_E_INVALID; }
  size_t off = 0;
  for (auto& x : src) {
    UFVM_CUDA(cudaMemcpyAsync(host + off, x.first, x.second * sizeof(double), cudaMemcpyDeviceToHost, stream));
    off += x.second;
  }
  UFVM_CUDA(cudaStreamSynchronize(stream));
  return UFVM_OK;
}

int ufvm_service_release(ufvm_service* h, int64_t ticket) {
  if (!h) return UFVM_E_INVALID;
  AllocStreamScope alloc_scope(h->impl.svc.stream);  // the service allocates on its stream
  auto it = h->impl.rec.find(ticket);
  if (it == h->impl.rec.end()) return UFVM_OK;
  if (it->second.state == 1) { set_error("ticket is still resident"); return UFVM_E_INVALID; }
  Record& r = it->second;
  if (r.released) { set_error("unknown ticket"); return UFVM_E_INVALID; }
  ServiceImpl& S = h->impl;
  if (r.snap.U) {
    S.snap_bytes -= r.snap.bytes();
    for (double** q : {&r.snap.U, &r.snap.p, &r.snap.mdot})
      if (*q) { cudaFreeAsync(*q, S.svc.stream); *q = nullptr; }
    r.snap.nU = r.snap.np = r.snap.nm = 0;
  }
  bool in_slot = false;
  for (Case* c : S.svc.cases) in_slot = in_slot || (r.c && c == r.c);
  if (in_slot) {  // still a frozen slot: it leaves the batch with the next departures
    r.released = true;
    return UFVM_OK;
  }
  if (r.c) delete r.c;  // a case without a snapshot belongs to its record
  r.c = nullptr;
  S.rec.erase(it);
  return UFVM_OK;
}

int ufvm_service_stats(ufvm_service* h, double* out, int n) {
  if (!h || !out) return UFVM_E_INVALID;
  const Service& V = h->impl.svc;
  std::vector<double> v(V.ph_ms, V.ph_ms + Service::PH_N);
  v.push_back((double)V.n_usweeps);
  v.push_back((double)V.n_pcycles);
  v.push_back((double)V.n_iter_calls);
  v.push_back(h->impl.clock_ms);
  v.push_back((double)V.n_graph_ticks);
  v.push_back((double)V.n_captures);
  v.push_back((double)V.launches_total);
  v.push_back((double)V.cta_rows);
  v.push_back((double)V.n_tunes);
  v.push_back((double)(h->impl.slot_bytes() + h->impl.snap_bytes));
  v.push_back((double)h->impl.max_bytes);
  v.push_back((double)h->impl.n_deferred_mem);
  v.push_back((double)h->impl.n_oom_requeue);
  v.push_back((double)h->impl.n_drops);
  v.push_back(h->impl.est_scale);
  v.push_back((double)V.loops_seen[0]);  // U smoother loop bodies run by replayed ticks
  v.push_back((double)V.loops_seen[1]);  // p V-cycle loop bodies run by replayed ticks
  v.push_back(V.host_rebuild_ms);
  v.push_back(V.host_capture_ms);
  v.push_back(h->impl.host_drop_ms);
  v.push_back(V.build_wall_ms);
  for (int k = 0; k < 4; ++k) v.push_back(V.build_ms[k]);
  v.push_back(h->impl.host_admit_ms);
  for (int i = 0; i < n; ++i) out[i] = i < (int)v.size() ? v[i] : 0.0;
  return UFVM_OK;
}

int ufvm_service_profile(ufvm_service* h, int32_t kernel, int32_t reps, double* ms_per_unit,
                         double* bytes_per_unit) {
  if (!h || !ms_per_unit || !bytes_per_unit) return UFVM_E_INVALID;
  AllocStreamScope alloc_scope(h->impl.svc.stream);  // the service allocates on its stream
  return h->impl.svc.profile(kernel, reps, ms_per_unit, bytes_per_unit);
}

int ufvm_service_poll(ufvm_service* h, int64_t* tickets, int64_t capacity, int64_t* n_out) {
  if (!h || !n_out || capacity < 0 || (capacity > 0 && !tickets)) return UFVM_E_INVALID;
  auto& f = h->impl.finished_unpolled;
  const int64_t n = std::min<int64_t>(capacity, (int64_t)f.size());
  for (int64_t i = 0; i < n; ++i) tickets[i] = f[i];
  f.erase(f.begin(), f.begin() + n);
  *n_out = n;
  return UFVM_OK;
}

int ufvm_service_admit(ufvm_service* h, int32_t* n_resident) {
  if (!h) return UFVM_E_INVALID;
  AllocStreamScope alloc_scope(h->impl.svc.stream);  // the service allocates on its stream
  ServiceImpl& S = h->impl;
  S.steps_since_admit = 1 << 30;  // due now
  UFVM_CHECK(admit(S));
  int active = 0;
  for (char f : S.frozen) active += f ? 0 : 1;
  if (n_resident) *n_resident = active;
  return UFVM_OK;
}

int ufvm_service_inject_admit_oom(ufvm_service* h, int64_t ticket, int32_t count) {
  if (!h || count < 0) return UFVM_E_INVALID;
  h->impl.inject_oom[ticket] = count;
  return UFVM_OK;
}

int ufvm_service_set_memory_budget(ufvm_service* h, int64_t bytes) {
  if (!h || bytes <= 0) { set_error("the memory budget must be positive"); return UFVM_E_INVALID; }
  h->impl.max_bytes = bytes;
  return UFVM_OK;
}

int ufvm_service_set_admit_interval(ufvm_service* h, int32_t steps) {
  if (!h || steps < 1) return UFVM_E_INVALID;
  h->impl.admit_interval = steps;
  return UFVM_OK;
}

int ufvm_service_set_schedule(ufvm_service* h, int32_t cta_rows, int32_t packed) {
  if (!h || cta_rows < 0 || packed < 0 || packed > 1) return UFVM_E_INVALID;
  if (h->impl.svc.use_packing != packed) {
    h->impl.svc.use_packing = packed;
    h->impl.svc.tables_dirty = true;
  }
  if (cta_rows == 0) {  // hand the schedule back to the autotuner
    h->impl.tune_on = true;
    h->impl.next_tune = h->impl.steps;
    return UFVM_OK;
  }
  h->impl.tune_on = false;
  h->impl.tune_pos = -1;
  if (h->impl.svc.cta_rows != cta_rows) {
    h->impl.svc.cta_rows = cta_rows;
    h->impl.svc.tables_dirty = true;
  }
  return UFVM_OK;
}

int ufvm_service_stream(ufvm_service* h, void** stream) {
  if (!h || !stream) return UFVM_E_INVALID;
  *stream = (void*)h->impl.svc.stream;
  return UFVM_OK;
}

int ufvm_service_destroy(ufvm_service* h) {
  if (!h) return UFVM_OK;
  {
    AllocStreamScope alloc_scope(h->impl.svc.stream);
  // cases in slots (active or frozen) are owned by the Service; the rest by their records
  for (auto& kv : h->impl.rec)
    for (Case* c : h->impl.svc.cases)
      if (kv.second.c == c) kv.second.c = nullptr;
    delete h;
  }
  // give the memory the service's arrays held in the device's default pool back to the device
  int dev = 0;
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess || cudaMemPoolTrimTo(pool, 0) != cudaSuccess)
    cudaGetLastError();
  return UFVM_OK;
}

}  // extern "C"
