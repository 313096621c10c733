// service_api.cu -- extern "C" entry points of the batched steady-case service.
//
// Admission policy: first come, first served, while the sum of resident cells stays within
// max_resident_cells; a case that alone exceeds the budget is admitted when the service is
// empty. Each ufvm_service_step advances every resident case by one SIMPLE iteration
// (fast.cu), then retires finished cases and admits queued ones, so requests that arrive
// while others run join the batch as soon as cells free up (continuous batching).
#include <deque>
#include <map>
#include <memory>

#include "fast.cuh"

namespace ufvm {

struct Pending {
  long long ticket;
  int max_iter;
  double nu;
  std::vector<double> points, bvu, bvp;
  std::vector<int32_t> fs, fn, own, nei, ptype, pstart, pn, bcu, bcp;
  double t_submit;  // service clock (ms) at submission
};

struct Record {
  int state = 0;  // 0 queued, 1 resident, 2 converged, 3 stopped
  int status = UFVM_OK;
  int iterations = 0, max_iter = 0;
  double res[16] = {0};
  double t_submit = 0, t_admit = 0, t_done = 0;
  Case* c = nullptr;  // owned while resident or finished-unreleased
  long long cells = 0;
  std::string err;    // why admission or a step failed
};

struct ServiceImpl {
  Service svc;
  long long max_cells = 0, resident_cells = 0, next_ticket = 1, finished = 0;
  std::deque<Pending> queue;
  std::map<long long, Record> rec;
  double clock_ms = 0;  // accumulated device time of all steps
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // admission runs at most every admit_interval steps unless the resident cells fall to half
  // the budget: a newly admitted case's first iteration builds its AMG hierarchy, a step that
  // cannot be replayed from the captured graph, so admissions are gathered into few steps
  int admit_interval = 8;
  long long steps_since_admit = 1 << 30;
  // schedule autotuner: times the candidate CTA thresholds of the V-cycle on the live batch
  // (graph-replayed steps only; the first step after each switch, which re-captures the graph,
  // is not timed), interleaved over two rounds, and keeps the fastest. The threshold does not
  // change any result, only which launches run the small levels. Re-tunes every tune_every steps.
  bool tune_on = true;
  long long tune_every = 2000, next_tune = 24, steps = 0;
  std::vector<int> tune_cand = {2048, 4096, 8192, 16384, 65536};
  int tune_pos = -1, tune_in_cand = 0;  // position in the candidate sequence; steps at it
  std::vector<double> tune_ms;
  std::vector<int> tune_n;
  std::vector<long long> finished_unpolled;  // tickets finished since the last poll
  ~ServiceImpl() {
    for (auto& kv : rec)
      if (kv.second.c && kv.second.state >= 2) { delete kv.second.c; kv.second.c = nullptr; }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

static int admit(ServiceImpl& S) {
  if (S.queue.empty()) return UFVM_OK;
  if (!S.svc.cases.empty() && S.steps_since_admit < S.admit_interval && 2 * S.resident_cells > S.max_cells)
    return UFVM_OK;
  const size_t before = S.svc.cases.size();
  while (!S.queue.empty()) {
    Pending& p = S.queue.front();
    const long long nc_est = (long long)(p.own.empty() ? 0 : 1);
    long long ncell = 0;
    for (int32_t o : p.own) ncell = std::max<long long>(ncell, o + 1);
    for (int32_t o : p.nei) ncell = std::max<long long>(ncell, o + 1);
    (void)nc_est;
    if (!S.svc.cases.empty() && S.resident_cells + ncell > S.max_cells) break;
    ufvm_mesh_desc d;
    d.n_points = (int32_t)(p.points.size() / 3); d.points = p.points.data();
    d.n_faces = (int32_t)p.own.size(); d.face_start = p.fs.data(); d.face_nodes = p.fn.data();
    d.n_interior = (int32_t)p.nei.size(); d.owner = p.own.data(); d.neighbour = p.nei.data();
    d.n_patches = (int32_t)p.ptype.size(); d.patch_type = p.ptype.data(); d.patch_start = p.pstart.data();
    d.patch_n = p.pn.data();
    ufvm_settings cs = S.svc.S;
    cs.nu = p.nu;
    // the pressure reference cell is per case, as in cfdReadSystem.m:238-252: a case whose
    // boundaries are all walls, empty or symmetry planes pins p at the settings' pRefCell
    // (cell 0 when the shared settings carry none); any other case has no reference cell
    bool closed = true;
    for (int32_t t : p.ptype)
      if (t != UFVM_PATCH_WALL && t != UFVM_PATCH_EMPTY && t != UFVM_PATCH_SYMMETRY) closed = false;
    cs.fixed_element = closed ? std::max(0, S.svc.S.fixed_element) : -1;
    Case* c = new Case();
    const int st = create_case_into(*c, &d, cs, p.bcu.data(), p.bcp.data(), p.bvu.data(), p.bvp.data(), nullptr,
                                    nullptr, nullptr, S.svc.stream);
    Record& r = S.rec[p.ticket];
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
    r.cells = ncell;
    S.resident_cells += ncell;
    S.svc.cases.push_back(c);
    S.svc.tickets.push_back(p.ticket);
    S.svc.tables_dirty = true;
    S.queue.pop_front();
  }
  if (S.svc.cases.size() != before) S.steps_since_admit = 0;
  return UFVM_OK;
}

// One step of the schedule autotuner (called after every timed step).
static void tune_step(ServiceImpl& S, double ms, bool graph_step) {
  if (!S.tune_on) return;
  const int nc = (int)S.tune_cand.size();
  if (S.tune_pos < 0) {
    if (S.steps < S.next_tune || S.svc.cases.size() < 2) return;
    S.tune_ms.assign(nc, 0.0);
    S.tune_n.assign(nc, 0);
    S.tune_pos = 0;
    S.tune_in_cand = 0;
    S.svc.cta_rows = S.tune_cand[0];
    S.svc.tables_dirty = true;
    return;
  }
  const int cand = S.tune_pos % nc;
  // step 0 at a candidate re-captures the graph; steps 1-2 are timed
  if (S.tune_in_cand >= 1 && graph_step) {
    S.tune_ms[cand] += ms;
    S.tune_n[cand] += 1;
  }
  if (++S.tune_in_cand < 3) return;
  S.tune_in_cand = 0;
  if (++S.tune_pos < 2 * nc) {
    S.svc.cta_rows = S.tune_cand[S.tune_pos % nc];
    S.svc.tables_dirty = true;
    return;
  }
  int best = -1;
  double best_ms = 0;
  for (int k = 0; k < nc; ++k)
    if (S.tune_n[k] > 0 && (best < 0 || S.tune_ms[k] / S.tune_n[k] < best_ms)) {
      best = k;
      best_ms = S.tune_ms[k] / S.tune_n[k];
    }
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
  ServiceImpl& S = h->impl;
  Service& V = S.svc;
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
    std::vector<Case*> keep;
    std::vector<long long> keept;
    for (size_t q = 0; q < V.cases.size(); ++q) {
      Record& r = S.rec[V.tickets[q]];
      r.iterations += 1;
      std::copy(&res[q * 16], &res[q * 16] + 16, r.res);
      bool done = false;
      if (conv[q] == 1) { r.state = 2; r.status = UFVM_OK; done = true; }
      else if (conv[q] < 0) { r.state = 3; r.status = -conv[q]; done = true; }
      else if (r.max_iter > 0 && r.iterations >= r.max_iter) { r.state = 3; r.status = UFVM_E_NOT_CONVERGED; done = true; }
      if (done) {
        r.t_done = S.clock_ms;
        S.resident_cells -= r.cells;
        ++S.finished;
        S.finished_unpolled.push_back(V.tickets[q]);
        V.tables_dirty = true;
      } else {
        keep.push_back(V.cases[q]);
        keept.push_back(V.tickets[q]);
      }
    }
    V.cases = keep;
    V.tickets = keept;
  }
  ++S.steps_since_admit;
  UFVM_CHECK(admit(S));
  if (n_resident) *n_resident = (int32_t)V.cases.size();
  if (n_queued) *n_queued = (int32_t)S.queue.size();
  if (n_finished_total) *n_finished_total = S.finished;
  return UFVM_OK;
}

int ufvm_service_status(ufvm_service* h, int64_t ticket, int32_t* state, int32_t* status, int32_t* iterations,
                        double* res16, double* latency_ms, double* queue_ms) {
  if (!h) return UFVM_E_INVALID;
  auto it = h->impl.rec.find(ticket);
  if (it == h->impl.rec.end()) { set_error("unknown ticket"); return UFVM_E_INVALID; }
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
  if (it == h->impl.rec.end()) { set_error("unknown ticket"); return UFVM_E_INVALID; }
  if (!it->second.c) {
    set_error("ticket has no resident or finished case" +
              (it->second.err.empty() ? std::string() : " (admission failed: " + it->second.err + ")"));
    return UFVM_E_INVALID;
  }
  // borrow the case through a temporary handle-free path
  Case& C = *it->second.c;
  const size_t R = C.M.Nc + C.M.Fb;
  std::string s(name ? name : "");
  std::vector<std::pair<const double*, size_t>> src;
  if (s == "U") { for (int c = 0; c < 3; ++c) src.push_back({C.U[c].p, (size_t)C.rowsU}); }
  else if (s == "p") src.push_back({C.p.p, R});
  else if (s == "mdot") src.push_back({C.mdot.p, (size_t)C.M.F});
  else { set_error("unknown field " + s); return UFVM_E_INVALID; }
  size_t tot = 0;
  for (auto& x : src) tot += x.second;
  if (written) *written = (int64_t)tot;
  if (!host) return UFVM_OK;
  if ((int64_t)tot > n) { set_error("host buffer too small"); return UFVM_E_INVALID; }
  size_t off = 0;
  for (auto& x : src) {
    UFVM_CUDA(cudaMemcpyAsync(host + off, x.first, x.second * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    off += x.second;
  }
  UFVM_CUDA(cudaStreamSynchronize(C.stream));
  return UFVM_OK;
}

int ufvm_service_release(ufvm_service* h, int64_t ticket) {
  if (!h) return UFVM_E_INVALID;
  auto it = h->impl.rec.find(ticket);
  if (it == h->impl.rec.end()) return UFVM_OK;
  if (it->second.state == 1) { set_error("ticket is still resident"); return UFVM_E_INVALID; }
  if (it->second.c) { delete it->second.c; it->second.c = nullptr; }
  h->impl.rec.erase(it);
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
  for (int i = 0; i < n; ++i) out[i] = i < (int)v.size() ? v[i] : 0.0;
  return UFVM_OK;
}

int ufvm_service_profile(ufvm_service* h, int32_t kernel, int32_t reps, double* ms_per_unit,
                         double* bytes_per_unit) {
  if (!h || !ms_per_unit || !bytes_per_unit) return UFVM_E_INVALID;
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
  // resident cases are owned by the Service; finished ones by their records
  for (auto& kv : h->impl.rec)
    if (kv.second.state == 1) kv.second.c = nullptr;
  delete h;
  return UFVM_OK;
}

}  // extern "C"
