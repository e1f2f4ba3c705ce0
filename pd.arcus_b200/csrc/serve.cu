// Request loop: continuous batching of single-point, minimisation and MD
// jobs of different sizes on one GPU (pdgpu_serve_*, include/pdgpu.h).
//
// No reference counterpart: the reference runs one protocol on one
// WorkSpace at a time (protocols/protocolbase.cpp, md.cpp:202-267,
// minimise.cpp:99-179, energy.cpp:14-20).  Here a worker thread owns the
// device side of every admitted job.  Each job gets its own CUDA stream and
// device state (coordinates, neighbour list, Born radii, integrator or
// minimiser state stay resident until it finishes) and advances as a small
// state machine: the worker enqueues one phase of work (a tile search or a
// list sizing pass, a single-point evaluation, a chunk of minimiser steps, an
// MD block replayed
// from a CUDA graph), records an event, and moves on to the other jobs; the
// next phase is enqueued when the event has completed.  Kernels of different
// jobs therefore overlap on the device, and a job that arrives while others
// run is admitted as soon as a stream slot and its memory estimate fit under
// the HBM budget (in arrival order, or least work first with jobs that
// waited over a second ahead of the rest).  Every job runs the kernels the
// plain calls run, with one fixed pair-pass layout, so its results do not
// depend on what else is on the device.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "entry.cuh"

using namespace pdgpu;

namespace {

using Clock = std::chrono::steady_clock;
double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Page-locked host blocks reused across jobs (cudaHostAlloc is slow).
class PinnedPool {
 public:
  void *get(size_t bytes, size_t *cap) {
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    {
      std::lock_guard<std::mutex> lk(m_);
      auto it = free_.find(c);
      if (it != free_.end()) {
        void *p = it->second;
        free_.erase(it);
        *cap = c;
        return p;
      }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, c, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    *cap = c;
    return p;
  }
  void put(void *p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(m_);
    free_.emplace(cap, p);
  }
  ~PinnedPool() {
    for (auto &kv : free_) cudaFreeHost(kv.second);
  }

 private:
  std::multimap<size_t, void *> free_;
  std::mutex m_;
};

enum Phase { PH_QUEUED, PH_SIZE, PH_MIN, PH_MD, PH_FINISH, PH_DONE, PH_FAILED };

constexpr double kAgeMs = 1000.0;  // least-work admission: a job queued this long goes first

// what the device writes back between phases (page-locked)
struct PinHead {
  long long total;     // list entries after a count pass
  int flags[F_COUNT];  // device flags (overflow, NaN)
  int step;            // MD: step of the block start (host -> device)
  int pad;
};

struct Job {
  int64_t id = 0;
  pdgpu_job spec;
  std::shared_ptr<SystemHost> host;
  int natoms = 0;
  std::vector<double> x0;  // SoA start positions
  Clock::time_point t_submit, t_admit, t_done;
  int state = PDGPU_JOB_QUEUED;
  int status = PDGPU_OK;
  std::string error;
  int steps_done = 0;
  int64_t est_bytes = 0, charged = 0;
  // device side
  std::unique_ptr<SysEntry> e;
  cudaStream_t st = nullptr;
  int slot = -1;
  cudaEvent_t ev = nullptr;
  Phase phase = PH_QUEUED, after_size = PH_QUEUED;
  PinHead *pin = nullptr;
  size_t pin_cap = 0;
  double *res = nullptr;  // x,y,z | fixed fx,fy,fz | gx,gy,gz | energies | MD history
  size_t res_cap = 0;
  bool have_results = false;
  // progress
  int counter = 0;   // list cadence counter
  int iter = 0;      // minimiser iterations the device took
  int taken = 0;     // minimiser steps of the system
  int chunk = 0;     // minimiser steps in the chunk in flight
  int md_done = 0;   // MD steps completed
  int block = 0;     // MD steps in the block in flight
  int regrow = 0;
  MDCoef k;
  unsigned char *min_host = nullptr;  // minimiser state read-back (inside pin)
  // a group: single-point, minimisation or MD jobs admitted together share
  // one device pack (a batch, one launch sequence for all of them).  The
  // leader owns the pack, the stream slot and the phases; `group` lists
  // every member in pack order (the leader first), empty for a lone job.
  std::vector<Job *> group;
  int gpos = 0;            // position in the leader's pack
  bool member_failed = false;
};

constexpr int kGroupMax = 64;              // jobs per group
constexpr long long kGroupAtoms = 262144;  // atoms per group

size_t res_doubles(const Job &j) {
  size_t n = (size_t)j.natoms;
  size_t d = 12 * n + E_COUNT;
  if (j.spec.kind == PDGPU_JOB_MD) d += 3 * (size_t)j.spec.steps;
  return d;
}

}  // namespace

struct pdgpu_server {
  int device = 0;
  pdgpu_ctx *ctx = nullptr;
  pdgpu_serve_params prm;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<Job *> incoming;                     // guarded by m
  std::map<int64_t, std::unique_ptr<Job>> jobs;   // guarded by m
  bool stop = false;                              // guarded by m
  int64_t next_id = 1;                            // guarded by m
  // worker-owned
  std::vector<Job *> queue, active;
  std::vector<cudaStream_t> streams;
  // slots [0, n_short) run on streams of the device's highest priority and
  // take single-point jobs only, so a short job never queues behind the
  // long minimisation and MD jobs holding the other slots, and its kernels
  // are scheduled ahead of theirs
  int n_short = 0;
  std::vector<int> free_slots, free_short;
  int64_t bytes_in_use = 0;
  PinnedPool pool;
  std::thread worker;
  // statistics (guarded by m)
  pdgpu_serve_stats stats;
  // host time of the worker's steps (PDGPU_SERVE_TRACE=1: a summary on
  // stderr when the server is destroyed): [job kind][phase the step left,
  // kTraceAdmit for the admission], and the worker loop's iterations
  static constexpr int kTraceAdmit = 7;
  struct StepClock {
    long long n = 0;
    double total_ms = 0.0, max_ms = 0.0;
    void add(double ms) {
      n++;
      total_ms += ms;
      max_ms = std::max(max_ms, ms);
    }
  };
  bool trace = false;
  StepClock trace_step[3][8], trace_loop;
  void trace_add(const Job *j, int phase, Clock::time_point t0) {
    if (!trace) return;
    const int k = j->spec.kind == PDGPU_JOB_ENERGY ? 0 : j->spec.kind == PDGPU_JOB_MINIMISE ? 1 : 2;
    trace_step[k][phase].add(ms_between(t0, Clock::now()));
  }
  void trace_print() const;

  void run();
  void admit(Job *j, const std::vector<Job *> &more);
  std::vector<Job *> group_with(Job *j);
  void advance(Job *j);
  void retire(Job *j);
  void fail(Job *j, int status, const std::string &msg);
  void enqueue_size(Job *j, Phase then);
  void start(Job *j, Phase then);
  void enqueue_min_chunk(Job *j);
  void enqueue_md_block(Job *j);
  void enqueue_results(Job *j);
  bool record(Job *j, Phase next);
};

bool pdgpu_server::record(Job *j, Phase next) {
  cudaError_t e = cudaEventRecord(j->ev, j->st);
  if (e != cudaSuccess) {
    fail(j, PDGPU_ERR_CUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
    return false;
  }
  j->phase = next;
  return true;
}

void pdgpu_server::fail(Job *j, int status, const std::string &msg) {
  j->status = status;
  j->error = msg;
  j->phase = PH_FAILED;
}

// A job on the tile layout (systems within the search limit) rebuilds by
// tile search: no list, no size read-back.
static bool tile_search_job(const Pack &P) {
  return P.v.tile_mode && P.v.tile_meta && P.v.n_sc > 0 && P.v.max_sys_atoms <= kTileSearchMaxAtoms && !P.slow();
}
static void rebuild_pairs(Pack &P, cudaStream_t st) {
  if (tile_search_job(P)) {
    launch_tiles_search(P.v, st);
    P.csr_stale = true;
  } else {
    launch_nlist_count(P, st);
    launch_nlist_fill(P, st);
    P.csr_stale = false;
  }
}

// count pass of a list rebuild, its size back to the host (on the tile
// layout: the tile search, and straight on to the next phase)
void pdgpu_server::enqueue_size(Job *j, Phase then) {
  Pack &P = *j->e->pack;
  if (tile_search_job(P)) {
    rebuild_pairs(P, j->st);
    P.have_list = true;
    start(j, then);
    return;
  }
  launch_nlist_count(P, j->st);
  cudaMemcpyAsync(&j->pin->total, P.v.row_start + P.v.n_atoms, sizeof(long long), cudaMemcpyDeviceToHost, j->st);
  j->after_size = then;
  record(j, PH_SIZE);
}

// The job's work once its pairs exist: one evaluation and the results, or
// the first minimiser chunk, or the first MD block.
void pdgpu_server::start(Job *j, Phase then) {
  if (then == PH_FINISH) {
    calc_forces_enqueue(j->st, j->e.get(), true);
    enqueue_results(j);
  } else if (then == PH_MIN) {
    enqueue_min_chunk(j);
  } else {
    enqueue_md_block(j);
  }
}

// Up to 16 minimiser steps without a host round trip (as pdgpu_minimise_run),
// replayed from a graph of the job's (cached by chunk length and the steps
// of the chunk that rebuild the pairs): one launch instead of some ten per
// step from the worker thread, whose launch rate bounds the loop.
void pdgpu_server::enqueue_min_chunk(Job *j) {
  SysEntry *e = j->e.get();
  Pack &P = *e->pack;
  const pdgpu_min_params &p = j->spec.min;
  const Consts &k = consts();
  double J2k = k.J2kcal * k.Na;
  double slope = p.SlopeCutoff > 0 ? p.SlopeCutoff * J2k : -1.0;
  int steps = j->spec.steps;
  j->chunk = std::min(16, steps - j->iter);
  std::string key = "min" + std::to_string(j->chunk) + ":";
  for (int q = 0; q < j->chunk; q++) {
    int cnt = j->counter + j->iter + q;
    key += (p.UpdateNList > 0 && (cnt % p.UpdateNList) == 0) ? '1' : '0';
  }
  auto enqueue = [&]() {
    for (int q = 0; q < j->chunk; q++) {
      if (key[key.size() - j->chunk + q] == '1') rebuild_pairs(P, j->st);
      calc_forces_enqueue(j->st, e, true, min_step_src(e->min_state, false));
      launch_min_step(P.v, j->st, e->min_state, p.Algorithm, slope, p.Strictness, p.StepSize, steps);
    }
  };
  SysEntry::GraphSlot *g = nullptr;
  for (auto &x : e->gslots)
    if (x.key == key) g = &x;
  if (!g && (int)e->gslots.size() < SysEntry::kGraphSlots) {
    SysEntry::GraphSlot ng;
    begin_capture_count();
    cudaError_t ce = cudaStreamBeginCapture(j->st, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      enqueue();
      ce = cudaStreamEndCapture(j->st, &ng.graph);
    }
    ng.nodes = end_capture_count();
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ng.exec, ng.graph, 0);
    if (ce != cudaSuccess) {
      e->drop_slot(ng);
      fail(j, PDGPU_ERR_CUDA, std::string("minimiser graph: ") + cudaGetErrorString(ce));
      return;
    }
    ng.key = key;
    e->gslots.push_back(ng);
    g = &e->gslots.back();
  }
  if (g) {
    cudaGraphLaunch(g->exec, j->st);
    launch_counter() += g->nodes;
  } else {
    enqueue();
  }
  cudaMemcpyAsync(j->pin->flags, P.v.flags, sizeof(int) * F_COUNT, cudaMemcpyDeviceToHost, j->st);
  cudaMemcpyAsync(j->min_host, j->e->min_state, min_state_size() * std::max<size_t>(1, j->group.size()),
                  cudaMemcpyDeviceToHost, j->st);
  record(j, PH_MIN);
}

// One list period of MD (as pdgpu_md_run): [rebuild] + UpdateNList steps,
// replayed from the job's CUDA graph when it is a full period.
void pdgpu_server::enqueue_md_block(Job *j) {
  SysEntry *e = j->e.get();
  Pack &P = *e->pack;
  PackView &v = P.v;
  const pdgpu_md_params &p = j->spec.md;
  int every = p.UpdateNList;
  int steps = j->spec.steps;
  bool rebuild = every > 0 && (j->counter % every) == 0;
  int block = 1;
  if (rebuild && every > 1) block = std::min(every, steps - j->md_done);
  bool use_graph = p.UseGraph && rebuild && block == every && every > 1;
  j->block = block;
  j->pin->step = j->md_done;
  cudaMemsetAsync(v.flags + F_NL_OVERFLOW, 0, sizeof(int), j->st);
  // a group goes on past a member's NaN energy (the member is marked failed
  // from its energy history at the end)
  if (!j->group.empty()) cudaMemsetAsync(v.flags + F_NAN, 0, sizeof(int), j->st);
  cudaMemcpyAsync(e->step_dev, &j->pin->step, sizeof(int), cudaMemcpyHostToDevice, j->st);
  if (use_graph) {
    if (!e->gexec || e->gkey != "md") {
      e->drop_graph();
      begin_capture_count();
      cudaError_t ce = cudaStreamBeginCapture(j->st, cudaStreamCaptureModeThreadLocal);
      if (ce != cudaSuccess) {
        end_capture_count();
        fail(j, PDGPU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        return;
      }
      rebuild_pairs(P, j->st);
      for (int q = 0; q < block; q++) md_step_enqueue(j->st, e, j->k, q);
      md_steps_end(j->st, e);
      ce = cudaStreamEndCapture(j->st, &e->graph);
      e->gnodes = end_capture_count();
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->gexec, e->graph, 0);
      if (ce != cudaSuccess) {
        fail(j, PDGPU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        return;
      }
      e->gkey = "md";  // the job's list buffer and settings are fixed while the graph lives
    }
    cudaGraphLaunch(e->gexec, j->st);
    launch_counter() += e->gnodes;
  } else {
    if (rebuild) rebuild_pairs(P, j->st);
    for (int q = 0; q < block; q++) md_step_enqueue(j->st, e, j->k, q);
    md_steps_end(j->st, e);
  }
  cudaMemcpyAsync(j->pin->flags, v.flags, sizeof(int) * F_COUNT, cudaMemcpyDeviceToHost, j->st);
  record(j, PH_MD);
}

void pdgpu_server::enqueue_results(Job *j) {
  Pack &P = *j->e->pack;
  PackView &v = P.v;
  const std::vector<Job *> lone(1, j);
  const std::vector<Job *> &members = j->group.empty() ? lone : j->group;
  for (size_t s = 0; s < members.size(); s++) {
    Job *m = members[s];
    const size_t n = (size_t)m->natoms, o = (size_t)P.atom_off[s];
    double *r = m->res;
    cudaMemcpyAsync(r, v.x + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + n, v.y + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 2 * n, v.z + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 3 * n, v.fx + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 4 * n, v.fy + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 5 * n, v.fz + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 6 * n, v.gx + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 7 * n, v.gy + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 8 * n, v.gz + o, sizeof(double) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 9 * n, v.hx + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 10 * n, v.hy + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 11 * n, v.hz + o, sizeof(long long) * n, cudaMemcpyDeviceToHost, j->st);
    cudaMemcpyAsync(r + 12 * n, v.ene + s * E_COUNT, sizeof(double) * E_COUNT, cudaMemcpyDeviceToHost, j->st);
    if (m->spec.kind == PDGPU_JOB_MD && j->md_done > 0)  // member s of the [step][member][3] history
      cudaMemcpy2DAsync(r + 12 * n + E_COUNT, sizeof(double) * 3, j->e->hist + 3 * s,
                        sizeof(double) * 3 * members.size(), sizeof(double) * 3, (size_t)j->md_done,
                        cudaMemcpyDeviceToHost, j->st);
    m->have_results = true;
  }
  record(j, PH_FINISH);
}

// MD settings that must agree for jobs to share a pack (the seed is per
// system: each member keeps its own random stream)
static bool same_md(const pdgpu_job &a, const pdgpu_job &b) {
  const pdgpu_md_params &p = a.md, &q = b.md;
  return a.steps == b.steps && a.init_temp == b.init_temp && p.Integrator == q.Integrator &&
         p.UpdateNList == q.UpdateNList && p.LangevinOnHydrogens == q.LangevinOnHydrogens &&
         p.UseGraph == q.UseGraph && p.Timestep == q.Timestep && p.FricCoeff == q.FricCoeff &&
         p.TargetTemp == q.TargetTemp;
}

// Queued jobs that can share a pack with j: the same kind (single point;
// minimisation with the same settings and step count; MD with the same
// settings, step count and start temperature), the same surface-term
// cadence, on the tile layout within the tile search's size limit, fitting
// the budget; at most kGroupMax jobs and kGroupAtoms atoms.  A member's
// results do not depend on the others (the tile passes, the minimiser and
// the integrator with its per-system random stream are per system), so
// grouping changes no result.
std::vector<Job *> pdgpu_server::group_with(Job *j) {
  std::vector<Job *> more;
  const int kind = j->spec.kind;
  if (!prm.tiles || j->natoms > kTileSearchMaxAtoms) return more;
  long long atoms = j->natoms;
  int64_t bytes = bytes_in_use + j->est_bytes;
  for (Job *c : queue) {
    if ((int)more.size() + 1 >= kGroupMax) break;
    if (c == j || c->spec.kind != kind || c->natoms > kTileSearchMaxAtoms) continue;
    if (c->host->lcpo_update != j->host->lcpo_update) continue;
    if (c->host->params.FastMode != j->host->params.FastMode) continue;  // one pair-term path per pack
    if (kind == PDGPU_JOB_MINIMISE &&
        (c->spec.steps != j->spec.steps || std::memcmp(&c->spec.min, &j->spec.min, sizeof j->spec.min) != 0))
      continue;
    if (kind == PDGPU_JOB_MD && !same_md(c->spec, j->spec)) continue;
    if (atoms + c->natoms > kGroupAtoms || bytes + c->est_bytes > prm.hbm_budget) continue;
    atoms += c->natoms;
    bytes += c->est_bytes;
    more.push_back(c);
  }
  return more;
}

void pdgpu_server::admit(Job *j, const std::vector<Job *> &more) {
  if (!more.empty()) {
    j->group.push_back(j);
    for (Job *m : more) j->group.push_back(m);
  }
  const std::vector<Job *> lone(1, j);
  const std::vector<Job *> &members = j->group.empty() ? lone : j->group;
  const int S = (int)members.size();
  if (j->spec.kind == PDGPU_JOB_ENERGY && !free_short.empty()) {
    j->slot = free_short.back();
    free_short.pop_back();
  } else {
    j->slot = free_slots.back();
    free_slots.pop_back();
  }
  j->st = streams[j->slot];
  const auto now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(m);
    for (Job *x : members) {
      x->t_admit = now;
      x->state = PDGPU_JOB_RUNNING;
      stats.active++;
      stats.queued--;
    }
    if (S > 1) stats.groups++;
    stats.peak_active = std::max(stats.peak_active, stats.active);
  }
  for (int q = 0; q < S; q++) {
    Job *x = members[q];
    x->gpos = q;
    x->charged = x->est_bytes;
    bytes_in_use += x->charged;
    x->res = (double *)pool.get(sizeof(double) * res_doubles(*x), &x->res_cap);
    if (!x->res) {
      fail(j, PDGPU_ERR_NOMEM, "page-locked host allocation failed");
      return;
    }
  }
  // page-locked scratch (the leader's): flags and every member's minimiser state
  j->pin = (PinHead *)pool.get(sizeof(PinHead) + min_state_size() * S, &j->pin_cap);
  if (!j->pin) {
    fail(j, PDGPU_ERR_NOMEM, "page-locked host allocation failed");
    return;
  }
  j->min_host = (unsigned char *)(j->pin + 1);
  if (cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming) != cudaSuccess) {
    fail(j, PDGPU_ERR_CUDA, "cudaEventCreate failed");
    return;
  }
  // device state: the template's topology, the job's positions
  j->e = std::make_unique<SysEntry>();
  SysEntry *e = j->e.get();
  e->host = j->host;
  for (Job *x : members) e->members.push_back(x->host);
  e->st = j->st;
  int r = entry_materialize(device, e, false);
  if (r) {
    fail(j, r, last_error_cstr());
    return;
  }
  Pack &P = *e->pack;
  for (int q = 0; q < 3; q++) P.v.lpa[q] = prm.lanes[q];
  P.v.tile_mode = prm.tiles ? 1 : 0;
  P.tuned = true;
  P.coop = false;  // jobs run side by side on their own streams: no cooperative launches
  P.coop_md = false;
  if (prm.tiles && (r = pack_ensure_tiles(&P))) {
    fail(j, r, last_error_cstr());
    return;
  }
  for (int q = 0; q < S; q++) {  // every member's start positions into its slice of the pack
    Job *x = members[q];
    const size_t n = (size_t)x->natoms, o = (size_t)P.atom_off[q];
    std::memcpy(x->res, x->x0.data(), sizeof(double) * 3 * n);
    cudaMemcpyAsync(P.v.x + o, x->res, sizeof(double) * n, cudaMemcpyHostToDevice, j->st);
    cudaMemcpyAsync(P.v.y + o, x->res + n, sizeof(double) * n, cudaMemcpyHostToDevice, j->st);
    cudaMemcpyAsync(P.v.z + o, x->res + 2 * n, sizeof(double) * n, cudaMemcpyHostToDevice, j->st);
  }
  const size_t n = (size_t)P.v.n_atoms;
  launch_pack_positions(P.v, j->st);
  cudaMemsetAsync(P.v.flags, 0, sizeof(int) * F_COUNT, j->st);
  if (j->spec.kind == PDGPU_JOB_MINIMISE) {
    unsigned char *ms = nullptr;
    if (xalloc(e, &ms, min_state_size() * S) != cudaSuccess) {
      fail(j, PDGPU_ERR_NOMEM, "device allocation failed (minimiser state)");
      return;
    }
    e->min_state = ms;
    min_state_init(j->min_host, S);
    cudaMemcpyAsync(ms, j->min_host, min_state_size() * S, cudaMemcpyHostToDevice, j->st);
    // WorkSpace::old = cur (minimise.cpp:114)
    cudaMemcpyAsync(P.v.ox, P.v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, j->st);
    cudaMemcpyAsync(P.v.oy, P.v.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, j->st);
    cudaMemcpyAsync(P.v.oz, P.v.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, j->st);
    enqueue_size(j, PH_MIN);
  } else if (j->spec.kind == PDGPU_JOB_MD) {
    // history [step][member][3]
    if (xalloc(e, &e->hist, (size_t)3 * j->spec.steps * S) != cudaSuccess) {
      fail(j, PDGPU_ERR_NOMEM, "device allocation failed (MD history)");
      return;
    }
    e->hist_cap = j->spec.steps;
    j->pin->step = 0;
    // every member's seed, staged through the pinned block (the minimiser
    // state's room, which an MD job does not use)
    static_assert(sizeof(unsigned long long) <= 8, "seed size");
    unsigned long long *seeds = reinterpret_cast<unsigned long long *>(j->min_host);
    if (min_state_size() < sizeof(unsigned long long)) {
      fail(j, PDGPU_ERR_STATE, "pinned staging too small for the MD seeds");
      return;
    }
    for (int q = 0; q < S; q++) {
      const unsigned long long seed = members[q]->spec.md.Seed;
      std::memcpy(seeds + q, &seed, sizeof seed);
    }
    cudaMemcpyAsync(e->seeds, seeds, sizeof(unsigned long long) * S, cudaMemcpyHostToDevice, j->st);
    launch_vel_init_impl(P.v, j->st, j->spec.init_temp, e->seeds);
    j->k = md_coef(&j->spec.md, 0, j->spec.steps);
    enqueue_size(j, PH_MD);
  } else {
    enqueue_size(j, PH_FINISH);
  }
}

void pdgpu_server::advance(Job *j) {
  SysEntry *e = j->e.get();
  Pack &P = *e->pack;
  switch (j->phase) {
    case PH_SIZE: {
      long long total = j->pin->total;
      int r = nlist_reserve(P, total, j->st);
      if (r) {
        fail(j, r, last_error_cstr());
        return;
      }
      P.nl_total = total;
      cudaMemsetAsync(P.v.flags + F_NL_OVERFLOW, 0, sizeof(int), j->st);
      launch_nlist_fill(P, j->st);
      P.have_list = true;
      int64_t actual = P.bytes + 64 * 1024;
      if (actual > j->charged) {
        bytes_in_use += actual - j->charged;
        j->charged = actual;
      }
      e->drop_graph();  // a regrown list buffer invalidates a captured block
      start(j, j->after_size);
      return;
    }
    case PH_MIN: {
      // every member's state; the group goes on while one still advances
      // (a member that converged or met a NaN sits the rest out, as in
      // pdgpu_minimise_run on a batch)
      const std::vector<Job *> lone(1, j);
      const std::vector<Job *> &members = j->group.empty() ? lone : j->group;
      int advanced = 0, alive = 0;
      for (size_t q = 0; q < members.size(); q++) {
        Job *x = members[q];
        int taken, nan;
        double mult;
        min_state_read(j->min_host, (int)q, &taken, &nan, &mult);
        advanced = std::max(advanced, taken - x->taken);
        x->taken = taken;
        if (nan && !x->member_failed) {
          x->steps_done = -1;
          x->member_failed = true;
          x->status = PDGPU_ERR_UNSTABLE;
          x->error = "Simulation unstable (NaN energy during minimisation)";
        }
        if (!x->member_failed) alive++;
      }
      if (!alive) {
        fail(j, PDGPU_ERR_UNSTABLE, "Simulation unstable (NaN energy during minimisation)");
        return;
      }
      if (j->pin->flags[F_LCPO_CAND]) {
        fail(j, PDGPU_ERR_STATE, kLcpoCandMsg);
        return;
      }
      bool overflow = j->pin->flags[F_NL_OVERFLOW] != 0;
      bool finished = advanced < j->chunk && !overflow;
      j->iter += advanced;
      if (overflow) {
        if (++j->regrow > 8) {
          fail(j, PDGPU_ERR_STATE, "neighbour list kept overflowing during minimisation");
          return;
        }
        enqueue_size(j, PH_MIN);  // sized rebuild at the current positions, then go on
        return;
      }
      if (finished || j->iter >= j->spec.steps) {
        for (Job *x : members)
          if (!x->member_failed) x->steps_done = x->taken;
        // cur = old; recompute the energies (minimise.cpp:172-176)
        launch_min_finish(P.v, j->st);
        calc_forces_enqueue(j->st, e, true, min_step_src(e->min_state, true));
        enqueue_results(j);
        return;
      }
      enqueue_min_chunk(j);
      return;
    }
    case PH_MD: {
      if (j->pin->flags[F_NL_OVERFLOW]) {
        // state untouched since the block start: grow the list, run it again
        if (++j->regrow > 8) {
          fail(j, PDGPU_ERR_STATE, "neighbour list kept overflowing after regrowth");
          return;
        }
        enqueue_size(j, PH_MD);
        return;
      }
      if (j->pin->flags[F_LCPO_CAND]) {
        fail(j, PDGPU_ERR_STATE, kLcpoCandMsg);
        return;
      }
      if (j->pin->flags[F_NAN] && j->group.empty()) {
        j->steps_done = j->md_done;
        fail(j, PDGPU_ERR_UNSTABLE, "Simulation unstable or division by zero (NaN energy)");
        return;
      }
      j->md_done += j->block;
      j->counter += j->block;
      if (j->md_done >= j->spec.steps) {
        j->steps_done = j->md_done;
        enqueue_results(j);
        return;
      }
      enqueue_md_block(j);
      return;
    }
    case PH_FINISH:
      if (j->spec.kind == PDGPU_JOB_ENERGY) {
        j->steps_done = 1;
        for (Job *x : j->group) x->steps_done = 1;
      }
      if (j->spec.kind == PDGPU_JOB_MD && !j->group.empty()) {
        // a member whose energy went NaN failed at that step, as alone
        // (md.cpp's run_core stops at an unstable step)
        for (Job *x : j->group) {
          const double *h = x->res + 12 * (size_t)x->natoms + E_COUNT;
          int bad = -1;
          for (int k = 0; k < j->md_done && bad < 0; k++)
            if (!(h[3 * k] == h[3 * k])) bad = k;
          x->steps_done = bad < 0 ? j->md_done : bad;
          if (bad >= 0) {
            x->member_failed = true;
            x->status = PDGPU_ERR_UNSTABLE;
            x->error = "Simulation unstable or division by zero (NaN energy)";
          }
        }
      }
      j->phase = PH_DONE;
      return;
    default:
      return;
  }
}

void pdgpu_server::retire(Job *j) {
  if (j->e) {
    j->e->free_device();  // stream-ordered frees
    j->e.reset();
  }
  if (j->ev) {
    cudaEventDestroy(j->ev);
    j->ev = nullptr;
  }
  if (j->slot >= 0) (j->slot < n_short ? free_short : free_slots).push_back(j->slot);
  j->slot = -1;
  const std::vector<Job *> lone(1, j);
  const std::vector<Job *> members = j->group.empty() ? lone : j->group;
  for (Job *x : members) {
    bytes_in_use -= x->charged;
    x->charged = 0;
  }
  std::lock_guard<std::mutex> lk(m);
  const auto now = Clock::now();
  for (Job *x : members) {
    x->t_done = now;
    bool ok = j->phase == PH_DONE && !x->member_failed;
    if (x != j && !ok && !x->member_failed) {  // the group failed as a whole
      x->status = j->status;
      x->error = j->error;
    }
    if (x != j) x->phase = ok ? PH_DONE : PH_FAILED;
    x->state = ok ? PDGPU_JOB_DONE : PDGPU_JOB_FAILED;
    stats.active--;
    if (ok)
      stats.completed++;
    else
      stats.failed++;
  }
  stats.bytes_in_use = bytes_in_use;
  cv_done.notify_all();
}

void pdgpu_server::run() {
  cudaSetDevice(device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(m);
      while (!incoming.empty()) {
        queue.push_back(incoming.front());
        incoming.pop_front();
      }
      if (stop) {
        for (Job *j : queue) {
          j->status = PDGPU_ERR_STATE;
          j->error = "server shut down before the job was admitted";
          j->state = PDGPU_JOB_FAILED;
          j->t_done = Clock::now();
          stats.queued--;
          stats.failed++;
        }
        queue.clear();
        cv_done.notify_all();
        if (active.empty()) break;
      }
      if (active.empty() && queue.empty()) {
        cv_work.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
    }
    bool progressed = false;
    const auto t_loop = Clock::now();
    for (size_t a = 0; a < active.size();) {
      Job *j = active[a];
      cudaError_t q = cudaEventQuery(j->ev);
      if (q == cudaErrorNotReady) {
        a++;
        continue;
      }
      progressed = true;
      const auto t_step = Clock::now();
      const int ph_step = j->phase;
      if (q != cudaSuccess)
        fail(j, PDGPU_ERR_CUDA, std::string("job stream: ") + cudaGetErrorString(q));
      else
        advance(j);
      trace_add(j, ph_step, t_step);
      if (j->phase == PH_DONE || j->phase == PH_FAILED) {
        retire(j);
        active.erase(active.begin() + a);
      } else {
        a++;
      }
    }
    // Admission order: arrival (policy 0), or jobs that have waited longer
    // than kAgeMs first (in arrival order) and then the least work (atoms x
    // steps) first (policy 1); a job is admitted when a slot is free and its
    // estimate fits the budget.
    while (!free_slots.empty() || !free_short.empty()) {
      const auto now = Clock::now();
      int pick = -1;
      double best = 0;
      for (size_t q = 0; q < queue.size(); q++) {
        Job *c = queue[q];
        if (bytes_in_use + c->est_bytes > prm.hbm_budget) continue;
        if (free_slots.empty() && c->spec.kind != PDGPU_JOB_ENERGY) continue;  // only short slots left
        double waited = ms_between(c->t_submit, now);
        // a minimisation or MD job waits for like jobs to share its pack
        if (prm.group && c->spec.kind != PDGPU_JOB_ENERGY && waited < prm.batch_ms) continue;
        double key = (prm.policy == 0 || waited > kAgeMs)
                         ? -1e30 + (double)q
                         : (double)c->natoms * (double)std::max(1, c->spec.steps);
        if (pick < 0 || key < best) {
          pick = (int)q;
          best = key;
        }
      }
      if (pick < 0) break;
      Job *j = queue[pick];
      std::vector<Job *> more = prm.group ? group_with(j) : std::vector<Job *>();
      queue.erase(queue.begin() + pick);
      for (Job *x : more) queue.erase(std::find(queue.begin(), queue.end(), x));
      const auto t_admit = Clock::now();
      admit(j, more);
      trace_add(j, kTraceAdmit, t_admit);
      progressed = true;
      if (j->phase == PH_FAILED)
        retire(j);
      else
        active.push_back(j);
      std::lock_guard<std::mutex> lk(m);
      stats.bytes_in_use = bytes_in_use;
      stats.peak_bytes = std::max(stats.peak_bytes, bytes_in_use);
    }
    if (trace && progressed) trace_loop.add(ms_between(t_loop, Clock::now()));
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

void pdgpu_server::trace_print() const {
  static const char *kinds[3] = {"energy", "minimise", "md"};
  static const char *phases[8] = {"queued", "size", "min", "md", "finish", "done", "failed", "admit"};
  std::fprintf(stderr, "pdgpu serve trace: worker loop iterations with progress %lld, mean %.3f ms, max %.3f ms\n",
               trace_loop.n, trace_loop.n ? trace_loop.total_ms / trace_loop.n : 0.0, trace_loop.max_ms);
  for (int k = 0; k < 3; k++)
    for (int p = 0; p < 8; p++) {
      const StepClock &c = trace_step[k][p];
      if (c.n)
        std::fprintf(stderr, "  %-8s %-6s steps %6lld  total %9.3f ms  mean %7.3f ms  max %8.3f ms\n", kinds[k],
                     phases[p], c.n, c.total_ms, c.total_ms / c.n, c.max_ms);
    }
}

// ------------------------------------------------------------------ C ABI
// (declared in include/pdgpu.h)
struct pdgpu_ctx;
namespace pdgpu {
int ctx_device(pdgpu_ctx *c);
int ctx_system_host(pdgpu_ctx *c, int sys, std::shared_ptr<SystemHost> *out);
}  // namespace pdgpu

extern "C" {

void pdgpu_serve_params_default(pdgpu_serve_params *p) {
  std::memset(p, 0, sizeof *p);
  p->hbm_budget = 120LL * 1000 * 1000 * 1000;
  p->max_active = 16;
  p->lanes[0] = p->lanes[1] = p->lanes[2] = 8;
  p->tiles = 1;   // tile passes; rebuilds by tile search, no list (systems within the search limit)
  p->policy = 1;  // least work first: short jobs do not queue behind long MD runs
  p->group = 1;   // queued single-point / like minimisation / like MD jobs share a pack
  p->batch_ms = 60;  // like minimisation / MD jobs gather into groups (a few % of an MD job's run)
}

int pdgpu_serve_create(pdgpu_ctx *ctx, const pdgpu_serve_params *p, pdgpu_server **out) {
  if (!ctx || !out) {
    set_error("pdgpu_serve_create: NULL argument");
    return PDGPU_ERR_ARG;
  }
  pdgpu_serve_params prm;
  pdgpu_serve_params_default(&prm);
  if (p) prm = *p;
  if (prm.hbm_budget <= 0 || prm.max_active <= 0 || prm.max_active > 1024) {
    set_error("pdgpu_serve_create: budget must be > 0 and max_active in [1, 1024]");
    return PDGPU_ERR_ARG;
  }
  for (int q = 0; q < 3; q++)
    if (prm.lanes[q] != 4 && prm.lanes[q] != 8 && prm.lanes[q] != 16 && prm.lanes[q] != 32) {
      set_error("pdgpu_serve_create: lanes per atom must be 4, 8, 16 or 32");
      return PDGPU_ERR_ARG;
    }
  auto *s = new pdgpu_server();
  s->ctx = ctx;
  s->device = ctx_device(ctx);
  s->prm = prm;
  std::memset(&s->stats, 0, sizeof s->stats);
  const char *trace = std::getenv("PDGPU_SERVE_TRACE");
  s->trace = trace && trace[0] == '1';
  cudaSetDevice(s->device);
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  s->n_short = prm.max_active >= 4 ? std::max(2, prm.max_active / 4) : 0;
  for (int q = 0; q < prm.max_active; q++) {
    cudaStream_t st;
    const bool short_slot = q < s->n_short;
    cudaError_t e = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, short_slot ? greatest : least);
    if (e != cudaSuccess) {
      for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
      delete s;
      return cuda_fail(e, "pdgpu_serve_create: stream");
    }
    s->streams.push_back(st);
  }
  for (int q = prm.max_active - 1; q >= 0; q--) (q < s->n_short ? s->free_short : s->free_slots).push_back(q);
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return PDGPU_OK;
}

int pdgpu_serve_submit(pdgpu_server *s, int32_t sys, const pdgpu_job *job, const double *xyz, int64_t *job_id) {
  if (!s || !job || !xyz || !job_id) {
    set_error("pdgpu_serve_submit: NULL argument");
    return PDGPU_ERR_ARG;
  }
  if (job->kind < PDGPU_JOB_ENERGY || job->kind > PDGPU_JOB_MD ||
      (job->kind != PDGPU_JOB_ENERGY && job->steps <= 0)) {
    set_error("pdgpu_serve_submit: unknown job kind or steps <= 0");
    return PDGPU_ERR_ARG;
  }
  if (job->kind == PDGPU_JOB_MD) {
    int r = validate_md(&job->md);
    if (r) return r;
  }
  if (job->kind == PDGPU_JOB_MINIMISE && job->min.Algorithm != PDGPU_MIN_STEEPEST_DESCENT &&
      job->min.Algorithm != PDGPU_MIN_CONJUGATE_GRADIENTS) {
    set_error("pdgpu_serve_submit: unknown minimiser");
    return PDGPU_ERR_ARG;
  }
  std::shared_ptr<SystemHost> host;
  int r = ctx_system_host(s->ctx, sys, &host);
  if (r) return r;
  auto j = std::make_unique<Job>();
  j->spec = *job;
  j->host = host;
  j->natoms = host->natoms;
  size_t n = (size_t)j->natoms;
  j->x0.resize(3 * n);
  for (size_t i = 0; i < n; i++) {
    j->x0[i] = xyz[3 * i];
    j->x0[n + i] = xyz[3 * i + 1];
    j->x0[2 * n + i] = xyz[3 * i + 2];
  }
  // device bytes before the list is sized: per-atom arrays, a list of 256
  // entries per atom and the worst-case tile store (48 bytes per tile of
  // 32 x 8 atoms), the LCPO overlap lists where the system has the term;
  // the pack is charged its real size once sized
  {
    int64_t nsc = ((int64_t)n + 31) / 32, njc = ((int64_t)n + 7) / 8, tiles = 0;
    for (int64_t k = 0; k < nsc; k++) tiles += njc - 4 * k;
    j->est_bytes = (int64_t)n * (1024 + 256 * 4) + tiles * 48 + nsc * 16 * 64 + (int64_t)4 * 1024 * 1024;
    if (host->lcpo_update > 0) j->est_bytes += (int64_t)n * (kLcpoMax * 12 + kLcpoCand * 4 + 96);
  }
  if (j->est_bytes > s->prm.hbm_budget) {
    set_error("pdgpu_serve_submit: the job alone exceeds the HBM budget");
    return PDGPU_ERR_BUDGET;
  }
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->m);
  if (s->stop) {
    set_error("pdgpu_serve_submit: server is shutting down");
    return PDGPU_ERR_STATE;
  }
  j->id = s->next_id++;
  *job_id = j->id;
  s->incoming.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  s->stats.submitted++;
  s->stats.queued++;
  s->cv_work.notify_one();
  return PDGPU_OK;
}

static Job *find_job(pdgpu_server *s, int64_t id) {
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) {
    set_error("unknown job id " + std::to_string(id));
    return nullptr;
  }
  return it->second.get();
}

int pdgpu_serve_wait(pdgpu_server *s, int64_t job_id, double timeout_s) {
  if (!s) return PDGPU_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->m);
  Job *j = find_job(s, job_id);
  if (!j) return PDGPU_ERR_ARG;
  auto done = [&] { return j->state == PDGPU_JOB_DONE || j->state == PDGPU_JOB_FAILED; };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    set_error("pdgpu_serve_wait: timed out");
    return PDGPU_ERR_STATE;
  }
  if (j->state == PDGPU_JOB_FAILED) {
    set_error(j->error);
    return j->status;
  }
  return PDGPU_OK;
}

int pdgpu_serve_info(pdgpu_server *s, int64_t job_id, pdgpu_job_info *info) {
  if (!s || !info) return PDGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  Job *j = find_job(s, job_id);
  if (!j) return PDGPU_ERR_ARG;
  std::memset(info, 0, sizeof *info);
  info->state = j->state;
  info->status = j->status;
  info->natoms = j->natoms;
  info->kind = j->spec.kind;
  bool admitted = j->state != PDGPU_JOB_QUEUED && j->t_admit != Clock::time_point();
  bool finished = j->state == PDGPU_JOB_DONE || j->state == PDGPU_JOB_FAILED;
  if (finished) info->steps_done = j->steps_done;
  info->t_queue_ms = admitted ? ms_between(j->t_submit, j->t_admit) : -1.0;
  info->t_run_ms = admitted && finished ? ms_between(j->t_admit, j->t_done) : -1.0;
  info->t_total_ms = finished ? ms_between(j->t_submit, j->t_done) : -1.0;
  return PDGPU_OK;
}

int pdgpu_serve_result(pdgpu_server *s, int64_t job_id, double *xyz, double *f, double *ene, double *history) {
  if (!s) return PDGPU_ERR_ARG;
  Job *j;
  {
    std::lock_guard<std::mutex> lk(s->m);
    j = find_job(s, job_id);
    if (!j) return PDGPU_ERR_ARG;
    if (j->state != PDGPU_JOB_DONE && j->state != PDGPU_JOB_FAILED) {
      set_error("pdgpu_serve_result: job not finished");
      return PDGPU_ERR_STATE;
    }
    if (!j->have_results || j->phase != PH_DONE) {
      set_error("pdgpu_serve_result: the job failed before producing results: " + j->error);
      return j->status ? j->status : PDGPU_ERR_STATE;
    }
  }
  size_t n = (size_t)j->natoms;
  const double *r = j->res;
  const Consts &k = consts();
  if (xyz)
    for (size_t i = 0; i < n; i++) {
      xyz[3 * i] = r[i];
      xyz[3 * i + 1] = r[n + i];
      xyz[3 * i + 2] = r[2 * n + i];
    }
  if (f) {
    // as the integrator sums them: fixed point, FP64 pair, tile j side
    const long long *fx = (const long long *)(r + 3 * n);
    const long long *hx = (const long long *)(r + 9 * n);
    for (size_t i = 0; i < n; i++)
      for (int c = 0; c < 3; c++)
        f[3 * i + c] = ((double)fx[c * n + i] * kInvForceScale + r[(6 + c) * n + i] +
                        (double)hx[c * n + i] * kInvJScale) *
                       k.N_per_kcalmolA;
  }
  if (ene)
    for (int q = 0; q < E_COUNT; q++) ene[q] = r[12 * n + q] * k.J_per_kcalmol;
  if (history && j->spec.kind == PDGPU_JOB_MD)
    for (size_t q = 0; q < 3 * (size_t)j->steps_done; q++)
      history[q] = r[12 * n + E_COUNT + q] * k.J_per_kcalmol;
  return PDGPU_OK;
}

int pdgpu_serve_release(pdgpu_server *s, int64_t job_id) {
  if (!s) return PDGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  Job *j = find_job(s, job_id);
  if (!j) return PDGPU_ERR_ARG;
  if (j->state != PDGPU_JOB_DONE && j->state != PDGPU_JOB_FAILED) {
    set_error("pdgpu_serve_release: job not finished");
    return PDGPU_ERR_STATE;
  }
  s->pool.put(j->pin, j->pin_cap);
  s->pool.put(j->res, j->res_cap);
  s->jobs.erase(job_id);
  return PDGPU_OK;
}

int pdgpu_serve_get_stats(pdgpu_server *s, pdgpu_serve_stats *out) {
  if (!s || !out) return PDGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  *out = s->stats;
  return PDGPU_OK;
}

int pdgpu_serve_destroy(pdgpu_server *s) {
  if (!s) return PDGPU_OK;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
    s->cv_work.notify_one();
  }
  if (s->worker.joinable()) s->worker.join();
  if (s->trace) s->trace_print();
  cudaSetDevice(s->device);
  for (cudaStream_t st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto &kv : s->jobs) {
    s->pool.put(kv.second->pin, kv.second->pin_cap);
    s->pool.put(kv.second->res, kv.second->res_cap);
  }
  delete s;
  return PDGPU_OK;
}

}  // extern "C"
