// Handles behind the C ABI: a system, a batch of systems, or a served job.
// Shared by the ABI (api.cu) and the request loop (serve.cu).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "internal.cuh"

namespace pdgpu {
const char *last_error_cstr();
// load the allocation-free list build's static scratch on the current
// device and look up its address (noalloc.cu)
int noalloc_prepare_current_device();
void launch_md_step_impl(const PackView &v, cudaStream_t st, const MDCoef &c, const double *normals,
                         const int *step_dev, const unsigned char *is_h, const unsigned long long *seeds,
                         double *frames = nullptr, int frame_every = 0, int frame_cap = 0);
// one MD step of every atom fused with the step's energy record (the
// integrator's work done by the energy reduction's blocks; step_dev needed)
void launch_md_step_energy(const PackView &v, cudaStream_t st, const MDCoef &c, const unsigned char *is_h,
                           const unsigned long long *seeds, int mode, double *hist, int *step_dev);
void launch_pair_counts(const PackView &v, cudaStream_t st, unsigned long long *out);
void launch_ke_from_velocities(const PackView &v, cudaStream_t st);
void launch_vel_init_impl(const PackView &v, cudaStream_t st, double temp, const unsigned long long *seeds);
void launch_min_step(const PackView &v, cudaStream_t st, void *ms, int algorithm, double slope_kcal,
                     double strict_kcal, double step_size, int nsteps);
void launch_min_finish(const PackView &v, cudaStream_t st);
// where the LCPO term reads each system's WorkSpace::Step inside a
// minimisation: the step being evaluated, or (last) the last step taken
StepSrc min_step_src(const void *ms, bool last);
int min_state_last(const void *host_buf, int s);
// Monte Carlo (moves.cu): per-system Metropolis state
size_t mc_state_size();
void launch_mc_accept(const PackView &v, cudaStream_t st, void *m, int step, double inv_kT,
                      const unsigned long long *keys, int keep_lowest);
void launch_mc_restore(const PackView &v, cudaStream_t st);
void mc_state_read(const void *buf, int s, int *accepted, int *done, double *lowest_kcal, int *low_step);
size_t min_state_size();
void min_state_init(void *host_buf, int n);
void min_state_read(const void *host_buf, int s, int *taken, int *nan, double *mult);
}  // namespace pdgpu

// A handle: one system (a WorkSpace), or a batch of many packed into one
// device Pack.  `host` is the first member; a batch shares its members'
// host data with the systems it was made from.  The device side (`pack` and
// the small buffers) is created on first use and lives on stream `st`;
// every allocation is stream-ordered so that creating and dropping handles
// never synchronises the device.
struct SysEntry {
  std::shared_ptr<pdgpu::SystemHost> host;
  std::vector<std::shared_ptr<pdgpu::SystemHost>> members;
  std::unique_ptr<pdgpu::Pack> pack;
  cudaStream_t st = nullptr;
  unsigned long long *seeds = nullptr;  // [S] RNG keys
  bool custom_seeds = false;
  // the keys hold base + s from the last default upload (skip re-uploading)
  bool seeds_default = false;
  unsigned long long seeds_base = 0;
  int nsys() const { return (int)members.size(); }
  std::vector<const pdgpu::SystemHost *> member_ptrs() const {
    std::vector<const pdgpu::SystemHost *> m;
    for (auto &h : members) m.push_back(h.get());
    return m;
  }
  int *step_dev = nullptr;
  int ws_step = 0;  // WorkSpace::Step outside the protocols (pdgpu_set_step; a protocol leaves its last step)
  double *hist = nullptr;
  int hist_cap = 0;
  // trajectory snapshots (pdgpu_md_set_trajectory): a device ring written by
  // the integrator, mirrored into a page-locked host ring on the pack's
  // second stream after each list period
  int traj_every = 0, traj_dev_cap = 0, traj_host_cap = 0;
  double *traj_dev = nullptr;
  double *traj_host = nullptr;
  std::vector<long long> traj_step;   // [traj_host_cap] step of each host slot
  long long traj_copied = 0, traj_read = 0;  // frames copied to the host ring / handed out
  cudaEvent_t traj_ev = nullptr;      // the last copy
  bool traj_pending = false;
  void free_trajectory() {
    if (traj_host) cudaFreeHost(traj_host);
    if (traj_ev) cudaEventDestroy(traj_ev);
    traj_host = nullptr;
    traj_ev = nullptr;
    traj_dev = nullptr;  // an `extra` allocation, freed with the entry
    traj_every = traj_dev_cap = traj_host_cap = 0;
    traj_step.clear();
    traj_copied = traj_read = 0;
    traj_pending = false;
  }
  void *min_state = nullptr;
  void *mc_state = nullptr;
  std::vector<void *> extra;
  // page-locked: an MD run's flag read-back and step-counter upload
  // ([F_COUNT] flags, then 3 ints); pdgpu_md_run_io's energies
  int *pin_flags = nullptr;
  double *pin_ene = nullptr;
  double *io_stage = nullptr;  // [6N] device staging of pdgpu_md_run_io's state (an `extra` allocation)
  // cached MD block graph (the request loop's job graph)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::string gkey;
  long long gnodes = 0;
  // MD step-block graphs of pdgpu_md_run, keyed by everything baked into
  // them (block length, whether the block starts with a list rebuild,
  // buffers, integrator settings).  A run that starts inside a list period,
  // or ends inside one, replays a graph for its partial head or tail block
  // as well as the whole-period graph; the few most recent stay cached.
  struct GraphSlot {
    std::string key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;
    long long used = 0;
  };
  static constexpr int kGraphSlots = 4;
  std::vector<GraphSlot> gslots;
  long long gclock = 0;
  long long graph_replays = 0;  // step-block graph launches (pdgpu_graph_replays)
  void drop_slot(GraphSlot &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = GraphSlot();
  }
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    gexec = nullptr;
    graph = nullptr;
    gkey.clear();
    for (auto &g : gslots) drop_slot(g);
    gslots.clear();
  }
  void free_device() {
    drop_graph();
    if (traj_pending && pack) cudaStreamSynchronize(pack->side);
    free_trajectory();
    if (pin_flags || pin_ene) cudaStreamSynchronize(st);  // no copy in flight into them
    if (pin_flags) cudaFreeHost(pin_flags);
    if (pin_ene) cudaFreeHost(pin_ene);
    pin_flags = nullptr;
    pin_ene = nullptr;
    io_stage = nullptr;
    for (void *p : extra) cudaFreeAsync(p, st);
    extra.clear();
    seeds = nullptr;
    step_dev = nullptr;
    hist = nullptr;
    hist_cap = 0;
    min_state = nullptr;
    mc_state = nullptr;
    pack.reset();
  }
  ~SysEntry() { free_device(); }
};

// stream-ordered, zero-filled allocation owned by the entry
template <typename T>
static inline cudaError_t xalloc(SysEntry *e, T **p, size_t n) {
  size_t bytes = sizeof(T) * (n ? n : 1);
  cudaError_t r = cudaMallocAsync((void **)p, bytes, e->st);
  if (r == cudaSuccess) {
    e->extra.push_back(*p);
    r = cudaMemsetAsync(*p, 0, bytes, e->st);
  }
  return r;
}

namespace pdgpu {
// Device side of a handle: the pack of its members, the RNG keys and the
// step counters, enqueued on e->st (with `sync`, waited for).
int entry_materialize(int device, SysEntry *e, bool sync = true);
bool has_bonded(const Pack &P);
// Forcefield::calcForces for {FF_Bonded, FF_GeneralizedBorn_Still} and the
// LCPO term where the handle has it: zero, Born radii, bonded, fused pair,
// chain rule, surface term; one energy reduction if reduce.  `step` is
// where the surface term reads WorkSpace::Step (default: e->ws_step).
void calc_forces_enqueue(cudaStream_t st, SysEntry *e, bool reduce);
// (coop: -1 = the pack's single-evaluation launch form, else 0/1)
void calc_forces_enqueue(cudaStream_t st, SysEntry *e, bool reduce, StepSrc step, int ebuf = 0, int coop = -1);
// one MD step: forces, integrator, energy record (+ step counter advance);
// q = the step's index in its block (its energy buffer is q & 1 on tiles)
void md_step_enqueue(cudaStream_t st, SysEntry *e, const MDCoef &k, int q);
void md_steps_end(cudaStream_t st, SysEntry *e);
MDCoef md_coef(const pdgpu_md_params *p, int step, int steps);
// grow a pack's list buffer to hold `total` entries (stream-ordered)
int nlist_reserve(Pack &P, long long total, cudaStream_t st);
int validate_md(const pdgpu_md_params *p);
}  // namespace pdgpu
