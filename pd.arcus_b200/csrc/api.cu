// C ABI of libpdgpu (declared in include/pdgpu.h) and the protocol runners.
#include <algorithm>
#include <functional>
#include <limits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>

#include "entry.cuh"

using namespace pdgpu;

struct pdgpu_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  std::map<int, std::unique_ptr<SysEntry>> sys;
  int next_id = 1;
  double last_ms = 0.0;
};

#define CHECK_CTX(c)                        \
  do {                                      \
    if (!(c)) {                             \
      set_error("null context");            \
      return PDGPU_ERR_ARG;                 \
    }                                       \
    cudaSetDevice((c)->device);             \
  } while (0)

// Look a handle up; with `device` its device side is created on first use.
static int get_sys(pdgpu_ctx *c, int id, bool device, SysEntry **out) {
  auto it = c->sys.find(id);
  if (it == c->sys.end()) {
    set_error("unknown system id " + std::to_string(id));
    return PDGPU_ERR_ARG;
  }
  SysEntry *e = it->second.get();
  if (device && !e->pack) {
    int r = entry_materialize(c->device, e);
    if (r) {
      e->free_device();
      return r;
    }
  }
  *out = e;
  return PDGPU_OK;
}
#define GET_SYS(e, c, id)                  \
  SysEntry *e = nullptr;                   \
  do {                                     \
    int r_ = get_sys((c), (id), true, &e); \
    if (r_) return r_;                     \
  } while (0)
#define GET_SYS_HOST(e, c, id)              \
  SysEntry *e = nullptr;                    \
  do {                                      \
    int r_ = get_sys((c), (id), false, &e); \
    if (r_) return r_;                      \
  } while (0)


static int sync_check(pdgpu_ctx *c, const char *what) {
  cudaError_t e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return cuda_fail(e, what);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  return PDGPU_OK;
}

// After an evaluation on the tile layout: a grid barrier of the evaluation
// kernel that ran out of time (F_BARRIER) is reported, and its counters are
// cleared so the next evaluation starts clean.
static int barrier_check(pdgpu_ctx *c, pdgpu::Pack &P, const int *flags_host = nullptr) {
  using namespace pdgpu;
  int f = 0;
  if (flags_host) {
    f = flags_host[F_BARRIER];
  } else if (P.v.tile_mode) {
    PDGPU_CUDA(cudaMemcpyAsync(&f, P.v.flags + F_BARRIER, sizeof f, cudaMemcpyDeviceToHost, c->st));
    int r = sync_check(c, "evaluation flags");
    if (r) return r;
  }
  if (!f) return PDGPU_OK;
  cudaMemsetAsync(P.v.flags + F_BARRIER, 0, sizeof(int), c->st);
  if (P.v.tile_count) cudaMemsetAsync(P.v.tile_count + 2, 0, 2 * sizeof(int), c->st);
  cudaStreamSynchronize(c->st);
  set_error("the evaluation kernel's grid barrier timed out (blocks not co-resident); "
            "set PDGPU_FUSED=0 to run the three passes as separate launches");
  return PDGPU_ERR_CUDA;
}

namespace pdgpu {
int entry_materialize(int device, SysEntry *e, bool sync) {
  std::string err;
  Pack *p = pack_create(device, e->st, e->member_ptrs(), &err, sync);
  if (!p) {
    set_error(err);
    return PDGPU_ERR_NOMEM;
  }
  e->pack.reset(p);
  if (xalloc(e, &e->seeds, e->nsys()) != cudaSuccess || xalloc(e, &e->step_dev, 3) != cudaSuccess) {
    set_error("device allocation failed");
    return PDGPU_ERR_NOMEM;
  }
  return PDGPU_OK;
}
}  // namespace pdgpu

extern "C" int pdgpu_get_positions(pdgpu_ctx *c, int32_t sys, double *xyz);
extern "C" int pdgpu_set_positions(pdgpu_ctx *c, int32_t sys, const double *xyz);
extern "C" int pdgpu_get_velocities(pdgpu_ctx *c, int32_t sys, double *v);
extern "C" int pdgpu_set_velocities(pdgpu_ctx *c, int32_t sys, const double *v);

namespace pdgpu {
int ctx_device(pdgpu_ctx *c) { return c->device; }
// the host data of a single system (for the request loop's job templates)
int ctx_system_host(pdgpu_ctx *c, int sys, std::shared_ptr<SystemHost> *out) {
  auto it = c->sys.find(sys);
  if (it == c->sys.end()) {
    set_error("unknown system id " + std::to_string(sys));
    return PDGPU_ERR_ARG;
  }
  if (it->second->nsys() != 1) {
    set_error("a job runs on a single system, not a batch");
    return PDGPU_ERR_ARG;
  }
  *out = it->second->host;
  return PDGPU_OK;
}
}  // namespace pdgpu

// Topology and settings are edited on single systems; a batch takes its
// members' topology, settings and state when it is created.
static int need_single(SysEntry *e, const char *what) {
  if (e->nsys() != 1) {
    set_error(std::string(what) + ": not allowed on a batch (edit the member systems, then re-create the batch)");
    return PDGPU_ERR_STATE;
  }
  return PDGPU_OK;
}

// Re-create a handle's pack after its host topology changed (re-setup),
// keeping positions and velocities.
static int rebuild_pack(pdgpu_ctx *c, SysEntry *e, int sys) {
  if (!e->pack) return PDGPU_OK;  // built from the host data on first use
  int n = e->pack->v.n_atoms;
  std::vector<double> x(3 * (size_t)n), vv(3 * (size_t)n);
  int r = pdgpu_get_positions(c, sys, x.data());
  if (r) return r;
  r = pdgpu_get_velocities(c, sys, vv.data());
  if (r) return r;
  std::string err;
  Pack *p = pack_create(c->device, e->st, e->member_ptrs(), &err);
  if (!p) {
    set_error(err);
    return PDGPU_ERR_NOMEM;
  }
  e->drop_graph();
  e->pack.reset(p);
  r = pdgpu_set_positions(c, sys, x.data());
  if (r) return r;
  return pdgpu_set_velocities(c, sys, vv.data());
}

extern "C" {

const char *pdgpu_last_error(void) { return last_error_cstr(); }

void pdgpu_ff_params_default(pdgpu_ff_params *p) {
  memset(p, 0, sizeof *p);
  // FF_NonBonded::settodefault (nonbonded.cpp:968-1004), then the
  // FF_GeneralizedBorn_Still constructor overrides (gbff.cpp:17-38)
  p->Cutoff = 15;
  p->InnerCutoff = 12;
  p->VdwCutoff = 15;
  p->VdwInnerCutoff = 12;
  p->Vdw14Scaling = 1.0;
  p->Elec14Scaling = 1.0;
  p->Dielectric = 1.0;
  p->DDDielectricAlpha = 1.0;
  p->DielectricSolute = 1.0;
  p->DielectricSolvent = 80.0;
  p->GbsaStillCutoff = 10;
  p->ExpApproxThreshold = -4.0;
  p->DielectricOffset = -0.090;
  p->BornRadiusOffset = 0.0;
  p->P1 = 0.073;
  p->P2 = 0.921;
  p->P3 = 6.211;
  p->P4 = 15.236;
  p->P5 = 1.254;
  p->Padding = 0.5;
  p->FastMode = 1;
  p->EnergySwitch = 1;
  p->ForceSwitch = 0;
  p->DDDielectric = 0;
  p->DoVdw = 1;
  p->DoElec = 1;
  p->VdwCor = 0;
}

void pdgpu_md_params_default(pdgpu_md_params *p) {
  memset(p, 0, sizeof *p);
  // MolecularDynamics::settodefault (md.cpp:39-70)
  p->Integrator = PDGPU_INTEGRATOR_BEEMAN;
  p->UpdateNList = 10;
  p->LangevinOnHydrogens = 1;
  p->UseGraph = 1;
  p->Timestep = 1e-15;
  p->FricCoeff = 10e12;
  p->TargetTemp = 300;
  p->Seed = 0;
}

void pdgpu_min_params_default(pdgpu_min_params *p) {
  // Minimisation::settodefault (minimise.cpp:34-41); UpdateNList from
  // ProtocolBase (protocolbase.cpp:20)
  p->Algorithm = PDGPU_MIN_CONJUGATE_GRADIENTS;
  p->UpdateNList = 1;
  p->StepSize = 2e5;
  p->SlopeCutoff = -1.0;
  p->Strictness = 0.0;
}

int pdgpu_ctx_create(int device, pdgpu_ctx **out) {
  if (!out) {
    set_error("out is NULL");
    return PDGPU_ERR_ARG;
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count 0"));
    return PDGPU_ERR_NODEVICE;
  }
  if (device < 0 || device >= n) {
    set_error("device index out of range");
    return PDGPU_ERR_ARG;
  }
  PDGPU_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  PDGPU_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_error("libpdgpu is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
              std::to_string(prop.minor));
    return PDGPU_ERR_NODEVICE;
  }
  pdgpu_ctx *c = new pdgpu_ctx();
  c->device = device;
  // keep freed pack memory in the device pool (packs come and go with
  // batches and served jobs); the threshold only stops trimming at syncs
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaStreamCreate");
  }
  // the allocation-free list build's static scratch: loaded now, so a
  // caller that reserves its device memory after creating a context finds
  // the array already in place
  int r = noalloc_prepare_current_device();
  if (r) {
    cudaStreamDestroy(c->st);
    delete c;
    return r;
  }
  *out = c;
  return PDGPU_OK;
}

int pdgpu_ctx_destroy(pdgpu_ctx *c) {
  if (!c) return PDGPU_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  c->sys.clear();
  cudaStreamSynchronize(c->st);
  cudaStreamDestroy(c->st);
  delete c;
  return PDGPU_OK;
}

int pdgpu_ctx_mem_used(pdgpu_ctx *c, int64_t *bytes) {
  CHECK_CTX(c);
  int64_t b = 0;
  for (auto &kv : c->sys)
    if (kv.second->pack) b += kv.second->pack->bytes;
  *bytes = b;
  return PDGPU_OK;
}

// ------------------------------------------------------------ systems
static int validate_params(const pdgpu_ff_params *p) {
  if (!p) return PDGPU_OK;
  if (!(p->Cutoff > 0) || !(p->InnerCutoff >= 0) || !(p->InnerCutoff < p->Cutoff) ||
      !(p->VdwCutoff > 0) || !(p->VdwInnerCutoff < p->VdwCutoff) || !(p->Padding >= 0) ||
      !(p->GbsaStillCutoff > 0) || !(p->DielectricSolute > 0) || !(p->DielectricSolvent > 0) ||
      !(p->Dielectric > 0) || !(p->P5 > 0)) {
    set_error("invalid forcefield settings (cutoffs must satisfy 0 <= Inner < Cutoff, dielectrics > 0)");
    return PDGPU_ERR_ARG;
  }
  return PDGPU_OK;
}

int pdgpu_system_create(pdgpu_ctx *c, int32_t natoms, const double *charge, const double *radius,
                        const double *epsilon, const double *mass, const double *gb_radius,
                        const int32_t *residue, const int32_t *c12p, const int32_t *c12i,
                        const double *c12d, const int32_t *c13p, const int32_t *c13i,
                        const double *c13d, const int32_t *c14p, const int32_t *c14i,
                        const pdgpu_ff_params *params, int32_t *sys_id) {
  CHECK_CTX(c);
  if (natoms <= 0 || natoms >= (1 << 24) || !charge || !radius || !epsilon || !mass || !gb_radius ||
      !residue || !c12p || !c13p || !c14p || !sys_id) {
    set_error("pdgpu_system_create: bad arguments (natoms must be in [1, 2^24), arrays non-NULL)");
    return PDGPU_ERR_ARG;
  }
  int r = validate_params(params);
  if (r) return r;
  auto e = std::make_unique<SysEntry>();
  e->host = std::make_shared<SystemHost>();
  e->members.push_back(e->host);
  SystemHost &h = *e->host;
  h.natoms = natoms;
  if (params)
    h.params = *params;
  else
    pdgpu_ff_params_default(&h.params);
  h.charge.assign(charge, charge + natoms);
  h.radius.assign(radius, radius + natoms);
  h.epsilon.assign(epsilon, epsilon + natoms);
  h.mass.assign(mass, mass + natoms);
  h.gbR.assign(gb_radius, gb_radius + natoms);
  h.residue.assign(residue, residue + natoms);
  for (int i = 0; i < natoms; i++)
    if (!(mass[i] > 0)) {
      set_error("pdgpu_system_create: masses must be positive");
      return PDGPU_ERR_ARG;
    }
  auto csr = [&](const int32_t *p, const int32_t *idx, std::vector<int> &P, std::vector<int> &I) -> bool {
    P.assign(p, p + natoms + 1);
    if (P[0] != 0) return false;
    for (int i = 0; i < natoms; i++)
      if (P[i + 1] < P[i]) return false;
    if (P[natoms] > 0 && !idx) return false;
    I.assign(idx, idx + P[natoms]);
    return true;
  };
  if (!csr(c12p, c12i, h.c12p, h.c12i) || !csr(c13p, c13i, h.c13p, h.c13i) ||
      !csr(c14p, c14i, h.c14p, h.c14i)) {
    set_error("pdgpu_system_create: malformed covalent CSR lists");
    return PDGPU_ERR_ARG;
  }
  if ((h.c12p[natoms] && !c12d) || (h.c13p[natoms] && !c13d)) {
    set_error("pdgpu_system_create: 1-2 and 1-3 equilibrium distances required");
    return PDGPU_ERR_ARG;
  }
  if (h.c12p[natoms]) h.c12d.assign(c12d, c12d + h.c12p[natoms]);
  if (h.c13p[natoms]) h.c13d.assign(c13d, c13d + h.c13p[natoms]);
  std::string err;
  r = host_bondorder(h, &err);
  if (r) {
    set_error(err);
    return r;
  }
  host_gb_fixed_terms(h);
  e->st = c->st;  // the device side is created on first use
  int id = c->next_id++;
  c->sys[id] = std::move(e);
  *sys_id = id;
  return PDGPU_OK;
}

int pdgpu_batch_create(pdgpu_ctx *c, const int32_t *sys_ids, int32_t nsys, int32_t *batch_id) {
  CHECK_CTX(c);
  if (!sys_ids || nsys <= 0 || !batch_id) {
    set_error("pdgpu_batch_create: bad arguments");
    return PDGPU_ERR_ARG;
  }
  auto e = std::make_unique<SysEntry>();
  long long total = 0;
  std::vector<SysEntry *> src;
  for (int k = 0; k < nsys; k++) {
    GET_SYS(m, c, sys_ids[k]);
    if (m->nsys() != 1) {
      set_error("pdgpu_batch_create: members must be single systems, not batches");
      return PDGPU_ERR_ARG;
    }
    e->members.push_back(m->host);
    src.push_back(m);
    total += m->host->natoms;
  }
  if (total >= (1 << 24)) {
    set_error("pdgpu_batch_create: a batch holds fewer than 2^24 atoms");
    return PDGPU_ERR_ARG;
  }
  e->host = e->members[0];
  e->st = c->st;
  int r = entry_materialize(c->device, e.get());
  if (r) return r;
  // the batch starts from its members' current positions, velocities and
  // RNG keys (device to device, no host round trip)
  Pack &B = *e->pack;
  std::vector<unsigned long long> keys(nsys);
  for (int k = 0; k < nsys; k++) {
    const PackView &s = src[k]->pack->v;
    size_t o = B.atom_off[k], n = s.n_atoms;
    double *dst[6] = {B.v.x, B.v.y, B.v.z, B.v.vx, B.v.vy, B.v.vz};
    const double *from[6] = {s.x, s.y, s.z, s.vx, s.vy, s.vz};
    for (int q = 0; q < 6; q++)
      PDGPU_CUDA(cudaMemcpyAsync(dst[q] + o, from[q], sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    PDGPU_CUDA(cudaMemcpyAsync(&keys[k], src[k]->seeds, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
  }
  r = sync_check(c, "batch_create");
  if (r) return r;
  PDGPU_CUDA(cudaMemcpyAsync(e->seeds, keys.data(), sizeof(unsigned long long) * nsys, cudaMemcpyHostToDevice,
                             c->st));
  e->custom_seeds = false;
  e->seeds_default = false;
  launch_pack_positions(B.v, c->st);
  r = sync_check(c, "batch_create");
  if (r) return r;
  int id = c->next_id++;
  c->sys[id] = std::move(e);
  *batch_id = id;
  return PDGPU_OK;
}

int pdgpu_batch_info(pdgpu_ctx *c, int32_t batch, int32_t *nsys, int32_t *atom_offset) {
  CHECK_CTX(c);
  GET_SYS(e, c, batch);
  if (nsys) *nsys = e->nsys();
  if (atom_offset)
    for (int s = 0; s <= e->nsys(); s++) atom_offset[s] = e->pack->atom_off[s];
  return PDGPU_OK;
}

int pdgpu_set_seeds(pdgpu_ctx *c, int32_t sys, const uint64_t *seeds) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  e->seeds_default = false;
  if (!seeds) {
    e->custom_seeds = false;
    return PDGPU_OK;
  }
  PDGPU_CUDA(cudaMemcpyAsync(e->seeds, seeds, sizeof(unsigned long long) * e->nsys(), cudaMemcpyHostToDevice,
                             c->st));
  e->custom_seeds = true;
  return sync_check(c, "set_seeds");
}

int pdgpu_system_destroy(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  cudaStreamSynchronize(c->st);
  if (!c->sys.erase(sys)) {
    set_error("unknown system id");
    return PDGPU_ERR_ARG;
  }
  return PDGPU_OK;
}

int pdgpu_system_set_params(pdgpu_ctx *c, int32_t sys, const pdgpu_ff_params *params) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  int r = validate_params(params);
  if (r) return r;
  if (!params) {
    set_error("params is NULL");
    return PDGPU_ERR_ARG;
  }
  r = need_single(e, "pdgpu_system_set_params");
  if (r) return r;
  SystemHost &h = *e->host;
  bool fixed_changed = params->P1 != h.params.P1 || params->P2 != h.params.P2 || params->P3 != h.params.P3 ||
                       params->P4 != h.params.P4 || params->DielectricOffset != h.params.DielectricOffset;
  h.params = *params;
  if (fixed_changed) {
    // the Still fixed terms depend on P1-P4: rebuild the pack (re-setup)
    host_gb_fixed_terms(h);
    return rebuild_pack(c, e, sys);
  }
  if (!e->pack) return PDGPU_OK;
  e->drop_graph();
  Pack &P = *e->pack;
  pack_set_params(&P, 0, *params);
  PDGPU_CUDA(cudaMemcpyAsync((void *)P.v.sp, P.sp.data(), sizeof(SysParams), cudaMemcpyHostToDevice, c->st));
  P.have_list = false;  // the list radius may have changed
  P.csr_stale = false;
  return sync_check(c, "set_params");
}

int pdgpu_system_set_bonded(pdgpu_ctx *c, int32_t sys, int32_t nb, const int32_t *bij, const double *blk,
                            int32_t na, const int32_t *aiaj, const double *akt, int32_t nt,
                            const int32_t *tidx, const int32_t *tterms, const double *tpar, int32_t ni,
                            const int32_t *iidx, const int32_t *iterms, const double *ipar) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  if (nb < 0 || na < 0 || nt < 0 || ni < 0 || (nb && (!bij || !blk)) || (na && (!aiaj || !akt)) ||
      (nt && (!tidx || !tterms || !tpar)) || (ni && (!iidx || !iterms || !ipar))) {
    set_error("pdgpu_system_set_bonded: bad arguments");
    return PDGPU_ERR_ARG;
  }
  int r = need_single(e, "pdgpu_system_set_bonded");
  if (r) return r;
  SystemHost &h = *e->host;
  int n = h.natoms;
  auto inrange = [&](const int32_t *a, long cnt) {
    for (long k = 0; k < cnt; k++)
      if (a[k] < 0 || a[k] >= n) return false;
    return true;
  };
  if (!inrange(bij, 2L * nb) || !inrange(aiaj, 3L * na) || !inrange(tidx, 4L * nt) || !inrange(iidx, 4L * ni)) {
    set_error("pdgpu_system_set_bonded: atom index out of range");
    return PDGPU_ERR_ARG;
  }
  for (int k = 0; k < nt; k++)
    if (tterms[k] < 0 || tterms[k] > 4) {
      set_error("pdgpu_system_set_bonded: torsion term count must be 0..4");
      return PDGPU_ERR_ARG;
    }
  for (int k = 0; k < ni; k++)
    if (iterms[k] < 0 || iterms[k] > 4) {
      set_error("pdgpu_system_set_bonded: improper term count must be 0..4");
      return PDGPU_ERR_ARG;
    }
  h.nb = nb;
  h.na = na;
  h.nt = nt;
  h.ni = ni;
  h.bij.assign(bij, bij + 2 * nb);
  h.blk.assign(blk, blk + 2 * nb);
  h.aiaj.assign(aiaj, aiaj + 3 * na);
  h.akt.assign(akt, akt + 2 * na);
  h.tidx.assign(tidx, tidx + 4 * nt);
  h.tidx.insert(h.tidx.end(), iidx, iidx + 4 * ni);
  h.tterms.assign(tterms, tterms + nt);
  h.tterms.insert(h.tterms.end(), iterms, iterms + ni);
  h.tpar.assign(tpar, tpar + 12 * nt);
  h.tpar.insert(h.tpar.end(), ipar, ipar + 12 * ni);
  dihedral_sets(h);
  // rebuild the pack with the bonded terms, keeping the state
  return rebuild_pack(c, e, sys);
}

int pdgpu_system_set_hydrogens(pdgpu_ctx *c, int32_t sys, const int8_t *is_h) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  if (!is_h) {
    set_error("is_h is NULL");
    return PDGPU_ERR_ARG;
  }
  int r = need_single(e, "pdgpu_system_set_hydrogens");
  if (r) return r;
  e->host->is_h.assign(is_h, is_h + e->host->natoms);
  if (!e->pack) return PDGPU_OK;
  PDGPU_CUDA(cudaMemcpyAsync(e->pack->is_h, is_h, e->host->natoms, cudaMemcpyHostToDevice, c->st));
  return sync_check(c, "set_hydrogens");
}

// FF_SASA_LCPO::setup's per-atom parameters (lcpo.cpp:16-111), formed by
// the caller; update_sasa <= 0 removes the term.
int pdgpu_sasa_lcpo_set(pdgpu_ctx *c, int32_t sys, const double *radius, const double *p1234,
                        const double *sigma, const uint8_t *use, int32_t update_sasa) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  int r = need_single(e, "pdgpu_sasa_lcpo_set");
  if (r) return r;
  SystemHost &h = *e->host;
  const size_t n = (size_t)h.natoms;
  if (update_sasa > 0) {
    if (!radius || !p1234 || !sigma || !use) {
      set_error("pdgpu_sasa_lcpo_set: NULL parameter array");
      return PDGPU_ERR_ARG;
    }
    for (size_t i = 0; i < n; i++)
      if (use[i] && !(radius[i] > 0.0)) {
        set_error("pdgpu_sasa_lcpo_set: an atom in use has a radius <= 0");
        return PDGPU_ERR_ARG;
      }
    h.lcpo_r.assign(radius, radius + n);
    h.lcpo_p.assign(p1234, p1234 + 4 * n);
    h.lcpo_sigma.assign(sigma, sigma + n);
    h.lcpo_use.assign(use, use + n);
    h.lcpo_update = update_sasa;
  } else {
    h.lcpo_update = 0;
    h.lcpo_r.clear();
    h.lcpo_p.clear();
    h.lcpo_sigma.clear();
    h.lcpo_use.clear();
  }
  if (!e->pack) return PDGPU_OK;
  e->drop_graph();
  // the term reads the list rows: the calls that run it build them first
  // when the last rebuild made only the tiles
  return pack_upload_lcpo(e->pack.get(), e->member_ptrs());
}

int pdgpu_set_step(pdgpu_ctx *c, int32_t sys, int32_t step) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  if (step < 0) {
    set_error("pdgpu_set_step: step < 0");
    return PDGPU_ERR_ARG;
  }
  e->ws_step = step;
  return PDGPU_OK;
}

int pdgpu_get_step(pdgpu_ctx *c, int32_t sys, int32_t *step) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  if (!step) {
    set_error("step is NULL");
    return PDGPU_ERR_ARG;
  }
  *step = e->ws_step;
  return PDGPU_OK;
}

int pdgpu_system_set_torsions(pdgpu_ctx *c, int32_t sys, int32_t nrot, const int32_t *axis) {
  CHECK_CTX(c);
  GET_SYS_HOST(e, c, sys);
  int r = need_single(e, "pdgpu_system_set_torsions");
  if (r) return r;
  SystemHost &h = *e->host;
  const int n = h.natoms;
  if (nrot < 0 || (nrot && !axis)) {
    set_error("pdgpu_system_set_torsions: bad arguments");
    return PDGPU_ERR_ARG;
  }
  // The atoms each rotation moves: MoleculeBase::rotateBond(bi, bj)
  // (system/molecule.cpp:1099-1175) walks the covalent graph from bj and
  // never steps onto bi.  Consecutive rotations must nest (each moves a
  // subset of what the previous one moves) or start a new nest on atoms no
  // earlier rotation moves; each atom records the last rotation moving it.
  std::vector<int> last(n, -1), queue;
  std::vector<unsigned char> start(nrot, 0), mark(n, 0);
  for (int k = 0; k < nrot; k++) {
    int bi = axis[2 * k], bj = axis[2 * k + 1];
    if (bi < 0 || bi >= n || bj < 0 || bj >= n) {
      set_error("pdgpu_system_set_torsions: axis atom out of range");
      return PDGPU_ERR_ARG;
    }
    bool bonded = false;
    for (int q = h.c12p[bi]; q < h.c12p[bi + 1]; q++) bonded |= h.c12i[q] == bj;
    if (!bonded) {
      set_error("pdgpu_system_set_torsions: rotation " + std::to_string(k) + " is not about a covalent bond");
      return PDGPU_ERR_ARG;
    }
    queue.assign(1, bj);
    std::fill(mark.begin(), mark.end(), 0);
    mark[bi] = mark[bj] = 1;
    for (size_t q = 0; q < queue.size(); q++) {
      int a = queue[q];
      for (int t = h.c12p[a]; t < h.c12p[a + 1]; t++) {
        int nb = h.c12i[t];
        if (!mark[nb]) {
          mark[nb] = 1;
          queue.push_back(nb);
        }
      }
    }
    bool inner = true, fresh = true;
    for (int a : queue) {
      inner &= k > 0 && last[a] == k - 1;
      fresh &= last[a] == -1;
    }
    if (!inner && !fresh) {
      set_error("pdgpu_system_set_torsions: rotation " + std::to_string(k) +
                " neither nests inside the previous one nor moves only atoms no earlier rotation moves");
      return PDGPU_ERR_ARG;
    }
    start[k] = !inner;
    for (int a : queue) last[a] = k;
  }
  h.rot_axis.assign(axis, axis + 2 * nrot);
  h.rot_start = start;
  if (nrot)
    h.rot_last = last;
  else
    h.rot_last.clear();
  return rebuild_pack(c, e, sys);
}

int pdgpu_save_base_positions(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  PackView &v = e->pack->v;
  size_t n = v.n_atoms;
  PDGPU_CUDA(cudaMemcpyAsync(v.bx, v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.by, v.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.bz, v.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  return sync_check(c, "save_base_positions");
}

int pdgpu_perturb_torsions(pdgpu_ctx *c, int32_t sys, double sigma, uint64_t trial, const double *angles) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (!(sigma >= 0)) {
    set_error("pdgpu_perturb_torsions: sigma must be >= 0");
    return PDGPU_ERR_ARG;
  }
  double *ang = nullptr;
  size_t R = P.rot_total;
  if (angles && R) {
    PDGPU_CUDA(cudaMallocAsync((void **)&ang, sizeof(double) * R, c->st));
    PDGPU_CUDA(cudaMemcpyAsync(ang, angles, sizeof(double) * R, cudaMemcpyHostToDevice, c->st));
  }
  launch_torsion_moves(P.v, c->st, sigma, trial, e->seeds, ang);
  if (ang) cudaFreeAsync(ang, c->st);
  return sync_check(c, "perturb_torsions");
}

// ------------------------------------------------------------ state
// The caller's interleaved [n][3] buffer moves as one block to or from a
// device staging array; the device reshuffles it (a page-locked caller
// buffer is copied by DMA straight from or into its own memory).
static int copy_soa_in(pdgpu_ctx *c, Pack &P, const double *xyz, double *X, double *Y, double *Z) {
  const int n = P.v.n_atoms;
  int r = pack_ensure_stage(&P);
  if (r) return r;
  PDGPU_CUDA(cudaMemcpyAsync(P.stage, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, c->st));
  launch_aos_to_soa(P.stage, X, Y, Z, n, c->st);
  return PDGPU_OK;
}
static int copy_soa_out(pdgpu_ctx *c, Pack &P, double *xyz, const double *X, const double *Y,
                        const double *Z) {
  const int n = P.v.n_atoms;
  int r = pack_ensure_stage(&P);
  if (r) return r;
  launch_soa_to_aos(P.stage, X, Y, Z, n, c->st);
  PDGPU_CUDA(cudaMemcpyAsync(xyz, P.stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c->st));
  return sync_check(c, "copy out");
}

int pdgpu_set_positions(pdgpu_ctx *c, int32_t sys, const double *xyz) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!xyz) {
    set_error("xyz is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  int r = copy_soa_in(c, P, xyz, P.v.x, P.v.y, P.v.z);
  if (r) return r;
  launch_pack_positions(P.v, c->st);
  return sync_check(c, "set_positions");
}
int pdgpu_get_positions(pdgpu_ctx *c, int32_t sys, double *xyz) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!xyz) {
    set_error("xyz is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  return copy_soa_out(c, P, xyz, P.v.x, P.v.y, P.v.z);
}
int pdgpu_set_velocities(pdgpu_ctx *c, int32_t sys, const double *v) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!v) {
    set_error("v is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  int r = copy_soa_in(c, P, v, P.v.vx, P.v.vy, P.v.vz);
  if (r) return r;
  return sync_check(c, "set_velocities");
}
int pdgpu_get_velocities(pdgpu_ctx *c, int32_t sys, double *v) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!v) {
    set_error("v is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  return copy_soa_out(c, P, v, P.v.vx, P.v.vy, P.v.vz);
}

int pdgpu_get_forces(pdgpu_ctx *c, int32_t sys, double *f) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!f) {
    set_error("f is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  int n = P.v.n_atoms;
  std::vector<long long> a(3 * (size_t)n), h(3 * (size_t)n);
  std::vector<double> g(3 * (size_t)n);
  const long long *fs[3] = {P.v.fx, P.v.fy, P.v.fz};
  const double *gs[3] = {P.v.gx, P.v.gy, P.v.gz};
  const long long *hs[3] = {P.v.hx, P.v.hy, P.v.hz};
  for (int k = 0; k < 3; k++) {
    size_t o = (size_t)k * n;
    PDGPU_CUDA(cudaMemcpyAsync(a.data() + o, fs[k], sizeof(long long) * n, cudaMemcpyDeviceToHost, c->st));
    PDGPU_CUDA(cudaMemcpyAsync(g.data() + o, gs[k], sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    PDGPU_CUDA(cudaMemcpyAsync(h.data() + o, hs[k], sizeof(long long) * n, cudaMemcpyDeviceToHost, c->st));
  }
  int r = sync_check(c, "get_forces");
  if (r) return r;
  // the integrator's sum: fixed-point scattered terms, FP64 pair forces,
  // fixed-point j side of the tile passes
  double s = consts().N_per_kcalmolA;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      size_t q = (size_t)k * n + i;
      f[3 * i + k] = ((double)a[q] * kInvForceScale + g[q] + (double)h[q] * kInvJScale) * s;
    }
  return PDGPU_OK;
}

int pdgpu_get_born_radii(pdgpu_ctx *c, int32_t sys, double *born) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!born) {
    set_error("born is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  PDGPU_CUDA(cudaMemcpyAsync(born, P.v.born_d, sizeof(double) * P.v.n_atoms, cudaMemcpyDeviceToHost, c->st));
  return sync_check(c, "get_born_radii");
}

int pdgpu_get_atom_epot(pdgpu_ctx *c, int32_t sys, double *epot) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!epot) {
    set_error("epot is NULL");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  int n = P.v.n_atoms;
  std::vector<double> ea((size_t)AE_COUNT * n);
  PDGPU_CUDA(cudaMemcpyAsync(ea.data(), P.v.e_atom, sizeof(double) * ea.size(), cudaMemcpyDeviceToHost, c->st));
  if (P.last_ebuf)  // the last evaluation wrote its pair slots to the second buffer
    PDGPU_CUDA(cudaMemcpyAsync(ea.data(), P.v.e_pair_alt, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost,
                               c->st));
  int r = sync_check(c, "get_atom_epot");
  if (r) return r;
  double J = consts().J_per_kcalmol;
  for (int i = 0; i < n; i++)
    epot[i] = (ea[(size_t)AE_VDW * n + i] + ea[(size_t)AE_ELEC * n + i] + ea[(size_t)AE_POL * n + i] +
               ea[(size_t)AE_POL_SELF * n + i]) *
              J;
  return PDGPU_OK;
}

int pdgpu_get_energies(pdgpu_ctx *c, int32_t sys, double *ene, int32_t n) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  const int S = e->nsys();
  if (!ene || n < PDGPU_ENE_COUNT * S) {
    set_error("ene must hold PDGPU_ENE_COUNT values per system");
    return PDGPU_ERR_ARG;
  }
  static_assert(E_COUNT == PDGPU_ENE_COUNT, "energy record layout");
  Pack &P = *e->pack;
  std::vector<double> tmp((size_t)E_COUNT * S);
  PDGPU_CUDA(cudaMemcpyAsync(tmp.data(), P.v.ene, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, c->st));
  int r = sync_check(c, "get_energies");
  if (r) return r;
  double J = consts().J_per_kcalmol;
  for (size_t k = 0; k < tmp.size(); k++) ene[k] = tmp[k] * J;
  return PDGPU_OK;
}

int pdgpu_zero_forces(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  launch_zero(e->pack->v, c->st);
  return sync_check(c, "zero_forces");
}

// ------------------------------------------------------------ kernels
// enqueue a full list rebuild; when `size_check` the host reads the count
// and grows the list buffer first (one synchronisation)
}  // extern "C"
// Grow the list buffer (stream-ordered) to hold `total` entries plus slack.
int pdgpu::nlist_reserve(Pack &P, long long total, cudaStream_t st) {
  PackView &v = P.v;
  if (total <= v.nl_cap) return PDGPU_OK;
  long long cap = total + total / 3 + 4096;
  unsigned *nl = nullptr;
  cudaError_t ce = cudaMallocAsync((void **)&nl, sizeof(unsigned) * cap, st);
  if (ce != cudaSuccess) return cuda_fail(ce, "grow neighbour list");
  auto it = std::find(P.allocs.begin(), P.allocs.end(), (void *)v.nl);
  if (it != P.allocs.end()) {
    cudaFreeAsync(*it, st);
    *it = nl;
  }
  P.bytes += (int64_t)(cap - v.nl_cap) * 4;
  v.nl = nl;
  v.nl_cap = cap;
  return PDGPU_OK;
}
extern "C" {

static int nlist_enqueue(pdgpu_ctx *c, SysEntry *e, bool size_check) {
  Pack &P = *e->pack;
  PackView &v = P.v;
  launch_nlist_count(P, c->st);
  if (size_check) {
    long long total = 0;
    PDGPU_CUDA(cudaMemcpyAsync(&total, v.row_start + v.n_atoms, sizeof total, cudaMemcpyDeviceToHost, c->st));
    int r = sync_check(c, "nlist count");
    if (r) return r;
    r = nlist_reserve(P, total, c->st);
    if (r) return r;
    P.nl_total = total;
    PDGPU_CUDA(cudaMemsetAsync(v.flags + F_NL_OVERFLOW, 0, sizeof(int), c->st));
  }
  launch_nlist_fill(P, c->st);
  P.have_list = true;
  P.csr_stale = false;
  return PDGPU_OK;
}

// A list rebuild for a pack that runs the tile passes makes the tiles
// straight from the positions (no list, no host synchronisation); the list
// itself is built later, only if something reads it, at the positions of
// that rebuild (saved by the search), so it is the list the rebuild would
// have made.  Packs on the row passes, or with a system too large for the
// search, rebuild the list (and from it the tiles).
static bool tile_search_ok(const Pack &P) {
  // (FastMode off needs the list rows for its stand-alone LJ/Coulomb pass)
  return P.v.tile_mode && P.v.tile_meta && P.v.n_sc > 0 && P.v.max_sys_atoms <= kTileSearchMaxAtoms && !P.slow();
}
// the energy-record bits of the pair terms of an evaluation
static int pair_energy_mode(const Pack &P) { return P.slow() ? (EM_PAIR_NB | EM_PAIR_GB_SLOW) : EM_PAIR_GB; }
static void rebuild_enqueue(Pack &P, cudaStream_t st) {
  if (tile_search_ok(P)) {
    launch_tiles_search(P.v, st);
    P.csr_stale = true;
  } else {
    launch_nlist_count(P, st);
    launch_nlist_fill(P, st);
    P.csr_stale = false;
  }
}
// The list (CSR rows), built now at the saved positions when only tiles
// were made since the last list build.
static int need_csr(pdgpu_ctx *c, SysEntry *e) {
  Pack &P = *e->pack;
  if (!P.have_list) {
    set_error("no neighbour list: call pdgpu_nlist_build first (NeighbourList::calcNewList)");
    return PDGPU_ERR_STATE;
  }
  if (!P.csr_stale) return PDGPU_OK;
  PackView &v = P.v;
  double *x = v.x, *y = v.y, *z = v.z;
  const size_t N = (size_t)v.n_atoms;
  v.x = v.xs;
  v.y = v.xs + N;
  v.z = v.xs + 2 * N;
  int r = nlist_enqueue(c, e, true);
  v.x = x;
  v.y = y;
  v.z = z;
  return r;
}
static int need_csr_if(pdgpu_ctx *c, SysEntry *e, bool csr) {
  if (!e->pack->have_list) {
    set_error("no neighbour list: call pdgpu_nlist_build first (NeighbourList::calcNewList)");
    return PDGPU_ERR_STATE;
  }
  return csr ? need_csr(c, e) : PDGPU_OK;
}

int pdgpu_nlist_build(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (P.have_list && tile_search_ok(P)) {
    rebuild_enqueue(P, c->st);
    return sync_check(c, "nlist_build");
  }
  int r = nlist_enqueue(c, e, true);
  if (r) return r;
  return sync_check(c, "nlist_build");
}

int pdgpu_nlist_export(pdgpu_ctx *c, int32_t sys, int32_t shadow, int32_t *ptr, int32_t *data, int64_t cap,
                       int64_t *count) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r0 = need_csr(c, e);
  if (r0) return r0;
  if (!ptr || !count) {
    set_error("ptr/count is NULL");
    return PDGPU_ERR_ARG;
  }
  int n = P.v.n_atoms;
  std::vector<long long> rs(n + 1);
  PDGPU_CUDA(cudaMemcpyAsync(rs.data(), P.v.row_start, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, c->st));
  int r = sync_check(c, "export");
  if (r) return r;
  std::vector<unsigned> raw(rs[n]);
  if (rs[n])
    PDGPU_CUDA(cudaMemcpyAsync(raw.data(), P.v.nl, sizeof(unsigned) * rs[n], cudaMemcpyDeviceToHost, c->st));
  r = sync_check(c, "export");
  if (r) return r;
  int64_t k = 0;
  std::vector<int> row;
  for (int i = 0; i < n; i++) {
    ptr[i] = (int32_t)k;
    row.clear();
    for (long long q = rs[i]; q < rs[i + 1]; q++) {
      int j = (int)(raw[q] >> 3);
      int bo = (int)(raw[q] & 7u);
      if (!shadow && j >= i) continue;
      row.push_back((j & 0x00FFFFFF) | (bo << 24));
    }
    std::sort(row.begin(), row.end(), [](int a, int b) { return (a & 0x00FFFFFF) < (b & 0x00FFFFFF); });
    for (int x : row) {
      if (data && k < cap) data[k] = x;
      k++;
    }
  }
  ptr[n] = (int32_t)k;
  *count = k;
  if (data && k > cap) {
    set_error("export buffer too small");
    return PDGPU_ERR_ARG;
  }
  return PDGPU_OK;
}

static int ensure_tuned(pdgpu_ctx *c, Pack &P);
// What an evaluation reads: the tiles on the tile passes (current after
// any rebuild), the list on the row passes and for the autotuner (which
// times the row passes too).
static int ready_pairs(pdgpu_ctx *c, SysEntry *e) {
  Pack &P = *e->pack;
  int r = need_csr_if(c, e, !P.tuned || !P.v.tile_mode);
  if (r) return r;
  return ensure_tuned(c, P);
}

// Autotuner: lanes per atom (4, 8, 16, 32) of the Born, fused-pair and
// chain-rule kernels, chosen once per pack by timing each candidate on the
// current list with CUDA events.  The timed launches write their forces and
// energies into scratch buffers; the Born radii and chain weights they also
// write are the values the next evaluation computes anyway.
static int ensure_tuned(pdgpu_ctx *c, Pack &P) {
  if (P.tuned || P.v.n_atoms == 0 || !P.have_list) return PDGPU_OK;
  const int N = P.v.n_atoms;
  int re = pack_ensure_tiles(&P);  // the tile layout is timed too
  if (re) return re;
  PackView t = P.v;
  t.tile_mode = 0;
  // scratch for every array the timed launches accumulate into
  double *f = nullptr;
  double *ea = nullptr, *en = nullptr;
  PDGPU_CUDA(cudaMalloc(&f, sizeof(double) * 12 * (size_t)N));
  if (cudaMalloc(&ea, sizeof(double) * AE_COUNT * (size_t)N) != cudaSuccess ||
      cudaMalloc(&en, sizeof(double) * E_COUNT * (size_t)P.v.n_sys) != cudaSuccess) {
    cudaFree(f);
    cudaFree(ea);
    set_error("autotune scratch allocation failed");
    return PDGPU_ERR_NOMEM;
  }
  cudaMemsetAsync(f, 0, sizeof(double) * 12 * (size_t)N, c->st);
  t.gx = f;
  t.gy = f + N;
  t.gz = f + 2 * N;
  t.hx = (long long *)(f + 3 * (size_t)N);
  t.hy = (long long *)(f + 4 * (size_t)N);
  t.hz = (long long *)(f + 5 * (size_t)N);
  t.ej = (long long *)(f + 6 * (size_t)N);
  t.bsum = (long long *)(f + 11 * (size_t)N);
  t.e_atom = ea;
  t.ene = en;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  static const int cand[4] = {4, 8, 16, 32};
  int r = PDGPU_OK;
  float row_total = 0.f;
  for (int kern = 0; kern < 3 && r == PDGPU_OK; kern++) {
    float best = 1e30f;
    int pick = 8;
    for (int q = 0; q < 4; q++) {
      float tot = 0;
      for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(a, c->st);
        if (kern == 0) launch_born_radii_lpa(t, c->st, false, cand[q]);
        if (kern == 1) launch_gb_pair_lpa(t, c->st, cand[q]);
        if (kern == 2) launch_gb_chain_lpa(t, c->st, cand[q]);
        cudaEventRecord(b, c->st);
        r = sync_check(c, "autotune");
        if (r) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) tot += ms;  // the first launch warms the caches
      }
      if (r) break;
      if (tot < best) {
        best = tot;
        pick = cand[q];
      }
    }
    P.v.lpa[kern] = t.lpa[kern] = pick;
    row_total += best;
    // leave valid inputs for the next kernel's timing
    if (kern == 0) launch_born_radii_lpa(t, c->st, false, pick);
    if (kern == 1) launch_gb_pair_lpa(t, c->st, pick);
  }
  // the cluster-pair tile path against the tuned row path (three passes)
  if (r == PDGPU_OK && P.v.n_sc > 0) {
    t.tile_mode = 1;
    // each layout's rebuild comes with every list period: counted at the MD
    // default cadence (one rebuild per 10 evaluations).  The row passes
    // rebuild the list; the tile passes search the tiles from the
    // positions (systems within the search limit), else build the list and
    // the tiles from it.  Every timed rebuild runs at the current positions
    // and remakes what is there.
    const bool search = P.v.max_sys_atoms <= kTileSearchMaxAtoms;
    float build = 0, list = 0;
    for (int rep = 0; rep < 2 && r == PDGPU_OK; rep++) {
      cudaEventRecord(a, c->st);
      launch_nlist_count(P, c->st);
      launch_nlist_fill(P, c->st);  // (on the tile layout also the tiles from it: the same pairs)
      cudaEventRecord(b, c->st);
      r = sync_check(c, "autotune list build");
      cudaEventElapsedTime(&list, a, b);
      cudaEventRecord(a, c->st);
      if (search)
        launch_tiles_search(t, c->st);
      else
        launch_tiles_build(t, c->st);
      cudaEventRecord(b, c->st);
      r = sync_check(c, "autotune tile build");
      cudaEventElapsedTime(&build, a, b);
    }
    if (!search) build += list;
    row_total += 0.1f * 3.f * list;  // the row timings are sums of three repetitions
    float tot = 0.1f * 3.f * build;  // three timed repetitions below
    for (int rep = 0; rep < 4 && r == PDGPU_OK; rep++) {
      cudaEventRecord(a, c->st);
      launch_eval_tiles(t, c->st, 0, P.coop);  // the evaluation as the protocols run it
      cudaEventRecord(b, c->st);
      r = sync_check(c, "autotune tiles");
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0) tot += ms;
    }
    P.v.tile_mode = (r == PDGPU_OK && tot < row_total) ? 1 : 0;
  }
  if (r == PDGPU_OK) r = sync_check(c, "autotune");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(f);
  cudaFree(ea);
  cudaFree(en);
  if (r == PDGPU_OK) P.tuned = true;
  return r;
}

// GB calcForces enqueue (no sync)
static void gb_forces_enqueue(pdgpu_ctx *c, Pack &P) {
  if (P.v.tile_mode) {
    launch_eval_tiles(P.v, c->st, 0, P.coop);
  } else {
    launch_born_radii(P.v, c->st);
    launch_gb_pair(P.v, c->st);
    launch_gb_chain(P.v, c->st);
  }
  // FastMode off: FF_NonBonded::calcForces beside calcBornForces
  // (gbff.cpp:176-177), after the GB passes (they zero what it adds to)
  if (P.slow()) launch_nonbonded(P.v, c->st, P.sp[0].elec_mode);
  launch_energy(P.v, c->st, pair_energy_mode(P));
}

}  // extern "C"
bool pdgpu::has_bonded(const Pack &P) { return P.v.bt.nb + P.v.bt.na + P.v.bt.nt + P.v.bt.ni > 0; }
extern "C" {

int pdgpu_gb_forces(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = ready_pairs(c, e);
  if (r) return r;
  if (P.slow() && (r = need_csr(c, e))) return r;  // the stand-alone LJ/Coulomb pass reads the rows
  gb_forces_enqueue(c, P);
  r = sync_check(c, "gb_forces");
  return r ? r : barrier_check(c, P);
}

int pdgpu_gb_energies(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = need_csr(c, e);
  if (r) return r;
  // calcEnergies: radii, FF_NonBonded::calcEnergies at Dielectric =
  // DielectricSolute (gbff.cpp:44), then calcBornEnergy
  const int S = e->nsys();
  std::vector<SysParams> saved = P.sp;
  for (int s = 0; s < S; s++) {
    pdgpu_ff_params q = e->members[s]->params;
    q.Dielectric = q.DielectricSolute;
    pack_set_params(&P, s, q);
  }
  PDGPU_CUDA(cudaMemcpyAsync((void *)P.v.sp, P.sp.data(), sizeof(SysParams) * S, cudaMemcpyHostToDevice, c->st));
  launch_born_radii(P.v, c->st);
  launch_nonbonded(P.v, c->st, P.sp[0].elec_mode);
  launch_born_energy(P.v, c->st);
  launch_energy(P.v, c->st, EM_PAIR_NB | EM_BORN_ENERGY);
  r = sync_check(c, "gb_energies");
  P.sp = saved;
  PDGPU_CUDA(cudaMemcpyAsync((void *)P.v.sp, P.sp.data(), sizeof(SysParams) * S, cudaMemcpyHostToDevice, c->st));
  int r2 = sync_check(c, "gb_energies");
  return r ? r : r2;
}

int pdgpu_nonbonded_forces(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = need_csr(c, e);
  if (r) return r;
  launch_nonbonded(P.v, c->st, P.sp[0].elec_mode);
  launch_energy(P.v, c->st, EM_PAIR_NB);
  return sync_check(c, "nonbonded_forces");
}

int pdgpu_bonded_forces(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (has_bonded(P)) {
    launch_bonded_terms(P.v, c->st);
    launch_energy(P.v, c->st, EM_BONDED);
  }
  return sync_check(c, "bonded_forces");
}

// Forcefield::calcForces for {FF_Bonded, FF_GeneralizedBorn_Still}: the
// Born-radius kernel zeroes forces and record first; one energy reduction.
// extra_mode adds EM_KINETIC / EM_RECORD inside an MD step.
}  // extern "C"
// The LCPO component alone: FF_SASA_LCPO::calcForces at WorkSpace::Step =
// step (lcpo.cpp:176-190) adds its forces and epot_surf; calcEnergies
// (lcpo.cpp:168-173) recomputes the areas and epot_surf only.
static int lcpo_ready(pdgpu_ctx *c, SysEntry *e) {
  Pack &P = *e->pack;
  if (P.v.lc.update <= 0) {
    set_error("this system has no LCPO term (pdgpu_sasa_lcpo_set)");
    return PDGPU_ERR_STATE;
  }
  if (!P.have_list) {
    set_error("no neighbour list: call pdgpu_nlist_build first (NeighbourList::calcNewList)");
    return PDGPU_ERR_STATE;
  }
  PDGPU_CUDA(cudaMemsetAsync(P.v.flags + F_LCPO_CAND, 0, sizeof(int), c->st));
  return PDGPU_OK;
}
static int lcpo_done(pdgpu_ctx *c, SysEntry *e, const char *what) {
  int flag = 0;
  PDGPU_CUDA(cudaMemcpyAsync(&flag, e->pack->v.flags + F_LCPO_CAND, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  int r = sync_check(c, what);
  if (r) return r;
  if (flag) {
    set_error(kLcpoCandMsg);
    return PDGPU_ERR_STATE;
  }
  return PDGPU_OK;
}
extern "C" {
int pdgpu_sasa_lcpo_forces(pdgpu_ctx *c, int32_t sys, int32_t step) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  int r = lcpo_ready(c, e);
  if (r) return r;
  StepSrc src;
  src.imm = step < 0 ? e->ws_step : step;
  launch_lcpo(e->pack->v, c->st, src, false, e->pack->csr_stale);
  launch_energy(e->pack->v, c->st, EM_SURF);
  return lcpo_done(c, e, "sasa_lcpo_forces");
}

int pdgpu_sasa_lcpo_energies(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  int r = lcpo_ready(c, e);
  if (r) return r;
  launch_lcpo(e->pack->v, c->st, StepSrc(), true, e->pack->csr_stale);
  launch_energy(e->pack->v, c->st, EM_SURF);
  return lcpo_done(c, e, "sasa_lcpo_energies");
}

int pdgpu_sasa_lcpo_get(pdgpu_ctx *c, int32_t sys, double *sasa, double *deriv) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  const LcpoView &lc = e->pack->v.lc;
  if (lc.update <= 0) {
    set_error("this system has no LCPO term (pdgpu_sasa_lcpo_set)");
    return PDGPU_ERR_STATE;
  }
  const size_t N = (size_t)e->pack->v.n_atoms;
  if (sasa) PDGPU_CUDA(cudaMemcpyAsync(sasa, lc.sasa, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
  std::vector<double> d;
  if (deriv) {
    d.resize(3 * N);
    PDGPU_CUDA(cudaMemcpyAsync(d.data(), lc.deriv, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->st));
  }
  int r = sync_check(c, "sasa_lcpo_get");
  if (r) return r;
  for (size_t i = 0; i < N && deriv; i++) {
    deriv[3 * i] = d[i];
    deriv[3 * i + 1] = d[N + i];
    deriv[3 * i + 2] = d[2 * N + i];
  }
  return PDGPU_OK;
}
}  // extern "C"

// Forcefield::calcForces for {FF_Bonded, GB[, FF_SASA_LCPO]}: the bonded
// terms and the surface term (zeroing their accumulators first) run on the
// pack's second stream beside the three pair passes; the stream joins
// before the energies are read.  The surface term reads the step counter
// after the previous step's energy record, which runs on that stream too.
void pdgpu::calc_forces_enqueue(cudaStream_t st, SysEntry *e, bool reduce) {
  StepSrc step;
  step.imm = e->ws_step;
  calc_forces_enqueue(st, e, reduce, step);
}
void pdgpu::calc_forces_enqueue(cudaStream_t st, SysEntry *e, bool reduce, StepSrc step, int ebuf, int coop) {
  Pack &P = *e->pack;
  const bool bonded = has_bonded(P);
  const bool surf = P.v.lc.update > 0;
  const bool side = bonded || surf;
  if (side) {
    const size_t bytes = sizeof(long long) * (size_t)P.v.n_atoms;
    cudaEventRecord(P.fork, st);
    cudaStreamWaitEvent(P.side, P.fork, 0);
    cudaMemsetAsync(P.v.fx, 0, bytes, P.side);
    cudaMemsetAsync(P.v.fy, 0, bytes, P.side);
    cudaMemsetAsync(P.v.fz, 0, bytes, P.side);
    if (bonded) launch_bonded_terms(P.v, P.side);
    if (surf) launch_lcpo(P.v, P.side, step, false, P.csr_stale);
    cudaEventRecord(P.join, P.side);
  }
  // with an MD step's energy record still running beside, the record is
  // left to it (it forms the record from zero) and the fused pass, which
  // writes what the record reads, waits for it
  const bool pending = P.energy_pending();
  const int zero = ZF_PAIRS | (side ? 0 : ZF_BONDED) | (pending ? 0 : ZF_RECORD);
  const bool slow = P.slow();
  if (P.v.tile_mode) {
    // the tile layout: the three passes as one evaluation into energy
    // buffer `ebuf`; only a record still reading that buffer is waited for
    // (FastMode off: every pending record, as its LJ/Coulomb pass writes
    // buffer 0)
    P.wait_energy(st, ebuf);
    if (slow) P.wait_energy(st, ebuf ^ 1);
    PackView vb = P.v;
    vb.ebuf = ebuf;
    launch_eval_tiles(vb, st, zero, coop < 0 ? P.coop : coop != 0);
    P.last_ebuf = ebuf;
  } else {
    launch_born_radii(P.v, st, zero);
    P.wait_energy(st, 0);
    P.wait_energy(st, 1);
    launch_gb_pair(P.v, st);
    launch_gb_chain(P.v, st);
    P.last_ebuf = 0;
  }
  // FastMode off: FF_NonBonded::calcForces beside calcBornForces
  if (slow) launch_nonbonded(P.v, st, P.sp[0].elec_mode);
  if (side) cudaStreamWaitEvent(st, P.join, 0);
  if (reduce) launch_energy(P.v, st, pair_energy_mode(P) | (bonded ? EM_BONDED : 0) | (surf ? EM_SURF : 0));
}
extern "C" {

int pdgpu_calc_forces(pdgpu_ctx *c, int32_t sys) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = ready_pairs(c, e);
  if (r) return r;
  calc_forces_enqueue(c->st, e, true);
  r = sync_check(c, "calc_forces");
  return r ? r : barrier_check(c, P);
}

// ------------------------------------------------------------ MD
// RNG keys: those given to pdgpu_set_seeds, else base + s for system s
static int default_seeds(pdgpu_ctx *c, SysEntry *e, unsigned long long base) {
  if (e->custom_seeds || (e->seeds_default && e->seeds_base == base)) return PDGPU_OK;
  std::vector<unsigned long long> k(e->nsys());
  for (int s = 0; s < e->nsys(); s++) k[s] = base + (unsigned long long)s;
  PDGPU_CUDA(cudaMemcpyAsync(e->seeds, k.data(), sizeof(unsigned long long) * k.size(), cudaMemcpyHostToDevice,
                             c->st));
  e->seeds_default = true;
  e->seeds_base = base;
  return PDGPU_OK;
}

}  // extern "C"
MDCoef pdgpu::md_coef(const pdgpu_md_params *p, int step, int steps) {
  // the coefficient branches of md.cpp:961-1000
  MDCoef c;
  memset(&c, 0, sizeof c);
  c.dt = p->Timestep;
  c.gamma = p->FricCoeff;
  c.temp = p->TargetTemp;
  c.integrator = p->Integrator;
  c.step = step;
  c.steps = steps;
  c.stochastic_h = p->LangevinOnHydrogens;
  c.seed = p->Seed;
  double gt = c.gamma * c.dt;
  double gt2 = gt * gt, gt3 = gt * gt2, gt4 = gt2 * gt2, gt5 = gt2 * gt3, gt6 = gt3 * gt3, gt7 = gt3 * gt4,
         gt8 = gt4 * gt4, gt9 = gt4 * gt5;
  if (gt > 0.05) {
    c.c0 = exp(-gt);
    c.c1 = (1 - c.c0) / gt;
    c.c2 = (1 - c.c1) / gt;
    double eg = exp(-gt);
    c.varv = (1.0 - eg * eg);
    c.varr = (2.0 * gt - 3.0 + (4.0 - eg) * eg);
    c.crv = (1.0 - eg) * (1.0 - eg) / (sqrt(c.varv * c.varr));
  } else {
    c.c0 = 1 - gt + 0.5 * gt2 - gt3 / 6.0 + gt4 / 24.0 - gt5 / 120.0 + gt6 / 720.0 - gt7 / 5040.0 +
           gt8 / 40320.0 - gt9 / 362880.0;
    c.c1 = 1 - (0.5 * gt - gt2 / 6.0 + gt3 / 24.0 - gt4 / 120.0 + gt5 / 720.0 - gt6 / 5040.0 + gt7 / 40320.0 -
                gt8 / 362880.0);
    c.c2 = 0.5 - gt / 6.0 + gt2 / 24.0 - gt3 / 120.0 + gt4 / 720.0 - gt5 / 5040.0 + gt6 / 40320.0 -
           gt7 / 362880.0;
    c.varr = 2.0 * gt3 / 3.0 - gt4 / 2.0 + 7.0 * gt5 / 30.0 - gt6 / 12.0 + 31.0 * gt7 / 1260.0 - gt8 / 160.0 +
             127.0 * gt9 / 90720.0;
    c.varv = 2.0 * gt - 2.0 * gt2 + 4.0 * gt3 / 3.0 - 2.0 * gt4 / 3.0 + 4.0 * gt5 / 15.0 - 4.0 * gt6 / 45.0 +
             8.0 * gt7 / 315.0 - 2.0 * gt8 / 315.0 + 4.0 * gt9 / 2835.0;
    c.crv = sqrt(3.0) * (0.5 - 3.0 * gt / 16.0 - 17.0 * gt2 / 1280.0 + 17.0 * gt3 / 6144.0 +
                         40967.0 * gt4 / 34406400.0 - 57203.0 * gt5 / 275251200.0 -
                         1429487.0 * gt6 / 13212057600.0);
  }
  if (gt > 0 && c.c1 != 0) {
    c.kick1 = (1.0 - c.c0 / c.c1) / gt;
    c.c0c2_c1 = c.c0 * c.c2 / c.c1;
    c.inv_gamma = 1.0 / c.gamma;
    c.sq_crv = sqrt(1.0 - c.crv * c.crv);
  }
  return c;
}
extern "C" {

}  // extern "C"
int pdgpu::validate_md(const pdgpu_md_params *p) {
  if (!p || !(p->Timestep > 0) || p->Integrator < 0 || p->Integrator > 3 || !(p->TargetTemp >= 0) ||
      (p->Integrator == PDGPU_INTEGRATOR_LANGEVIN && !(p->FricCoeff > 0))) {
    set_error("invalid MD parameters");
    return PDGPU_ERR_ARG;
  }
  return PDGPU_OK;
}
extern "C" {

int pdgpu_md_step_with_normals(pdgpu_ctx *c, int32_t sys, const pdgpu_md_params *p, int32_t step,
                               int32_t total_steps, const double *normals) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  int r = validate_md(p);
  if (r) return r;
  Pack &P = *e->pack;
  double *nd = nullptr;
  if (normals) {
    PDGPU_CUDA(cudaMalloc(&nd, sizeof(double) * 6 * P.v.n_atoms));
    PDGPU_CUDA(cudaMemcpyAsync(nd, normals, sizeof(double) * 6 * P.v.n_atoms, cudaMemcpyHostToDevice, c->st));
  }
  if ((r = default_seeds(c, e, p->Seed))) return r;
  MDCoef k = md_coef(p, step, total_steps);
  launch_md_step_impl(P.v, c->st, k, nd, nullptr, P.is_h, e->seeds);
  r = sync_check(c, "md_step");
  if (nd) cudaFree(nd);
  return r;
}

int pdgpu_md_init_velocities(pdgpu_ctx *c, int32_t sys, double temperature, uint64_t seed) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  int r = default_seeds(c, e, seed);
  if (r) return r;
  launch_vel_init_impl(e->pack->v, c->st, temperature, e->seeds);
  return sync_check(c, "init_velocities");
}

// one MD step enqueue: forces, integrate, one energy reduction that also
// records the step and advances the device step counter (7 launches)
}  // extern "C"
void pdgpu::md_step_enqueue(cudaStream_t st, SysEntry *e, const MDCoef &k, int q) {
  Pack &P = *e->pack;
  StepSrc step;
  step.p = e->step_dev;  // MolecularDynamics::run_core sets WorkSpace::Step = Step (md.cpp:214)
  const int b = (P.v.tile_mode && !P.slow()) ? (q & 1) : 0;  // this step's energy buffer
  calc_forces_enqueue(st, e, false, step, b, P.coop_md ? 1 : 0);
  // the integrator writes the kinetic energies the previous step's record
  // reads: that record must be done
  P.wait_energy(st, b ^ 1);
  P.wait_energy(st, b);
  launch_md_step_impl(P.v, st, k, nullptr, e->step_dev, P.is_h, e->seeds, e->traj_dev, e->traj_every,
                      e->traj_dev_cap);
  // the step's energy record on the second stream, beside the next step's
  // evaluation (its bonded terms queue behind it on that stream)
  cudaEventRecord(P.fork2, st);
  cudaStreamWaitEvent(P.side, P.fork2, 0);
  PackView vb = P.v;
  vb.ebuf = b;
  launch_energy(vb, P.side,
                pair_energy_mode(P) | (has_bonded(P) ? EM_BONDED : 0) | (P.v.lc.update > 0 ? EM_SURF : 0) |
                    EM_KINETIC | EM_RECORD | EM_ASSIGN,
                e->hist, e->step_dev);
  cudaEventRecord(P.ene_done[b], P.side);
  P.ene_pending[b] = true;
}
// Trajectory frames of steps [s0, s1) (absolute): mirrored from the device
// ring into the host ring on the pack's second stream once the steps are
// done.  The step graph of the next list period writes other ring slots
// (the device ring holds two periods of frames), and before the period
// after that the main stream waits for this copy.
static void trajectory_copy(pdgpu_ctx *c, SysEntry *e, int s0, int s1) {
  if (e->traj_every <= 0) return;
  Pack &P = *e->pack;
  const int ev = e->traj_every;
  const size_t frame = 3 * (size_t)P.v.n_atoms;
  if (e->traj_pending) cudaStreamWaitEvent(c->st, e->traj_ev, 0);  // the previous period's copy
  cudaEventRecord(P.fork2, c->st);
  cudaStreamWaitEvent(P.side, P.fork2, 0);
  for (int st = std::max(s0, 1); st < s1; st++) {
    if (st % ev) continue;
    const long long idx = st / ev - 1;
    const double *src = e->traj_dev + (size_t)(idx % e->traj_dev_cap) * frame;
    const long long slot = e->traj_copied % e->traj_host_cap;
    cudaMemcpyAsync(e->traj_host + (size_t)slot * frame, src, sizeof(double) * frame, cudaMemcpyDeviceToHost,
                    P.side);
    e->traj_step[slot] = st;
    e->traj_copied++;
  }
  cudaEventRecord(e->traj_ev, P.side);
  e->traj_pending = true;
  // fewer than two periods of frames fit the device ring: the next period
  // waits for this copy
  const int per_period = (s1 - s0 + ev - 1) / ev + 1;
  if (2 * per_period > e->traj_dev_cap) cudaStreamWaitEvent(c->st, e->traj_ev, 0);
}

// The end of a run of MD steps: the last step's energy record joins the
// main stream.
void pdgpu::md_steps_end(cudaStream_t st, SysEntry *e) {
  Pack &P = *e->pack;
  P.wait_energy(st, 0);
  P.wait_energy(st, 1);
}
extern "C" {

int pdgpu_md_set_trajectory(pdgpu_ctx *c, int32_t sys, int32_t every, int32_t capacity) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (every < 0 || (every > 0 && capacity <= 0)) {
    set_error("md_set_trajectory: need every >= 0 and capacity > 0");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  if (e->traj_pending) cudaStreamSynchronize(P.side);
  e->drop_graph();
  if (e->traj_dev) {
    auto it = std::find(e->extra.begin(), e->extra.end(), (void *)e->traj_dev);
    if (it != e->extra.end()) {
      cudaFreeAsync(*it, e->st);
      e->extra.erase(it);
    }
  }
  e->free_trajectory();
  if (every == 0) return PDGPU_OK;
  const size_t frame = 3 * (size_t)P.v.n_atoms;
  // the device ring: two list periods of frames at the most frequent
  // cadence a run can use (every step), or the host capacity if smaller
  const int dev_cap = std::max(2, std::min(capacity, 64));
  if (xalloc(e, &e->traj_dev, frame * dev_cap) != cudaSuccess) {
    set_error("device allocation failed (trajectory ring)");
    return PDGPU_ERR_NOMEM;
  }
  if (cudaHostAlloc((void **)&e->traj_host, sizeof(double) * frame * capacity, cudaHostAllocDefault) != cudaSuccess) {
    e->traj_host = nullptr;
    set_error("page-locked allocation failed (trajectory frames)");
    return PDGPU_ERR_NOMEM;
  }
  cudaEventCreateWithFlags(&e->traj_ev, cudaEventDisableTiming);
  e->traj_every = every;
  e->traj_dev_cap = dev_cap;
  e->traj_host_cap = capacity;
  e->traj_step.assign(capacity, -1);
  return sync_check(c, "md_set_trajectory");
}

int pdgpu_md_read_trajectory(pdgpu_ctx *c, int32_t sys, double *frames, int64_t *steps, int32_t max_frames,
                             int32_t *count, int32_t *dropped) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!count || max_frames < 0 || (max_frames > 0 && !frames)) {
    set_error("md_read_trajectory: bad arguments");
    return PDGPU_ERR_ARG;
  }
  *count = 0;
  if (dropped) *dropped = 0;
  if (e->traj_every <= 0) return PDGPU_OK;
  if (e->traj_pending) {
    PDGPU_CUDA(cudaEventSynchronize(e->traj_ev));
  }
  long long first = e->traj_read;
  if (e->traj_copied - first > e->traj_host_cap) {  // overwritten before being read
    if (dropped) *dropped = (int32_t)(e->traj_copied - e->traj_host_cap - first);
    first = e->traj_copied - e->traj_host_cap;
  }
  const size_t frame = 3 * (size_t)e->pack->v.n_atoms;
  int n = 0;
  for (long long q = first; q < e->traj_copied && n < max_frames; q++, n++) {
    const long long slot = q % e->traj_host_cap;
    std::memcpy(frames + (size_t)n * frame, e->traj_host + (size_t)slot * frame, sizeof(double) * frame);
    if (steps) steps[n] = e->traj_step[slot];
  }
  e->traj_read = first + n;
  *count = n;
  return PDGPU_OK;
}

// The step loop of pdgpu_md_run.  `tail` (may be empty) enqueues work that
// follows the run (pdgpu_md_run_io's state copies): it is enqueued behind
// the last block before that block's one synchronisation, and again behind
// a block that had to run again.
static int md_run_impl(pdgpu_ctx *c, SysEntry *e, const pdgpu_md_params *p, int32_t first_step, int32_t steps,
                       int32_t total_steps, double *history, const std::function<int()> &tail) {
  int r = validate_md(p);
  if (r) return r;
  if (steps < 0 || first_step < 0 || total_steps < first_step + steps) {
    set_error("md_run: need 0 <= first_step and first_step + steps <= total_steps");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  PackView &v = P.v;
  if (steps == 0) return PDGPU_OK;
  const int S = e->nsys();
  if (e->hist_cap < steps) {
    if (e->hist) {
      cudaFree(e->hist);
      e->extra.erase(std::find(e->extra.begin(), e->extra.end(), (void *)e->hist));
      e->hist = nullptr;
    }
    if (xalloc(e, &e->hist, (size_t)3 * steps * S) != cudaSuccess) {
      set_error("device allocation failed (history)");
      return PDGPU_ERR_NOMEM;
    }
    e->hist_cap = steps;
  }
  if ((r = default_seeds(c, e, p->Seed))) return r;
  PDGPU_CUDA(cudaMemsetAsync(v.flags, 0, sizeof(int) * F_COUNT, c->st));
  MDCoef k = md_coef(p, first_step, total_steps);
  int every = p->UpdateNList;
  // size the list once up front (one synchronisation); later rebuilds run
  // inside the step blocks and report overflow through a device flag
  if (!P.have_list || P.nl_total < 0) {
    r = nlist_enqueue(c, e, true);
    if (r) return r;
  }
  if ((r = ready_pairs(c, e))) return r;
  // A block is one list period: [rebuild] + UpdateNList steps.  If the
  // in-block rebuild overflows the list buffer, every kernel after it skips
  // (device flag), the state stays at the block start, and the host grows
  // the buffer and runs the block again.
  if (!e->pin_flags && cudaHostAlloc((void **)&e->pin_flags, sizeof(int) * (F_COUNT + 3), 0) != cudaSuccess) {
    e->pin_flags = nullptr;
    set_error("page-locked host allocation failed (MD flags)");
    return PDGPU_ERR_NOMEM;
  }
  int *steps0 = e->pin_flags + F_COUNT;  // step counter, first step, finished-system count
  steps0[0] = steps0[1] = first_step;
  steps0[2] = 0;
  PDGPU_CUDA(cudaMemcpyAsync(e->step_dev, steps0, sizeof(int) * 3, cudaMemcpyHostToDevice, c->st));
  cudaEventRecord(P.ev0, c->st);
  int s = 0;
  while (s < steps) {
    int step = first_step + s;
    // Blocks follow the list periods (protocolbase.cpp:113-122: a rebuild
    // when the step counter is a multiple of UpdateNList).  A run that
    // starts inside a period first finishes that period in one block
    // without a rebuild; a run that ends inside one ends with a shorter
    // block that begins with the rebuild.  Every block of more than one
    // step replays a cached graph of its own shape.
    bool rebuild = every > 0 && (P.nlist_counter % every) == 0;
    int block = 1;
    if (every > 1) {
      const int left = rebuild ? every : every - P.nlist_counter % every;
      block = std::min(left, steps - s);
    }
    bool use_graph = p->UseGraph && block > 1;
    int counter0 = P.nlist_counter;
    for (int attempt = 0;; attempt++) {
      if (attempt == 4) {
        set_error("neighbour list kept overflowing after regrowth");
        return PDGPU_ERR_STATE;
      }
      if (s > 0 || attempt > 0) {  // the first block starts from the run's own setup
        PDGPU_CUDA(cudaMemsetAsync(v.flags + F_NL_OVERFLOW, 0, sizeof(int), c->st));
        steps0[0] = step;
        PDGPU_CUDA(cudaMemcpyAsync(e->step_dev, steps0, sizeof(int), cudaMemcpyHostToDevice, c->st));
      }
      if (use_graph) {
        // graphs are cached per system; the key holds every value baked in
        char key[288];
        snprintf(key, sizeof key, "%d|%d|%p|%lld|%p|%d|%d|%.17g|%.17g|%.17g|%d|%d|%d|%d%d%d|%d%d%d|%p|%d|%d", block,
                 (int)rebuild, (void *)v.nl, v.nl_cap, (void *)e->hist, k.integrator, k.steps, k.dt, k.gamma,
                 k.temp, k.stochastic_h, P.radix_passes, (int)e->host->params.FastMode, v.lpa[0], v.lpa[1],
                 v.lpa[2], v.tile_mode, (int)tile_search_ok(P), (int)P.coop_md, (void *)e->traj_dev, e->traj_every,
                 e->traj_dev_cap);
        SysEntry::GraphSlot *g = nullptr;
        for (auto &q : e->gslots)
          if (q.key == key) g = &q;
        if (!g) {
          if ((int)e->gslots.size() >= SysEntry::kGraphSlots) {  // evict the least recently used
            auto lru = std::min_element(e->gslots.begin(), e->gslots.end(),
                                        [](const SysEntry::GraphSlot &a, const SysEntry::GraphSlot &b) {
                                          return a.used < b.used;
                                        });
            e->drop_slot(*lru);
            e->gslots.erase(lru);
          }
          SysEntry::GraphSlot ng;
          const bool pend0 = P.ene_pending[0], pend1 = P.ene_pending[1];  // both false between blocks
          begin_capture_count();
          PDGPU_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
          if (rebuild) rebuild_enqueue(P, c->st);
          for (int q = 0; q < block; q++) md_step_enqueue(c->st, e, k, q);
          md_steps_end(c->st, e);
          cudaError_t ce = cudaStreamEndCapture(c->st, &ng.graph);
          ng.nodes = end_capture_count();
          if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ng.exec, ng.graph, 0);
          if (ce != cudaSuccess) {
            e->drop_slot(ng);
            P.ene_pending[0] = pend0;
            P.ene_pending[1] = pend1;
            if (P.coop_md && P.v.tile_mode) {
              // a graph that cannot hold the cooperative evaluation: the
              // same phases as three launches from here on
              cudaGetLastError();
              P.coop_md = false;
              continue;
            }
            return cuda_fail(ce, "capture md block");
          }
          ng.key = key;
          e->gslots.push_back(ng);
          g = &e->gslots.back();
        }
        g->used = ++e->gclock;
        PDGPU_CUDA(cudaGraphLaunch(g->exec, c->st));
        launch_counter() += g->nodes;
        e->graph_replays++;
        if (rebuild) P.csr_stale = tile_search_ok(P);  // what the graph's rebuild made
      } else {
        if (rebuild) rebuild_enqueue(P, c->st);
        for (int q = 0; q < block; q++) md_step_enqueue(c->st, e, k, q);
        md_steps_end(c->st, e);
      }
      const bool last = s + block >= steps;
      if (last) {
        cudaEventRecord(P.ev1, c->st);
        if (tail && (r = tail())) return r;
      }
      int *flags = e->pin_flags;
      PDGPU_CUDA(cudaMemcpyAsync(flags, v.flags, sizeof(int) * F_COUNT, cudaMemcpyDeviceToHost, c->st));
      r = sync_check(c, "md block");
      if (r) return r;
      if ((r = barrier_check(c, P, flags))) return r;
      if (flags[F_LCPO_CAND]) {
        set_error(kLcpoCandMsg);
        return PDGPU_ERR_STATE;
      }
      if (flags[F_NL_OVERFLOW]) {
        // state untouched since the block start: grow the list and re-run
        r = nlist_enqueue(c, e, true);
        if (r) return r;
        e->drop_graph();
        continue;
      }
      if (flags[F_NAN]) {
        if (history) {
          std::vector<double> h((size_t)3 * (s + block) * S);
          cudaMemcpy(h.data(), e->hist, sizeof(double) * h.size(), cudaMemcpyDeviceToHost);
          for (size_t q = 0; q < h.size(); q++) history[q] = h[q] * consts().J_per_kcalmol;
        }
        set_error("Simulation unstable or division by zero (NaN energy)");
        return PDGPU_ERR_UNSTABLE;
      }
      break;
    }
    P.nlist_counter = counter0 + block;
    trajectory_copy(c, e, step, step + block);
    s += block;
  }
  if (e->traj_every > 0 && (r = sync_check(c, "md_run"))) return r;
  if (steps > 0) e->ws_step = first_step + steps - 1;  // WorkSpace::Step as run_core leaves it
  float ms = 0;
  cudaEventElapsedTime(&ms, P.ev0, P.ev1);
  P.last_run_ms = ms;
  c->last_ms = ms;
  if (history) {
    std::vector<double> h((size_t)3 * steps * S);
    PDGPU_CUDA(cudaMemcpy(h.data(), e->hist, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    double J = consts().J_per_kcalmol;
    for (size_t q = 0; q < h.size(); q++) history[q] = h[q] * J;
  }
  return PDGPU_OK;
}

extern "C" int pdgpu_md_run(pdgpu_ctx *c, int32_t sys, const pdgpu_md_params *p, int32_t first_step,
                            int32_t steps, int32_t total_steps, double *history) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  return md_run_impl(c, e, p, first_step, steps, total_steps, history, std::function<int()>());
}

// ------------------------------------------------------------ minimiser
int pdgpu_minimise_run(pdgpu_ctx *c, int32_t sys, const pdgpu_min_params *p, int32_t steps,
                       int32_t *steps_taken) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!p || steps < 0 || (p->Algorithm != 0 && p->Algorithm != 1)) {
    set_error("invalid minimiser parameters");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  PackView &v = P.v;
  const Consts &k = consts();
  const int S = e->nsys();
  if (!e->min_state) {
    unsigned char *m = nullptr;
    PDGPU_CUDA(xalloc(e, &m, min_state_size() * S));
    e->min_state = m;
  }
  std::vector<unsigned char> hs(min_state_size() * S);
  min_state_init(hs.data(), S);
  PDGPU_CUDA(cudaMemcpyAsync(e->min_state, hs.data(), hs.size(), cudaMemcpyHostToDevice, c->st));
  PDGPU_CUDA(cudaMemsetAsync(v.flags, 0, sizeof(int) * F_COUNT, c->st));
  // WorkSpace::old = cur (minimise.cpp:114)
  int n = v.n_atoms;
  PDGPU_CUDA(cudaMemcpyAsync(v.ox, v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.oy, v.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.oz, v.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  double J2k = k.J2kcal * k.Na;
  double slope = p->SlopeCutoff > 0 ? p->SlopeCutoff * J2k : -1.0;
  double strict = p->Strictness;  // kcal/mol (minimise.cpp:256)
  int every = p->UpdateNList;
  int r;
  if (!P.have_list || P.nl_total < 0) {
    r = nlist_enqueue(c, e, true);
    if (r) return r;
  }
  if ((r = ready_pairs(c, e))) return r;
  cudaEventRecord(P.ev0, c->st);
  // Chunks of up to 16 steps run without a host synchronisation.  A step
  // whose list rebuild overflowed does nothing on the device (flag); the
  // host grows the list and repeats it.  The list cadence follows the
  // iterations the device actually took; every system still running takes
  // one step per iteration, and a finished system (converged, out of
  // steps, NaN) sits the rest out.
  const int counter0 = P.nlist_counter;
  int iter = 0, regrow = 0;
  std::vector<int> taken(S, 0);
  while (iter < steps) {
    int chunk = std::min(16, steps - iter);
    for (int q = 0; q < chunk; q++) {
      int cnt = counter0 + iter + q;
      if (every > 0 && (cnt % every) == 0) rebuild_enqueue(P, c->st);
      calc_forces_enqueue(c->st, e, true, min_step_src(e->min_state, false));
      launch_min_step(v, c->st, e->min_state, p->Algorithm, slope, strict, p->StepSize, steps);
    }
    int flags[F_COUNT];
    PDGPU_CUDA(cudaMemcpyAsync(flags, v.flags, sizeof flags, cudaMemcpyDeviceToHost, c->st));
    r = sync_check(c, "minimise");
    if (r) return r;
    if ((r = barrier_check(c, P, flags))) return r;
    if (flags[F_LCPO_CAND]) {
      set_error(kLcpoCandMsg);
      return PDGPU_ERR_STATE;
    }
    PDGPU_CUDA(cudaMemcpy(hs.data(), e->min_state, hs.size(), cudaMemcpyDeviceToHost));
    int advanced = 0, nan_count = 0;
    for (int s = 0; s < S; s++) {
      int nan, done_taken;
      double mult;
      min_state_read(hs.data(), s, &done_taken, &nan, &mult);
      advanced = std::max(advanced, done_taken - taken[s]);
      taken[s] = done_taken;
      if (nan) {
        taken[s] = -1;
        nan_count++;
      }
    }
    if (S == 1 && nan_count) {
      if (steps_taken) *steps_taken = -1;
      set_error("Simulation unstable (NaN energy during minimisation)");
      return PDGPU_ERR_UNSTABLE;
    }
    // every system finished early (converged on SlopeCutoff, or NaN)
    bool finished = advanced < chunk && !flags[F_NL_OVERFLOW];
    iter += advanced;
    if (flags[F_NL_OVERFLOW]) {
      if (++regrow > 8) {
        set_error("neighbour list kept overflowing during minimisation");
        return PDGPU_ERR_STATE;
      }
      r = nlist_enqueue(c, e, true);  // sized rebuild at the current positions
      if (r) return r;
      continue;
    }
    if (finished) break;
  }
  P.nlist_counter = counter0 + iter;
  // cur = old; recompute the energies (minimise.cpp:172-176)
  launch_min_finish(v, c->st);
  calc_forces_enqueue(c->st, e, true, min_step_src(e->min_state, true));
  cudaEventRecord(P.ev1, c->st);
  r = sync_check(c, "minimise finish");
  if (r) return r;
  PDGPU_CUDA(cudaMemcpy(hs.data(), e->min_state, hs.size(), cudaMemcpyDeviceToHost));
  e->ws_step = min_state_last(hs.data(), 0);
  float ms = 0;
  cudaEventElapsedTime(&ms, P.ev0, P.ev1);
  P.last_run_ms = ms;
  c->last_ms = ms;
  if (steps_taken)
    for (int s = 0; s < S; s++) steps_taken[s] = taken[s];
  return PDGPU_OK;
}

// MolecularDynamics::run with the state in host memory: the positions and
// velocities go in, the steps run, and the positions, velocities and energy
// record come back, with one host synchronisation after the step loop's
// own (the state calls would add one each).
int pdgpu_md_run_io(pdgpu_ctx *c, int32_t sys, const pdgpu_md_params *p, int32_t first_step, int32_t steps,
                    int32_t total_steps, const double *x_in, const double *v_in, double *x_out, double *v_out,
                    double *ene_out) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  const int n = P.v.n_atoms;
  const size_t blk = sizeof(double) * 3 * (size_t)n;
  // the state in and out through one device staging block [x | v], one
  // copy each way per array, and the copies out enqueued behind the last
  // step block before its synchronisation: one synchronisation per call
  if ((x_in || v_in || x_out || v_out) && !e->io_stage && xalloc(e, &e->io_stage, 6 * (size_t)n) != cudaSuccess) {
    set_error("device allocation failed (state staging)");
    return PDGPU_ERR_NOMEM;
  }
  const size_t ne = (size_t)E_COUNT * e->nsys();
  if (ene_out && !e->pin_ene && cudaHostAlloc((void **)&e->pin_ene, sizeof(double) * ne, 0) != cudaSuccess) {
    e->pin_ene = nullptr;
    set_error("page-locked host allocation failed (energies)");
    return PDGPU_ERR_NOMEM;
  }
  double *const X = e->io_stage, *const V = e->io_stage ? e->io_stage + 3 * (size_t)n : nullptr;
  if (x_in) PDGPU_CUDA(cudaMemcpyAsync(X, x_in, blk, cudaMemcpyHostToDevice, c->st));
  if (v_in) PDGPU_CUDA(cudaMemcpyAsync(V, v_in, blk, cudaMemcpyHostToDevice, c->st));
  if (x_in || v_in) launch_state_in(P.v, x_in ? X : nullptr, v_in ? V : nullptr, c->st);
  auto tail = [&]() -> int {
    if (x_out || v_out) launch_state_out(P.v, x_out ? X : nullptr, v_out ? V : nullptr, c->st);
    if (x_out) PDGPU_CUDA(cudaMemcpyAsync(x_out, X, blk, cudaMemcpyDeviceToHost, c->st));
    if (v_out) PDGPU_CUDA(cudaMemcpyAsync(v_out, V, blk, cudaMemcpyDeviceToHost, c->st));
    if (ene_out) PDGPU_CUDA(cudaMemcpyAsync(e->pin_ene, P.v.ene, sizeof(double) * ne, cudaMemcpyDeviceToHost, c->st));
    return PDGPU_OK;
  };
  int r = md_run_impl(c, e, p, first_step, steps, total_steps, nullptr, tail);
  if (r) return r;
  if (steps == 0) {  // no block ran: the copies out on their own
    if ((r = tail()) || (r = sync_check(c, "md_run_io"))) return r;
  }
  if (ene_out) {
    const double J = consts().J_per_kcalmol;
    for (size_t q = 0; q < ne; q++) ene_out[q] = e->pin_ene[q] * J;
  }
  return PDGPU_OK;
}

// ------------------------------------------------------------ Monte Carlo
void pdgpu_mc_params_default(pdgpu_mc_params *p) {
  if (!p) return;
  p->Steps = 0;
  p->FinalState = PDGPU_MC_LAST_ACC;  // montecarlo.h:53
  p->Temperature = 300.0;             // ConstantProfile(300), montecarlo.h:52
  p->Sigma = 15.0 * 3.14159265358979323846 / 180.0;
  p->Seed = 0;
}

// MonteCarlo::run_core (protocols/montecarlo.cpp:24-141) for every system of
// the handle at once, on the device: each step perturbs the phi/psi of the
// last accepted state (step 0 evaluates it unperturbed), rebuilds the list,
// evaluates the forcefield and applies the Metropolis test per system.  The
// host reads one flag block per 16 steps.
int pdgpu_mc_run(pdgpu_ctx *c, int32_t sys, const pdgpu_mc_params *p, int32_t *accepted, double *lowest) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!p || p->Steps < 1 || !(p->Temperature > 0) || !(p->Sigma >= 0) || p->FinalState < 0 || p->FinalState > 2) {
    set_error("invalid Monte Carlo parameters (Steps >= 1, Temperature > 0, Sigma >= 0, FinalState 0..2)");
    return PDGPU_ERR_ARG;
  }
  Pack &P = *e->pack;
  PackView &v = P.v;
  const int S = e->nsys();
  const size_t n = (size_t)v.n_atoms;
  if (!e->mc_state) {
    unsigned char *m = nullptr;
    PDGPU_CUDA(xalloc(e, &m, mc_state_size() * S));
    e->mc_state = m;
  }
  PDGPU_CUDA(cudaMemsetAsync(e->mc_state, 0, mc_state_size() * S, c->st));
  int r = default_seeds(c, e, p->Seed);
  if (r) return r;
  if (!P.have_list || P.nl_total < 0) {
    if ((r = nlist_enqueue(c, e, true))) return r;
  }
  if ((r = ready_pairs(c, e))) return r;
  // the starting state is the first base (and lowest) state
  PDGPU_CUDA(cudaMemcpyAsync(v.bx, v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.by, v.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.bz, v.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.ox, v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.oy, v.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemcpyAsync(v.oz, v.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  PDGPU_CUDA(cudaMemsetAsync(v.flags, 0, sizeof(int) * F_COUNT, c->st));
  const Consts &k = consts();
  const double inv_kT = k.J_per_kcalmol / (k.kB * p->Temperature);  // per kcal/mol
  const int keep_lowest = p->FinalState == PDGPU_MC_LOWEST_EPOT;
  std::vector<unsigned char> hs(mc_state_size() * S);
  cudaEventRecord(P.ev0, c->st);
  int step = 0, regrow = 0;
  while (step < p->Steps) {
    const int chunk = std::min(16, p->Steps - step);
    for (int q = 0; q < chunk; q++) {
      const int t = step + q;
      if (t != 0) launch_torsion_moves(v, c->st, p->Sigma, (unsigned long long)t, e->seeds, nullptr);
      rebuild_enqueue(P, c->st);  // the evaluator's list refresh
      StepSrc ws;
      ws.imm = t;  // WorkSpace::Step = Step (montecarlo.cpp:37)
      calc_forces_enqueue(c->st, e, true, ws);
      launch_mc_accept(v, c->st, e->mc_state, t, inv_kT, e->seeds, keep_lowest);
    }
    int flags[F_COUNT];
    PDGPU_CUDA(cudaMemcpyAsync(flags, v.flags, sizeof flags, cudaMemcpyDeviceToHost, c->st));
    PDGPU_CUDA(cudaMemcpyAsync(hs.data(), e->mc_state, hs.size(), cudaMemcpyDeviceToHost, c->st));
    if ((r = sync_check(c, "mc_run"))) return r;
    if ((r = barrier_check(c, P, flags))) return r;
    if (flags[F_LCPO_CAND]) {
      set_error(kLcpoCandMsg);
      return PDGPU_ERR_STATE;
    }
    if (flags[F_NL_OVERFLOW]) {
      // the steps from the overflowing rebuild on did nothing: grow the list
      // and go on from the first of them (its base state is untouched)
      if (++regrow > 8) {
        set_error("neighbour list kept overflowing during Monte Carlo");
        return PDGPU_ERR_STATE;
      }
      int acc, done, ls;
      double low;
      mc_state_read(hs.data(), 0, &acc, &done, &low, &ls);
      if ((r = nlist_enqueue(c, e, true))) return r;
      PDGPU_CUDA(cudaMemsetAsync(v.flags + F_NL_OVERFLOW, 0, sizeof(int), c->st));
      step = done;
      continue;
    }
    step += chunk;
  }
  // the final state (montecarlo.cpp:113-133), evaluated again
  if (p->FinalState == PDGPU_MC_LAST_ACC)
    launch_mc_restore(v, c->st);
  else if (p->FinalState == PDGPU_MC_LOWEST_EPOT)
    launch_min_finish(v, c->st);
  rebuild_enqueue(P, c->st);
  StepSrc ws;
  ws.imm = p->Steps - 1;
  calc_forces_enqueue(c->st, e, true, ws);
  cudaEventRecord(P.ev1, c->st);
  int flags[F_COUNT];
  PDGPU_CUDA(cudaMemcpyAsync(flags, v.flags, sizeof flags, cudaMemcpyDeviceToHost, c->st));
  if ((r = sync_check(c, "mc_run final"))) return r;
  if ((r = barrier_check(c, P, flags))) return r;
  if (flags[F_NL_OVERFLOW]) {  // the final state's list: sized, then evaluated again
    if ((r = nlist_enqueue(c, e, true))) return r;
    calc_forces_enqueue(c->st, e, true, ws);
    if ((r = sync_check(c, "mc_run final"))) return r;
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, P.ev0, P.ev1);
  P.last_run_ms = ms;
  c->last_ms = ms;
  e->ws_step = p->Steps - 1;
  for (int s = 0; s < S; s++) {
    int acc, done, ls;
    double low;
    mc_state_read(hs.data(), s, &acc, &done, &low, &ls);
    if (accepted) accepted[s] = acc;
    if (lowest) lowest[s] = acc ? low * k.J_per_kcalmol : std::numeric_limits<double>::quiet_NaN();
  }
  return PDGPU_OK;
}

// ------------------------------------------------------------ instrumentation
int pdgpu_pair_counts(pdgpu_ctx *c, int32_t sys, int64_t *counts) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = need_csr(c, e);
  if (r) return r;
  if (!counts) {
    set_error("counts is NULL");
    return PDGPU_ERR_ARG;
  }
  unsigned long long *d = nullptr;
  PDGPU_CUDA(cudaMalloc(&d, 5 * sizeof(unsigned long long)));
  cudaMemsetAsync(d, 0, 5 * sizeof(unsigned long long), c->st);
  launch_pair_counts(P.v, c->st, d);
  if (!P.v.tile_mode) {  // the tiles of the current list, for the counts
    int re = pack_ensure_tiles(&P);
    if (re) {
      cudaFree(d);
      return re;
    }
    launch_tiles_build(P.v, c->st);
  }
  launch_tile_counts(P.v, c->st, d + 3);
  unsigned long long h[5];
  cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, c->st);
  r = sync_check(c, "pair_counts");
  cudaFree(d);
  if (r) return r;
  for (int q = 0; q < 5; q++) counts[q] = (int64_t)h[q];
  return PDGPU_OK;
}

int pdgpu_profile_pair_kernels(pdgpu_ctx *c, int32_t sys, int32_t reps, double *ms) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = ready_pairs(c, e);
  if (r) return r;
  if (!ms || reps <= 0) {
    set_error("ms is NULL or reps <= 0");
    return PDGPU_ERR_ARG;
  }
  cudaEvent_t ev[4];
  for (int q = 0; q < 4; q++) cudaEventCreate(&ev[q]);
  double acc[3] = {0, 0, 0};
  for (int it = 0; it < reps; it++) {
    launch_zero(P.v, c->st);
    cudaEventRecord(ev[0], c->st);
    launch_born_radii(P.v, c->st);
    cudaEventRecord(ev[1], c->st);
    launch_gb_pair(P.v, c->st);
    cudaEventRecord(ev[2], c->st);
    launch_gb_chain(P.v, c->st);
    cudaEventRecord(ev[3], c->st);
    r = sync_check(c, "profile");
    if (r) break;
    for (int q = 0; q < 3; q++) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      acc[q] += t;
    }
  }
  for (int q = 0; q < 4; q++) cudaEventDestroy(ev[q]);
  if (r) return r;
  for (int q = 0; q < 3; q++) ms[q] = acc[q] / reps;
  return PDGPU_OK;
}

// Device times of the LCPO term's two launches (full evaluations at step
// 0; the forces they add are left in the accumulators) and the work they
// did: out[0] list ms, out[1] evaluation ms, out[2] overlap partners kept,
// out[3] (atom, partner, partner's partner) triples of the inner loop,
// out[4] those whose third atom overlaps the first (the full inner body).
int pdgpu_profile_eval(pdgpu_ctx *c, int32_t sys, int32_t reps, double *ms, int64_t *counts) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = ready_pairs(c, e);
  if (r) return r;
  if (!ms || reps <= 0) {
    set_error("ms is NULL or reps <= 0");
    return PDGPU_ERR_ARG;
  }
  if (!P.v.tile_mode) {
    set_error("pdgpu_profile_eval: the handle is not on the cluster-pair tile layout");
    return PDGPU_ERR_STATE;
  }
  cudaError_t ce = profile_eval_tiles(P.v, c->st, reps, ms);
  if (ce != cudaSuccess) return cuda_fail(ce, "profile_eval");
  if ((r = sync_check(c, "profile_eval"))) return r;
  if ((r = barrier_check(c, P))) return r;
  if (counts) {
    // the still list a Born phase makes (an evaluation's chain phase
    // clears it, so it is counted after a Born phase alone)
    int h[4] = {0, 0, 0, 0};
    PDGPU_CUDA(cudaMemsetAsync(P.v.tile_count + 2, 0, 2 * sizeof(int), c->st));
    launch_born_phase_only(P.v, c->st);
    PDGPU_CUDA(cudaMemcpyAsync(h, P.v.tile_count, sizeof h, cudaMemcpyDeviceToHost, c->st));
    if ((r = sync_check(c, "profile_eval counts"))) return r;
    counts[0] = h[0];
    counts[1] = h[2];
    // clear the list the lone Born phase left, and the sums it added
    PDGPU_CUDA(cudaMemsetAsync(P.v.tile_count + 2, 0, 2 * sizeof(int), c->st));
    PDGPU_CUDA(cudaMemsetAsync(P.v.bsum, 0, sizeof(long long) * P.v.n_atoms, c->st));
    // tiles each phase redid in its careful form (a pair at a decision edge)
    int *stats = nullptr;
    PDGPU_CUDA(cudaMallocAsync((void **)&stats, 3 * sizeof(int), c->st));
    PDGPU_CUDA(cudaMemsetAsync(stats, 0, 3 * sizeof(int), c->st));
    ce = count_deferred_tiles(P.v, c->st, stats);
    int d[3] = {0, 0, 0};
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d, stats, sizeof d, cudaMemcpyDeviceToHost, c->st);
    cudaFreeAsync(stats, c->st);
    if (ce != cudaSuccess) return cuda_fail(ce, "profile_eval deferred");
    if ((r = sync_check(c, "profile_eval counts"))) return r;
    for (int k = 0; k < 3; k++) counts[2 + k] = d[k];
  }
  return PDGPU_OK;
}

int pdgpu_measure_pipe_peaks(pdgpu_ctx *c, double *out) {
  CHECK_CTX(c);
  if (!out) {
    set_error("out is NULL");
    return PDGPU_ERR_ARG;
  }
  cudaError_t ce = measure_pipe_peaks(c->st, out);
  if (ce != cudaSuccess) return cuda_fail(ce, "measure_pipe_peaks");
  return sync_check(c, "measure_pipe_peaks");
}

int pdgpu_eval_mode(pdgpu_ctx *c, int32_t sys, int32_t set, int32_t *current) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (set < -1 || set > 2) {
    set_error("pdgpu_eval_mode: set must be -1 (query), 0 (three launches), 1 (one cooperative launch) or 2 "
              "(cooperative for single evaluations, three launches inside MD step blocks)");
    return PDGPU_ERR_ARG;
  }
  if (set >= 0) {
    const bool one = set >= 1, md = set == 1;
    if (P.coop_md != md) e->drop_graph();
    P.coop = one;
    P.coop_md = md;
  }
  if (current) *current = P.coop ? (P.coop_md ? 1 : 2) : 0;
  return PDGPU_OK;
}

int pdgpu_profile_lcpo(pdgpu_ctx *c, int32_t sys, int32_t reps, double *out) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (!out || reps <= 0) {
    set_error("out is NULL or reps <= 0");
    return PDGPU_ERR_ARG;
  }
  int r = lcpo_ready(c, e);
  if (r) return r;
  cudaEvent_t ev[3];
  for (int q = 0; q < 3; q++) cudaEventCreate(&ev[q]);
  double acc[2] = {0, 0};
  for (int it = 0; it < reps; it++) {
    cudaEventRecord(ev[0], c->st);
    launch_lcpo_part(P.v, c->st, StepSrc(), false, P.csr_stale, 0);
    cudaEventRecord(ev[1], c->st);
    launch_lcpo_part(P.v, c->st, StepSrc(), false, P.csr_stale, 1);
    cudaEventRecord(ev[2], c->st);
    r = sync_check(c, "profile_lcpo");
    if (r) break;
    for (int q = 0; q < 2; q++) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      acc[q] += t;
    }
  }
  for (int q = 0; q < 3; q++) cudaEventDestroy(ev[q]);
  if (r) return r;
  if ((r = lcpo_done(c, e, "profile_lcpo"))) return r;
  const size_t N = (size_t)P.v.n_atoms;
  std::vector<int> cnt(N), idx(N * kLcpoMax);
  std::vector<double> x(N), y(N), z(N), rad(N);
  PDGPU_CUDA(cudaMemcpy(cnt.data(), P.v.lc.cnt, sizeof(int) * N, cudaMemcpyDeviceToHost));
  PDGPU_CUDA(cudaMemcpy(idx.data(), P.v.lc.idx, sizeof(int) * N * kLcpoMax, cudaMemcpyDeviceToHost));
  PDGPU_CUDA(cudaMemcpy(x.data(), P.v.x, sizeof(double) * N, cudaMemcpyDeviceToHost));
  PDGPU_CUDA(cudaMemcpy(y.data(), P.v.y, sizeof(double) * N, cudaMemcpyDeviceToHost));
  PDGPU_CUDA(cudaMemcpy(z.data(), P.v.z, sizeof(double) * N, cudaMemcpyDeviceToHost));
  PDGPU_CUDA(cudaMemcpy(rad.data(), P.v.lc.r, sizeof(double) * N, cudaMemcpyDeviceToHost));
  double pairs = 0, triples = 0, overlapping = 0;
  for (size_t i = 0; i < N; i++) {
    pairs += cnt[i];
    for (int q = 0; q < cnt[i]; q++) {
      const int j = idx[i * kLcpoMax + q];
      triples += cnt[j];
      for (int t = 0; t < cnt[j]; t++) {
        const int k = idx[(size_t)j * kLcpoMax + t];
        const double dx = x[k] - x[i], dy = y[k] - y[i], dz = z[k] - z[i];
        const double rs = rad[i] + rad[k];
        if (k != (int)i && dx * dx + dy * dy + dz * dz <= rs * rs) overlapping++;
      }
    }
  }
  out[0] = acc[0] / reps;
  out[1] = acc[1] / reps;
  out[2] = pairs;
  out[3] = triples;
  out[4] = overlapping;
  return PDGPU_OK;
}

int pdgpu_autotune(pdgpu_ctx *c, int32_t sys, int32_t *lpa) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  int r = need_csr(c, e);
  if (r) return r;
  P.tuned = false;
  if ((r = ensure_tuned(c, P))) return r;
  e->drop_graph();
  if (lpa)
    for (int q = 0; q < 3; q++) lpa[q] = P.v.lpa[q];
  return PDGPU_OK;
}

int pdgpu_set_lanes(pdgpu_ctx *c, int32_t sys, const int32_t *lpa) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  e->drop_graph();
  if (!lpa) {
    P.tuned = false;
    return PDGPU_OK;
  }
  for (int q = 0; q < 3; q++)
    if (lpa[q] != 4 && lpa[q] != 8 && lpa[q] != 16 && lpa[q] != 32) {
      set_error("lanes per atom must be 4, 8, 16 or 32");
      return PDGPU_ERR_ARG;
    }
  for (int q = 0; q < 3; q++) P.v.lpa[q] = lpa[q];
  P.v.tile_mode = 0;  // the row path, with these lanes
  P.tuned = true;
  return PDGPU_OK;
}

int pdgpu_pair_path(pdgpu_ctx *c, int32_t sys, int32_t set, int32_t *current) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  Pack &P = *e->pack;
  if (set < -2 || set > 1) {
    set_error("pdgpu_pair_path: set must be -2 (query), -1 (tune), 0 (rows) or 1 (tiles)");
    return PDGPU_ERR_ARG;
  }
  if (set != -2) {
    e->drop_graph();
    if (set == -1) {
      P.tuned = false;
    } else {
      P.v.tile_mode = set;
      P.tuned = true;
      if (set == 1) {
        int re = pack_ensure_tiles(&P);
        if (re) return re;
        // tiles for the current list (after a tile search they are current already)
        if (P.have_list && !P.csr_stale) launch_tiles_build(P.v, c->st);
      }
      int r = sync_check(c, "pair_path");
      if (r) return r;
    }
  }
  if (current) *current = P.v.tile_mode;
  return PDGPU_OK;
}

int pdgpu_launch_count(pdgpu_ctx *c, int64_t *count) {
  CHECK_CTX(c);
  if (!count) {
    set_error("count is NULL");
    return PDGPU_ERR_ARG;
  }
  *count = launch_counter().load();
  return PDGPU_OK;
}

int pdgpu_graph_replays(pdgpu_ctx *c, int32_t sys, int64_t *replays) {
  CHECK_CTX(c);
  GET_SYS(e, c, sys);
  if (!replays) {
    set_error("replays is NULL");
    return PDGPU_ERR_ARG;
  }
  replays[0] = e->graph_replays;
  replays[1] = (int64_t)e->gslots.size();
  return PDGPU_OK;
}

int pdgpu_last_run_ms(pdgpu_ctx *c, double *ms) {
  CHECK_CTX(c);
  if (!ms) {
    set_error("ms is NULL");
    return PDGPU_ERR_ARG;
  }
  *ms = c->last_ms;
  return PDGPU_OK;
}

}  // extern "C"
