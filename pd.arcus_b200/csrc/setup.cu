// Host-side setup: constants, bond-order band, Still fixed terms, per-system
// kernel parameters and Pack allocation.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "internal.cuh"

namespace pdgpu {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
const char *last_error_cstr() { return g_err.c_str(); }
int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? PDGPU_ERR_NOMEM : PDGPU_ERR_CUDA;
}

// forcefields/forcefield.cpp:18-38 -- same expressions, same order.
const Consts &consts() {
  static Consts c = [] {
    Consts k;
    double e_charge = 1.60217645E-19;
    double sqr_e_charge = e_charge * e_charge;
    double e0 = 8.854187817E-12;
    double _4pi_e0 = (3.14159265358979323846 * 4.0) * e0;
    k.kcal2J = 4184.0;
    k.J2kcal = 1.0 / k.kcal2J;
    k.Na = 6.0221418E23;
    k.kB = 1.38065E-23;
    k.Angstrom = 1E-10;
    k.econv = (k.J2kcal * k.Na * sqr_e_charge) / (_4pi_e0 * k.Angstrom);
    k.halfeconv = k.econv * 0.5;
    k.econv_joule = sqr_e_charge / (_4pi_e0 * k.Angstrom);
    k.halfeconv_joule = k.econv_joule * 0.5;
    k.J_per_kcalmol = k.kcal2J / k.Na;
    k.N_per_kcalmolA = k.J_per_kcalmol / k.Angstrom;
    return k;
  }();
  return c;
}

// BondOrder::reinit (workspace/bondorder.cpp:77-195).  Band width: largest
// index distance of a 1-2/1-3/1-4 partner in the same or an adjacent residue,
// plus one.  The band is filled 1-4, 1-3, 1-2 (later writes win); partners
// farther apart than the band go to a sparse list, whose last entry for a
// pair wins when the neighbour list is corrected (neighbourlist.cpp:162-203).
int host_bondorder(SystemHost &s, std::string *err) {
  const int n = s.natoms;
  const std::vector<int> *P[3] = {&s.c12p, &s.c13p, &s.c14p};
  const std::vector<int> *I[3] = {&s.c12i, &s.c13i, &s.c14i};
  int mid = 0;
  for (int i = 0; i < n; i++)
    for (int l = 0; l < 3; l++)
      for (int k = (*P[l])[i]; k < (*P[l])[i + 1]; k++) {
        int lookup = (*I[l])[k];
        if (lookup < 0 || lookup >= n) {
          if (err) *err = "covalent partner index out of range";
          return PDGPU_ERR_ARG;
        }
        if (std::abs(s.residue[i] - s.residue[lookup]) > 1) continue;
        mid = std::max(mid, std::abs(i - lookup));
      }
  mid += 1;
  s.mid = mid;
  s.band.assign((size_t)mid * (size_t)(n > 1 ? n - 1 : 0), (int8_t)7);
  std::map<std::pair<int, int>, int> sparse;  // last write wins
  const int lists[3] = {2, 1, 0};
  const int orders[3] = {3, 2, 1};
  for (int i = 0; i < n; i++)
    for (int t = 0; t < 3; t++) {
      int l = lists[t];
      for (int k = (*P[l])[i]; k < (*P[l])[i + 1]; k++) {
        int j = (*I[l])[k];
        if (j <= i) continue;
        int delta = j - i;
        int order = std::min(orders[t], 7);
        if (delta > mid)
          sparse[std::make_pair(i, j)] = order;
        else
          s.band[(size_t)i * mid + (delta - 1)] = (int8_t)order;
      }
    }
  s.off_i.clear();
  s.off_j.clear();
  s.off_o.clear();
  for (auto &kv : sparse) {
    s.off_i.push_back(kv.first.first);
    s.off_j.push_back(kv.first.second);
    s.off_o.push_back(kv.second);
  }
  return PDGPU_OK;
}

// FF_GeneralizedBorn_Still::calcFixedBornRadiiTerms (gbff.cpp:307-381).
void host_gb_fixed_terms(SystemHost &s) {
  const double PI = 3.14159265358979323846;
  const double FourPI = 4.0 * PI;
  const int n = s.natoms;
  const pdgpu_ff_params &p = s.params;
  s.vj.assign(n, 0.0);
  s.terms123.assign(n, 0.0);
  auto sq = [](double x) { return x * x; };
  for (int j = 0; j < n; j++) {
    double Rj = s.gbR[j];
    if (Rj <= 0.01) Rj = 1.15;
    double v = FourPI * Rj * Rj * Rj / 3;
    for (int nk = s.c12p[j]; nk < s.c12p[j + 1]; nk++) {
      int k = s.c12i[nk];
      double Rk = s.gbR[k];
      if (Rk <= 0.01) Rk = 1.15;
      double rjk = 1.01 * s.c12d[nk];
      double hjk = Rj * (1.0 + (sq(Rk) - sq(Rj) - sq(rjk)) / (2.0 * Rj * rjk));
      v -= PI * sq(hjk) * (3 * Rj - hjk) / 3;
    }
    s.vj[j] = v < 0 ? 0 : v;
  }
  for (int i = 0; i < n; i++) {
    double Rj = s.gbR[i];
    if (Rj <= 0.01) Rj = 1.15;
    double term1 = -166.0 / (Rj + p.DielectricOffset + p.P1);
    double term2 = 0, term3 = 0;
    for (int nj = s.c12p[i]; nj < s.c12p[i + 1]; nj++) {
      double rij = s.c12d[nj];
      term2 += p.P2 * s.vj[s.c12i[nj]] / (sq(rij) * sq(rij));
    }
    for (int nj = s.c13p[i]; nj < s.c13p[i + 1]; nj++) {
      double rij = s.c13d[nj];
      term3 += p.P3 * s.vj[s.c13i[nj]] / (sq(rij) * sq(rij));
    }
    s.terms123[i] = term1 + term2 + term3;
  }
}

// Kernel-unit settings for one system.
SysParams make_sys_params(const pdgpu_ff_params &p) {
  const Consts &c = consts();
  SysParams s;
  memset(&s, 0, sizeof s);
  auto sq = [](double x) { return x * x; };
  auto cube = [](double x) { return x * x * x; };
  double Rc = p.Cutoff, Ri = p.InnerCutoff;
  s.rc2 = (float)sq(Rc);
  s.rc2_d = sq(Rc);
  s.rc = (float)Rc;
  s.rin = (float)Ri;
  s.inv_sw2 = (float)sq(1.0 / (Rc - Ri));
  s.vdw_rc = (float)p.VdwCutoff;
  s.vdw_rin = (float)p.VdwInnerCutoff;
  s.vdw_inv_sw2 = (float)sq(1.0 / (p.VdwCutoff - p.VdwInnerCutoff));
  s.vdw14 = (float)p.Vdw14Scaling;
  s.elec14 = (float)p.Elec14Scaling;
  s.econv_in = (float)(c.econv / p.DielectricSolute);
  s.econv_out = (float)(c.econv / p.DielectricSolvent);
  double premul_kcal = -c.halfeconv * (1 / p.DielectricSolute - 1 / p.DielectricSolvent);
  s.premul = (float)premul_kcal;
  s.premul_d = premul_kcal;
  s.exp_thresh = (float)p.ExpApproxThreshold;
  s.exp_thresh_d = p.ExpApproxThreshold;
  s.still2 = (float)sq(p.GbsaStillCutoff);
  s.still2_d = sq(p.GbsaStillCutoff);
  s.P4 = (float)p.P4;
  s.P5 = (float)p.P5;
  s.invP5 = (float)(1 / p.P5);
  s.P5_d = p.P5;
  s.invP5_d = 1 / p.P5;
  s.piP5 = (float)(p.P5 * 3.14159265358979323846);
  s.halfeconv_d = c.halfeconv;
  s.born_offset_d = p.BornRadiusOffset;
  double lc = std::max(p.Cutoff, p.VdwCutoff) + p.Padding;
  s.nl_lim2_d = sq(lc);
  // stand-alone LJ/Coulomb (nonbonded.cpp:1205-1229 mode selection)
  s.dielectric = (float)p.Dielectric;
  s.ddd_alpha = (float)p.DDDielectricAlpha;
  s.econv_nb = (float)(c.econv / p.Dielectric);
  // (the DDDielectric flag is not consulted here by the reference: its
  // calcForces and calcEnergies pick plain, energy-switched or
  // force-switched Coulomb only)
  int em = 1;
  if (p.EnergySwitch) em = 3;
  if (p.ForceSwitch) em = 4;
  if (!p.DoElec) em = 0;
  s.elec_mode = em;
  s.vdw_mode = p.DoVdw ? 2 : 0;
  s.fast_mode = p.FastMode;
  double sA = 1.0 / cube(sq(Rc) - sq(Ri));
  double sB = -(cube(sq(Rc)) - 3.0 * sq(Rc) * sq(Rc) * sq(Ri));
  double sC = 6.0 * sq(Rc) * sq(Ri);
  double sD = -(sq(Rc) + sq(Ri));
  double sE = 2.0 / 5.0;
  double fin = sA * (sB * (1.0 / Ri) + sC * Ri + sD * cube(Ri) + sE * cube(Ri) * sq(Ri));
  double fcut = sA * (sB * (1.0 / Rc) + sC * Rc + sD * cube(Rc) + sE * cube(Rc) * sq(Rc));
  s.fs_A = (float)sA;
  s.fs_B = (float)sB;
  s.fs_C = (float)sC;
  s.fs_D = (float)sD;
  s.fs_E = (float)sE;
  s.fs_cutV = (float)fcut;
  s.fs_eshift = (float)(Ri < Rc ? 1 / Ri + (fin - fcut) : 0.0);
  if (p.VdwCor) {
    // nonbonded.cpp:845-857, J -> kcal/mol
    double vp = -0.5 * p.VdwCorDensity * p.VdwCorEpsilon * (8.0 / 3.0) * 3.14159265358979323846 *
                sq(p.VdwCorRadius) * sq(p.VdwCorRadius) * sq(p.VdwCorRadius) / cube(p.VdwCorCutoff);
    s.vdwcor_e_d = vp;
    s.vdwcor_e = (float)vp;
  }
  return s;
}

// ----------------------------------------------------------------- Pack
Pack::~Pack() {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  for (void *a : allocs) cudaFreeAsync(a, st);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  if (fork2) cudaEventDestroy(fork2);
  for (auto &ev : ene_done)
    if (ev) cudaEventDestroy(ev);
  if (side) cudaStreamDestroy(side);
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
}

template <typename T>
static cudaError_t palloc(Pack *p, T **ptr, size_t count) {
  // stream-ordered allocation from the device's memory pool: packs are
  // created and freed often (batches, served jobs) and the pool keeps the
  // memory instead of returning it to the driver each time
  size_t bytes = sizeof(T) * (count > 0 ? count : 1);
  cudaError_t e = cudaMallocAsync((void **)ptr, bytes, p->st);
  if (e == cudaSuccess) {
    p->allocs.push_back((void *)*ptr);
    p->bytes += (int64_t)bytes;
    e = cudaMemsetAsync(*ptr, 0, bytes, p->st);
  }
  return e;
}

// The cluster-pair tile store (worst-case capacity), allocated the first
// time a pack uses or times the tile layout.
int pack_ensure_tiles(Pack *p) {
  PackView &v = p->v;
  if (v.tile_meta || v.n_sc == 0) return PDGPU_OK;
  if (palloc(p, &v.tile_meta, (size_t)v.tile_cap) != cudaSuccess ||
      palloc(p, &v.tile_rows, 8 * (size_t)v.tile_cap) != cudaSuccess ||
      palloc(p, &v.spec_rows, 16 * (size_t)v.spec_cap) != cudaSuccess ||
      palloc(p, &v.cbox, 6 * (size_t)v.n_jc) != cudaSuccess ||
      palloc(p, &v.xs, 3 * (size_t)v.n_atoms) != cudaSuccess ||
      palloc(p, &v.still_list, (size_t)v.tile_cap) != cudaSuccess ||
      palloc(p, &v.defer_list, (size_t)v.tile_cap) != cudaSuccess) {
    set_error("device allocation failed (cluster-pair tiles)");
    return PDGPU_ERR_NOMEM;
  }
  return PDGPU_OK;
}

// FF_SASA_LCPO parameters of every member (members without the term have
// use 0 on every atom) and the term's state, allocated the first time;
// enqueued on p->st.  All members share one UpdateSasa.
int pack_upload_lcpo(Pack *p, const std::vector<const SystemHost *> &systems) {
  PackView &v = p->v;
  LcpoView &lc = v.lc;
  const size_t N = (size_t)v.n_atoms;
  int update = 0;
  for (auto *h : systems)
    if (h->lcpo_update > 0) {
      if (update && update != h->lcpo_update) {
        set_error("batch members have different UpdateSasa values");
        return PDGPU_ERR_ARG;
      }
      update = h->lcpo_update;
    }
  lc.update = 0;
  if (!update) return PDGPU_OK;
  if (!lc.r) {
    double *r = nullptr, *sig = nullptr;
    double4 *p4 = nullptr;
    unsigned char *use = nullptr;
    int *atoms = nullptr;
    if (palloc(p, &r, N) != cudaSuccess || palloc(p, &p4, N) != cudaSuccess || palloc(p, &sig, N) != cudaSuccess ||
        palloc(p, &use, N) != cudaSuccess || palloc(p, &atoms, N) != cudaSuccess || palloc(p, &lc.cnt, N) != cudaSuccess ||
        palloc(p, &lc.idx, N * kLcpoMax) != cudaSuccess || palloc(p, &lc.s, N * kLcpoMax) != cudaSuccess ||
        palloc(p, &lc.sasa, N) != cudaSuccess || palloc(p, &lc.deriv, 3 * N) != cudaSuccess ||
        palloc(p, &lc.cand_n, N) != cudaSuccess || palloc(p, &lc.cand, N * kLcpoCand) != cudaSuccess ||
        palloc(p, &lc.xr, N) != cudaSuccess) {
      set_error("device allocation failed (LCPO surface term)");
      return PDGPU_ERR_NOMEM;
    }
    lc.r = r;
    lc.p = p4;
    lc.sigma = sig;
    lc.use = use;
    lc.atoms = atoms;
  }
  std::vector<double> r(N, 0.0), sig(N, 0.0);
  std::vector<double4> p4(N, make_double4(0, 0, 0, 0));
  std::vector<unsigned char> use(N, 0);
  for (size_t k = 0; k < systems.size(); k++) {
    const SystemHost &h = *systems[k];
    if (h.lcpo_update <= 0) continue;
    const int o = p->atom_off[k];
    for (int i = 0; i < h.natoms; i++) {
      r[o + i] = h.lcpo_r[i];
      p4[o + i] = make_double4(h.lcpo_p[4 * i], h.lcpo_p[4 * i + 1], h.lcpo_p[4 * i + 2], h.lcpo_p[4 * i + 3]);
      sig[o + i] = h.lcpo_sigma[i];
      use[o + i] = h.lcpo_use[i];
    }
  }
  std::vector<int> atoms;
  for (size_t i = 0; i < N; i++)
    if (use[i]) atoms.push_back((int)i);
  cudaStream_t st = p->st;
  // an atom leaving the term keeps no stale area, energy or derivative
  cudaMemsetAsync(lc.cnt, 0, sizeof(int) * N, st);
  cudaMemsetAsync(lc.sasa, 0, sizeof(double) * N, st);
  cudaMemsetAsync(lc.deriv, 0, sizeof(double) * 3 * N, st);
  cudaMemsetAsync(v.e_atom + (size_t)AE_SURF * N, 0, sizeof(double) * N, st);
  if ((!atoms.empty() &&
       cudaMemcpyAsync((void *)lc.atoms, atoms.data(), sizeof(int) * atoms.size(), cudaMemcpyHostToDevice, st) !=
           cudaSuccess) ||
      cudaMemcpyAsync((void *)lc.r, r.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync((void *)lc.p, p4.data(), sizeof(double4) * N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync((void *)lc.sigma, sig.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync((void *)lc.use, use.data(), N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    set_error("LCPO parameter upload failed");
    return PDGPU_ERR_CUDA;
  }
  lc.n_used = (int)atoms.size();
  lc.update = update;
  return PDGPU_OK;
}

int pack_ensure_stage(Pack *p) {
  if (p->stage) return PDGPU_OK;
  if (palloc(p, &p->stage, 3 * (size_t)p->v.n_atoms) != cudaSuccess || cudaStreamSynchronize(p->st) != cudaSuccess) {
    set_error("device allocation failed (state staging)");
    return PDGPU_ERR_NOMEM;
  }
  return PDGPU_OK;
}

// The evaluation kernel's lean build serves a pack whose systems all run
// FastMode with the LJ switch equal to the GB/Coulomb one.
static void pack_update_lean(Pack *p) {
  p->v.ev_lean = 1;
  for (const SysParams &q : p->sp)
    if (q.fast_mode == 0 || q.vdw_rin != q.rin || q.vdw_inv_sw2 != q.inv_sw2) p->v.ev_lean = 0;
}

void pack_set_params(Pack *p, int s, const pdgpu_ff_params &prm) {
  p->sp[s] = make_sys_params(prm);
  pack_update_lean(p);
}

#define PALLOC(ptr, n)                                        \
  do {                                                        \
    cudaError_t e_ = palloc(p, &(ptr), (n));                  \
    if (e_ != cudaSuccess) {                                  \
      if (err) *err = std::string("cudaMalloc failed: ") + cudaGetErrorString(e_); \
      delete p;                                               \
      return nullptr;                                         \
    }                                                         \
  } while (0)

void dihedral_sets(SystemHost &h) {
  const int n = h.nt + h.ni;
  std::map<std::array<double, 13>, int> seen;
  h.dih_set.assign(n, 0);
  h.dih_sets.clear();
  for (int q = 0; q < n; q++) {
    std::array<double, 13> key;
    std::copy(h.tpar.begin() + 12 * (size_t)q, h.tpar.begin() + 12 * (size_t)q + 12, key.begin());
    key[12] = (double)h.tterms[q];
    auto it = seen.find(key);
    if (it == seen.end()) {
      it = seen.emplace(key, (int)(h.dih_sets.size() / 13)).first;
      h.dih_sets.insert(h.dih_sets.end(), key.begin(), key.end());
    }
    h.dih_set[q] = it->second;
  }
}

Pack *pack_create(int device, cudaStream_t st, const std::vector<const SystemHost *> &systems,
                  std::string *err, bool sync) {
  const Consts &c = consts();
  Pack *p = new Pack();
  p->device = device;
  p->st = st;
  int S = (int)systems.size();
  int N = 0;
  p->atom_off.push_back(0);
  for (auto *s : systems) {
    N += s->natoms;
    p->atom_off.push_back(N);
  }
  PackView &v = p->v;
  v.n_atoms = N;
  v.n_sys = S;
  // host staging
  std::vector<int> sys_of(N);
  std::vector<float4> pq(2 * (size_t)N, make_float4(0, 0, 0, 0)), chainp(N), prm(N);
  std::vector<double4> xyzp(N);
  std::vector<double> gbR(N), pv(N), t123(N), minv(N), mass(N), X(N), Y(N), Z(N);
  std::vector<int> mid(S);
  std::vector<long long> band_off(S);
  std::vector<int8_t> band;
  std::vector<int> off_ptr(N + 1, 0);
  std::vector<std::vector<int2>> offl(N);
  double sqrt_eps_scale = std::sqrt(c.J2kcal * c.Na);
  for (int s = 0; s < S; s++) {
    const SystemHost &h = *systems[s];
    p->sp.push_back(make_sys_params(h.params));
    int o = p->atom_off[s];
    for (int i = 0; i < h.natoms; i++) {
      int g = o + i;
      sys_of[g] = s;
      prm[g] = make_float4((float)h.radius[i], (float)(h.epsilon[i] * sqrt_eps_scale), (float)h.gbR[i],
                           (float)h.vj[i]);
      pq[2 * (size_t)g] = make_float4(0, 0, 0, (float)h.charge[i]);
      chainp[g] = make_float4((float)h.gbR[i], (float)h.vj[i], 0.f, 0.f);
      gbR[g] = h.gbR[i];
      pv[g] = h.params.P4 * h.vj[i];
      xyzp[g] = make_double4(0, 0, 0, pv[g]);
      t123[g] = h.terms123[i];
      minv[g] = 1.0 / h.mass[i];
      mass[g] = h.mass[i];
    }
    mid[s] = h.mid;
    band_off[s] = (long long)band.size();
    band.insert(band.end(), h.band.begin(), h.band.end());
    for (size_t k = 0; k < h.off_i.size(); k++) {
      int a = o + h.off_i[k], b = o + h.off_j[k];
      offl[a].push_back(make_int2(b, h.off_o[k]));
      offl[b].push_back(make_int2(a, h.off_o[k]));
    }
  }
  std::vector<int2> off_data;
  for (int i = 0; i < N; i++) {
    off_ptr[i] = (int)off_data.size();
    off_data.insert(off_data.end(), offl[i].begin(), offl[i].end());
  }
  off_ptr[N] = (int)off_data.size();

  // cluster-pair tiles: i-clusters of 32 and j-clusters of 8 atoms per
  // system in atom order; capacities are worst cases (no overflow path):
  // every j-cluster at or after an i-cluster, and for the bond-order rows
  // every tile within MaxIndexDelta of it plus one per off-diagonal pair
  std::vector<int> sc_atom0, sc_sys, sc_jc0, jc_atom0, jc_off(S + 1, 0);
  long long tile_cap = 0, spec_cap = 0;
  int max_sys = 0;
  for (int s = 0; s < S; s++) {
    int o = p->atom_off[s], n = systems[s]->natoms;
    max_sys = std::max(max_sys, n);
    int nsc = (n + 31) / 32, njc = (n + 7) / 8;
    jc_off[s] = (int)jc_atom0.size();
    for (int k = 0; k < nsc; k++) {
      sc_atom0.push_back(o + 32 * k);
      sc_sys.push_back(s);
      sc_jc0.push_back(jc_off[s] + 4 * k);
      tile_cap += njc - 4 * k;
    }
    for (int k = 0; k < njc; k++) jc_atom0.push_back(o + 8 * k);
    spec_cap += (long long)nsc * ((32 + systems[s]->mid) / 8 + 3);
  }
  jc_off[S] = (int)jc_atom0.size();
  spec_cap += (long long)off_data.size();

  // device allocations
  int *atom_off_d, *sys_of_d, *mid_d, *off_ptr_d;
  SysParams *sp_d;
  long long *band_off_d;
  int8_t *band_d;
  int2 *off_data_d;
  float4 *prm_d;
  double *gbR_d, *pv_d, *t123_d, *minv_d, *mass_d;
  PALLOC(atom_off_d, S + 1);
  PALLOC(sys_of_d, N);
  PALLOC(sp_d, S);
  PALLOC(mid_d, S);
  PALLOC(band_off_d, S);
  PALLOC(band_d, band.size());
  PALLOC(off_ptr_d, N + 1);
  PALLOC(off_data_d, off_data.size());
  PALLOC(prm_d, N);
  PALLOC(gbR_d, N);
  PALLOC(pv_d, N);
  PALLOC(t123_d, N);
  PALLOC(minv_d, N);
  PALLOC(mass_d, N);
  PALLOC(v.x, N);
  PALLOC(v.y, N);
  PALLOC(v.z, N);
  PALLOC(v.vx, N);
  PALLOC(v.vy, N);
  PALLOC(v.vz, N);
  PALLOC(v.ox, N);
  PALLOC(v.oy, N);
  PALLOC(v.oz, N);
  PALLOC(v.pq, 2 * (size_t)N);
  PALLOC(v.xyzp, N);
  PALLOC(v.chainp, N);
  PALLOC(v.born_d, N);
  PALLOC(v.gx, N);
  PALLOC(v.gy, N);
  PALLOC(v.gz, N);
  PALLOC(v.fx, N);
  PALLOC(v.fy, N);
  PALLOC(v.fz, N);
  PALLOC(v.fox, N);
  PALLOC(v.foy, N);
  PALLOC(v.foz, N);
  PALLOC(v.dirx, N);
  PALLOC(v.diry, N);
  PALLOC(v.dirz, N);
  PALLOC(v.odx, N);
  PALLOC(v.ody, N);
  PALLOC(v.odz, N);
  PALLOC(v.e_atom, (size_t)AE_COUNT * N);
  PALLOC(v.ene, (size_t)E_COUNT * S);
  PALLOC(v.row_start, N + 1);
  PALLOC(v.row_cnt, N);
  PALLOC(v.cell_key, N);
  PALLOC(v.sorted_atom, N);
  v.cell_cap = 2 * N + 64 * S;
  PALLOC(v.cell_start, v.cell_cap);
  PALLOC(v.cell_end, v.cell_cap);
  PALLOC(v.grid, (size_t)8 * S);
  PALLOC(v.bbox, (size_t)6 * S);
  PALLOC(v.flags, F_COUNT);
  PALLOC(v.sys_flags, S);
  PALLOC(v.e_pair_alt, (size_t)4 * N);
  PALLOC(v.sys_flags_alt, S);
  v.ebuf = 0;
  PALLOC(p->tmp_keys, N);
  PALLOC(p->tmp_vals, N);
  int tiles = (N + 2047) / 2048;
  PALLOC(p->sort_hist, 256 * (size_t)(tiles > 0 ? tiles : 1));
  p->scan_tmp_len = (N + 1023) / 1024 + 1;
  PALLOC(p->scan_tmp, p->scan_tmp_len + 1);
  PALLOC(p->red_tmp, 4096);
  v.nl_cap = (long long)N * 48 + 4096;
  PALLOC(v.nl, (size_t)v.nl_cap);
  int bits = 1;
  while ((1LL << bits) < (long long)v.cell_cap) bits++;
  p->radix_passes = (bits + 7) / 8;
  // cluster-pair tiles and the accumulators of the tile passes
  {
    int *sc_atom0_d, *sc_sys_d, *sc_jc0_d, *jc_atom0_d, *jc_off_d;
    v.n_sc = (int)sc_atom0.size();
    v.n_jc = (int)jc_atom0.size();
    v.max_sys_atoms = max_sys;
    v.tile_cap = tile_cap;
    v.spec_cap = spec_cap;
    tile_launch_shapes(v);
    PALLOC(sc_atom0_d, sc_atom0.size());
    PALLOC(sc_sys_d, sc_sys.size());
    PALLOC(sc_jc0_d, sc_jc0.size());
    PALLOC(jc_atom0_d, jc_atom0.size());
    PALLOC(jc_off_d, jc_off.size());
    if (!jc_atom0.empty()) {
      cudaMemcpyAsync(sc_jc0_d, sc_jc0.data(), sizeof(int) * sc_jc0.size(), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(jc_atom0_d, jc_atom0.data(), sizeof(int) * jc_atom0.size(), cudaMemcpyHostToDevice, st);
    }
    cudaMemcpyAsync(jc_off_d, jc_off.data(), sizeof(int) * jc_off.size(), cudaMemcpyHostToDevice, st);
    v.sc_jc0 = sc_jc0_d;
    v.jc_atom0 = jc_atom0_d;
    v.jc_off = jc_off_d;
    PALLOC(v.tile_count, 4);  // the tile store itself: pack_ensure_tiles, on first use
    PALLOC(v.bsum, N);
    PALLOC(v.hx, N);
    PALLOC(v.hy, N);
    PALLOC(v.hz, N);
    PALLOC(v.ej, 4 * (size_t)N);
    if (!sc_atom0.empty()) {
      cudaMemcpyAsync(sc_atom0_d, sc_atom0.data(), sizeof(int) * sc_atom0.size(), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(sc_sys_d, sc_sys.data(), sizeof(int) * sc_sys.size(), cudaMemcpyHostToDevice, st);
    }
    v.sc_atom0 = sc_atom0_d;
    v.sc_sys = sc_sys_d;
    v.tile_mode = 0;
  }

  cudaMemcpyAsync(atom_off_d, p->atom_off.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(sys_of_d, sys_of.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(sp_d, p->sp.data(), sizeof(SysParams) * S, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(mid_d, mid.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(band_off_d, band_off.data(), sizeof(long long) * S, cudaMemcpyHostToDevice, st);
  if (!band.empty()) cudaMemcpyAsync(band_d, band.data(), band.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(off_ptr_d, off_ptr.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st);
  if (!off_data.empty())
    cudaMemcpyAsync(off_data_d, off_data.data(), sizeof(int2) * off_data.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(prm_d, prm.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(v.pq, pq.data(), sizeof(float4) * pq.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(v.xyzp, xyzp.data(), sizeof(double4) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(v.chainp, chainp.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(gbR_d, gbR.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(pv_d, pv.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(t123_d, t123.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(minv_d, minv.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(mass_d, mass.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st);
  v.atom_off = atom_off_d;
  v.sys_of = sys_of_d;
  v.sp = sp_d;
  pack_update_lean(p);
  v.mid = mid_d;
  v.band_off = band_off_d;
  v.band = band_d;
  v.off_ptr = off_ptr_d;
  v.off_data = off_data_d;
  v.prm = prm_d;
  v.gbR_d = gbR_d;
  v.pv_d = pv_d;
  v.terms123 = t123_d;
  v.inv_mass_si = minv_d;
  v.mass_si = mass_d;

  // bonded terms (converted to kcal/mol)
  BondedTerms &bt = v.bt;
  std::vector<int2> bij;
  std::vector<double2> blk, akt;
  std::vector<int4> aiaj, tidx;
  std::vector<int> tterms, ttype;
  std::vector<double> tpar;
  // dihedral parameter sets (few per forcefield): the pack's table holds
  // each once, in order of first appearance over the systems' terms
  std::map<std::array<double, 13>, int> types;
  std::vector<std::vector<int>> set_type(S);  // per system: its local sets' pack types (-1 not yet)
  std::vector<SystemHost> dih_fallback;        // systems whose sets were not formed (none expected)
  std::vector<const SystemHost *> dih_src(S);
  for (int s = 0; s < S; s++) {
    const SystemHost &h = *systems[s];
    dih_src[s] = &h;
    if (h.dih_set.size() != (size_t)(h.nt + h.ni)) {
      dih_fallback.reserve(S);
      dih_fallback.push_back(h);
      dihedral_sets(dih_fallback.back());
      dih_src[s] = &dih_fallback.back();
    }
    set_type[s].assign(dih_src[s]->dih_sets.size() / 13, -1);
  }
  double J2k = c.J2kcal * c.Na;
  for (int s = 0; s < S; s++) {
    const SystemHost &h = *systems[s];
    int o = p->atom_off[s];
    for (int k = 0; k < h.nb; k++) {
      bij.push_back(make_int2(o + h.bij[2 * k], o + h.bij[2 * k + 1]));
      blk.push_back(make_double2(h.blk[2 * k], h.blk[2 * k + 1] * J2k));
    }
    for (int k = 0; k < h.na; k++) {
      aiaj.push_back(make_int4(o + h.aiaj[3 * k], o + h.aiaj[3 * k + 1], o + h.aiaj[3 * k + 2], s));
      akt.push_back(make_double2(h.akt[2 * k] * J2k, h.akt[2 * k + 1]));
    }
  }
  for (int pass = 0; pass < 2; pass++)
    for (int s = 0; s < S; s++) {
      const SystemHost &h = *systems[s];
      int o = p->atom_off[s];
      int base = pass == 0 ? 0 : h.nt;
      int cnt = pass == 0 ? h.nt : h.ni;
      for (int k = 0; k < cnt; k++) {
        int q = base + k;
        tidx.push_back(make_int4(o + h.tidx[4 * q], o + h.tidx[4 * q + 1], o + h.tidx[4 * q + 2],
                                 o + h.tidx[4 * q + 3]));
        // the dihedral's parameter set, stored once per distinct set: the
        // kernel reads a 4-byte index per term and the table from cache
        const SystemHost &hd = *dih_src[s];
        const int local = hd.dih_set[q];
        int &ty = set_type[s][local];
        if (ty < 0) {
          std::array<double, 13> key;
          std::copy(hd.dih_sets.begin() + 13 * (size_t)local, hd.dih_sets.begin() + 13 * (size_t)local + 13,
                    key.begin());
          auto it = types.find(key);
          if (it == types.end()) {
            it = types.emplace(key, (int)tterms.size()).first;
            tterms.push_back(h.tterms[q]);
            for (int m = 0; m < 12; m++) {
              double val = h.tpar[12 * q + m];
              tpar.push_back(m < 4 ? val * J2k : val);
            }
            // cos and sin of each phase, so the kernel needs no transcendental
            // for the integer periodicities
            for (int m = 0; m < 4; m++) tpar.push_back(std::cos(h.tpar[12 * q + 8 + m]));
            for (int m = 0; m < 4; m++) tpar.push_back(std::sin(h.tpar[12 * q + 8 + m]));
          }
          ty = it->second;
        }
        ttype.push_back(ty);
      }
    }
  bt.nb = (int)bij.size();
  bt.na = (int)aiaj.size();
  int ndih = (int)tidx.size();
  int nt_all = 0;
  for (auto *s : systems) nt_all += s->nt;
  bt.nt = nt_all;
  bt.ni = ndih - nt_all;
  // per-system term ranges: bonds, angles, torsions, impropers (the last two
  // index the shared dihedral array: all torsions first, then impropers)
  std::vector<int> toff(4 * (S + 1), 0);
  int max_range = 0;
  for (int s = 0; s < S; s++) {
    const SystemHost &h = *systems[s];
    toff[s + 1] = toff[s] + h.nb;
    toff[(S + 1) + s + 1] = toff[(S + 1) + s] + h.na;
    toff[2 * (S + 1) + s + 1] = toff[2 * (S + 1) + s] + h.nt;
    max_range = std::max(max_range, std::max(std::max(h.nb, h.na), std::max(h.nt, h.ni)));
    max_range = std::max(max_range, h.natoms);
  }
  toff[3 * (S + 1)] = nt_all;
  for (int s = 0; s < S; s++) toff[3 * (S + 1) + s + 1] = toff[3 * (S + 1) + s] + systems[s]->ni;
  int *toff_d;
  PALLOC(toff_d, toff.size());
  cudaMemcpyAsync(toff_d, toff.data(), sizeof(int) * toff.size(), cudaMemcpyHostToDevice, st);
  bt.term_off = toff_d;
  PALLOC(bt.e_bond, bt.nb);
  PALLOC(bt.vir_bond, bt.nb);
  PALLOC(bt.e_angle, bt.na);
  PALLOC(bt.e_dih, ndih);
  // backbone torsion moves and hydrogen flags
  {
    std::vector<int2> rax;
    std::vector<unsigned char> rst;
    std::vector<int> roff(S + 1, 0), rlast(N, -1);
    std::vector<unsigned char> ish(N, 0);
    for (int s = 0; s < S; s++) {
      const SystemHost &h = *systems[s];
      int o = p->atom_off[s], r0 = (int)rax.size();
      for (size_t k = 0; k + 1 < h.rot_axis.size(); k += 2) {
        rax.push_back(make_int2(o + h.rot_axis[k], o + h.rot_axis[k + 1]));
        rst.push_back(h.rot_start[k / 2]);
      }
      roff[s + 1] = (int)rax.size();
      for (int i = 0; i < h.natoms && !h.rot_last.empty(); i++)
        rlast[o + i] = h.rot_last[i] < 0 ? -1 : r0 + h.rot_last[i];
      for (int i = 0; i < h.natoms && !h.is_h.empty(); i++) ish[o + i] = (unsigned char)h.is_h[i];
    }
    int2 *rax_d;
    int *roff_d, *rlast_d;
    unsigned char *rst_d;
    PALLOC(rax_d, rax.size());
    PALLOC(rst_d, rst.size());
    PALLOC(roff_d, S + 1);
    PALLOC(rlast_d, N);
    PALLOC(v.rot_xf, 12 * rax.size());
    PALLOC(p->is_h, N);
    if (!rax.empty()) {
      cudaMemcpyAsync(rax_d, rax.data(), sizeof(int2) * rax.size(), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(rst_d, rst.data(), rst.size(), cudaMemcpyHostToDevice, st);
    }
    cudaMemcpyAsync(roff_d, roff.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(rlast_d, rlast.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(p->is_h, ish.data(), N, cudaMemcpyHostToDevice, st);
    v.rot_axis = rax_d;
    v.rot_off = roff_d;
    v.rot_start = rst_d;
    v.rot_last = rlast_d;
    p->rot_total = (long long)rax.size();
    PALLOC(v.bx, N);
    PALLOC(v.by, N);
    PALLOC(v.bz, N);
  }
  v.lpa[0] = v.lpa[1] = v.lpa[2] = 8;
  v.e_chunks = (max_range + kReduceChunk - 1) / kReduceChunk;
  if (v.e_chunks < 1) v.e_chunks = 1;
  PALLOC(v.e_part, (size_t)S * v.e_chunks * kPartSlots);
  PALLOC(v.e_done, S);
  PALLOC(bt.bij, bij.size());
  PALLOC(bt.blk, blk.size());
  PALLOC(bt.aiaj, aiaj.size());
  PALLOC(bt.akt, akt.size());
  PALLOC(bt.tidx, tidx.size());
  PALLOC(bt.tterms, tterms.size());
  PALLOC(bt.ttype, ttype.size());
  PALLOC(bt.tpar, tpar.size());
  if (!bij.empty()) {
    cudaMemcpyAsync(bt.bij, bij.data(), sizeof(int2) * bij.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bt.blk, blk.data(), sizeof(double2) * blk.size(), cudaMemcpyHostToDevice, st);
  }
  if (!aiaj.empty()) {
    cudaMemcpyAsync(bt.aiaj, aiaj.data(), sizeof(int4) * aiaj.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bt.akt, akt.data(), sizeof(double2) * akt.size(), cudaMemcpyHostToDevice, st);
  }
  if (!tidx.empty()) {
    cudaMemcpyAsync(bt.tidx, tidx.data(), sizeof(int4) * tidx.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bt.tterms, tterms.data(), sizeof(int) * tterms.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bt.ttype, ttype.data(), sizeof(int) * ttype.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bt.tpar, tpar.data(), sizeof(double) * tpar.size(), cudaMemcpyHostToDevice, st);
  }
  if (pack_upload_lcpo(p, systems) != PDGPU_OK) {
    if (err) *err = last_error_cstr();
    delete p;
    return nullptr;
  }
  cudaEventCreate(&p->ev0);
  cudaEventCreate(&p->ev1);
  cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&p->fork2, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&p->ene_done[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&p->ene_done[1], cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking);
  cudaError_t e = sync ? cudaStreamSynchronize(st) : cudaGetLastError();
  if (e != cudaSuccess) {
    if (err) *err = std::string("pack upload failed: ") + cudaGetErrorString(e);
    delete p;
    return nullptr;
  }
  return p;
}

}  // namespace pdgpu
