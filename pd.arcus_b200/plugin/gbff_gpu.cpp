// FF_GeneralizedBorn_Still_GPU (gbff_gpu.h): the Still GB component of PD
// evaluated by libpdgpu.  Compiled against the reference's own headers
// (src/mmlib) and linked with the reference library and libpdgpu.so.
#include "gbff_gpu.h"

#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "exception.h"
#include "pdgpu.h"
#include "workspace/neighbourlist.h"
#include "workspace/workspace.h"

namespace Physics {

namespace {
// One libpdgpu context per device, shared by every component of the
// process (a context owns one CUDA stream; PD's protocols are
// single-threaded, so calls on it are serialised as the C ABI requires).
std::map<int, pdgpu_ctx *> &contexts() {
  static std::map<int, pdgpu_ctx *> m;
  return m;
}
}  // namespace
pdgpu_ctx *plugin_context(int device) {
  std::map<int, pdgpu_ctx *> &m = contexts();
  std::map<int, pdgpu_ctx *>::iterator it = m.find(device);
  if (it != m.end()) return it->second;
  pdgpu_ctx *c = 0;
  if (pdgpu_ctx_create(device, &c) != PDGPU_OK)
    throw ProcedureException(std::string("libpdgpu: ") + pdgpu_last_error());
  m[device] = c;
  return c;
}

FF_GeneralizedBorn_Still_GPU::FF_GeneralizedBorn_Still_GPU(WorkSpace &newwspace, int device)
    : FF_GeneralizedBorn_Still(newwspace), Device(device), m_ctx(0), m_sys(-1), m_listCount(0),
      m_haveList(false) {
  name = "Generalised Born (Still), B200";
}

// A copy gets its own device system at its first setup.
FF_GeneralizedBorn_Still_GPU::FF_GeneralizedBorn_Still_GPU(const FF_GeneralizedBorn_Still_GPU &other)
    : FF_GeneralizedBorn_Still(other), Device(other.Device), m_ctx(0), m_sys(-1), m_listCount(0),
      m_haveList(false) {
  needsetup = true;
}

FF_GeneralizedBorn_Still_GPU::~FF_GeneralizedBorn_Still_GPU() { release(); }

void FF_GeneralizedBorn_Still_GPU::release() {
  if (m_ctx && m_sys >= 0) pdgpu_system_destroy(m_ctx, m_sys);
  m_sys = -1;
  m_haveList = false;
}

void FF_GeneralizedBorn_Still_GPU::check(int status, const char *what) const {
  if (status == PDGPU_OK) return;
  std::string msg = std::string("libpdgpu ") + what + ": " + pdgpu_last_error();
  if (status == PDGPU_ERR_UNSTABLE) msg = "Simulation unstable or division by zero: " + msg;
  throw ProcedureException(msg);
}

void FF_GeneralizedBorn_Still_GPU::setup() {
  // the reference's own setup: parameter tables, GB radii per type, the
  // list cutoff request and shadow neighbours (gbff.cpp:40-87)
  FF_GeneralizedBorn_Still::setup();
  WorkSpace &wspace = getWSpace();
  const int n = (int)wspace.atom.size();
  release();
  m_ctx = plugin_context(Device);

  std::vector<double> q(n), rad(n), eps(n), mass(n), gbr(n);
  std::vector<int32_t> ir(n);
  std::vector<int32_t> c12p(1, 0), c13p(1, 0), c14p(1, 0), c12i, c13i, c14i;
  std::vector<double> c12d, c13d;
  for (int i = 0; i < n; i++) {
    const Particle &a = wspace.atom[i];
    q[i] = a.charge;
    rad[i] = a.radius;
    eps[i] = a.epsilon;
    mass[i] = a.mass;
    gbr[i] = GBtype[a.FFType].radius;
    ir[i] = a.ir;
    for (size_t k = 0; k < a.cov12atom.size(); k++) {
      c12i.push_back(a.cov12atom[k].i);
      c12d.push_back(a.cov12atom[k].d);
    }
    for (size_t k = 0; k < a.cov13atom.size(); k++) {
      c13i.push_back(a.cov13atom[k].i);
      c13d.push_back(a.cov13atom[k].d);
    }
    for (size_t k = 0; k < a.cov14atom.size(); k++) c14i.push_back(a.cov14atom[k].i);
    c12p.push_back((int32_t)c12i.size());
    c13p.push_back((int32_t)c13i.size());
    c14p.push_back((int32_t)c14i.size());
  }
  pdgpu_ff_params p;
  pdgpu_ff_params_default(&p);
  p.Cutoff = Cutoff;
  p.InnerCutoff = InnerCutoff;
  p.VdwCutoff = VdwCutoff;
  p.VdwInnerCutoff = VdwInnerCutoff;
  p.Vdw14Scaling = Vdw14Scaling;
  p.Elec14Scaling = Elec14Scaling;
  p.Dielectric = Dielectric;
  p.DielectricSolute = DielectricSolute;
  p.DielectricSolvent = DielectricSolvent;
  p.GbsaStillCutoff = GbsaStillCutoff;
  p.ExpApproxThreshold = ExpApproxThreshold;
  p.DielectricOffset = DielectricOffset;
  p.BornRadiusOffset = BornRadiusOffset;
  p.P1 = P1;
  p.P2 = P2;
  p.P3 = P3;
  p.P4 = P4;
  p.P5 = P5;
  p.DDDielectricAlpha = DDDielectricAlpha;
  p.VdwCorDensity = VdwCorDensity;
  p.VdwCorEpsilon = VdwCorEpsilon;
  p.VdwCorRadius = VdwCorRadius;
  p.VdwCorCutoff = VdwCorCutoff;
  p.FastMode = FastMode ? 1 : 0;
  p.EnergySwitch = EnergySwitch ? 1 : 0;
  p.ForceSwitch = ForceSwitch ? 1 : 0;
  p.DDDielectric = DDDielectric ? 1 : 0;
  p.DoVdw = DoVdw ? 1 : 0;
  p.DoElec = DoElec ? 1 : 0;
  p.VdwCor = VdwCor ? 1 : 0;
  int32_t sys = -1;
  check(pdgpu_system_create(m_ctx, n, &q[0], &rad[0], &eps[0], &mass[0], &gbr[0], &ir[0], &c12p[0],
                            c12i.empty() ? 0 : &c12i[0], c12d.empty() ? 0 : &c12d[0], &c13p[0],
                            c13i.empty() ? 0 : &c13i[0], c13d.empty() ? 0 : &c13d[0], &c14p[0],
                            c14i.empty() ? 0 : &c14i[0], &p, &sys),
        "system_create");
  m_sys = sys;
  m_haveList = false;
  m_buf.assign(3 * (size_t)n, 0.0);
  m_ene.assign(PDGPU_ENE_COUNT, 0.0);
  m_epot.assign(n, 0.0);
}

void FF_GeneralizedBorn_Still_GPU::upload_positions() {
  WorkSpace &wspace = getWSpace();
  const size_t n = wspace.atom.size();
  for (size_t i = 0; i < n; i++) {
    m_buf[3 * i] = wspace.cur.atom[i].p.x;
    m_buf[3 * i + 1] = wspace.cur.atom[i].p.y;
    m_buf[3 * i + 2] = wspace.cur.atom[i].p.z;
  }
  check(pdgpu_set_positions(m_ctx, m_sys, &m_buf[0]), "set_positions");
}

// The device list is rebuilt, at the positions just uploaded, whenever the
// workspace's own list was rebuilt since the last evaluation.
void FF_GeneralizedBorn_Still_GPU::refresh_list() {
  const unsigned count = getWSpace().nlist().getFullUpdateCount();
  if (m_haveList && count == m_listCount) return;
  check(pdgpu_nlist_build(m_ctx, m_sys), "nlist_build");
  m_listCount = count;
  m_haveList = true;
}

// Forces (N) of the evaluation added to the workspace's, and each atom's
// share of the energy to Particle::epot.
void FF_GeneralizedBorn_Still_GPU::apply_forces() {
  WorkSpace &wspace = getWSpace();
  const size_t n = wspace.atom.size();
  check(pdgpu_get_forces(m_ctx, m_sys, &m_buf[0]), "get_forces");
  for (size_t i = 0; i < n; i++) {
    wspace.cur.atom[i].f.x += m_buf[3 * i];
    wspace.cur.atom[i].f.y += m_buf[3 * i + 1];
    wspace.cur.atom[i].f.z += m_buf[3 * i + 2];
  }
  check(pdgpu_get_atom_epot(m_ctx, m_sys, &m_epot[0]), "get_atom_epot");
  for (size_t i = 0; i < n; i++) wspace.atom[i].epot += m_epot[i];
  // the component's own Born radii (GB_atom_param[i].bornradius) as the
  // device formed them
  check(pdgpu_get_born_radii(m_ctx, m_sys, &m_epot[0]), "get_born_radii");
  for (size_t i = 0; i < n && i < GB_atom_param.size(); i++) GB_atom_param[i].bornradius = m_epot[i];
}

void FF_GeneralizedBorn_Still_GPU::calcForces() {
  if (!Active) return;
  WorkSpace &wspace = getWSpace();
  upload_positions();
  refresh_list();
  check(pdgpu_zero_forces(m_ctx, m_sys), "zero_forces");
  check(pdgpu_gb_forces(m_ctx, m_sys), "gb_forces");
  apply_forces();
  check(pdgpu_get_energies(m_ctx, m_sys, &m_ene[0], PDGPU_ENE_COUNT), "get_energies");
  // the bookkeeping of calcForcesIncludingVacuo (gbff.cpp:1731-1736,
  // 1810-1816): the LJ/Coulomb slots are assigned, the GB terms added
  epot_vdw = m_ene[PDGPU_ENE_VDW];
  epot_elec = m_ene[PDGPU_ENE_ELEC];
  epot_pol = m_ene[PDGPU_ENE_POL];
  epot_pol_cross = m_ene[PDGPU_ENE_POL_CROSS];
  epot_pol_self = m_ene[PDGPU_ENE_POL_SELF];
  epot = m_ene[PDGPU_ENE_EPOT];
  wspace.ene.epot_vdw = epot_vdw;
  wspace.ene.epot_elec = epot_elec;
  wspace.ene.epot_pol += epot_pol;
  wspace.ene.epot_pol_cross += epot_pol_cross;
  wspace.ene.epot_pol_self += epot_pol_self;
  wspace.ene.epot += epot;
}

void FF_GeneralizedBorn_Still_GPU::calcEnergies() {
  if (!Active) return;
  WorkSpace &wspace = getWSpace();
  upload_positions();
  refresh_list();
  check(pdgpu_zero_forces(m_ctx, m_sys), "zero_forces");
  check(pdgpu_gb_energies(m_ctx, m_sys), "gb_energies");
  apply_forces();  // the vacuum LJ/Coulomb forces of the energy path
  check(pdgpu_get_energies(m_ctx, m_sys, &m_ene[0], PDGPU_ENE_COUNT), "get_energies");
  // FF_NonBonded::calcEnergies assigns the LJ/Coulomb slots and adds them
  // to epot; calcBornEnergy adds the Born energy to epot alone
  // (gbff.cpp:161-166, 574-578)
  epot_vdw = m_ene[PDGPU_ENE_VDW];
  epot_elec = m_ene[PDGPU_ENE_ELEC];
  epot_pol = m_ene[PDGPU_ENE_GB_COMPONENT];
  epot_pol_cross = m_ene[PDGPU_ENE_GB_COMPONENT + 1];
  epot_pol_self = m_ene[PDGPU_ENE_GB_COMPONENT + 2];
  epot = m_ene[PDGPU_ENE_EPOT];
  wspace.ene.epot_vdw = epot_vdw;
  wspace.ene.epot_elec = epot_elec;
  wspace.ene.InternalVirial += m_ene[PDGPU_ENE_VIRIAL];
  wspace.ene.epot += epot;
}

}  // namespace Physics
