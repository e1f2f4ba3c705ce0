// FF_SASA_LCPO_GPU (lcpo_gpu.h): the LCPO surface-area term of PD evaluated
// by libpdgpu.  Compiled against the reference's own headers (src/mmlib) and
// linked with the reference library and libpdgpu.so.
#include "lcpo_gpu.h"

#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

#include "exception.h"
#include "forcefields/ffparam.h"
#include "pdgpu.h"
#include "tools/stringtool.h"
#include "workspace/neighbourlist.h"
#include "workspace/workspace.h"

namespace Physics {

pdgpu_ctx *plugin_context(int device);  // gbff_gpu.cpp: one context per device

FF_SASA_LCPO_GPU::FF_SASA_LCPO_GPU(WorkSpace &newwspace, int device)
    : FF_SASA_LCPO(newwspace), Device(device), m_ctx(0), m_sys(-1), m_listCount(0), m_haveList(false),
      m_slack(0.0) {
  name = "LCPO SASA, B200";
}

FF_SASA_LCPO_GPU::FF_SASA_LCPO_GPU(const FF_SASA_LCPO_GPU &other)
    : FF_SASA_LCPO(other), Device(other.Device), m_ctx(0), m_sys(-1), m_listCount(0), m_haveList(false),
      m_slack(0.0) {
  needsetup = true;
}

FF_SASA_LCPO_GPU::~FF_SASA_LCPO_GPU() { release(); }

void FF_SASA_LCPO_GPU::release() {
  if (m_ctx && m_sys >= 0) pdgpu_system_destroy(m_ctx, m_sys);
  m_sys = -1;
  m_haveList = false;
}

void FF_SASA_LCPO_GPU::check(int status, const char *what) const {
  if (status == PDGPU_OK) return;
  throw ProcedureException(std::string("libpdgpu ") + what + ": " + pdgpu_last_error());
}

namespace {
struct LcpoLine {
  int attype, neighbors;
  double radius, p[4];
};
}  // namespace

void FF_SASA_LCPO_GPU::setup() {
  if (!cmpstring(ASPsection_name, ""))
    throw ProcedureException("FF_SASA_LCPO_GPU: per-type ASP sections are not supported; set GlobalASP");
  FF_SASA_LCPO::setup();  // the reference's own: the 7 A list request, the type checks
  WorkSpace &wspace = getWSpace();
  const int n = (int)wspace.atom.size();
  // the LCPO types of the parameter set, in file order (lcpo.cpp:200-260)
  Section sec;
  if (wspace.ffps().getSection("LCPOSASAPARAMETERS", sec) != 0)
    throw ProcedureException("FF_SASA_LCPO_GPU: no LCPOSASAPARAMETERS section in the parameter set");
  std::vector<LcpoLine> types;
  for (size_t l = 0; l < sec.sectionline.size(); l++) {
    std::string line = sec.sectionline[l];
    removecomments(line, "#\12\15");
    std::vector<std::string> tok = chopstr(line, " \12\15\t");
    if (tok.size() < 8 || !cmpstring(tok[0], "LCPOSASATYPE")) continue;
    LcpoLine t;
    t.attype = wspace.ffps().findAtomType(tok[1]);
    t.neighbors = atoi(tok[2].c_str());
    t.radius = strtod(tok[3].c_str(), NULL);
    for (int k = 0; k < 4; k++) t.p[k] = strtod(tok[4 + k].c_str(), NULL);
    types.push_back(t);
  }
  std::vector<double> rad(n), p4(4 * (size_t)n), sigma(n, GlobalASP);
  std::vector<uint8_t> use(n);
  for (int i = 0; i < n; i++) {
    const Particle &a = wspace.atom[i];
    int heavy = 0;
    for (size_t k = 0; k < a.cov12atom.size(); k++)
      if (wspace.atom[a.cov12atom[k].i].Z != 1) heavy++;
    size_t t = 0;
    for (; t < types.size(); t++)
      if (types[t].attype == a.FFType && (types[t].neighbors < 0 || types[t].neighbors == heavy)) break;
    if (t == types.size()) throw ProcedureException("FF_SASA_LCPO_GPU: no LCPO type for an atom");
    rad[i] = types[t].radius + 1.4;
    for (int k = 0; k < 4; k++) p4[4 * (size_t)i + k] = types[t].p[k];
    use[i] = a.Z == 1 ? 0 : 1;
  }
  // a device system of the component's own: the atoms and their covalent
  // lists (the list's bond orders), a 7 A list radius
  release();
  m_ctx = plugin_context(Device);
  std::vector<double> q(n), r(n), e(n), m(n), gbr(n, 1.0);
  std::vector<int32_t> ir(n), c12p(1, 0), c13p(1, 0), c14p(1, 0), c12i, c13i, c14i;
  std::vector<double> c12d, c13d;
  for (int i = 0; i < n; i++) {
    const Particle &a = wspace.atom[i];
    q[i] = a.charge;
    r[i] = a.radius;
    e[i] = a.epsilon;
    m[i] = a.mass;
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
  p.Cutoff = p.VdwCutoff = 7.0;  // FF_SASA_LCPO::setup's list request (lcpo.cpp:20)
  p.InnerCutoff = p.VdwInnerCutoff = 4.0;
  int32_t sys = -1;
  check(pdgpu_system_create(m_ctx, n, &q[0], &r[0], &e[0], &m[0], &gbr[0], &ir[0], &c12p[0],
                            c12i.empty() ? 0 : &c12i[0], c12d.empty() ? 0 : &c12d[0], &c13p[0],
                            c13i.empty() ? 0 : &c13i[0], c13d.empty() ? 0 : &c13d[0], &c14p[0],
                            c14i.empty() ? 0 : &c14i[0], &p, &sys),
        "system_create");
  m_sys = sys;
  double reach = 0.0;  // the largest overlap distance r_i + r_j
  for (int i = 0; i < n; i++)
    if (use[i] && 2.0 * rad[i] > reach) reach = 2.0 * rad[i];
  m_slack = std::max(p.Cutoff, p.VdwCutoff) + p.Padding - reach;
  m_ref.assign(3 * (size_t)n, 0.0);
  check(pdgpu_sasa_lcpo_set(m_ctx, m_sys, &rad[0], &p4[0], &sigma[0], &use[0], UpdateSasa), "sasa_lcpo_set");
  m_haveList = false;
  m_buf.assign(3 * (size_t)n, 0.0);
  m_ene.assign(PDGPU_ENE_COUNT, 0.0);
}

void FF_SASA_LCPO_GPU::upload_and_list() {
  WorkSpace &wspace = getWSpace();
  const size_t n = wspace.atom.size();
  for (size_t i = 0; i < n; i++) {
    m_buf[3 * i] = wspace.cur.atom[i].p.x;
    m_buf[3 * i + 1] = wspace.cur.atom[i].p.y;
    m_buf[3 * i + 2] = wspace.cur.atom[i].p.z;
  }
  check(pdgpu_set_positions(m_ctx, m_sys, &m_buf[0]), "set_positions");
  const unsigned count = wspace.nlist().getFullUpdateCount();
  bool stale = !m_haveList || count != m_listCount;
  if (!stale) {
    // a pair that was beyond the list cutoff at the build and is now inside
    // the largest overlap distance has closed by more than the slack: no
    // atom may have moved by half of it
    const double lim = 0.25 * m_slack * m_slack;
    for (size_t i = 0; i < n && !stale; i++) {
      const double dx = m_buf[3 * i] - m_ref[3 * i], dy = m_buf[3 * i + 1] - m_ref[3 * i + 1],
                   dz = m_buf[3 * i + 2] - m_ref[3 * i + 2];
      stale = m_slack <= 0.0 || dx * dx + dy * dy + dz * dz >= lim;
    }
  }
  if (stale) {
    check(pdgpu_nlist_build(m_ctx, m_sys), "nlist_build");
    m_ref = m_buf;
    m_listCount = count;
    m_haveList = true;
  }
  check(pdgpu_zero_forces(m_ctx, m_sys), "zero_forces");
}

// The forces (N) added to the workspace's; epot_cav added to epot and
// epot_surf (lcpo.cpp:186-189).
void FF_SASA_LCPO_GPU::finish() {
  WorkSpace &wspace = getWSpace();
  const size_t n = wspace.atom.size();
  check(pdgpu_get_forces(m_ctx, m_sys, &m_buf[0]), "get_forces");
  for (size_t i = 0; i < n; i++) {
    wspace.cur.atom[i].f.x += m_buf[3 * i];
    wspace.cur.atom[i].f.y += m_buf[3 * i + 1];
    wspace.cur.atom[i].f.z += m_buf[3 * i + 2];
  }
  check(pdgpu_get_energies(m_ctx, m_sys, &m_ene[0], PDGPU_ENE_COUNT), "get_energies");
  epot = m_ene[PDGPU_ENE_SURF];
  wspace.ene.epot_surf += epot;
  wspace.ene.epot += epot;
}

void FF_SASA_LCPO_GPU::calcForces() {
  if (!Active) return;
  upload_and_list();
  check(pdgpu_sasa_lcpo_forces(m_ctx, m_sys, (int32_t)getWSpace().Step), "sasa_lcpo_forces");
  finish();
}

void FF_SASA_LCPO_GPU::calcEnergies() {
  if (!Active) return;
  upload_and_list();
  check(pdgpu_sasa_lcpo_energies(m_ctx, m_sys), "sasa_lcpo_energies");
  finish();
}

}  // namespace Physics
