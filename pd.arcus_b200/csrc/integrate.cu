// MD integrators, kinetic energy, velocity initialisation and the
// minimiser's device-side control flow.
//
//   Langevin        MolecularDynamics::applyForces_LangevinIntegration (md.cpp:906-1042)
//   Langevin non-H  applyForces_LangevinIntegration_NonHydrogens        (md.cpp:1048-1218)
//   VelocityVerlet  applyForces_VelocityVerletIntegration               (md.cpp:788-838)
//   Beeman          applyForces_BeemanIntegration                       (md.cpp:841-902)
//   Verlet          applyForces_VerletIntegration                       (md.cpp:748-786)
//   KE              calcKineticEnergy                                   (md.cpp:504-539)
//   init velocities setInitialSpeeds                                    (md.cpp:342-363)
//   SD / CG         Minimisation::doSteepestDescentStep / doConjugateGradientStep
//                   (minimise.cpp:181-318) and the runcore bookkeeping (:99-179)
//
// State is FP64 (positions in Angstrom, velocities in m/s, forces converted
// from the fixed-point accumulators to N), as in the reference.  Random
// normals come from a counter-based Philox4x32-10 generator keyed by the
// system's seed and indexed by (system-local atom, step), so a system's
// trajectory does not depend on which other systems share its launch.
// Roofline: HBM-bound, 152 B/atom/step algorithmic traffic.
#include <cuda_runtime.h>
#include <cstddef>

#include "mdatom.cuh"

namespace pdgpu {

// One integrator step for every atom of the pack.  KE per atom goes to
// e_atom[AE_KIN] and is reduced per system afterwards.
// The thermostat's normals depend on the step, the atom and its system's key
// only, so they are drawn before the wait for the force passes (under a
// programmatic dependent launch, beside the last pass's tail).  The step
// counter is final by then: the step's launch waits on the event of the
// energy record that advanced it, a full dependency.
__global__ void k_md_step(PackView v, MDDev d, const double *normals, const int *step_dev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < v.n_atoms;
  const int step = !live ? 0 : step_dev ? *step_dev : d.c.step;
  double nr[6];
  const bool pre = live && !normals && md_draws_normals(v, d, step, i);
  if (pre) md_normals(v, d, step, i, nr);
  PDGPU_DEP_ENTRY();
  if (!live || v.flags[F_NL_OVERFLOW]) return;  // forces incomplete: keep the state, host re-plans
  v.e_atom[(size_t)AE_KIN * v.n_atoms + i] = md_atom(v, d, normals, step, i, pre ? nr : nullptr);  // J
}

// per-atom kinetic energy from the current velocities (J)
__global__ void k_kinetic_atoms(PackView v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  double vx = v.vx[i], vy = v.vy[i], vz = v.vz[i];
  v.e_atom[(size_t)AE_KIN * v.n_atoms + i] = 0.5 * v.mass_si[i] * (vx * vx + vy * vy + vz * vz);
}

// setInitialSpeeds: Boltzmann draw (two nrand pairs, the second overwriting
// vy as the reference does, md.cpp:353-356); then rescale to 3/2 N kB T.
__global__ void k_vel_init(PackView v, double kB, double temp, const unsigned long long *sys_seed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  int s = v.sys_of[i];
  double nr[6];
  six_normals(sys_seed[s] ^ 0x5EEDull, i - v.atom_off[s], -1, nr);
  double sigma = sqrt(kB * temp / v.mass_si[i]);
  double vx = nr[0] * sigma, vy = nr[1] * sigma;
  vy = nr[2] * sigma;  // nrand(vy, vz): second pair overwrites vy
  double vz = nr[3] * sigma;
  v.vx[i] = vx;
  v.vy[i] = vy;
  v.vz[i] = vz;
}
__global__ void k_vel_scale(PackView v, double kB, double temp, double kcal2J_per_mol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  int s = v.sys_of[i];
  int n = v.atom_off[s + 1] - v.atom_off[s];
  double ekin = v.ene[(size_t)s * E_COUNT + E_EKIN] * kcal2J_per_mol;  // J
  double edes = 3 * n * kB * temp / 2;
  double chi = sqrt(edes / ekin);
  v.vx[i] *= chi;
  v.vy[i] *= chi;
  v.vz[i] *= chi;
}

// --------------------------------------------------------------- minimiser
struct MinState {
  double mult, old_energy, local_old, gamma, fmagold, fmagnew;
  int step, breakcount, done, action;  // action: 0 step, 1 restore-and-skip, 2 restore-then-step
  int taken, nan;
  int last;  // the last step the loop evaluated (WorkSpace::Step when the loop ends)
};

// CG dot products: per (chunk, system) partials of fmagold = sum of.of and
// fmagnew = sum (of-f).f into e_part slots 0 and 1; the last block of each
// system adds them in a fixed order for k_min_control.
__global__ void k_min_dots(PackView v, double N_per_unit, int C) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int c = blockIdx.x, s = blockIdx.y;
  int a0 = v.atom_off[s] + c * kReduceChunk, a1 = min(a0 + kReduceChunk, v.atom_off[s + 1]);
  __shared__ double sa[256], sb[256];
  double A = 0, B = 0;
  for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
    double f[3] = {force_N(v.fx[i], v.gx[i], v.hx[i]) * N_per_unit, force_N(v.fy[i], v.gy[i], v.hy[i]) * N_per_unit,
                   force_N(v.fz[i], v.gz[i], v.hz[i]) * N_per_unit};
    double of[3] = {v.fox[i], v.foy[i], v.foz[i]};
    A += of[0] * of[0] + of[1] * of[1] + of[2] * of[2];
    B += (of[0] - f[0]) * f[0] + (of[1] - f[1]) * f[1] + (of[2] - f[2]) * f[2];
  }
  sa[threadIdx.x] = A;
  sb[threadIdx.x] = B;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  double *part = v.e_part + (size_t)s * C * 10;
  if (threadIdx.x == 0) {
    part[(size_t)c * 10] = sa[0];
    part[(size_t)c * 10 + 1] = sb[0];
  }
  // the last block of the system adds the chunk partials (lanes strided over
  // the chunks, then a fixed shuffle tree) into slots 2 and 3 of chunk 0
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&v.e_done[s], 1) == C - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < 2) {
    double t = 0.0;
    for (int q = lane; q < C; q += 32) t += __ldcg(part + (size_t)q * 10 + warp);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) part[2 + warp] = t;
  }
  if (threadIdx.x == 0) v.e_done[s] = 0;
}

// One thread per system: the accept / restore decision of the step.
// Energies here are kcal/mol; one joule per molecule (the reference's
// "m_OldEnergy += 1" after a rejected SD step) is J_unit kcal/mol.
__global__ void k_min_control(PackView v, MinState *ms, int algorithm, double slope_cutoff_kcal,
                              double strictness_kcal, double J_unit, int nsteps, int C) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= v.n_sys) return;
  MinState &m = ms[s];
  if (algorithm == PDGPU_MIN_CONJUGATE_GRADIENTS && !v.flags[F_NL_OVERFLOW]) {
    const double *o = v.e_part + (size_t)s * C * 10;  // totals of k_min_dots
    m.fmagold = o[2];
    m.fmagnew = o[3];
  }
  if (v.flags[F_NL_OVERFLOW]) {  // no valid forces this step: do nothing, retry
    m.action = -1;
    return;
  }
  if (m.done) {
    m.action = -1;
    return;
  }
  m.last = m.step;
  double epot = v.ene[(size_t)s * E_COUNT + E_EPOT];
  if (!(epot == epot)) {
    m.nan = 1;
    m.done = 1;
    m.action = -1;
    atomicExch(&v.flags[F_NAN], 1);
    return;
  }
  if (m.step == 0) m.local_old = epot;
  if (m.step > 0 && slope_cutoff_kcal > 0.0) {
    double d = m.local_old - epot;
    if (d >= 0.0 && d < slope_cutoff_kcal) m.breakcount++;
    m.local_old = epot;
  }
  if (m.breakcount > 10) {
    m.done = 1;
    m.action = -1;
    return;
  }
  if (algorithm == PDGPU_MIN_STEEPEST_DESCENT) {
    if (m.step != 0) {
      if (epot <= m.old_energy) {
        m.mult *= 1.2;
        m.old_energy = epot;
        m.action = 0;  // save then step
      } else {
        m.mult *= 0.5 / 1.2;
        m.old_energy += J_unit;
        m.action = 1;  // restore, no step
      }
    } else {
      m.old_energy = epot;
      m.action = 0;
    }
  } else {
    if (m.step != 0) {
      if ((m.mult < 0.05 && (epot - m.old_energy) < strictness_kcal) || epot < m.old_energy) {
        m.mult *= 1.2;
        double g = m.fmagold != 0 ? m.fmagnew / m.fmagold : 0.0;
        if (g < 0) g = 0;
        m.gamma = g;
        m.old_energy = epot;
        m.action = 3;  // new direction, save, step
      } else {
        m.mult *= 0.5 / 1.2;
        m.action = 2;  // restore positions, step along the old direction
      }
    } else {
      m.old_energy = epot;
      m.action = 4;  // first step: direction = force
    }
  }
  m.step++;
  m.taken = m.step;
  if (m.step >= nsteps) m.done = 1;
}

__global__ void k_min_update(PackView v, const MinState *ms, double N_per_unit, double step_size) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  int s = v.sys_of[i];
  const MinState &m = ms[s];
  int a = m.action;
  if (a < 0) return;
  double f[3] = {force_N(v.fx[i], v.gx[i], v.hx[i]) * N_per_unit, force_N(v.fy[i], v.gy[i], v.hy[i]) * N_per_unit,
                 force_N(v.fz[i], v.gz[i], v.hz[i]) * N_per_unit};
  double p[3] = {v.x[i], v.y[i], v.z[i]};
  double sc = step_size * m.mult;
  if (a == 0) {  // SD accept (or first step): save p, f; step along f
    v.ox[i] = p[0];
    v.oy[i] = p[1];
    v.oz[i] = p[2];
    v.fox[i] = f[0];
    v.foy[i] = f[1];
    v.foz[i] = f[2];
    for (int k = 0; k < 3; k++) p[k] += f[k] * sc;
  } else if (a == 1) {  // SD reject: restore p (the restored force is recomputed next step)
    p[0] = v.ox[i];
    p[1] = v.oy[i];
    p[2] = v.oz[i];
  } else if (a == 2) {  // CG reject: restore p, step along the current direction
    p[0] = v.ox[i] + v.dirx[i] * sc;
    p[1] = v.oy[i] + v.diry[i] * sc;
    p[2] = v.oz[i] + v.dirz[i] * sc;
  } else {  // 3: CG accept (new direction), 4: first CG step
    double d[3];
    if (a == 3) {
      d[0] = v.odx[i] * m.gamma + f[0];
      d[1] = v.ody[i] * m.gamma + f[1];
      d[2] = v.odz[i] * m.gamma + f[2];
    } else {
      d[0] = f[0];
      d[1] = f[1];
      d[2] = f[2];
    }
    v.dirx[i] = d[0];
    v.diry[i] = d[1];
    v.dirz[i] = d[2];
    v.odx[i] = d[0];
    v.ody[i] = d[1];
    v.odz[i] = d[2];
    v.ox[i] = p[0];
    v.oy[i] = p[1];
    v.oz[i] = p[2];
    v.fox[i] = f[0];
    v.foy[i] = f[1];
    v.foz[i] = f[2];
    for (int k = 0; k < 3; k++) p[k] += d[k] * sc;
  }
  store_pos(v, i, p[0], p[1], p[2]);
}

// end of runcore: cur = old (the last accepted positions)
__global__ void k_min_restore_best(PackView v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  store_pos(v, i, v.ox[i], v.oy[i], v.oz[i]);
}

// --------------------------------------------------------------- launchers
void launch_md_step_impl(const PackView &v, cudaStream_t st, const MDCoef &c, const double *normals,
                         const int *step_dev, const unsigned char *is_h, const unsigned long long *seeds,
                         double *frames, int frame_every, int frame_cap) {
  MDDev d = make_md_dev(c, is_h, seeds);
  d.frames = frames;
  d.frame_every = frames ? frame_every : 0;
  d.frame_cap = frame_cap;
  // 64-thread blocks: a 20k-atom system spreads over every SM
  if (v.n_atoms) PDGPU_LAUNCH_DEP(k_md_step, (v.n_atoms + 63) / 64, 64, 0, st, v, d, normals, step_dev);
}

std::atomic<long long> &launch_counter() {
  static std::atomic<long long> n{0};
  return n;
}
static thread_local long long tl_captured = -1;  // -1: this thread is not capturing
void count_launch() {
  if (tl_captured >= 0)
    tl_captured++;
  else
    launch_counter()++;
}
bool pdl_enabled() {
  static const bool on = [] {
    const char *e = getenv("PDGPU_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
void begin_capture_count() { tl_captured = 0; }
long long end_capture_count() {
  long long n = tl_captured;
  tl_captured = -1;
  return n;
}
void launch_ke_from_velocities(const PackView &v, cudaStream_t st) {
  if (!v.n_atoms) return;
  PDGPU_LAUNCH(k_kinetic_atoms, (v.n_atoms + 255) / 256, 256, 0, st, v);
  launch_energy(v, st, EM_KINETIC);
}
void launch_vel_init_impl(const PackView &v, cudaStream_t st, double temp, const unsigned long long *seeds) {
  const Consts &k = consts();
  if (!v.n_atoms) return;
  PDGPU_LAUNCH(k_vel_init, (v.n_atoms + 255) / 256, 256, 0, st, v, k.kB, temp, seeds);
  launch_ke_from_velocities(v, st);
  PDGPU_LAUNCH(k_vel_scale, (v.n_atoms + 255) / 256, 256, 0, st, v, k.kB, temp, k.kcal2J / k.Na);
  launch_ke_from_velocities(v, st);
}
void launch_min_step(const PackView &v, cudaStream_t st, void *ms, int algorithm, double slope_kcal,
                     double strict_kcal, double step_size, int nsteps) {
  const Consts &k = consts();
  MinState *m = (MinState *)ms;
  int C = v.e_chunks;
  if (algorithm == PDGPU_MIN_CONJUGATE_GRADIENTS)
    PDGPU_LAUNCH(k_min_dots, dim3(C, v.n_sys), 256, 0, st, v, k.N_per_kcalmolA, C);
  PDGPU_LAUNCH(k_min_control, (v.n_sys + 127) / 128, 128, 0, st, v, m, algorithm, slope_kcal, strict_kcal,
               k.J2kcal * k.Na, nsteps, C);
  PDGPU_LAUNCH(k_min_update, (v.n_atoms + 63) / 64, 64, 0, st, v, m, k.N_per_kcalmolA, step_size);
}
void launch_min_finish(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_min_restore_best, (v.n_atoms + 255) / 256, 256, 0, st, v);
}
size_t min_state_size() { return sizeof(MinState); }
int min_state_last(const void *host_buf, int s) { return ((const MinState *)host_buf)[s].last; }
StepSrc min_step_src(const void *ms, bool last) {
  static_assert(sizeof(MinState) % sizeof(int) == 0, "MinState is a whole number of ints");
  StepSrc r;
  r.p = (const int *)((const char *)ms + (last ? offsetof(MinState, last) : offsetof(MinState, step)));
  r.stride = (int)(sizeof(MinState) / sizeof(int));
  return r;
}
void min_state_init(void *host_buf, int n) {
  MinState *m = (MinState *)host_buf;
  for (int s = 0; s < n; s++) {
    m[s] = MinState{};
    m[s].mult = 1.0;
  }
}
void min_state_read(const void *host_buf, int s, int *taken, int *nan, double *mult) {
  const MinState *m = (const MinState *)host_buf;
  *taken = m[s].taken;
  *nan = m[s].nan;
  *mult = m[s].mult;
}

}  // namespace pdgpu
