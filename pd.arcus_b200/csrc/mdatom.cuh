// One MD integrator step for one atom (md.cpp:748-1218), shared by the
// step kernel and the fused step-and-energy kernel.  State is FP64
// (positions in Angstrom, velocities in m/s, forces converted from the
// fixed-point accumulators to N), as in the reference.  Random normals come
// from a counter-based Philox4x32-10 generator keyed by the system's seed
// and indexed by (system-local atom, step), so a system's trajectory does
// not depend on which other systems share its launch.
#pragma once
#include "internal.cuh"

namespace pdgpu {

// (Philox4x32-10 and the Box-Muller pair live in internal.cuh)
// Box-Muller pair in single precision for the thermostat noise: the
// variates need the normal distribution, not particular bits (24-bit
// uniforms; the tails are cut at 5.8 sigma, probability 8e-9)
__device__ __forceinline__ void nrand_pair_f(unsigned ua, unsigned ub, double &n1, double &n2) {
  const float z1 = ((float)(ua >> 8) + 1.0f) * (1.0f / 16777216.0f);  // (0, 1]
  const float z2 = (float)(ub >> 8) * (1.0f / 16777216.0f);           // [0, 1)
  const float l = sqrtf(-2.0f * logf(z1));
  float s, c;
  sincospif(-2.0f * z2, &s, &c);
  n1 = (double)(l * c);
  n2 = (double)(l * s);
}
// six normals for atom `local` at `step`, in the reference's draw order
// n1x n2y n2x n1z n1y n2z
__device__ __forceinline__ void six_normals(unsigned long long seed, int local, int step, double *o) {
  unsigned k0 = (unsigned)seed, k1 = (unsigned)(seed >> 32);
  U4 r1 = philox(U4{(unsigned)local, (unsigned)step, 0u, 0x4D44u}, k0, k1);
  U4 r2 = philox(U4{(unsigned)local, (unsigned)step, 1u, 0x4D44u}, k0, k1);
  nrand_pair_f(r1.a, r1.b, o[0], o[1]);
  nrand_pair_f(r1.c, r1.d, o[2], o[3]);
  nrand_pair_f(r2.a, r2.b, o[4], o[5]);
}

// Total force on atom i along one axis in kcal/mol/A (the caller scales to
// N): the fixed-point scattered terms, the atom's FP64 pair force and the
// fixed-point j side of the tile passes, added in this order.
__device__ __forceinline__ double force_N(long long f, double g, long long h) {
  return (double)f * kInvForceScale + g + (double)h * kInvJScale;
}

__device__ __forceinline__ void store_pos(const PackView &v, int i, double x, double y, double z) {
  v.x[i] = x;
  v.y[i] = y;
  v.z[i] = z;
  float hx = __double2float_rn(x), hy = __double2float_rn(y), hz = __double2float_rn(z);
  float4 a = v.pq[2 * (size_t)i];
  a.x = hx;
  a.y = hy;
  a.z = hz;
  v.pq[2 * (size_t)i] = a;
  // the Born radius slot (.w) is refreshed by the next Born-radius pass
  v.pq[2 * (size_t)i + 1] = make_float4(__double2float_rn(x - (double)hx), __double2float_rn(y - (double)hy),
                                        __double2float_rn(z - (double)hz), 0.f);
  v.xyzp[i] = make_double4(x, y, z, v.pv_d[i]);
}

struct MDDev {
  MDCoef c;
  double N_per_unit;   // kcal/mol/A -> N
  double inv_angstrom; // 1 / 1e-10 as the reference forms it
  double kB;
  const unsigned char *is_h;
  const unsigned long long *sys_seed;
  // trajectory snapshots: with frame_every > 0, the positions after step s
  // (s > 0, s % frame_every == 0) go to ring slot (s / frame_every - 1) %
  // frame_cap of frames[frame_cap][N][3]
  double *frames;
  int frame_every, frame_cap;
};
inline MDDev make_md_dev(const MDCoef &c, const unsigned char *is_h, const unsigned long long *seeds) {
  const Consts &k = consts();
  MDDev d;
  d.c = c;
  d.N_per_unit = k.N_per_kcalmolA;
  d.inv_angstrom = 1 / k.Angstrom;
  d.kB = k.kB;
  d.is_h = is_h;
  d.sys_seed = seeds;
  d.frames = nullptr;
  d.frame_every = 0;
  d.frame_cap = 0;
  return d;
}

// Whether atom i draws thermostat normals at `step` (md_atom's Langevin
// branch for it).
__device__ __forceinline__ bool md_draws_normals(const PackView &v, const MDDev &d, int step, int i) {
  const MDCoef &c = d.c;
  if (c.integrator != PDGPU_INTEGRATOR_LANGEVIN || c.gamma * c.dt < 0.00001) return false;
  const bool hyd = d.is_h && d.is_h[i];
  return (c.stochastic_h || !hyd) && step < c.steps - 1;
}
// The six normals of atom i at `step` (its system's key, its local index).
__device__ __forceinline__ void md_normals(const PackView &v, const MDDev &d, int step, int i, double *nr) {
  const int s = v.sys_of[i];
  six_normals(d.sys_seed[s], i - v.atom_off[s], step, nr);
}

// Advance atom i by one step of the integrator in d.c at `step`; returns
// its kinetic energy (J) at the point the reference measures it.  `pre`:
// the atom's thermostat normals drawn already (md_normals), or NULL.
__device__ __forceinline__ double md_atom(const PackView &v, const MDDev &d, const double *normals, int step,
                                          int i, const double *pre = nullptr) {
  const MDCoef &c = d.c;
  double m = v.mass_si[i];
  double f[3] = {force_N(v.fx[i], v.gx[i], v.hx[i]) * d.N_per_unit, force_N(v.fy[i], v.gy[i], v.hy[i]) * d.N_per_unit,
                 force_N(v.fz[i], v.gz[i], v.hz[i]) * d.N_per_unit};
  double vel[3] = {v.vx[i], v.vy[i], v.vz[i]};
  double pos[3] = {v.x[i], v.y[i], v.z[i]};
  double t = c.dt;
  int integ = c.integrator;
  bool hyd = d.is_h && d.is_h[i];
  bool langevin = integ == PDGPU_INTEGRATOR_LANGEVIN;
  if (langevin && c.gamma * t < 0.00001) integ = PDGPU_INTEGRATOR_VELOCITY_VERLET, langevin = false;
  bool vv_like = integ == PDGPU_INTEGRATOR_VELOCITY_VERLET || (langevin && !c.stochastic_h && hyd);
  double ke = 0;
  if (vv_like && integ == PDGPU_INTEGRATOR_VELOCITY_VERLET) {
    // md.cpp:788-838 as written: kick, KE, kick, drift with v+dv, kick
    double tim = 0.5 * t / m;
    for (int k = 0; k < 3; k++) vel[k] += f[k] * tim;
    ke = 0.5 * m * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    for (int k = 0; k < 3; k++) {
      double dv = f[k] * tim;
      vel[k] += dv;
      double dr = t * (vel[k] + dv);
      dr *= d.inv_angstrom;
      pos[k] += dr;
      vel[k] += dv;
    }
  } else if (langevin && vv_like) {
    // hydrogens in the non-hydrogen Langevin variant (md.cpp:1135-1183)
    double tim = 0.5 * t / m;
    if (step > 0)
      for (int k = 0; k < 3; k++) vel[k] += f[k] * tim;
    ke = 0.5 * m * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    if (step < c.steps - 1)
      for (int k = 0; k < 3; k++) {
        double dv = f[k] * tim;
        double dr = t * (vel[k] + dv);
        dr *= d.inv_angstrom;
        pos[k] += dr;
        vel[k] += dv;
      }
  } else if (langevin) {
    // md.cpp:1003-1040 with the step's constant quotients formed on the host
    const double im = 1.0 / m;
    double tim = t * im;
    if (step > 0)
      for (int k = 0; k < 3; k++) vel[k] += c.kick1 * f[k] * tim;
    ke = 0.5 * m * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    if (step < c.steps - 1) {
      double nr[6];
      if (normals) {
        for (int k = 0; k < 6; k++) nr[k] = normals[6 * (size_t)i + k];
      } else if (pre) {
        for (int k = 0; k < 6; k++) nr[k] = pre[k];
      } else {
        md_normals(v, d, step, i, nr);
      }
      double n1x = nr[0], n2y = nr[1], n2x = nr[2], n1z = nr[3], n1y = nr[4], n2z = nr[5];
      double kTdivm = d.kB * c.temp * im;
      double sigmav = sqrt(kTdivm * c.varv);
      double sigmar = sqrt(kTdivm * c.varr) * c.inv_gamma;
      double sq = c.sq_crv;
      double dvr[3] = {sigmav * (c.crv * n1x + sq * n2x), sigmav * (c.crv * n1y + sq * n2y),
                       sigmav * (c.crv * n1z + sq * n2z)};
      double drr[3] = {sigmar * n1x, sigmar * n1y, sigmar * n1z};
      for (int k = 0; k < 3; k++) {
        double dr = t * (c.c1 * vel[k] + c.c2 * f[k] * tim) + drr[k];
        dr *= d.inv_angstrom;
        double dv = c.c0c2_c1 * f[k] * tim + dvr[k];
        pos[k] += dr;
        vel[k] *= c.c0;
        vel[k] += dv;
      }
    }
  } else if (integ == PDGPU_INTEGRATOR_BEEMAN) {
    double tim = t / (6.0 * m);
    double fo[3] = {v.fox[i], v.foy[i], v.foz[i]};
    if (step > 0)
      for (int k = 0; k < 3; k++) vel[k] += (2.0 * f[k]) * tim;
    ke = 0.5 * m * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    if (step < c.steps - 1) {
      for (int k = 0; k < 3; k++) {
        double dr = t * (vel[k] + (4.0 * f[k] - fo[k]) * tim);
        dr *= d.inv_angstrom;
        double dv = (5.0 * f[k] - fo[k]) * tim;
        pos[k] += dr;
        vel[k] += dv;
      }
      v.fox[i] = f[0];
      v.foy[i] = f[1];
      v.foz[i] = f[2];
    }
  } else {  // Verlet (md.cpp:748-786): needs the previous position in o*
    double op[3] = {v.ox[i], v.oy[i], v.oz[i]};
    double np[3];
    for (int k = 0; k < 3; k++) {
      double t2a = f[k] * (t * t / 1e-10 / m);
      np[k] = pos[k] * 2 - op[k] + t2a;
      vel[k] = (np[k] - op[k]) / (2 * t / 1e-10);
    }
    v.ox[i] = pos[0];
    v.oy[i] = pos[1];
    v.oz[i] = pos[2];
    v.fox[i] = f[0];
    v.foy[i] = f[1];
    v.foz[i] = f[2];
    pos[0] = np[0];
    pos[1] = np[1];
    pos[2] = np[2];
    ke = 0.5 * m * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  }
  v.vx[i] = vel[0];
  v.vy[i] = vel[1];
  v.vz[i] = vel[2];
  store_pos(v, i, pos[0], pos[1], pos[2]);
  if (d.frame_every > 0 && step > 0 && step % d.frame_every == 0) {
    // WorkSpace::outtra.append after the step (md.cpp:260)
    double *fr = d.frames + (size_t)((step / d.frame_every - 1) % d.frame_cap) * 3 * (size_t)v.n_atoms + 3 * (size_t)i;
    fr[0] = pos[0];
    fr[1] = pos[1];
    fr[2] = pos[2];
  }
  return ke;
}

}  // namespace pdgpu
