// Backbone phi/psi trial moves on the device (Monte Carlo trial
// conformations; the reference does this on the host with
// MoleculeBase::setResiduePhiPsi, system/molecule.cpp:677-744, and the
// Metropolis loop in protocols/montecarlo.cpp:16-159).
//
// A chain's backbone rotations, ordered from the N terminus (phi_0, psi_0,
// phi_1, ...), move nested sets of atoms (a nest): rotation k moves the
// side of its bond away from the N terminus, a subset of what rotation k-1
// moves, so every atom of the chain is moved by a leading run of the nest's
// rotations, ending at the last rotation that moves it (the host finds it
// per atom).  Applying the rotations from the C terminus backwards, every
// rotation axis is made of atoms that no later-applied rotation moves, so
// all axes come from the base coordinates and an atom's final position is
// the prefix composition R_first o ... o R_last applied to its base
// position.  The reference applies them from the N terminus forwards with
// each axis taken from the already-rotated coordinates; both orders give
// the same rigid motions.  One thread per system composes the prefix
// transforms (restarting at each nest); one thread per atom applies its
// transform.
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

// x -> M x + t, stored as 12 doubles (row-major M, then t)
struct Affine {
  double m[9], t[3];
};

__global__ void k_torsion_prefix(PackView v, double sigma, unsigned long long trial,
                                 const unsigned long long *keys, const double *angles) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= v.n_sys) return;
  int r0 = v.rot_off[s], r1 = v.rot_off[s + 1];
  Affine P = {{1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 0}};
  // the stream of a system depends only on its own key and the trial
  // number, so a system draws the same angles alone and in any batch
  unsigned long long key = keys[s];
  unsigned k0 = (unsigned)key, k1 = (unsigned)(key >> 32);
  for (int r = r0; r < r1; r++) {
    if (v.rot_start[r]) P = Affine{{1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 0}};
    int2 ax = v.rot_axis[r];
    double a[3] = {v.bx[ax.x], v.by[ax.x], v.bz[ax.x]};
    double u[3] = {v.bx[ax.y] - a[0], v.by[ax.y] - a[1], v.bz[ax.y] - a[2]};
    double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (int k = 0; k < 3; k++) u[k] /= nu;
    double th;
    if (angles) {
      th = angles[r];
    } else {
      U4 q = philox(U4{(unsigned)(r - r0), (unsigned)trial, (unsigned)(trial >> 32), 0x70524Fu}, k0, k1);
      double n1, n2;
      nrand_pair(q.a, q.b, n1, n2);
      th = sigma * n1;
    }
    // Rodrigues rotation matrix Q about unit axis u by th
    double c = cos(th), sn = sin(th), C = 1 - c;
    double Q[9] = {c + u[0] * u[0] * C,        u[0] * u[1] * C - u[2] * sn, u[0] * u[2] * C + u[1] * sn,
                   u[1] * u[0] * C + u[2] * sn, c + u[1] * u[1] * C,        u[1] * u[2] * C - u[0] * sn,
                   u[2] * u[0] * C - u[1] * sn, u[2] * u[1] * C + u[0] * sn, c + u[2] * u[2] * C};
    // R(x) = Q x + (a - Q a);  P <- P o R
    double qa[3];
    for (int i = 0; i < 3; i++) qa[i] = a[i] - (Q[3 * i] * a[0] + Q[3 * i + 1] * a[1] + Q[3 * i + 2] * a[2]);
    Affine N;
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++)
        N.m[3 * i + j] = P.m[3 * i] * Q[j] + P.m[3 * i + 1] * Q[3 + j] + P.m[3 * i + 2] * Q[6 + j];
      N.t[i] = P.m[3 * i] * qa[0] + P.m[3 * i + 1] * qa[1] + P.m[3 * i + 2] * qa[2] + P.t[i];
    }
    P = N;
    double *o = v.rot_xf + 12 * (size_t)r;
    for (int k = 0; k < 9; k++) o[k] = P.m[k];
    for (int k = 0; k < 3; k++) o[9 + k] = P.t[k];
  }
}

__device__ __forceinline__ void store_pos_mv(const PackView &v, int i, double x, double y, double z) {
  v.x[i] = x;
  v.y[i] = y;
  v.z[i] = z;
  float hx = __double2float_rn(x), hy = __double2float_rn(y), hz = __double2float_rn(z);
  float4 a = v.pq[2 * (size_t)i];
  a.x = hx;
  a.y = hy;
  a.z = hz;
  v.pq[2 * (size_t)i] = a;
  v.pq[2 * (size_t)i + 1] = make_float4(__double2float_rn(x - (double)hx), __double2float_rn(y - (double)hy),
                                        __double2float_rn(z - (double)hz), 0.f);
  v.xyzp[i] = make_double4(x, y, z, v.pv_d[i]);
}

__global__ void k_torsion_apply(PackView v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  int last = v.rot_last[i];
  double x = v.bx[i], y = v.by[i], z = v.bz[i];
  if (last >= 0) {
    const double *T = v.rot_xf + 12 * (size_t)last;
    double nx = T[0] * x + T[1] * y + T[2] * z + T[9];
    double ny = T[3] * x + T[4] * y + T[5] * z + T[10];
    double nz = T[6] * x + T[7] * y + T[8] * z + T[11];
    x = nx;
    y = ny;
    z = nz;
  }
  store_pos_mv(v, i, x, y, z);
}

void launch_torsion_moves(const PackView &v, cudaStream_t st, double sigma, unsigned long long trial,
                          const unsigned long long *keys, const double *angles) {
  if (!v.n_atoms) return;
  PDGPU_LAUNCH(k_torsion_prefix, (v.n_sys + 63) / 64, 64, 0, st, v, sigma, trial, keys, angles);
  PDGPU_LAUNCH(k_torsion_apply, (v.n_atoms + 255) / 256, 256, 0, st, v);
}

// ------------------------------------------------------------ Metropolis
// MonteCarlo::accept (protocols/montecarlo.cpp:143-159) for every system of
// the pack, on the energy record of the step's evaluation: a non-finite
// energy is rejected; a lower one accepted; otherwise d = (E_old - E_new) /
// kB T, rejected when d < -50, else accepted when u < e^d with u uniform in
// [0, 1) from Philox keyed by the system's key and the step (the reference
// draws it with rand()).  Step 0 (no move) is accepted when finite.
// An accepted step moves the system's base positions (the state the next
// trial perturbs) to the current ones; with keep_lowest the lowest-energy
// state also goes to the saved positions (o*).
struct MCSys {
  double old_e, low_e;  // kcal/mol
  int acc, last, done, low_step;
};
size_t mc_state_size() { return sizeof(MCSys); }

__global__ void k_mc_accept(PackView v, MCSys *m, int step, double inv_kT, const unsigned long long *keys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= v.n_sys || v.flags[F_NL_OVERFLOW]) return;
  MCSys &q = m[s];
  const double e = v.ene[(size_t)s * E_COUNT + E_EPOT];
  bool ok = e == e && fabs(e) <= 1.79e308;
  if (ok && step != 0 && !(e < q.old_e)) {
    const double d = (q.old_e - e) * inv_kT;
    if (d < -50.0) {
      ok = false;
    } else {
      const unsigned long long k = keys[s];
      U4 r = philox(U4{(unsigned)step, 0x4D43u, 0x5452u, 0u}, (unsigned)k, (unsigned)(k >> 32));
      const double u = (double)(((unsigned long long)r.a << 21) ^ (unsigned long long)(r.b >> 11)) *
                       (1.0 / 9007199254740992.0);  // 53 bits
      ok = u < exp(d);
    }
  }
  q.last = ok ? 1 : 0;
  q.done = step + 1;
  if (ok) {
    q.old_e = e;
    q.acc++;
    if (step == 0 || e < q.low_e) {
      q.low_e = e;
      q.low_step = step;
      q.last = 3;  // accepted and the lowest so far
    }
  }
}

__global__ void k_mc_commit(PackView v, const MCSys *m, int keep_lowest) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms || v.flags[F_NL_OVERFLOW]) return;
  const int last = m[v.sys_of[i]].last;
  if (!last) return;
  const double x = v.x[i], y = v.y[i], z = v.z[i];
  v.bx[i] = x;
  v.by[i] = y;
  v.bz[i] = z;
  if (keep_lowest && last == 3) {
    v.ox[i] = x;
    v.oy[i] = y;
    v.oz[i] = z;
  }
}

// the state a Monte Carlo run ends in: the base positions (last accepted)
__global__ void k_mc_restore(PackView v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  store_pos_mv(v, i, v.bx[i], v.by[i], v.bz[i]);
}
void launch_mc_restore(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_mc_restore, (v.n_atoms + 255) / 256, 256, 0, st, v);
}

void launch_mc_accept(const PackView &v, cudaStream_t st, void *m, int step, double inv_kT,
                      const unsigned long long *keys, int keep_lowest) {
  if (!v.n_sys) return;
  PDGPU_LAUNCH(k_mc_accept, (v.n_sys + 127) / 128, 128, 0, st, v, (MCSys *)m, step, inv_kT, keys);
  if (v.n_atoms) PDGPU_LAUNCH(k_mc_commit, (v.n_atoms + 255) / 256, 256, 0, st, v, (const MCSys *)m, keep_lowest);
}
// the host's view of one system's state
void mc_state_read(const void *buf, int s, int *accepted, int *done, double *lowest_kcal, int *low_step) {
  const MCSys &q = ((const MCSys *)buf)[s];
  *accepted = q.acc;
  *done = q.done;
  *lowest_kcal = q.low_e;
  *low_step = q.low_step;
}

}  // namespace pdgpu
