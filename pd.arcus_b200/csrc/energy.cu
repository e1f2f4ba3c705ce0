// Energy record (Hamiltonian, workspace/hamiltonian.h:23-49) from the
// per-atom and per-term energies the force kernels write.
//
// One kernel, two stages, both in a fixed order so every total is
// bit-reproducible: each block of the grid (chunks, systems) sums one
// kReduceChunk-item chunk of each range of one system (per-atom terms and the bond
// / angle / dihedral term arrays); the last block of a system to finish
// adds the chunk partials in chunk order, applies them to the record with
// the reference's semantics (the GB and stand-alone LJ/Coulomb components
// assign epot_vdw / epot_elec, everything else accumulates), and in a step
// loop records the step's energies and advances the step.
#include <cuda_runtime.h>

#include "mdatom.cuh"

namespace pdgpu {

constexpr int kChunk = kReduceChunk;
constexpr int kEnergyThreads = 384;  // twelve warps: one per partial slot in the final sum, one for the record
// partial slots
enum { P_VDW = 0, P_ELEC, P_POL, P_SELF, P_NBVIR, P_KIN, P_BOND, P_BVIR, P_ANGLE, P_DIH, P_SURF, P_COUNT };
static_assert(kEnergyThreads / 32 >= P_COUNT, "one warp per partial slot");
static_assert(P_COUNT <= kPartSlots, "partials fit the reduction buffer");

// hist: [step][sys][3] (epot, ekin, etot); step_dev[0] current step,
// step_dev[1] first step of the run, step_dev[2] finished-system counter.
// MD: the block first advances its chunk's atoms by one integrator step
// (the step kernel's work, md_atom) and sums their kinetic energies, so a
// step needs no separate integrator launch.
template <bool MD>
__global__ void __launch_bounds__(kEnergyThreads) k_energy(PackView v, int mode, int C, double J2kcalmol,
                                                           double *hist, int *step_dev, MDDev md) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  const int c = blockIdx.x, s = blockIdx.y, N = v.n_atoms;
  const int md_step = MD ? *step_dev : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double sh[kEnergyThreads / 32][P_COUNT];
  __shared__ double tot[P_COUNT];
  __shared__ int last;
  double acc[P_COUNT];
#pragma unroll
  for (int k = 0; k < P_COUNT; k++) acc[k] = 0.0;
  int a0 = v.atom_off[s] + c * kChunk, a1 = min(a0 + kChunk, v.atom_off[s + 1]);
  bool atoms = mode & (EM_PAIR_GB | EM_PAIR_NB | EM_BORN_ENERGY | EM_KINETIC | EM_SURF);
  const double *ep = v.ebuf ? v.e_pair_alt : v.e_atom;  // the pair slots of this energy buffer
  int *sflags = v.ebuf ? v.sys_flags_alt : v.sys_flags;
  if (atoms)
    for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
      if (mode & (EM_PAIR_GB | EM_PAIR_NB)) {
        acc[P_VDW] += ep[(size_t)AE_VDW * N + i];
        acc[P_ELEC] += ep[(size_t)AE_ELEC * N + i];
      }
      if (mode & (EM_PAIR_GB | EM_BORN_ENERGY | EM_PAIR_GB_SLOW)) {
        acc[P_POL] += ep[(size_t)AE_POL * N + i];
        acc[P_SELF] += ep[(size_t)AE_POL_SELF * N + i];
      }
      if (mode & EM_PAIR_NB) acc[P_NBVIR] += v.e_atom[(size_t)AE_VIR * N + i];
      if (mode & EM_SURF) acc[P_SURF] += v.e_atom[(size_t)AE_SURF * N + i];
      if (MD) {
        const double ke = md_atom(v, md, nullptr, md_step, i);  // J
        v.e_atom[(size_t)AE_KIN * N + i] = ke;
        acc[P_KIN] += ke;
      } else if (mode & EM_KINETIC) {
        acc[P_KIN] += v.e_atom[(size_t)AE_KIN * N + i];
      }
    }
  if (mode & EM_BONDED) {
    const int S1 = v.n_sys + 1;
    const int *off = v.bt.term_off;
    int b0 = off[s] + c * kChunk, b1 = min(b0 + kChunk, off[s + 1]);
    for (int t = b0 + threadIdx.x; t < b1; t += blockDim.x) {
      acc[P_BOND] += v.bt.e_bond[t];
      acc[P_BVIR] += v.bt.vir_bond[t];
    }
    int g0 = off[S1 + s] + c * kChunk, g1 = min(g0 + kChunk, off[S1 + s + 1]);
    for (int t = g0 + threadIdx.x; t < g1; t += blockDim.x) acc[P_ANGLE] += v.bt.e_angle[t];
    // torsions and impropers share the dihedral array: two ranges
    for (int r = 2; r < 4; r++) {
      int d0 = off[r * S1 + s] + c * kChunk, d1 = min(d0 + kChunk, off[r * S1 + s + 1]);
      for (int t = d0 + threadIdx.x; t < d1; t += blockDim.x) acc[P_DIH] += v.bt.e_dih[t];
    }
  }
  // block partials: warp trees, then the warps in order
#pragma unroll
  for (int k = 0; k < P_COUNT; k++)
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < P_COUNT; k++) sh[warp][k] = acc[k];
  __syncthreads();
  double *part = v.e_part + (size_t)s * C * P_COUNT;
  if (threadIdx.x < P_COUNT) {
    double t = 0.0;
    for (int w = 0; w < kEnergyThreads / 32; w++) t += sh[w][threadIdx.x];
    part[(size_t)c * P_COUNT + threadIdx.x] = t;
  }
  // the last block of this system to finish forms the record
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&v.e_done[s], 1) == C - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // warp w adds slot w over the chunks: lane l takes chunks l, l+32, ...
  // (loads in parallel), then a fixed shuffle tree; the record, the step
  // counters and the system's flags are read in parallel meanwhile
  __shared__ double sE[E_COUNT];
  __shared__ int sflag, sk;
  double *E = v.ene + (size_t)s * E_COUNT;
  if (warp < P_COUNT) {
    double t = 0.0;
    for (int q = lane; q < C; q += 32) t += __ldcg(part + (size_t)q * P_COUNT + warp);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) tot[warp] = t;
  } else if (warp == P_COUNT) {
    static_assert(E_COUNT <= 30, "one lane per record slot");
    if (lane < E_COUNT) sE[lane] = __ldcg(E + lane);
    if (lane == 30) sflag = __ldcg(sflags + s);
    if (lane == 31 && (mode & EM_RECORD)) sk = __ldcg(step_dev) - __ldcg(step_dev + 1);
  } else {
    static_assert(kEnergyThreads / 32 > P_COUNT, "a spare warp reads the record");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.e_done[s] = 0;
    double *R = sE;
    if (mode & EM_ASSIGN)  // as WorkSpace::zeroForces left it
      for (int k = 0; k < E_COUNT; k++)
        if (k != E_EKIN) R[k] = 0.0;
    if (mode & (EM_PAIR_GB | EM_PAIR_NB)) {
      R[E_VDW] = tot[P_VDW];
      R[E_ELEC] = tot[P_ELEC];
      R[E_EPOT] += tot[P_VDW] + tot[P_ELEC];
    }
    if (mode & EM_PAIR_GB) {
      R[E_POL] += tot[P_POL] + tot[P_SELF];
      R[E_POL_CROSS] += tot[P_POL];
      R[E_POL_SELF] += tot[P_SELF];
      R[E_EPOT] += tot[P_POL] + tot[P_SELF];
    }
    if (mode & EM_PAIR_NB) R[E_VIRIAL] += tot[P_NBVIR];
    if (mode & EM_PAIR_GB_SLOW) {
      // calcBornForces adds its energy to epot alone (gbff.cpp:1340); the
      // component's own totals go to the extra slots
      R[E_EPOT] += tot[P_POL] + tot[P_SELF];
      R[E_GB_COMPONENT] = tot[P_POL] + tot[P_SELF];
      R[E_GB_COMPONENT + 1] = tot[P_POL];
      R[E_GB_COMPONENT + 2] = tot[P_SELF];
    }
    if (mode & EM_BORN_ENERGY) {
      // the energy-only path adds the Born energy to epot alone
      // (gbff.cpp:574-578); the component's own totals go to extra slots
      R[E_EPOT] += tot[P_POL] + tot[P_SELF];
      R[E_GB_COMPONENT] = tot[P_POL] + tot[P_SELF];
      R[E_GB_COMPONENT + 1] = tot[P_POL];
      R[E_GB_COMPONENT + 2] = tot[P_SELF];
    }
    if (mode & EM_BONDED) {
      R[E_BOND] += tot[P_BOND];
      R[E_ANGLE] += tot[P_ANGLE];
      R[E_TORSION] += tot[P_DIH];
      R[E_VIRIAL] += tot[P_BVIR];
      R[E_EPOT] += tot[P_BOND] + tot[P_ANGLE] + tot[P_DIH];
    }
    if (mode & EM_SURF) {  // FF_SASA_LCPO adds epot_cav to epot and epot_surf
      R[E_SURF] += tot[P_SURF];
      R[E_EPOT] += tot[P_SURF];
    }
    if (mode & EM_KINETIC) {
      R[E_EKIN] = tot[P_KIN] * J2kcalmol;
      R[E_ETOT] = R[E_EPOT] + R[E_EKIN];
    }
    if (sflag & SF_NONFINITE) R[E_EPOT] = __longlong_as_double(0x7ff8000000000000LL);  // NaN
    if (!(R[E_EPOT] == R[E_EPOT])) atomicExch(&v.flags[F_NAN], 1);
  }
  __syncthreads();
  if (warp == 0) {
    if (lane < E_COUNT) E[lane] = sE[lane];
    if (lane == 31) sflags[s] = 0;  // consumed
    if ((mode & EM_RECORD) && lane < 3) {
      double *h = hist + ((size_t)sk * v.n_sys + s) * 3;
      h[lane] = sE[lane == 0 ? E_EPOT : lane == 1 ? E_EKIN : E_ETOT];
    }
    // the last system to finish advances the step (every block has read
    // step_dev[0] before it counts itself finished)
    if ((mode & EM_RECORD) && lane == 0) {
      __threadfence();
      int done = atomicAdd(&step_dev[2], 1);
      if (done == v.n_sys - 1) {
        step_dev[2] = 0;
        __threadfence();
        atomicAdd(&step_dev[0], 1);
      }
    }
  }
}

int energy_chunks(const PackView &v) { return v.e_chunks; }

void launch_energy(const PackView &v, cudaStream_t st, int mode, double *hist, int *step_dev) {
  if (!v.n_sys) return;
  const Consts &k = consts();
  int C = v.e_chunks;
  PDGPU_LAUNCH_DEP(k_energy<false>, dim3(C, v.n_sys), kEnergyThreads, 0, st, v, mode, C, k.J2kcal * k.Na, hist,
                   step_dev, MDDev{});
}
void launch_md_step_energy(const PackView &v, cudaStream_t st, const MDCoef &c, const unsigned char *is_h,
                           const unsigned long long *seeds, int mode, double *hist, int *step_dev) {
  if (!v.n_sys || !v.n_atoms) return;
  const Consts &k = consts();
  int C = v.e_chunks;
  PDGPU_LAUNCH_DEP(k_energy<true>, dim3(C, v.n_sys), kEnergyThreads, 0, st, v, mode | EM_KINETIC, C,
                   k.J2kcal * k.Na, hist, step_dev, make_md_dev(c, is_h, seeds));
}

}  // namespace pdgpu
