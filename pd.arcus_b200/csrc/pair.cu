// Pair kernels of the Still GB + LJ + Coulomb evaluation.
//
//   K2 k_born        calcBornRadii_PairwiseApprox     (gbff.cpp:415-466)
//   K3 k_gb_pair     calcForcesIncludingVacuo loop 1  (gbff.cpp:1529-1736)
//   K4 k_gb_chain    calcForcesIncludingVacuo loop 2  (gbff.cpp:1751-1818)
//      k_born_energy calcBornEnergy                   (gbff.cpp:520-579)
//      k_nonbonded   FF_NonBonded_CalcForces_T_fast2  (nonbonded.cpp:548-893)
//
// Layout: a group of LPA lanes (4, 8, 16 or 32; chosen per system by the
// autotuner) walks atom i's full neighbour row, so one warp serves 32/LPA
// atoms.  Rows are contiguous uint32 (j<<3|bondorder) entries.  Every atom
// accumulates only its own force, so no atomics touch j: per-lane FP32
// partials are summed in FP64 with a fixed shuffle tree inside the group and
// added to the atom's FP64 pair force by the group's first lane, kernel
// after kernel in stream order.  Results are bit-reproducible run to run for
// a given lanes-per-atom, and FP64 keeps the range of clashing trial
// structures.  Each neighbour costs one 32-byte record gather per kernel plus
// one 16-byte parameter gather.  The fused pass evaluates the GB and the
// vacuum Coulomb terms without branches (both computed, one selected), so
// the lanes of a group stay converged.
//
// Precision: pair arithmetic in FP32 on coordinates split as hi+lo floats
// (dx = (xi_hi - xj_hi) + (xi_lo - xj_lo), i.e. the FP64 difference rounded
// once).  The two discontinuous predicates of the reference -- the Still
// cutoff (Born sums, chain rule) and the GB exp-approximation threshold
// (uGB > -4 switches the solvent term off and Coulomb to eps=80) -- are
// decided in FP64 with the reference's exact expressions whenever the FP32
// value lies within a guard band of the threshold.  Born sums are FP64 per
// term (they feed the threshold through a_i*a_j) and fixed point across
// lanes; energies are FP64 sums of per-lane FP32 partials.
//
// Roofline: FP32/SFU-bound.  Algorithmic work per interaction: K2 21 flop +
// 3 SFU (directed pairs r<=10A, bo>=3), K3 90 flop + 5 SFU (unordered pairs
// r<=Rc), K4 36 flop + 4 SFU (as K2).
#include <cuda_runtime.h>

#include "pairmath.cuh"

namespace pdgpu {

// --------------------------------------------------------------- positions
// FP64 state -> the pair-kernel records (hi/lo floats, FP64 AoS copy).
__global__ void k_pack_positions(PackView v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  double x = v.x[i], y = v.y[i], z = v.z[i];
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

void launch_pack_positions(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_pack_positions, (v.n_atoms + 255) / 256, 256, 0, st, v);
}

// Interleaved [n][3] <-> three arrays, on the device: the state transfer
// calls move one contiguous block between the caller's buffer and a device
// staging array, with no host-side reshuffle.
__global__ void k_aos_to_soa(const double *aos, double *X, double *Y, double *Z, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  X[i] = aos[3 * (size_t)i];
  Y[i] = aos[3 * (size_t)i + 1];
  Z[i] = aos[3 * (size_t)i + 2];
}
__global__ void k_soa_to_aos(double *aos, const double *X, const double *Y, const double *Z, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  aos[3 * (size_t)i] = X[i];
  aos[3 * (size_t)i + 1] = Y[i];
  aos[3 * (size_t)i + 2] = Z[i];
}
// The MD state in and out of pdgpu_md_run_io in one launch each: positions
// (with the pair-kernel records) and velocities from / to interleaved
// [n][3] staging blocks (either may be absent).
__global__ void k_state_in(PackView v, const double *X, const double *V) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  if (X) {
    const double x = X[3 * (size_t)i], y = X[3 * (size_t)i + 1], z = X[3 * (size_t)i + 2];
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
  if (V) {
    v.vx[i] = V[3 * (size_t)i];
    v.vy[i] = V[3 * (size_t)i + 1];
    v.vz[i] = V[3 * (size_t)i + 2];
  }
}
__global__ void k_state_out(PackView v, double *X, double *V) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  if (X) {
    X[3 * (size_t)i] = v.x[i];
    X[3 * (size_t)i + 1] = v.y[i];
    X[3 * (size_t)i + 2] = v.z[i];
  }
  if (V) {
    V[3 * (size_t)i] = v.vx[i];
    V[3 * (size_t)i + 1] = v.vy[i];
    V[3 * (size_t)i + 2] = v.vz[i];
  }
}
void launch_state_in(const PackView &v, const double *X, const double *V, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_state_in, (v.n_atoms + 255) / 256, 256, 0, st, v, X, V);
}
void launch_state_out(const PackView &v, double *X, double *V, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_state_out, (v.n_atoms + 255) / 256, 256, 0, st, v, X, V);
}

void launch_aos_to_soa(const double *aos, double *X, double *Y, double *Z, int n, cudaStream_t st) {
  if (n > 0) PDGPU_LAUNCH(k_aos_to_soa, (n + 255) / 256, 256, 0, st, aos, X, Y, Z, n);
}
void launch_soa_to_aos(double *aos, const double *X, const double *Y, const double *Z, int n, cudaStream_t st) {
  if (n > 0) PDGPU_LAUNCH(k_soa_to_aos, (n + 255) / 256, 256, 0, st, aos, X, Y, Z, n);
}

__global__ void k_zero(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < v.n_atoms) {
    v.fx[i] = 0;
    v.fy[i] = 0;
    v.fz[i] = 0;
    v.gx[i] = 0.0;
    v.gy[i] = 0.0;
    v.gz[i] = 0.0;
    v.hx[i] = 0;
    v.hy[i] = 0;
    v.hz[i] = 0;
    v.bsum[i] = 0;
    for (int k = 0; k < 4; k++) v.ej[(size_t)k * v.n_atoms + i] = 0;
#pragma unroll
    for (int k = 0; k < AE_COUNT; k++) v.e_atom[(size_t)k * v.n_atoms + i] = 0.0;
  }
  if (i < v.n_sys * E_COUNT) {
    // keep the kinetic slots; zero the potential record (WorkSpace::zeroForces)
    int slot = i % E_COUNT;
    if (slot != E_EKIN) v.ene[i] = 0.0;
  }
}

void launch_zero(const PackView &v, cudaStream_t st) {
  int n = max(v.n_atoms, v.n_sys * E_COUNT);
  if (n) PDGPU_LAUNCH(k_zero, (n + 255) / 256, 256, 0, st, v);
}

// --------------------------------------------------------------- K2 radii
// Born-radius sums in FP32 per term (hi/lo coordinate differences), each
// term converted to 64-bit fixed point (2^40) before it is added, so the
// sum is exact in integers: independent of the order of the row, of the
// lanes per atom and of the batch the system sits in.  The Still cutoff
// (r <= GbsaStillCutoff, a jump in the sum) is decided in FP64 with the
// reference's expression when the FP32 distance lies within a guard band;
// the close-contact factor CCF is continuous at its threshold.  The
// inversion a_i = -halfeconv / Gpol_i is FP64.
template <int LPA>
__global__ void __launch_bounds__(256) k_born(PackView v, int zero_first) {
  if (v.flags[F_NL_OVERFLOW]) return;  // list incomplete: the host re-plans
  const int sub = threadIdx.x % LPA;
  constexpr int G = 256 / LPA;  // atoms per block and pass
  for (int i0 = blockIdx.x * G; i0 < v.n_atoms; i0 += gridDim.x * G) {
    const int i = i0 + (int)threadIdx.x / LPA;
    const bool valid = i < v.n_atoms;
    const int ii = valid ? i : 0;
    const int s = v.sys_of[ii];
    const SysParams &P = v.sp[s];
    if (valid && zero_first && sub < 3) {
      // WorkSpace::zeroForces for this atom (and the record, by the first atom)
      long long *f = sub == 0 ? v.fx : (sub == 1 ? v.fy : v.fz);
      double *g = sub == 0 ? v.gx : (sub == 1 ? v.gy : v.gz);
      long long *h = sub == 0 ? v.hx : (sub == 1 ? v.hy : v.hz);
      if (zero_first & ZF_BONDED) f[i] = 0;
      g[i] = 0.0;
      h[i] = 0;
      if ((zero_first & ZF_RECORD) && i == v.atom_off[s]) {
        for (int k = sub; k < E_COUNT; k += 3)
          if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
        if (sub == 0) v.sys_flags[s] = 0;
      }
    }
    const float4 ia = v.pq[2 * (size_t)ii], ib = v.pq[2 * (size_t)ii + 1];
    const float Ri = v.chainp[ii].x;
    const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
    const float invP5 = P.invP5, piP5 = P.piP5, P4s = P.P4 * (float)kBornScale;
    const double still2_d = P.still2_d;
    long long acc = 0;
    const long long e = valid ? v.row_start[i + 1] : 0;
#pragma unroll 2
    for (long long k = (valid ? v.row_start[i] : 0) + sub; k < e; k += LPA) {
      const unsigned ent = v.nl[k];
      if ((ent & 7u) > 2u) {  // 1-2 and 1-3 partners carry no Born term
        const int j = (int)(ent >> 3);
        const float4 ja = v.pq[2 * (size_t)j], jb = v.pq[2 * (size_t)j + 1], jc = v.chainp[j];
        const Dx d = diff(ia, ib, ja, jb);
        bool in = d.r2 <= s_lo;
        if (!in && d.r2 <= s_hi) in = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > still2_d);
        if (in) acc += __float2ll_rn(__fmul_rn(born_term_noV(d, Ri, jc.x, invP5, piP5, P4s), jc.y));
      }
    }
    const long long fixed = group_sum<LPA>(acc);
    if (valid && sub == 0) {
      double Gpol = v.terms123[i] + (double)fixed * kInvBornScale;
      double a = -P.halfeconv_d / Gpol + P.born_offset_d;
      v.born_d[i] = a;
      reinterpret_cast<float *>(&v.pq[2 * (size_t)i + 1])[3] = (float)a;
    }
  }
}

// Blocks for a persistent pass over the atoms: every SM holds the same
// number of resident blocks, each walking atoms block-strided.
template <typename K>
static int persistent_blocks(K kern, int n_atoms, int lpa) {
  static int sms = 0, occ = 0;  // per kernel instantiation
  if (!occ) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, 0) != cudaSuccess || occ <= 0) occ = 1;
  }
  long long need = ((long long)n_atoms * lpa + 255) / 256;
  long long cap = (long long)sms * occ;
  return (int)(need < cap ? need : cap);
}

void launch_born_radii_lpa(const PackView &v, cudaStream_t st, int zero_first, int lpa) {
  if (!v.n_atoms) return;
  switch (lpa) {
    case 4: PDGPU_LAUNCH(k_born<4>, persistent_blocks(k_born<4>, v.n_atoms, 4), 256, 0, st, v, zero_first); break;
    case 16: PDGPU_LAUNCH(k_born<16>, persistent_blocks(k_born<16>, v.n_atoms, 16), 256, 0, st, v, zero_first); break;
    case 32: PDGPU_LAUNCH(k_born<32>, persistent_blocks(k_born<32>, v.n_atoms, 32), 256, 0, st, v, zero_first); break;
    default: PDGPU_LAUNCH(k_born<8>, persistent_blocks(k_born<8>, v.n_atoms, 8), 256, 0, st, v, zero_first); break;
  }
}

// --------------------------------------------------------------- K3 pair
template <int LPA>
__global__ void __launch_bounds__(256, 4) k_gb_pair(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sub = threadIdx.x % LPA;
  constexpr int G = 256 / LPA;
  for (int i0 = blockIdx.x * G; i0 < v.n_atoms; i0 += gridDim.x * G) {
  const int i = i0 + (int)threadIdx.x / LPA;
  const bool valid = i < v.n_atoms;
  const int ii = valid ? i : 0;
  const SysParams &P = v.sp[v.sys_of[ii]];
  const float4 ia = v.pq[2 * (size_t)ii], ib = v.pq[2 * (size_t)ii + 1], ip = v.prm[ii];
  const float ai = ib.w;
  const float qi = ia.w, radi = ip.x, epsi = ip.y;
  GbSettings gs;  // every setting in registers for the whole row
  gs.load(P);
  float fx = 0.f, fy = 0.f, fz = 0.f;  // -dE/dr_i, kcal/mol/A
  float e_vdw = 0.f, e_el = 0.f, e_pol = 0.f, deda = 0.f;
  const long long e = valid ? v.row_start[i + 1] : 0;
#pragma unroll 2
  for (long long k = (valid ? v.row_start[i] : 0) + sub; k < e; k += LPA) {
    const unsigned ent = v.nl[k];
    const int j = (int)(ent >> 3);
    const float4 ja = v.pq[2 * (size_t)j], jb = v.pq[2 * (size_t)j + 1], jp = v.prm[j];
    const Dx d = diff(ia, ib, ja, jb);
    if (d.r2 <= gs.rc2) {
      const int bo = (int)(ent & 7u);
      // LJ and vacuum Coulomb apply from bond order 3 (1-4, scaled) on
      const GbPair t = gb_pair_term(gs, d, bo >= 3, bo == 3, ai, jb.w, qi, ja.w, radi, jp.x, epsi, jp.y, v, i, j);
      e_pol += t.epol;
      deda += t.dedal * jb.w;
      e_vdw += t.vdw;
      e_el += t.elec;
      fx -= t.fscal * d.x;
      fy -= t.fscal * d.y;
      fz -= t.fscal * d.z;
    }
  }
  const double sx = group_sum<LPA>((double)fx);
  const double sy = group_sum<LPA>((double)fy);
  const double sz = group_sum<LPA>((double)fz);
  const double dv = group_sum<LPA>((double)e_vdw);
  const double de = group_sum<LPA>((double)e_el);
  const double dp = group_sum<LPA>((double)e_pol);
  const double dd = group_sum<LPA>((double)deda);
  if (valid && sub == 0) {
    v.gx[i] += sx;
    v.gy[i] += sy;
    v.gz[i] += sz;
    const int N = v.n_atoms;
    double ai_d = v.born_d[i];
    double qd = (double)qi;
    double eself = P.premul_d * qd * qd / ai_d;
    v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv;
    v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
    v.e_atom[(size_t)AE_POL * N + i] = dp;
    v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
    double deda_i = dd - eself / ai_d;
    double gpi = ai_d * ai_d / 166.0;  // gbff.cpp:1755 uses the literal 166.0
    reinterpret_cast<float *>(&v.chainp[i])[2] = (float)(gpi * deda_i);
  }
  }
}

void launch_gb_pair_lpa(const PackView &v, cudaStream_t st, int lpa) {
  if (!v.n_atoms) return;
  switch (lpa) {
    case 4: PDGPU_LAUNCH(k_gb_pair<4>, persistent_blocks(k_gb_pair<4>, v.n_atoms, 4), 256, 0, st, v); break;
    case 16: PDGPU_LAUNCH(k_gb_pair<16>, persistent_blocks(k_gb_pair<16>, v.n_atoms, 16), 256, 0, st, v); break;
    case 32: PDGPU_LAUNCH(k_gb_pair<32>, persistent_blocks(k_gb_pair<32>, v.n_atoms, 32), 256, 0, st, v); break;
    default: PDGPU_LAUNCH(k_gb_pair<8>, persistent_blocks(k_gb_pair<8>, v.n_atoms, 8), 256, 0, st, v); break;
  }
}

// --------------------------------------------------------------- K4 chain
template <int LPA>
__global__ void __launch_bounds__(256) k_gb_chain(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sub = threadIdx.x % LPA;
  constexpr int G = 256 / LPA;
  for (int i0 = blockIdx.x * G; i0 < v.n_atoms; i0 += gridDim.x * G) {
  const int i = i0 + (int)threadIdx.x / LPA;
  const bool valid = i < v.n_atoms;
  const int ii = valid ? i : 0;
  const SysParams &P = v.sp[v.sys_of[ii]];
  const float4 ia = v.pq[2 * (size_t)ii], ib = v.pq[2 * (size_t)ii + 1], ic = v.chainp[ii];
  const float Ri = ic.x, Vi = ic.y, wi = ic.z;
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  const float invP5 = P.invP5, piP5 = P.piP5, P4 = P.P4;
  const double still2_d = P.still2_d;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  const long long e = valid ? v.row_start[i + 1] : 0;
#pragma unroll 2
  for (long long k = (valid ? v.row_start[i] : 0) + sub; k < e; k += LPA) {
    const unsigned ent = v.nl[k];
    const int j = (int)(ent >> 3);
    const float4 ja = v.pq[2 * (size_t)j], jb = v.pq[2 * (size_t)j + 1], jc = v.chainp[j];
    if ((ent & 7u) > 2u) {
      const Dx d = diff(ia, ib, ja, jb);
      bool in = d.r2 <= s_lo;
      if (!in && d.r2 <= s_hi) {
        double d2 = ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]);
        in = !(d2 > still2_d);
      }
      if (in) {
        const float tt = chain_term(d, Ri, jc.x, Vi, jc.y, wi, jc.z, invP5, piP5, P4);
        fx += tt * d.x;
        fy += tt * d.y;
        fz += tt * d.z;
      }
    }
  }
  const double sx = group_sum<LPA>((double)fx);
  const double sy = group_sum<LPA>((double)fy);
  const double sz = group_sum<LPA>((double)fz);
  if (valid && sub == 0) {
    v.gx[i] += sx;
    v.gy[i] += sy;
    v.gz[i] += sz;
  }
  }
}

void launch_gb_chain_lpa(const PackView &v, cudaStream_t st, int lpa) {
  if (!v.n_atoms) return;
  switch (lpa) {
    case 4: PDGPU_LAUNCH(k_gb_chain<4>, persistent_blocks(k_gb_chain<4>, v.n_atoms, 4), 256, 0, st, v); break;
    case 16: PDGPU_LAUNCH(k_gb_chain<16>, persistent_blocks(k_gb_chain<16>, v.n_atoms, 16), 256, 0, st, v); break;
    case 32: PDGPU_LAUNCH(k_gb_chain<32>, persistent_blocks(k_gb_chain<32>, v.n_atoms, 32), 256, 0, st, v); break;
    default: PDGPU_LAUNCH(k_gb_chain<8>, persistent_blocks(k_gb_chain<8>, v.n_atoms, 8), 256, 0, st, v); break;
  }
}

void launch_born_radii(const PackView &v, cudaStream_t st, int zero_first) {
  if (v.tile_mode)
    launch_born_radii_tile(v, st, zero_first);
  else
    launch_born_radii_lpa(v, st, zero_first, v.lpa[0]);
}
void launch_gb_pair(const PackView &v, cudaStream_t st) {
  if (v.tile_mode)
    launch_gb_pair_tile(v, st);
  else
    launch_gb_pair_lpa(v, st, v.lpa[1]);
}
void launch_gb_chain(const PackView &v, cudaStream_t st) {
  if (v.tile_mode)
    launch_gb_chain_tile(v, st);
  else
    launch_gb_chain_lpa(v, st, v.lpa[2]);
}

// --------------------------------------------------------------- Born energy
// Energy-only Born term: all pairs r <= Rc, no exp threshold, energy switch.
__global__ void __launch_bounds__(256) k_born_energy(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1];
  float acc = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int j = (int)(ent >> 3);
    float4 ja = v.pq[2 * (size_t)j], jb = v.pq[2 * (size_t)j + 1];
    Dx d = diff(ia, ib, ja, jb);
    if (d.r2 > P.rc2) continue;
    float r = sqrtf(d.r2);
    float S = 1.f;
    if (!(r < P.rin)) {
      float dd = r - P.rin;
      float s = 1.f - P.inv_sw2 * dd * dd;
      S = s * s;
    }
    float aiaj = ib.w * jb.w;
    float t = __expf(__fdividef(-d.r2 * 0.25f, aiaj));
    acc += S * ia.w * ja.w * rsqrtf(d.r2 + aiaj * t);
  }
  double sum = group_sum<32>((double)acc);
  if (lane == 0) {
    const int N = v.n_atoms;
    double ai = v.born_d[i];
    double q = (double)ia.w;
    double eself = P.premul_d * q * q / ai;
    v.e_atom[(size_t)AE_POL * N + i] = P.premul_d * sum;
    v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
  }
}

void launch_born_energy(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_born_energy, (v.n_atoms + 7) / 8, 256, 0, st, v);
}

// --------------------------------------------------------------- LJ/Coulomb
// FF_NonBonded fast2 kernel: all unordered pairs r <= Rc (each atom sums its
// own side, energies weighted 1/2).  Modes as selected by calcForces.
template <int EM>
__device__ __forceinline__ void nb_elec(const SysParams &P, float r, float r2, float invr, float qq,
                                        float &pot, float &frc) {
  pot = 0.f;
  frc = 0.f;
  if (EM == 1) {
    pot = P.econv_nb * qq * invr;
    frc = -pot * invr;
  } else if (EM == 2) {
    float inc = (P.dielectric + P.ddd_alpha * r) * r;
    pot = P.econv_nb * P.dielectric * qq / inc;  // econv * qq / inc
    frc = -pot * (P.dielectric + 2.f * P.ddd_alpha * r) / inc;
  } else if (EM == 3) {
    pot = P.econv_nb * qq * invr;
    frc = -pot * invr;
    if (r > P.rin) {
      float d = r - P.rin;
      float s = 1.f - P.inv_sw2 * d * d;
      float ds = -4.f * P.inv_sw2 * d * s;
      s = s * s;
      frc = s * frc + pot * ds;
      pot *= s;
    }
  } else if (EM == 4) {
    float base = P.econv_nb * qq;
    float rc2 = P.rc2, ri2 = P.rin * P.rin;
    if (r > P.rin) {
      float w = rc2 - r2;
      frc = -base * P.fs_A * invr * invr * w * w * (rc2 - 3.f * ri2 + 2.f * r2);
      pot = -base * (P.fs_A * r * (P.fs_B * invr * invr + P.fs_C + P.fs_D * r2 + P.fs_E * r2 * r2) -
                     P.fs_cutV);
    } else {
      frc = -base * invr * invr;
      pot = base * (invr - P.fs_eshift);
    }
  }
}

template <int EM>
__global__ void __launch_bounds__(256) k_nonbonded(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ip = v.prm[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, e_vdw = 0.f, e_el = 0.f, vir = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int bo = (int)(ent & 7u);
    if (bo < 3) continue;  // the 1-4 scaling table zeroes 1-2 and 1-3 pairs
    int j = (int)(ent >> 3);
    float4 ja = v.pq[2 * (size_t)j], jb = v.pq[2 * (size_t)j + 1];
    Dx d = diff(ia, ib, ja, jb);
    float r2 = d.r2;
    if (EM == 1 || EM == 2) {
      // unswitched Coulomb is discontinuous at Rc: decide boundary pairs
      // with the reference's FP64 expression (fv = p_j - p_i; innerdot)
      if (fabsf(r2 - P.rc2) <= 4e-6f * P.rc2) {
        double d2 = ref_d2(v.x[j], v.y[j], v.z[j], v.x[i], v.y[i], v.z[i]);
        if (d2 > P.rc2_d) continue;
      } else if (r2 > P.rc2) {
        continue;
      }
    } else if (r2 > P.rc2) {
      continue;
    }
    float invr = rsqrtf(r2);
    float r = r2 * invr;
    float vdw = 0.f, vdwf = 0.f;
    if (P.vdw_mode && r < P.vdw_rc) {
      float4 jp = v.prm[j];
      float rr = (ip.x + jp.x) * invr;
      float rr2 = rr * rr;
      float B = rr2 * rr2 * rr2;
      float A = B * B;
      float eps = ((bo == 3) ? P.vdw14 : 1.f) * ip.y * jp.y;
      vdw = (2.f * eps) * (0.5f * A - B);
      vdwf = -(12.f * eps * invr) * (A - B);
      if (r > P.vdw_rin) {
        float dd = r - P.vdw_rin;
        float s = 1.f - P.vdw_inv_sw2 * dd * dd;
        float ds = -4.f * P.vdw_inv_sw2 * dd * s;
        s = s * s;
        vdwf = s * vdwf + vdw * ds;
        vdw *= s;
      }
    }
    float pot, frc;
    float qq = ia.w * ja.w * ((bo == 3) ? P.elec14 : 1.f);
    nb_elec<EM>(P, r, r2, invr, qq, pot, frc);
    float fm = vdwf + frc;
    e_vdw += vdw;
    e_el += pot;
    vir += r * fm;
    float s = fm * invr;  // force on i along (p_j - p_i): f_i += s * (p_j - p_i)
    fx -= s * d.x;
    fy -= s * d.y;
    fz -= s * d.z;
  }
  double sx = group_sum<32>((double)fx);
  double sy = group_sum<32>((double)fy);
  double sz = group_sum<32>((double)fz);
  double dv = group_sum<32>((double)e_vdw);
  double de = group_sum<32>((double)e_el);
  double dw = group_sum<32>((double)vir);
  if (lane == 0) {
    v.gx[i] += sx;
    v.gy[i] += sy;
    v.gz[i] += sz;
    const int N = v.n_atoms;
    v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv + P.vdwcor_e_d;
    v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
    v.e_atom[(size_t)AE_VIR * N + i] = 0.5 * dw;
  }
}

void launch_nonbonded(const PackView &v, cudaStream_t st, int elec_mode) {
  if (!v.n_atoms) return;
  // the mode is per system; a pack holds systems of one mode (checked when
  // the pack is built)
  int blocks = (v.n_atoms + 7) / 8;
  switch (elec_mode) {
    case 0: PDGPU_LAUNCH((k_nonbonded<0>), blocks, 256, 0, st, v); break;
    case 1: PDGPU_LAUNCH((k_nonbonded<1>), blocks, 256, 0, st, v); break;
    case 2: PDGPU_LAUNCH((k_nonbonded<2>), blocks, 256, 0, st, v); break;
    case 3: PDGPU_LAUNCH((k_nonbonded<3>), blocks, 256, 0, st, v); break;
    default: PDGPU_LAUNCH((k_nonbonded<4>), blocks, 256, 0, st, v); break;
  }
}

// --------------------------------------------------------------- pair counts
// Instrumentation: the pair sets the roofline counts use, decided exactly as
// the kernels decide them.  out[0] P_B (directed, r <= still cutoff, bo >= 3),
// out[1] P_H (unordered, r <= Rc), out[2] list entries.
__global__ void k_pair_counts(PackView v, unsigned long long *out) {
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1];
  unsigned long long pb = 0, ph = 0;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int j = (int)(ent >> 3);
    Dx d = diff(ia, ib, v.pq[2 * (size_t)j], v.pq[2 * (size_t)j + 1]);
    if (j < i && d.r2 <= P.rc2) ph++;
    if ((ent & 7u) > 2u && ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) <= P.still2_d) pb++;
  }
  pb = group_sum<32>(pb);
  ph = group_sum<32>(ph);
  if (lane == 0) {
    atomicAdd(&out[0], pb);
    atomicAdd(&out[1], ph);
    atomicAdd(&out[2], (unsigned long long)(e - b));
  }
}

void launch_pair_counts(const PackView &v, cudaStream_t st, unsigned long long *out) {
  if (v.n_atoms) PDGPU_LAUNCH(k_pair_counts, (v.n_atoms + 7) / 8, 256, 0, st, v, out);
}

}  // namespace pdgpu
