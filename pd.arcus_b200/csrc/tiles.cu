// Cluster-pair tiles: the neighbour pair set re-cut into 32 x 8 blocks so
// the three pair passes read their partners with coalesced loads and each
// unordered pair is evaluated once.
//
// Atoms of a system are cut, in their own order (residue order: bonded and
// spatially close atoms are neighbours in memory), into i-clusters of 32
// (one per lane of a warp) and j-clusters of 8.  A tile is an (i-cluster,
// j-cluster) pair of one system whose bounding boxes lie within the list
// radius, with j-cluster start >= i-cluster start; its 32 x 8 bit mask holds
// exactly the pairs of the reference's neighbour list (the same FP64
// distance predicate, neighbourlist.cpp:263-266) with j > i where the
// j-cluster lies inside the i-cluster, so every unordered list pair sits in
// exactly one tile.  Tiles with 1-2, 1-3 or 1-4 partners (the bond-order
// band and the off-diagonal list) carry two more masks: bond order <= 2 and
// bond order == 3.
//
// Each pass runs one block per i-cluster; its warps take the cluster's
// tiles in turn.  A warp stages the tile's 8 j atoms in shared memory, then
// every lane (one i atom) walks them: the i side accumulates in registers,
// the j side is summed over the warp with shuffles and added to the j atom
// with 64-bit fixed-point atomics (order-independent).  Per-lane i sums are
// added in fixed warp order.  Pass results:
//   K2 k_born_tile   Born sums, i and j side, fixed point 2^40 (exact);
//                    k_born_finish inverts them (FP64) and zeroes the j-side
//                    accumulators of the next passes
//   K3 k_gb_tile     forces (i: FP64 pair force, j: fixed point 2^24),
//                    per-atom LJ / Coulomb / GB energies and dE/da (i side
//                    FP64, j side fixed point); k_gb_finish forms the
//                    reference's per-atom values and the chain-rule weights
//   K4 k_chain_tile  chain-rule forces (i and j side as K3)
// The per-pair arithmetic is the row kernels' (pairmath.cuh).
#include <cuda_runtime.h>

#include "pairmath.cuh"

namespace pdgpu {

constexpr int kTileWarps = 4;  // warps per block (one block per i-cluster)

// --------------------------------------------------------------- boxes
// FP64 bounding box of every cluster; a cluster with a NaN coordinate gets
// an infinite box, so its pairs are decided by the exact test as in the
// neighbour list (which keeps pairs whose distance compares false).
__global__ void k_cluster_bbox(PackView v) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.n_sc + v.n_jc) return;
  bool is_i = c < v.n_sc;
  int k = is_i ? c : c - v.n_sc;
  int a0 = is_i ? v.sc_atom0[k] : v.jc_atom0[k];
  int s = is_i ? v.sc_sys[k] : v.jc_sys[k];
  int n = min(is_i ? 32 : 8, v.atom_off[s + 1] - a0);
  double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
  bool nan = false;
  for (int a = a0; a < a0 + n; a++) {
    double p[3] = {v.x[a], v.y[a], v.z[a]};
    for (int q = 0; q < 3; q++) {
      if (!(p[q] == p[q])) nan = true;
      lo[q] = fmin(lo[q], p[q]);
      hi[q] = fmax(hi[q], p[q]);
    }
  }
  double *b = (is_i ? v.sc_bb : v.jc_bb) + 6 * (size_t)k;
  for (int q = 0; q < 3; q++) {
    b[q] = nan ? -INFINITY : lo[q];
    b[3 + q] = nan ? INFINITY : hi[q];
  }
}

__device__ __forceinline__ double box_gap2(const double *a, const double *b) {
  double g2 = 0.0;
  for (int q = 0; q < 3; q++) {
    double g = fmax(0.0, fmax(a[q] - b[3 + q], b[q] - a[3 + q]));
    g2 += g * g;
  }
  return g2;
}

// --------------------------------------------------------------- tile list
// One warp per i-cluster: candidates by box distance, then the exact pair
// masks.  Two passes over the candidates (count, then fill after one atomic
// reservation), so a cluster's tiles are contiguous and ordered by j-cluster.
__global__ void k_tile_build(PackView v) {
  const int lane = threadIdx.x & 31;
  const int sc = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (sc >= v.n_sc) return;
  if (v.flags[F_NL_OVERFLOW]) return;
  const int s = v.sc_sys[sc];
  const int a0 = v.sc_atom0[sc];
  const int na = min(32, v.atom_off[s + 1] - a0);
  const double lim = v.sp[s].nl_lim2_d;
  const int mid = v.mid[s];
  const bool has_off = v.off_ptr[v.atom_off[s + 1]] > v.off_ptr[v.atom_off[s]];
  const int i = a0 + lane;
  const bool vi = lane < na;
  const double xi = vi ? v.x[i] : 0.0, yi = vi ? v.y[i] : 0.0, zi = vi ? v.z[i] : 0.0;
  double bbi[6];
  for (int q = 0; q < 6; q++) bbi[q] = v.sc_bb[6 * (size_t)sc + q];
  const int j_first = v.jc_off[s] + (a0 - v.atom_off[s]) / 8;  // first j-cluster at or after a0
  const int j_end = v.jc_off[s + 1];
  int base = 0, count = 0;
  for (int pass = 0; pass < 2; pass++) {
    int k = 0;
    for (int J0 = j_first; J0 < j_end; J0 += 32) {
      const int Jl = J0 + lane;
      bool cand = false;
      if (Jl < j_end) cand = box_gap2(bbi, v.jc_bb + 6 * (size_t)Jl) <= lim;
      unsigned cm = __ballot_sync(0xffffffffu, cand);
      while (cm) {
        const int J = J0 + __ffs(cm) - 1;
        cm &= cm - 1;
        const int b0 = v.jc_atom0[J];
        const int nb = min(8, v.atom_off[s + 1] - b0);
        const bool inside = b0 < a0 + 32;  // the j-cluster lies in this i-cluster
        unsigned m[8];
        unsigned any = 0;
#pragma unroll
        for (int t = 0; t < 8; t++) {
          const int j = b0 + t;
          bool in = false;
          if (vi && t < nb && j != i && (!inside || j > i)) {
            double d2 = ref_d2(xi, yi, zi, v.x[j], v.y[j], v.z[j]);
            in = !(d2 > lim);
          }
          m[t] = __ballot_sync(0xffffffffu, in);
          any |= m[t];
        }
        if (!any) continue;
        if (pass == 1) {
          const int e = base + k;
          if (lane < 8) v.tile_mask[8 * (size_t)e + lane] = m[lane & 7];
          // bond orders other than 7 inside the tile
          int spec = -1;
          const bool near = b0 - (a0 + na - 1) < mid;  // some |i-j| < MaxIndexDelta
          if (near || has_off) {
            unsigned ex[8], b14[8], anyb = 0;
#pragma unroll
            for (int t = 0; t < 8; t++) {
              int bo = 7;
              if ((m[t] >> lane) & 1u) bo = bond_order(v, s, i, b0 + t);
              ex[t] = __ballot_sync(0xffffffffu, bo <= 2);
              b14[t] = __ballot_sync(0xffffffffu, bo == 3);
              anyb |= ex[t] | b14[t];
            }
            if (anyb) {
              if (lane == 0) spec = atomicAdd(&v.tile_count[1], 1);
              spec = __shfl_sync(0xffffffffu, spec, 0);
              if (spec < v.spec_cap) {
                if (lane < 8) {
                  v.spec_mask[16 * (size_t)spec + lane] = ex[lane & 7];
                  v.spec_mask[16 * (size_t)spec + 8 + lane] = b14[lane & 7];
                }
              } else {
                if (lane == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
                spec = -1;
              }
            }
          }
          if (lane == 0) {
            v.tile_jc[e] = J;
            v.tile_spec[e] = spec;
          }
        }
        k++;
      }
    }
    if (pass == 0) {
      count = k;
      if (lane == 0) base = atomicAdd(&v.tile_count[0], count);
      base = __shfl_sync(0xffffffffu, base, 0);
      if ((long long)base + count > v.tile_cap) {  // cannot happen: capacity is the worst case
        if (lane == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
        return;
      }
    }
  }
  if (lane == 0) {
    v.tile_e0[sc] = base;
    v.tile_e1[sc] = base + count;
  }
}

// --------------------------------------------------------------- K2 tiles
__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ float warp_sum_f(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ long long to_fixed_j(float f) {
  // saturate far outside any physical range (clashing trial structures
  // stay well inside: 2^39 kcal/mol/A)
  float s = fminf(fmaxf(f * (float)kJScale, -9.0e18f), 9.0e18f);
  return __float2ll_rn(s);
}

__global__ void __launch_bounds__(32 * kTileWarps) k_born_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  const int a0 = v.sc_atom0[sc];
  const int na = min(32, v.atom_off[s + 1] - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ic = v.chainp[i];
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  const float invP5 = P.invP5, piP5 = P.piP5, P4s = P.P4 * (float)kBornScale;
  const double still2_d = P.still2_d;
  long long acc_i = 0;
  const int e1 = v.tile_e1[sc];
  for (int e = v.tile_e0[sc] + warp; e < e1; e += kTileWarps) {
    const int J = v.tile_jc[e];
    const int b0 = v.jc_atom0[J];
    const int nb = min(8, v.atom_off[s + 1] - b0);
    if (lane < nb) {
      sA[warp][lane] = v.pq[2 * (size_t)(b0 + lane)];
      sB[warp][lane] = v.pq[2 * (size_t)(b0 + lane) + 1];
      sC[warp][lane] = v.chainp[b0 + lane];
    }
    const unsigned mine = v.tile_mask[8 * (size_t)e + (lane & 7)];
    const int spec = v.tile_spec[e];
    const unsigned exl = spec >= 0 ? v.spec_mask[16 * (size_t)spec + (lane & 7)] : 0u;
    __syncwarp();
    long long jsum = 0;  // lane t keeps j atom t's total
    for (int t = 0; t < nb; t++) {
      const unsigned mt = __shfl_sync(0xffffffffu, mine, t);
      const unsigned xt = __shfl_sync(0xffffffffu, exl, t);
      bool in = ((mt & ~xt) >> lane) & 1u;  // in the list, bond order > 2
      const float4 ja = sA[warp][t], jb = sB[warp][t], jc = sC[warp][t];
      long long ti = 0, tj = 0;
      if (in) {
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi)
          ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[b0 + t], v.y[b0 + t], v.z[b0 + t]) > still2_d);
        if (ok) {
          const float term = born_term_noV(d, ic.x, jc.x, invP5, piP5, P4s);
          ti = __float2ll_rn(term * jc.y);
          tj = __float2ll_rn(term * ic.y);
        }
      }
      acc_i += ti;
      const long long tot = warp_sum_ll(tj);
      if (lane == t) jsum = tot;
    }
    if (lane < nb && jsum) atomicAdd((unsigned long long *)&v.bsum[b0 + lane], (unsigned long long)jsum);
    __syncwarp();
  }
  if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
}

// a_i = -halfeconv / (terms123_i + sum) (FP64); zero the accumulators the
// following passes add into (and, first in an evaluation, the forces)
__global__ void k_born_finish(PackView v, int zero_first) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  const int s = v.sys_of[i];
  const SysParams &P = v.sp[s];
  long long sum = v.bsum[i];
  v.bsum[i] = 0;
  double Gpol = v.terms123[i] + (double)sum * kInvBornScale;
  double a = -P.halfeconv_d / Gpol + P.born_offset_d;
  v.born_d[i] = a;
  reinterpret_cast<float *>(&v.pq[2 * (size_t)i + 1])[3] = (float)a;
  const int N = v.n_atoms;
  for (int q = 0; q < 4; q++) v.ej[(size_t)q * N + i] = 0;
  if (zero_first) {
    v.fx[i] = 0;
    v.fy[i] = 0;
    v.fz[i] = 0;
    v.gx[i] = 0.0;
    v.gy[i] = 0.0;
    v.gz[i] = 0.0;
    v.hx[i] = 0;
    v.hy[i] = 0;
    v.hz[i] = 0;
    if (i == v.atom_off[s])
      for (int k = 0; k < E_COUNT; k++)
        if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
  }
}

// --------------------------------------------------------------- K3 tiles
__global__ void __launch_bounds__(32 * kTileWarps) k_gb_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sP[kTileWarps][8];
  __shared__ float red[kTileWarps][7][32];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  GbSettings gs;
  gs.load(P);
  const int a0 = v.sc_atom0[sc];
  const int na = min(32, v.atom_off[s + 1] - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ip = v.prm[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, e_vdw = 0.f, e_el = 0.f, e_pol = 0.f, deda = 0.f;
  const int N = v.n_atoms;
  const int e1 = v.tile_e1[sc];
  for (int e = v.tile_e0[sc] + warp; e < e1; e += kTileWarps) {
    const int J = v.tile_jc[e];
    const int b0 = v.jc_atom0[J];
    const int nb = min(8, v.atom_off[s + 1] - b0);
    if (lane < nb) {
      sA[warp][lane] = v.pq[2 * (size_t)(b0 + lane)];
      sB[warp][lane] = v.pq[2 * (size_t)(b0 + lane) + 1];
      sP[warp][lane] = v.prm[b0 + lane];
    }
    const unsigned mine = v.tile_mask[8 * (size_t)e + (lane & 7)];
    const int spec = v.tile_spec[e];
    const unsigned exl = spec >= 0 ? v.spec_mask[16 * (size_t)spec + (lane & 7)] : 0u;
    const unsigned b14l = spec >= 0 ? v.spec_mask[16 * (size_t)spec + 8 + (lane & 7)] : 0u;
    __syncwarp();
    float jv[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // lane t: j atom t's totals
    for (int t = 0; t < nb; t++) {
      const unsigned mt = __shfl_sync(0xffffffffu, mine, t);
      const unsigned xt = __shfl_sync(0xffffffffu, exl, t);
      const unsigned bt = __shfl_sync(0xffffffffu, b14l, t);
      const float4 ja = sA[warp][t], jb = sB[warp][t], jp = sP[warp][t];
      const Dx d = diff(ia, ib, ja, jb);
      const bool in = ((mt >> lane) & 1u) && d.r2 <= gs.rc2;
      float c[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (in) {
        const bool nb3 = !((xt >> lane) & 1u);  // bond order >= 3
        const bool b14 = (bt >> lane) & 1u;
        const GbPair g = gb_pair_term(gs, d, nb3, b14, ib.w, jb.w, ia.w, ja.w, ip.x, jp.x, ip.y, jp.y, v, i,
                                      b0 + t);
        e_pol += g.epol;
        deda += g.dedal * jb.w;
        e_vdw += g.vdw;
        e_el += g.elec;
        fx -= g.fscal * d.x;
        fy -= g.fscal * d.y;
        fz -= g.fscal * d.z;
        c[0] = g.fscal * d.x;
        c[1] = g.fscal * d.y;
        c[2] = g.fscal * d.z;
        c[3] = g.vdw;
        c[4] = g.elec;
        c[5] = g.epol;
        c[6] = g.dedal * ib.w;
      }
#pragma unroll
      for (int q = 0; q < 7; q++) {
        const float tot = warp_sum_f(c[q]);
        if (lane == t) jv[q] = tot;
      }
    }
    if (lane < nb) {
      const int j = b0 + lane;
      atomicAdd((unsigned long long *)&v.hx[j], (unsigned long long)to_fixed_j(jv[0]));
      atomicAdd((unsigned long long *)&v.hy[j], (unsigned long long)to_fixed_j(jv[1]));
      atomicAdd((unsigned long long *)&v.hz[j], (unsigned long long)to_fixed_j(jv[2]));
#pragma unroll
      for (int q = 0; q < 4; q++)
        atomicAdd((unsigned long long *)&v.ej[(size_t)q * N + j], (unsigned long long)to_fixed_j(jv[3 + q]));
    }
    __syncwarp();
  }
  // i side: the warps' partials in fixed order
  red[warp][0][lane] = fx;
  red[warp][1][lane] = fy;
  red[warp][2][lane] = fz;
  red[warp][3][lane] = e_vdw;
  red[warp][4][lane] = e_el;
  red[warp][5][lane] = e_pol;
  red[warp][6][lane] = deda;
  __syncthreads();
  if (warp == 0 && lane < na) {
    double t[7];
    for (int q = 0; q < 7; q++) {
      t[q] = 0.0;
      for (int w = 0; w < kTileWarps; w++) t[q] += (double)red[w][q][lane];
    }
    v.gx[i] += t[0];
    v.gy[i] += t[1];
    v.gz[i] += t[2];
    v.e_atom[(size_t)AE_VDW * N + i] = t[3];
    v.e_atom[(size_t)AE_ELEC * N + i] = t[4];
    v.e_atom[(size_t)AE_POL * N + i] = t[5];
    v.deda[i] = t[6];
  }
}

// Per-atom values of the fused pass from its i and j sides, as the row
// kernel leaves them: LJ and Coulomb halves, the GB pair sum, the self term,
// and the chain-rule weight gpi * dE/da_i (gbff.cpp:1731-1757).
__global__ void k_gb_finish(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  const int N = v.n_atoms;
  const SysParams &P = v.sp[v.sys_of[i]];
  double dv = v.e_atom[(size_t)AE_VDW * N + i] + (double)v.ej[i] * kInvJScale;
  double de = v.e_atom[(size_t)AE_ELEC * N + i] + (double)v.ej[(size_t)N + i] * kInvJScale;
  double dp = v.e_atom[(size_t)AE_POL * N + i] + (double)v.ej[(size_t)2 * N + i] * kInvJScale;
  double dd = v.deda[i] + (double)v.ej[(size_t)3 * N + i] * kInvJScale;
  double ai_d = v.born_d[i];
  double qd = (double)v.pq[2 * (size_t)i].w;
  double eself = P.premul_d * qd * qd / ai_d;
  v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv;
  v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
  v.e_atom[(size_t)AE_POL * N + i] = dp;
  v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
  double deda_i = dd - eself / ai_d;
  double gpi = ai_d * ai_d / 166.0;  // gbff.cpp:1755 uses the literal 166.0
  reinterpret_cast<float *>(&v.chainp[i])[2] = (float)(gpi * deda_i);
}

// --------------------------------------------------------------- K4 tiles
__global__ void __launch_bounds__(32 * kTileWarps) k_chain_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  __shared__ float red[kTileWarps][3][32];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  const int a0 = v.sc_atom0[sc];
  const int na = min(32, v.atom_off[s + 1] - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ic = v.chainp[i];
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  const float invP5 = P.invP5, piP5 = P.piP5, P4 = P.P4;
  const double still2_d = P.still2_d;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  const int e1 = v.tile_e1[sc];
  for (int e = v.tile_e0[sc] + warp; e < e1; e += kTileWarps) {
    const int J = v.tile_jc[e];
    const int b0 = v.jc_atom0[J];
    const int nb = min(8, v.atom_off[s + 1] - b0);
    if (lane < nb) {
      sA[warp][lane] = v.pq[2 * (size_t)(b0 + lane)];
      sB[warp][lane] = v.pq[2 * (size_t)(b0 + lane) + 1];
      sC[warp][lane] = v.chainp[b0 + lane];
    }
    const unsigned mine = v.tile_mask[8 * (size_t)e + (lane & 7)];
    const int spec = v.tile_spec[e];
    const unsigned exl = spec >= 0 ? v.spec_mask[16 * (size_t)spec + (lane & 7)] : 0u;
    __syncwarp();
    float jv[3] = {0.f, 0.f, 0.f};
    for (int t = 0; t < nb; t++) {
      const unsigned mt = __shfl_sync(0xffffffffu, mine, t);
      const unsigned xt = __shfl_sync(0xffffffffu, exl, t);
      const bool in = ((mt & ~xt) >> lane) & 1u;  // in the list, bond order > 2
      const float4 ja = sA[warp][t], jb = sB[warp][t], jc = sC[warp][t];
      float c0 = 0.f, c1 = 0.f, c2 = 0.f;
      if (in) {
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi)
          ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[b0 + t], v.y[b0 + t], v.z[b0 + t]) > still2_d);
        if (ok) {
          const float tt = chain_term(d, ic.x, jc.x, ic.y, jc.y, ic.z, jc.z, invP5, piP5, P4);
          fx += tt * d.x;
          fy += tt * d.y;
          fz += tt * d.z;
          c0 = -tt * d.x;
          c1 = -tt * d.y;
          c2 = -tt * d.z;
        }
      }
      const float t0 = warp_sum_f(c0), t1 = warp_sum_f(c1), t2 = warp_sum_f(c2);
      if (lane == t) {
        jv[0] = t0;
        jv[1] = t1;
        jv[2] = t2;
      }
    }
    if (lane < nb) {
      const int j = b0 + lane;
      atomicAdd((unsigned long long *)&v.hx[j], (unsigned long long)to_fixed_j(jv[0]));
      atomicAdd((unsigned long long *)&v.hy[j], (unsigned long long)to_fixed_j(jv[1]));
      atomicAdd((unsigned long long *)&v.hz[j], (unsigned long long)to_fixed_j(jv[2]));
    }
    __syncwarp();
  }
  red[warp][0][lane] = fx;
  red[warp][1][lane] = fy;
  red[warp][2][lane] = fz;
  __syncthreads();
  if (warp == 0 && lane < na) {
    double t[3];
    for (int q = 0; q < 3; q++) {
      t[q] = 0.0;
      for (int w = 0; w < kTileWarps; w++) t[q] += (double)red[w][q][lane];
    }
    v.gx[i] += t[0];
    v.gy[i] += t[1];
    v.gz[i] += t[2];
  }
}

// instrumentation: out[0] += list pairs held by the tiles, out[1] += tiles
__global__ void k_tile_counts(PackView v, unsigned long long *out) {
  const int n = v.tile_count[0];
  unsigned long long p = 0, t = 0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    for (int w = 0; w < 8; w++) p += __popc(v.tile_mask[8 * (size_t)e + w]);
    t++;
  }
  p = group_sum<32>(p);
  t = group_sum<32>(t);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], p);
    atomicAdd(&out[1], t);
  }
}
void launch_tile_counts(const PackView &v, cudaStream_t st, unsigned long long *out) {
  PDGPU_LAUNCH(k_tile_counts, 296, 256, 0, st, v, out);
}

// --------------------------------------------------------------- launchers
void launch_tiles_build(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_cluster_bbox, (v.n_sc + v.n_jc + 127) / 128, 128, 0, st, v);
  cudaMemsetAsync(v.tile_count, 0, 2 * sizeof(int), st);
  PDGPU_LAUNCH(k_tile_build, (v.n_sc + 3) / 4, 128, 0, st, v);
}
void launch_born_radii_tile(const PackView &v, cudaStream_t st, bool zero_first) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_born_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH(k_born_finish, (v.n_atoms + 255) / 256, 256, 0, st, v, (int)zero_first);
}
void launch_gb_pair_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_gb_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH(k_gb_finish, (v.n_atoms + 255) / 256, 256, 0, st, v);
}
void launch_gb_chain_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_chain_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
}

}  // namespace pdgpu
