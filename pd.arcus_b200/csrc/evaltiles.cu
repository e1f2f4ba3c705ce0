// One GB evaluation on the cluster-pair tiles in one persistent launch.
//
// FF_GeneralizedBorn_Still::calcForces in FastMode (gbff.cpp:168-180) has
// three passes over the pairs with a global dependency between each:
//   A  Born-radius sums (calcBornRadii_PairwiseApprox, gbff.cpp:415-466);
//      every pair term must be in before a radius can be formed
//   B  GB + LJ + Coulomb (calcForcesIncludingVacuo loop 1, :1529-1736);
//      needs every radius, and leaves each atom's dE/da complete only when
//      every pair is in
//   C  Born-radius chain rule (loop 2, :1751-1818); needs every dE/da.
// Here the three are phases of one cooperative launch (every block
// resident), separated by two grid barriers.  The per-atom steps between
// them are folded into the phases: phase B forms each atom's Born radius
// from its fixed-point sum when it stages the atom (the FP64 expression of
// k_born_finish, so the same bits), and phase C forms each atom's chain
// weight gpi * dE/da the same way.  The per-atom outputs (Born radii, the
// per-atom energies) are written by grid-stride epilogues that nothing in
// the same phase reads.
//
// Every warp keeps one contiguous tile range for phases A and B (an equal
// share of the pack's tiles).  Phase A also notes the tiles that hold a
// pair inside the Still cutoff (within the guard band); phase C runs over
// that compacted list only, in equal shares.  As in the separate passes
// (tiles.cu), a tile's sums depend on the tile alone and are added in
// 64-bit fixed point, so results do not depend on how the tiles are spread
// over warps, on the grid, or on the batch a system sits in.
//
// The barriers spin with a bounded number of naps; a barrier that runs out
// sets F_BARRIER, and every block then returns (the host reports it and
// clears the counter).  The same kernel runs one phase per launch where a
// cooperative launch is not available (PDGPU_FUSED=0, or a grid that cannot
// be resident): three launches, the same arithmetic, the same results.
//
// Pair arithmetic: the phase-A Born terms are those of the row and tile
// passes (born_term_noV, explicit roundings: the same Born radii bit for
// bit); phases B and C follow gb_pair_term and chain_term with every
// selection branch-free except the GB cross term and the rare FP64
// re-decisions.  The j records of a tile are stored twice in shared memory
// (slots 0-7 and 8-15) so lane a reads j atom (a + t) mod 8 at slot a + t
// with a fixed offset per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "tilecommon.cuh"

namespace pdgpu {

constexpr int kEvWarps = 4;  // warps per block
// resident blocks per SM the register allocation must allow: 4 (up to 128
// registers a thread; the default), or 5 (PDGPU_EV_BLOCKS=5; 102 registers)
constexpr unsigned kBarrierNaps = 1u << 22;  // about half a second of 100 ns naps

// ------------------------------------------------------------- barrier
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned x;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
  return x;
}
// The wait of a programmatic dependent launch: every earlier kernel of the
// stream has completed and its memory is visible; then the next kernel may
// be scheduled (PDGPU_DEP_ENTRY's two steps, after a launch's static loads).
__device__ __forceinline__ void griddep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Grid barrier over a counter that counts arrivals; every block waits for
// `target` arrivals.  False when the wait ran out (the flag is set).
__device__ __forceinline__ bool grid_barrier(unsigned *ctr, unsigned target, int *flags) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    int ok = 1;
    unsigned naps = 0;
    while (ld_acquire_u32(ctr) < target) {
      if (++naps > kBarrierNaps) {
        ok = 0;
        atomicExch(&flags[F_BARRIER], 1);
        break;
      }
      __nanosleep(100);
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// This warp's share [e0, e1) of T work items.
__device__ __forceinline__ void ev_range(long long T, int warp, int &e0, int &e1) {
  const long long G = (long long)gridDim.x * kEvWarps;
  const long long g = (long long)blockIdx.x * kEvWarps + warp;
  e0 = (int)(T * g / G);
  e1 = (int)(T * (g + 1) / G);
}

// Born radius of atom i from its fixed-point sum (k_born_finish's FP64
// expression, gbff.cpp:463-465).
__device__ __forceinline__ double born_radius(const PackView &v, const SysParams &P, int i) {
  const double Gpol = v.terms123[i] + (double)v.bsum[i] * kInvBornScale;
  return -P.halfeconv_d / Gpol + P.born_offset_d;
}

// A lane's bond-order rows rotated so bit t is j atom (a + t) mod 8.
__device__ __forceinline__ unsigned rot8(unsigned row, int a) {
  row &= 0xffu;
  return ((row >> a) | (row << (8 - a))) & 0xffu;
}

// Tile staging shared by the phases: the tile's metadata, this lane's row
// bits and bond-order rows and, in lanes 0..7, the j atom's records and the
// per-atom inputs the phase forms from them.  Records are loaded one tile
// ahead of their use and the metadata two tiles ahead (the records' address
// depends on it), so no tile waits for a load chain.
struct EvStage {
  int4 m;
  unsigned row, x0, x1;  // list bits; bond order <= 2 rows; == 3 rows
  float4 a, b, c;
  double u;              // phase B: terms123[j]; phase C: born_d[j]
  long long w;           // phase B: bsum[j]; phase C: the dE/da sum of j
};
// PH: the phase (1 A, 2 B, 4 C) the stage is for.  The static part reads
// only what the list build and the integrator wrote (the tile records,
// coordinates, per-atom parameters); the dynamic part what the evaluation's
// earlier phases wrote (the Born sums; the Born radii and dE/da sums).
template <int PH>
__device__ __forceinline__ void ev_stage_static(const PackView &v, int t, int lane, EvStage &q) {
  q.row = tile_row(v, t, lane);
  q.x0 = q.x1 = 0;
  if (q.m.y >= 0) {
    q.x0 = spec_row(v, q.m.y, 0, lane);
    if (PH == 2) q.x1 = spec_row(v, q.m.y, 1, lane);
  }
  if (lane <= (q.m.w & 7)) {
    const int j = q.m.x + lane;
    q.a = v.pq[2 * (size_t)j];
    q.b = v.pq[2 * (size_t)j + 1];
    q.c = v.prm[j];
    if (PH == 2) q.u = v.terms123[j];
  }
}
template <int PH>
__device__ __forceinline__ void ev_stage_dyn(const PackView &v, int lane, EvStage &q) {
  if (lane <= (q.m.w & 7)) {
    const int j = q.m.x + lane;
    if (PH == 2) q.w = v.bsum[j];
    if (PH == 4) {
      q.u = v.born_d[j];
      q.w = v.ej[(size_t)3 * v.n_atoms + j];
    }
  }
}
template <int PH>
__device__ __forceinline__ void ev_stage(const PackView &v, int t, int lane, EvStage &q) {
  ev_stage_static<PH>(v, t, lane, q);
  ev_stage_dyn<PH>(v, lane, q);
}
// Walks a warp's tiles [e, e1) (PH 1, 2) or still-list entries (PH 4) with
// the two-deep prefetch: next() returns the stage of the current tile and
// its index, and issues the loads for the tiles after it.  start() is in
// two parts: the static loads of the first items (which a launch may issue
// before the earlier phases of its evaluation are done), then the dynamic
// part of the first item's stage.
template <int PH>
struct EvWalk {
  int e, e1;
  int t0, t1, t2;  // tiles of items e, e+1, e+2
  int4 m1;         // metadata of item e+1
  EvStage nx;      // stage of item e
  __device__ __forceinline__ int tile_of(const PackView &v, int k) const {
    return PH == 4 ? v.still_list[k] : k;
  }
  __device__ __forceinline__ void start_static(const PackView &v, int lane, int b, int end) {
    e = b;
    e1 = end;
    t0 = t1 = t2 = 0;
    if (e < e1) {
      t0 = tile_of(v, e);
      nx.m = v.tile_meta[t0];
      ev_stage_static<PH>(v, t0, lane, nx);
    }
    if (e + 1 < e1) {
      t1 = tile_of(v, e + 1);
      m1 = v.tile_meta[t1];
    }
    if (e + 2 < e1) t2 = tile_of(v, e + 2);
  }
  __device__ __forceinline__ void start_dyn(const PackView &v, int lane) {
    if (e < e1) ev_stage_dyn<PH>(v, lane, nx);
  }
  __device__ __forceinline__ void start(const PackView &v, int lane, int b, int end) {
    start_static(v, lane, b, end);
    start_dyn(v, lane);
  }
  // the current item's stage and tile; advances the prefetch by one item
  __device__ __forceinline__ EvStage next(const PackView &v, int lane, int &tile) {
    const EvStage cur = nx;
    tile = t0;
    if (e + 1 < e1) {
      nx.m = m1;
      ev_stage<PH>(v, t1, lane, nx);
    }
    if (e + 2 < e1) m1 = v.tile_meta[t2];
    t0 = t1;
    t1 = t2;
    if (e + 3 < e1) t2 = tile_of(v, e + 3);
    e++;
    return cur;
  }
};
// One tile staged on its own (the deferred tiles' second pass).
template <int PH>
__device__ __forceinline__ EvStage ev_stage_one(const PackView &v, int t, int lane) {
  EvStage q;
  q.m = v.tile_meta[t];
  ev_stage<PH>(v, t, lane, q);
  return q;
}

// A tile with a pair at a decision edge (the Still cutoff's, or the
// exp-approximation range's) is not added in a phase's main loop: its index
// goes to the warp's slots of defer_list ([first, first + n) for a warp
// whose items start at `first`), and the warp redoes those tiles in the
// careful form after its main loop, adding their sums then.  A tile's
// result therefore depends on the tile alone, and the main loop carries
// neither the FP64 decisions nor the registers they need.
__device__ __forceinline__ void defer_tile(const PackView &v, int lane, int first, int &n, int t) {
  if (lane == 0) v.defer_list[first + n] = t;
  n++;
}

// ============================================================= phase A
// Born sums.  Each term is converted to fixed point and added exactly
// (the row and tile passes' arithmetic).  Tiles with a pair inside the
// Still cutoff's guard band are appended to the still list in runs of up
// to 32 (per-warp order inside a run).
//
// One tile's terms: the i side's sum (this lane's i atom) and the j side's
// (lane (g,a): j atom a, this group's i atoms).  A pair in the guard band
// of the Still cutoff is decided by its FP64 distance: the fast form
// (CAREFUL false) leaves such pairs out and reports them in `band`, and the
// caller then redoes the tile in the careful form, which decides them; a
// tile's result therefore depends on the tile alone.
// The FP64 inputs of the guard-band decisions (passed by value to the
// careful forms, which are out of line).
struct ExactIn {
  const double *x, *y, *z;
  const double *terms123;
  const long long *bsum;
};
__device__ __forceinline__ ExactIn exact_in(const PackView &v) {
  ExactIn x;
  x.x = v.x;
  x.y = v.y;
  x.z = v.z;
  x.terms123 = v.terms123;
  x.bsum = v.bsum;
  return x;
}
struct BornTileIn {
  float4 ia, ib;
  float Ri, Vi, s_lo, s_hi, invP5, piP5, P4s;
  double still2_d;
  int i, b0;
};
struct BornTileOut {
  long long tile_i, jacc;
  bool any;
};
// born_term_noV's value with every step taken on every lane and the
// results selected (the same bits; no divergent branches, so the eight
// steps of a tile interleave).
__device__ __forceinline__ float born_term_sel(const Dx &d, float Ri, float Rj, float invP5, float piP5,
                                               float P4scaled) {
  const float Rs = __fadd_rn(Ri, Rj);
  const float ir2 = __fdividef(1.f, d.r2);
  const float term = __fmul_rn(__fmul_rn(P4scaled, ir2), ir2);
  const float rdivR = __fdividef(d.r2, __fmul_rn(Rs, Rs));
  const float sh = __sinf(__fmul_rn(__fmul_rn(0.5f, piP5), rdivR));
  const float c = __fmul_rn(sh, sh);
  const float tc = __fmul_rn(term, __fmul_rn(c, c));
  return rdivR > invP5 ? term : tc;
}
template <bool CAREFUL>
__device__ __forceinline__ BornTileOut born_tile(const ExactIn &v, const BornTileIn &q, const float4 *sA,
                                                 const float4 *sB, const float4 *sC, unsigned rows, int a, int g8,
                                                 bool &band) {
  long long tile_i = 0, jacc = 0;
  bool any = false;
#pragma unroll(CAREFUL ? 1 : 8)
  for (int t = 0; t < 8; t++) {
    const bool row = (rows >> t) & 1u;
    const float4 ja = sA[a + t], jb = sB[a + t], jc = sC[a + t];
    const Dx d = diff(q.ia, q.ib, ja, jb);
    bool ok = row && d.r2 <= q.s_lo;
    const bool edge = row && !(d.r2 <= q.s_lo) && d.r2 <= q.s_hi;
    if (CAREFUL) {
      if (edge) {
        const int j = q.b0 + ((a + t) & 7), i = q.i;
        ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > q.still2_d);
      }
    } else {
      band |= edge;
    }
    any |= row && d.r2 <= q.s_hi;
    const float term = born_term_sel(d, q.Ri, jc.x, q.invP5, q.piP5, q.P4s);
    // the j side's term is made fixed point by the lane that owns j (the same bits)
    const float tJ = ok ? __fmul_rn(term, q.Vi) : 0.f;
    tile_i += __float2ll_rn(ok ? __fmul_rn(term, jc.y) : 0.f);
    jacc += __float2ll_rn(__shfl_sync(0xffffffffu, tJ, g8 | ((a - t) & 7)));
  }
  BornTileOut o;
  o.tile_i = tile_i;
  o.jacc = jacc;
  o.any = any;
  return o;
}
// The i-side inputs of atom i of the tile's i-cluster (this lane's).
__device__ __forceinline__ void born_i_side(const PackView &v, const TileInfo &ti, int lane, BornTileIn &q) {
  q.i = ti.a0 + (lane < ti.na ? lane : 0);
  q.ia = v.pq[2 * (size_t)q.i];
  q.ib = v.pq[2 * (size_t)q.i + 1];
  const float4 pi = v.prm[q.i];
  q.Ri = pi.z;
  q.Vi = pi.w;
  const SysParams &P = v.sp[ti.s];
  q.s_hi = P.still2 * (1.f + 4e-6f);
  q.s_lo = P.still2 * (1.f - 4e-6f);
  q.invP5 = P.invP5;
  q.piP5 = P.piP5;
  q.P4s = P.P4 * (float)kBornScale;
  q.still2_d = P.still2_d;
}
// A tile's j records into this warp's slots.
__device__ __forceinline__ void born_stage_j(const TileInfo &ti, const EvStage &cur, int lane, float4 *sA,
                                             float4 *sB, float4 *sC) {
  if (lane < ti.nb) {
    sA[lane] = sA[lane + 8] = cur.a;
    sB[lane] = sB[lane + 8] = cur.b;
    sC[lane] = sC[lane + 8] = make_float4(cur.c.z, cur.c.w, 0.f, 0.f);
  }
}
// The j side's sums of a tile over the i groups, added to the Born sums.
__device__ __forceinline__ void born_add_j(const PackView &v, const TileInfo &ti, int lane, long long jacc) {
  jacc += __shfl_xor_sync(0xffffffffu, jacc, 8);
  jacc += __shfl_xor_sync(0xffffffffu, jacc, 16);
  if (lane < ti.nb && jacc) atomicAdd((unsigned long long *)&v.bsum[ti.b0 + lane], (unsigned long long)jacc);
}

__device__ __forceinline__ void phase_born(const PackView &v, int warp, int lane, float4 (*sA)[16],
                                           float4 (*sB)[16], float4 (*sC)[16]) {
  int e, e1;
  ev_range(v.tile_count[0], warp, e, e1);
  const int first = e;
  const int g8 = lane & ~7, a = lane & 7;
  int a0 = -1, na = 0, nd = 0;
  BornTileIn q;
  q.ia = q.ib = make_float4(0, 0, 0, 0);
  q.Ri = q.Vi = q.s_lo = q.s_hi = q.invP5 = q.piP5 = q.P4s = 0.f;
  q.still2_d = 0.0;
  q.i = 0;
  long long acc_i = 0;
  unsigned near = 0;
  int run0 = e;
  const ExactIn xin = exact_in(v);
  EvWalk<1> walk;
  walk.start(v, lane, e, e1);
  auto flush_near = [&](int upto) {
    // tiles [run0, upto) with their bits in `near`
    const int cnt = __popc(near);
    if (cnt) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&v.tile_count[2], cnt);
      base = __shfl_sync(0xffffffffu, base, 0);
      if ((near >> lane) & 1u) v.still_list[base + __popc(near & ((1u << lane) - 1u))] = run0 + lane;
    }
    near = 0;
    run0 = upto;
  };
  for (; e < e1; e++) {
    int te;
    const EvStage cur = walk.next(v, lane, te);
    const TileInfo ti = tile_info(cur.m);
    if (ti.a0 != a0) {
      if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
      acc_i = 0;
      a0 = ti.a0;
      na = ti.na;
      born_i_side(v, ti, lane, q);
    }
    q.b0 = ti.b0;
    born_stage_j(ti, cur, lane, sA[warp], sB[warp], sC[warp]);
    const unsigned rows = rot8(cur.row & ~cur.x0, a);  // bond order > 2 only
    __syncwarp();
    bool band = false;  // a pair whose inclusion the FP64 distance decides
    const BornTileOut o = born_tile<false>(xin, q, sA[warp], sB[warp], sC[warp], rows, a, g8, band);
    // a pair inside the Still cutoff's guard band: the tile goes to the chain-rule phase
    const bool any = __any_sync(0xffffffffu, o.any);
    if (any) near |= 1u << (e - run0);
    if (__any_sync(0xffffffffu, band)) {
      defer_tile(v, lane, first, nd, e);
    } else {
      acc_i += o.tile_i;
      if (any) born_add_j(v, ti, lane, o.jacc);  // no pair inside the cutoff: no j terms
    }
    if (e - run0 == 31) flush_near(e + 1);
    __syncwarp();
  }
  if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
  flush_near(e1);
  if (v.defer_stats && lane == 0 && nd) atomicAdd(&v.defer_stats[0], nd);
  // the deferred tiles in the careful form
  __syncwarp();
  for (int k = 0; k < nd; k++) {
    const int t = v.defer_list[first + k];
    const EvStage cur = ev_stage_one<1>(v, t, lane);
    const TileInfo ti = tile_info(cur.m);
    born_i_side(v, ti, lane, q);
    q.b0 = ti.b0;
    born_stage_j(ti, cur, lane, sA[warp], sB[warp], sC[warp]);
    const unsigned rows = rot8(cur.row & ~cur.x0, a);
    __syncwarp();
    bool band = false;
    const BornTileOut o = born_tile<true>(xin, q, sA[warp], sB[warp], sC[warp], rows, a, g8, band);
    if (lane < ti.na && o.tile_i) atomicAdd((unsigned long long *)&v.bsum[q.i], (unsigned long long)o.tile_i);
    born_add_j(v, ti, lane, o.jacc);
    __syncwarp();
  }
}

// ============================================================= phase B
// GB + LJ + Coulomb for one pair (gb_pair_term's expressions), every
// output zero unless `in`.  Selections are branch-free except the GB cross
// term (skipped by a warp with no pair inside the exp-approximation range)
// and the FP64 re-decision of that range's edge.
struct PairOut {
  float fscal, epol, dedal, vdw, elec;
};
// The exp-approximation range's edge is decided by the FP64 predicate: the
// fast form (CAREFUL false) takes the FP32 decision and reports a pair
// inside the edge's guard band in `band` (the caller then redoes the tile
// in the careful form).
// LEAN: every system of the pack runs FastMode and switches LJ with the
// GB/Coulomb switch (the same parameters, so the same values): the slow
// branch and the second switch are left out.  Both builds give the same
// bits for such a system.
template <bool CAREFUL, bool LEAN>
__device__ __forceinline__ PairOut pair_gb(const GbSettings &g, float r2, bool in, bool nb, bool b14, float ai,
                                           float aj, float qiqj, float radsum, float epsij, const ExactIn &v,
                                           int i, int j, double ai_d, const SysParams *P, bool &band) {
  const float invr = rsqrtf(r2);
  const float r = r2 * invr;
  const float aiaj = ai * aj;
  const float u = __fdividef(-0.25f * r2, aiaj);
  bool gb = u > g.thr;
  const bool edge = in && fabsf(u - g.thr) <= g.band;
  if (CAREFUL) {
    if (edge) {
      // the FP64 predicate of gbff.cpp:1553-1575 with both radii formed
      // from their sums (the same values the epilogue stores)
      const double aj_d = -P->halfeconv_d / (v.terms123[j] + (double)v.bsum[j] * kInvBornScale) + P->born_offset_d;
      const double srij = ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]);
      gb = -srij * 0.25 / (ai_d * aj_d) > g.thr_d;
    }
  } else {
    band |= edge;
  }
  gb = gb && in;
  const float dr = r - g.rin;
  const bool on = r >= g.rin;
  const float sw = 1.f - g.inv_sw2 * dr * dr;
  const float S = on ? sw * sw : 1.f;
  const float dSdd = on ? -4.f * g.inv_sw2 * dr * sw : 0.f;
  float dedr = 0.f, epol = 0.f, dedal = 0.f;
  if (gb) {
    const float tg = __expf(u);
    const float fgb = rsqrtf(r2 + tg * aiaj);
    const float l = fgb * fgb;
    const float epol0 = g.premul * qiqj * fgb;
    const float dedr0 = -epol0 * (r - 0.25f * r * tg) * l;
    const float dedal0 = -epol0 * tg * (1.f - u) * l;
    epol = epol0 * S;
    dedr = S * dedr0 + dSdd * epol0;
    dedal = dedal0 * S;
  } else if (!LEAN && g.slow && in) {
    // FastMode off (calcBornForces, gbff.cpp:1292-1324): the GB term's
    // t = 0 limit q_i q_j / r beyond the exp-approximation range
    const float epol0 = g.premul * qiqj * invr;
    epol = epol0 * S;
    dedr = S * (-epol0 * invr) + dSdd * epol0;
  }
  if (!LEAN) nb = nb && !g.slow;  // FastMode off: the vacuum terms come from FF_NonBonded::calcForces
  const float ec = (gb ? g.econv_in : g.econv_out) * (b14 ? g.elec14 : 1.f) * qiqj * invr;
  const float elf = S * (-ec * invr) + ec * dSdd;
  // Lennard-Jones 12-6 with its own switch
  const float rr = radsum * invr;
  const float rr2 = rr * rr;
  const float B = rr2 * rr2 * rr2;
  const float A = B * B;
  const float eps = epsij * (b14 ? g.vdw14 : 1.0f);
  float vdw = (2.f * eps) * (0.5f * A - B);
  float vdwf = -(12.f * eps * invr) * (A - B);
  float vS = S, vdS = dSdd;
  if (!LEAN) {
    const float vd = r - g.vdw_rin;
    const float vs = 1.f - g.vdw_inv_sw2 * vd * vd;
    const bool von = r > g.vdw_rin;
    vS = von ? vs * vs : 1.f;
    vdS = von ? -4.f * g.vdw_inv_sw2 * vd * vs : 0.f;
  }
  vdwf = vS * vdwf + vdw * vdS;
  vdw *= vS;
  const bool lj = in && nb && r < g.vdw_rc;
  const bool el = in && nb;
  vdw = lj ? vdw : 0.f;
  vdwf = lj ? vdwf : 0.f;
  PairOut o;
  o.elec = el ? ec * S : 0.f;
  const float fel = el ? elf : 0.f;
  o.fscal = in ? dedr * 2.f * invr + (vdwf + fel) * invr : 0.f;
  o.epol = epol;
  o.dedal = dedal;
  o.vdw = vdw;
  return o;
}

// The i side of a tile is converted to fixed point per tile (so its sums
// depend on the tile alone) and kept in this lane's shared-memory slots
// while the warp's range stays in one i-cluster; the sums go to memory when
// the range moves to the next cluster.  Exact integer sums: the same bits
// as adding every tile's share to memory at once.
struct ISide {
  long long (*f)[32];  // [7][32]: this warp's slots
  int lane;
  bool bad;
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int q = 0; q < 7; q++) f[q][lane] = 0;
    bad = false;
  }
  __device__ __forceinline__ void add(int q, float x) {
    bad |= !(fabsf(x) <= 3.0e38f);
    f[q][lane] += to_fixed_j(x);
  }
  __device__ __forceinline__ void flush(const PackView &v, int i, int s, int N) {
    long long *dst[7] = {v.hx + i, v.hy + i, v.hz + i, v.ej + i, v.ej + (size_t)N + i, v.ej + (size_t)2 * N + i,
                         v.ej + (size_t)3 * N + i};
#pragma unroll
    for (int q = 0; q < 7; q++) {
      const long long x = f[q][lane];
      if (x) atomicAdd((unsigned long long *)dst[q], (unsigned long long)x);
    }
    if (bad) atomicOr(&(v.ebuf ? v.sys_flags_alt : v.sys_flags)[s], SF_NONFINITE);
  }
};

// One tile's GB + LJ + Coulomb terms: the i side's sums of this lane's i
// atom (io: force x, y, z, vdw, elec, pol, dE/da) and the j side's (jo,
// lane (g,a): j atom a, this group's i atoms, before the sum over groups).
struct PairTileIn {
  float4 ia, ib, ip;
  double ai_d;
  int i, b0;
};
struct PairTileOut {
  float io[7], jo[7];
};
template <bool CAREFUL, bool LEAN>
__device__ __forceinline__ PairTileOut pair_tile(const ExactIn &v, const GbSettings &gs, const SysParams *P,
                                                 const PairTileIn &q, const float4 *sA, const float4 *sB,
                                                 const float4 *sP, unsigned rows, unsigned xrows, unsigned brows,
                                                 int a, int g8, bool &band) {
  float io[7], jo[7];
#pragma unroll
  for (int k = 0; k < 7; k++) io[k] = jo[k] = 0.f;
#pragma unroll(CAREFUL ? 1 : 8)
  for (int t = 0; t < 8; t++) {
    const float4 ja = sA[a + t], jb = sB[a + t], jp = sP[a + t];
    const Dx d = diff(q.ia, q.ib, ja, jb);
    const bool in = ((rows >> t) & 1u) && d.r2 <= gs.rc2;
    const bool nb3 = !((xrows >> t) & 1u);
    const bool b14 = (brows >> t) & 1u;
    const PairOut o = pair_gb<CAREFUL, LEAN>(gs, d.r2, in, nb3, b14, q.ib.w, jb.w, q.ia.w * ja.w, q.ip.x + jp.x,
                                       q.ip.y * jp.y, v, q.i, q.b0 + ((a + t) & 7), q.ai_d, P, band);
    io[5] += o.epol;
    io[6] += o.dedal * jb.w;
    io[3] += o.vdw;
    io[4] += o.elec;
    const float cx = o.fscal * d.x, cy = o.fscal * d.y, cz = o.fscal * d.z;
    io[0] -= cx;
    io[1] -= cy;
    io[2] -= cz;
    const float c[7] = {cx, cy, cz, o.vdw, o.elec, o.epol, o.dedal * q.ib.w};
    const int src = g8 | ((a - t) & 7);
#pragma unroll
    for (int k = 0; k < 7; k++) jo[k] += __shfl_sync(0xffffffffu, c[k], src);
  }
  PairTileOut o;
#pragma unroll
  for (int k = 0; k < 7; k++) {
    o.io[k] = io[k];
    o.jo[k] = jo[k];
  }
  return o;
}
// The i-side inputs of this lane's atom of the tile's i-cluster.
__device__ __forceinline__ void pair_i_side(const PackView &v, const TileInfo &ti, const SysParams *P, int lane,
                                            PairTileIn &q) {
  q.i = ti.a0 + (lane < ti.na ? lane : 0);
  q.ia = v.pq[2 * (size_t)q.i];
  q.ib = v.pq[2 * (size_t)q.i + 1];
  q.ip = v.prm[q.i];
  q.ai_d = born_radius(v, *P, q.i);
  q.ib.w = (float)q.ai_d;
}
// A tile's j records into this warp's slots, with each j atom's Born
// radius formed from its staged sum: -halfeconv / G + offset with 1/G from
// the FP32 reciprocal and one Newton step in FP64 (about 48 bits, so the
// FP32 radius is born_radius's rounded in all but tie cases; decisions at
// the exp-approximation edge use the FP64 radii themselves).
__device__ __forceinline__ void pair_stage_j(const TileInfo &ti, const EvStage &cur, int lane, double hec,
                                             double boff, float4 *sA, float4 *sB, float4 *sP) {
  if (lane < ti.nb) {
    float4 b = cur.b;
    const double G = cur.u + (double)cur.w * kInvBornScale;
    const double r0 = (double)__frcp_rn((float)G);
    const double r1 = fma(r0, fma(-G, r0, 1.0), r0);
    b.w = (float)fma(hec, r1, boff);
    sA[lane] = sA[lane + 8] = cur.a;
    sB[lane] = sB[lane + 8] = b;
    sP[lane] = sP[lane + 8] = cur.c;
  } else if (lane < 8) {
    // a j-cluster shorter than 8 atoms: its empty slots hold zero records,
    // so the masked-out terms of those slots multiply finite numbers
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    sA[lane] = sA[lane + 8] = z;
    sB[lane] = sB[lane + 8] = z;
    sP[lane] = sP[lane + 8] = z;
  }
}
// The j side's sums of a tile over the i groups, added to the j atoms.
__device__ __forceinline__ void pair_add_j(const PackView &v, const TileInfo &ti, int lane, float (&jacc)[7]) {
  const int N = v.n_atoms;
#pragma unroll
  for (int k = 0; k < 7; k++) {
    jacc[k] += __shfl_xor_sync(0xffffffffu, jacc[k], 8);
    jacc[k] += __shfl_xor_sync(0xffffffffu, jacc[k], 16);
  }
  if (lane < ti.nb) {
    const int j = ti.b0 + lane;
    add_fixed(v, &v.hx[j], jacc[0], ti.s);
    add_fixed(v, &v.hy[j], jacc[1], ti.s);
    add_fixed(v, &v.hz[j], jacc[2], ti.s);
#pragma unroll
    for (int k = 0; k < 4; k++) add_fixed(v, &v.ej[(size_t)k * N + j], jacc[3 + k], ti.s);
  }
}

template <bool LEAN>
__device__ __forceinline__ void phase_pair(const PackView &v, int warp, int lane, float4 (*sA)[16],
                                           float4 (*sB)[16], float4 (*sP)[16], long long (*sI)[7][32],
                                           bool early) {
  int e, e1;
  ev_range(v.tile_count[0], warp, e, e1);
  const int first = e;
  const int N = v.n_atoms;
  const int g8 = lane & ~7, a = lane & 7;
  int a0 = -1, s_cur = -1, na = 0, s_i = 0, nd = 0;
  ISide acc;
  acc.f = sI[warp];
  acc.lane = lane;
  acc.clear();
  PairTileIn q;
  q.ia = q.ib = q.ip = make_float4(0, 0, 0, 0);
  q.ai_d = 0.0;
  q.i = 0;
  const SysParams *P = nullptr;
  double hec = 0.0, boff = 0.0;  // -halfeconv and the Born radius offset
  GbSettings gs;
  const ExactIn xin = exact_in(v);
  EvWalk<2> walk;
  walk.start_static(v, lane, e, e1);
  if (early) griddep_wait();
  walk.start_dyn(v, lane);
  for (; e < e1; e++) {
    int te;
    const EvStage cur = walk.next(v, lane, te);
    const TileInfo ti = tile_info(cur.m);
    if (ti.s != s_cur) {
      s_cur = ti.s;
      P = &v.sp[ti.s];
      gs.load(*P);
      hec = -P->halfeconv_d;
      boff = P->born_offset_d;
    }
    if (ti.a0 != a0) {
      if (lane < na) acc.flush(v, q.i, s_i, N);
      acc.clear();
      a0 = ti.a0;
      na = ti.na;
      s_i = ti.s;
      pair_i_side(v, ti, P, lane, q);
    }
    q.b0 = ti.b0;
    pair_stage_j(ti, cur, lane, hec, boff, sA[warp], sB[warp], sP[warp]);
    const unsigned rows = rot8(cur.row, a);
    const unsigned xrows = rot8(cur.x0, a), brows = rot8(cur.x1, a);  // bond order <= 2, == 3
    __syncwarp();
    bool band = false;
    PairTileOut o = pair_tile<false, LEAN>(xin, gs, P, q, sA[warp], sB[warp], sP[warp], rows, xrows, brows, a, g8, band);
    if (__any_sync(0xffffffffu, band)) {
      defer_tile(v, lane, first, nd, e);
    } else {
      pair_add_j(v, ti, lane, o.jo);
#pragma unroll
      for (int k = 0; k < 7; k++) acc.add(k, o.io[k]);
    }
    __syncwarp();
  }
  if (lane < na) acc.flush(v, q.i, s_i, N);
  if (v.defer_stats && lane == 0 && nd) atomicAdd(&v.defer_stats[1], nd);
  // the deferred tiles in the careful form; their i sums go to memory at once
  __syncwarp();
  for (int k = 0; k < nd; k++) {
    const int t = v.defer_list[first + k];
    const EvStage cur = ev_stage_one<2>(v, t, lane);
    const TileInfo ti = tile_info(cur.m);
    P = &v.sp[ti.s];
    gs.load(*P);
    hec = -P->halfeconv_d;
    boff = P->born_offset_d;
    pair_i_side(v, ti, P, lane, q);
    q.b0 = ti.b0;
    pair_stage_j(ti, cur, lane, hec, boff, sA[warp], sB[warp], sP[warp]);
    const unsigned rows = rot8(cur.row, a);
    const unsigned xrows = rot8(cur.x0, a), brows = rot8(cur.x1, a);
    __syncwarp();
    bool band = false;
    PairTileOut o = pair_tile<true, LEAN>(xin, gs, P, q, sA[warp], sB[warp], sP[warp], rows, xrows, brows, a, g8, band);
    pair_add_j(v, ti, lane, o.jo);
    acc.clear();
#pragma unroll
    for (int c = 0; c < 7; c++) acc.add(c, o.io[c]);
    if (lane < ti.na) acc.flush(v, q.i, ti.s, N);
    __syncwarp();
  }
}

// ============================================================= phase C
// Chain-rule weight of an atom: gpi * dE/da with gpi = a^2 / 166.0 (the
// literal of gbff.cpp:1755) and dE/da = the pair sum - Eself / a, Eself =
// premul q^2 / a (gbff.cpp:1731-1757; k_gb_finish's expression), here as
// (a^2 * sum - premul q^2) / 166 in FP64: one rounding apart, and the
// weight is used in FP32.
__device__ __forceinline__ float chain_weight(const SysParams &P, double ai_d, long long dsum, float q) {
  const double dd = (double)dsum * kInvJScale;
  const double qd = (double)q;
  return (float)((ai_d * ai_d * dd - P.premul_d * qd * qd) * (1.0 / 166.0));
}

// One tile's chain-rule terms: the i side's force on this lane's i atom
// (io) and the j side's (jo, lane (g,a): j atom a, this group's i atoms,
// before the sum over groups); the Still cutoff's guard band as in phase A.
struct ChainTileIn {
  float4 ia, ib, ic;  // ic: R, V, the chain weight
  float s_lo, s_hi, invP5, piP5, P4;
  double still2_d;
  int i, b0;
};
struct ChainTileOut {
  float io[3], jo[3];
};
// chain_term's value with every step taken on every lane and the results
// selected (no divergent branches, so the eight steps of a tile interleave).
__device__ __forceinline__ float chain_term_sel(const Dx &d, float Ri, float Rj, float Vi, float Vj, float wi,
                                                float wj, float invP5, float piP5, float P4) {
  const float Rs = Ri + Rj;
  const float rdivR = __fdividef(d.r2, Rs * Rs);
  const float th = rdivR * piP5;
  float sn, cs;
  __sincosf(th, &sn, &cs);
  const float sq = 0.5f - 0.5f * cs;
  const float Xc = 4.f * sq * sq - 2.f * sq * sn * th;
  const float X = rdivR > invP5 ? 4.f : Xc;
  const float ir2 = __fdividef(1.f, d.r2);  // the fast reciprocal: deterministic, ~1 ulp
  const float ir6 = ir2 * ir2 * ir2;
  return P4 * X * ir6 * (wi * Vj + wj * Vi);
}
template <bool CAREFUL>
__device__ __forceinline__ ChainTileOut chain_tile(const ExactIn &v, const ChainTileIn &q, const float4 *sA,
                                                   const float4 *sB, const float4 *sC, unsigned rows, int a, int g8,
                                                   bool &band) {
  float io[3], jo[3];
#pragma unroll
  for (int k = 0; k < 3; k++) io[k] = jo[k] = 0.f;
#pragma unroll(CAREFUL ? 1 : 8)
  for (int t = 0; t < 8; t++) {
    const float4 ja = sA[a + t], jb = sB[a + t], jc = sC[a + t];
    const Dx d = diff(q.ia, q.ib, ja, jb);
    const bool row = (rows >> t) & 1u;
    bool ok = row && d.r2 <= q.s_lo;
    const bool edge = row && !ok && d.r2 <= q.s_hi;
    if (CAREFUL) {
      if (edge) {
        const int j = q.b0 + ((a + t) & 7), i = q.i;
        ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > q.still2_d);
      }
    } else {
      band |= edge;
    }
    // selected, not multiplied by zero: a lane without a pair may hold a
    // stale j slot of any value
    const float tt = chain_term_sel(d, q.ic.x, jc.x, q.ic.y, jc.y, q.ic.z, jc.z, q.invP5, q.piP5, q.P4);
    const float cx = ok ? tt * d.x : 0.f, cy = ok ? tt * d.y : 0.f, cz = ok ? tt * d.z : 0.f;
    io[0] += cx;
    io[1] += cy;
    io[2] += cz;
    const int src = g8 | ((a - t) & 7);
    jo[0] += __shfl_sync(0xffffffffu, -cx, src);
    jo[1] += __shfl_sync(0xffffffffu, -cy, src);
    jo[2] += __shfl_sync(0xffffffffu, -cz, src);
  }
  ChainTileOut o;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    o.io[k] = io[k];
    o.jo[k] = jo[k];
  }
  return o;
}
// The i-side inputs of this lane's atom of the tile's i-cluster.
__device__ __forceinline__ const SysParams *chain_i_side(const PackView &v, const TileInfo &ti, int lane,
                                                         ChainTileIn &q) {
  const int N = v.n_atoms;
  q.i = ti.a0 + (lane < ti.na ? lane : 0);
  q.ia = v.pq[2 * (size_t)q.i];
  q.ib = v.pq[2 * (size_t)q.i + 1];
  const float4 pi = v.prm[q.i];
  const SysParams *P = &v.sp[ti.s];
  q.ic = make_float4(pi.z, pi.w, chain_weight(*P, v.born_d[q.i], v.ej[(size_t)3 * N + q.i], q.ia.w), 0.f);
  q.s_hi = P->still2 * (1.f + 4e-6f);
  q.s_lo = P->still2 * (1.f - 4e-6f);
  q.invP5 = P->invP5;
  q.piP5 = P->piP5;
  q.P4 = P->P4;
  q.still2_d = P->still2_d;
  return P;
}
// A tile's j records (with each j atom's chain weight) into this warp's slots.
__device__ __forceinline__ void chain_stage_j(const TileInfo &ti, const EvStage &cur, const SysParams *P, int lane,
                                              float4 *sA, float4 *sB, float4 *sC) {
  if (lane < ti.nb) {
    const float4 c = make_float4(cur.c.z, cur.c.w, chain_weight(*P, cur.u, cur.w, cur.a.w), 0.f);
    sA[lane] = sA[lane + 8] = cur.a;
    sB[lane] = sB[lane + 8] = cur.b;
    sC[lane] = sC[lane + 8] = c;
  }
}
// A tile's forces: the j side summed over the i groups, and the i side.
__device__ __forceinline__ void chain_add(const PackView &v, const TileInfo &ti, int lane, int i,
                                          const ChainTileOut &o) {
  float jo[3] = {o.jo[0], o.jo[1], o.jo[2]};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    jo[c] += __shfl_xor_sync(0xffffffffu, jo[c], 8);
    jo[c] += __shfl_xor_sync(0xffffffffu, jo[c], 16);
  }
  if (lane < ti.nb) {
    const int j = ti.b0 + lane;
    add_fixed(v, &v.hx[j], jo[0], ti.s);
    add_fixed(v, &v.hy[j], jo[1], ti.s);
    add_fixed(v, &v.hz[j], jo[2], ti.s);
  }
  if (lane < ti.na) {
    add_fixed(v, &v.hx[i], o.io[0], ti.s);
    add_fixed(v, &v.hy[i], o.io[1], ti.s);
    add_fixed(v, &v.hz[i], o.io[2], ti.s);
  }
}

__device__ __forceinline__ void phase_chain(const PackView &v, int warp, int lane, float4 (*sA)[16],
                                            float4 (*sB)[16], float4 (*sC)[16], bool early) {
  int q0, q1;
  ev_range(v.tile_count[2], warp, q0, q1);
  const int g8 = lane & ~7, a = lane & 7;
  int a0 = -1, nd = 0;
  ChainTileIn q;
  q.ia = q.ib = q.ic = make_float4(0, 0, 0, 0);
  q.s_hi = q.s_lo = q.invP5 = q.piP5 = q.P4 = 0.f;
  q.still2_d = 0.0;
  q.i = 0;
  const SysParams *P = nullptr;
  const ExactIn xin = exact_in(v);
  EvWalk<4> walk;
  walk.start_static(v, lane, q0, q1);
  if (early) griddep_wait();
  walk.start_dyn(v, lane);
  for (int k = q0; k < q1; k++) {
    int t;
    const EvStage cur = walk.next(v, lane, t);
    const TileInfo ti = tile_info(cur.m);
    if (ti.a0 != a0) {
      a0 = ti.a0;
      P = chain_i_side(v, ti, lane, q);
    }
    q.b0 = ti.b0;
    chain_stage_j(ti, cur, P, lane, sA[warp], sB[warp], sC[warp]);
    const unsigned rows = rot8(cur.row & ~cur.x0, a);  // bond order > 2 only
    __syncwarp();
    bool band = false;
    const ChainTileOut o = chain_tile<false>(xin, q, sA[warp], sB[warp], sC[warp], rows, a, g8, band);
    if (__any_sync(0xffffffffu, band))
      defer_tile(v, lane, q0, nd, t);
    else
      chain_add(v, ti, lane, q.i, o);
    __syncwarp();
  }
  if (v.defer_stats && lane == 0 && nd) atomicAdd(&v.defer_stats[2], nd);
  // the deferred tiles in the careful form
  __syncwarp();
  for (int k = 0; k < nd; k++) {
    const int t = v.defer_list[q0 + k];
    const EvStage cur = ev_stage_one<4>(v, t, lane);
    const TileInfo ti = tile_info(cur.m);
    P = chain_i_side(v, ti, lane, q);
    q.b0 = ti.b0;
    chain_stage_j(ti, cur, P, lane, sA[warp], sB[warp], sC[warp]);
    const unsigned rows = rot8(cur.row & ~cur.x0, a);
    __syncwarp();
    bool band = false;
    const ChainTileOut o = chain_tile<true>(xin, q, sA[warp], sB[warp], sC[warp], rows, a, g8, band);
    chain_add(v, ti, lane, q.i, o);
    __syncwarp();
  }
}

// ============================================================= per-atom steps
// Before phase A: zero what phase B adds into (and, first in an
// evaluation, the forces and the record; ZeroFlags), as k_born_finish did.
__device__ __forceinline__ void prologue_zero(const PackView &v, int zero) {
  const int N = v.n_atoms;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    for (int q = 0; q < 4; q++) v.ej[(size_t)q * N + i] = 0;
    if (zero) {
      if (zero & ZF_BONDED) {
        v.fx[i] = 0;
        v.fy[i] = 0;
        v.fz[i] = 0;
      }
      v.gx[i] = 0.0;
      v.gy[i] = 0.0;
      v.gz[i] = 0.0;
      v.hx[i] = 0;
      v.hy[i] = 0;
      v.hz[i] = 0;
      const int s = v.sys_of[i];
      if ((zero & ZF_RECORD) && i == v.atom_off[s]) {
        for (int k = 0; k < E_COUNT; k++)
          if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
        v.sys_flags[s] = 0;
        v.sys_flags_alt[s] = 0;
      }
    }
  }
}
// After phase B (no phase-B reader of these): the Born radii.
__device__ __forceinline__ void epilogue_radii(const PackView &v) {
  const int N = v.n_atoms;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const double a = born_radius(v, v.sp[v.sys_of[i]], i);
    v.born_d[i] = a;
    reinterpret_cast<float *>(&v.pq[2 * (size_t)i + 1])[3] = (float)a;
  }
}
// After phase C: the per-atom energies (k_gb_finish's values) and the
// Born sums cleared for the next evaluation.
__device__ __forceinline__ void epilogue_energies(const PackView &v) {
  const int N = v.n_atoms;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const SysParams &P = v.sp[v.sys_of[i]];
    const double dv = (double)v.ej[i] * kInvJScale;
    const double de = (double)v.ej[(size_t)N + i] * kInvJScale;
    const double dp = (double)v.ej[(size_t)2 * N + i] * kInvJScale;
    const double ai_d = v.born_d[i];
    const double qd = (double)v.pq[2 * (size_t)i].w;
    double *ep = v.ebuf ? v.e_pair_alt : v.e_atom;  // the pair slots of this energy buffer
    ep[(size_t)AE_VDW * N + i] = 0.5 * dv;
    ep[(size_t)AE_ELEC * N + i] = 0.5 * de;
    ep[(size_t)AE_POL * N + i] = dp;
    ep[(size_t)AE_POL_SELF * N + i] = P.premul_d * qd * qd / ai_d;
    v.bsum[i] = 0;
  }
}

// ============================================================= the kernel
// ph: which phases (1 A, 2 B, 4 C); more than one needs a cooperative
// launch.  One compiled kernel serves the single launch and the three
// one-phase launches, so both forms run the same instructions and give the
// same bits whatever the compiler's contraction and scheduling choices.
// MINB: resident blocks per SM the register allocation must allow
// (PDGPU_EV_BLOCKS, 4 or 5, picks the build at run time; 4 by default).
// tile_count[2] is the still-list length, tile_count[3] the barrier / exit
// counter; the last block out clears both.
template <int MINB, bool LEAN>
__global__ void __launch_bounds__(32 * kEvWarps, MINB) k_eval_tiles(PackView v, int zero, int ph) {
  // a launch of phase B or C alone follows the launch of the phase before
  // it: it stages its first tiles while that one still runs, and waits for
  // it (griddep_wait) before it reads anything the evaluation writes
  const bool early = ph == 2 || ph == 4;
  if (!early) PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ float4 s0[kEvWarps][16], s1[kEvWarps][16], s2[kEvWarps][16];
  __shared__ long long si[kEvWarps][7][32];  // phase B's i-side sums
  unsigned *ctr = reinterpret_cast<unsigned *>(&v.tile_count[3]);
  const unsigned G = gridDim.x;
  unsigned passed = 0;  // barriers this launch has crossed
  if (ph & 1) {
    prologue_zero(v, zero);
    phase_born(v, warp, lane, s0, s1, s2);
  }
  if ((ph & 1) && (ph & 6)) {
    if (!grid_barrier(ctr, G * ++passed, v.flags)) return;
  }
  if (ph & 2) {
    phase_pair<LEAN>(v, warp, lane, s0, s1, s2, si, early);
    epilogue_radii(v);
  }
  if ((ph & 2) && (ph & 4)) {
    if (!grid_barrier(ctr, G * ++passed, v.flags)) return;
  }
  if (ph & 4) {
    phase_chain(v, warp, lane, s0, s1, s2, early);
    epilogue_energies(v);
    // the last block out clears the still list and the counter
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(ctr, 1u);
      if (prev == G * (passed + 1) - 1) {
        v.tile_count[2] = 0;
        atomicExch(ctr, 0u);
      }
    }
  }
}

// ============================================================= host side
static int fused_wanted() {
  static int w = -1;
  if (w < 0) {
    const char *s = getenv("PDGPU_FUSED");
    w = (s && s[0] == '0') ? 0 : 1;
  }
  return w;
}

// PDGPU_EV_LEAN=0 runs the general build for every pack (the lean build
// gives the same bits where it applies; tested)
static int lean_allowed() {
  static int w = -1;
  if (w < 0) {
    const char *s = getenv("PDGPU_EV_LEAN");
    w = (s && s[0] == '0') ? 0 : 1;
  }
  return w;
}

static int ev_minb() {
  static int m = 0;
  if (!m) {
    const char *s = getenv("PDGPU_EV_BLOCKS");
    m = (s && s[0] == '5') ? 5 : 4;
  }
  return m;
}

// Resident blocks of the evaluation kernel on this device (the grid of its
// cooperative launch), and no more warps than a pack can have tiles.
int eval_tiles_grid(long long tile_cap) {
  int dev = 0, sms = 148, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ev_minb() == 4)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_eval_tiles<4, false>, 32 * kEvWarps, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_eval_tiles<5, false>, 32 * kEvWarps, 0);
  const long long need = (tile_cap + kEvWarps - 1) / kEvWarps;
  return (int)std::max(1LL, std::min((long long)std::max(occ, 1) * sms, need));
}

static cudaError_t launch_ev(int ph, const PackView &v, cudaStream_t st, int zero, bool coop) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(v.ev_blocks);
  cfg.blockDim = dim3(32 * kEvWarps);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  int na = 0;
  if (coop) {
    attr[na].id = cudaLaunchAttributeCooperative;
    attr[na].val.cooperative = 1;
    na++;
  }
  // programmatic dependent launch for the one-phase launches (a
  // cooperative launch waits for the kernel before it in the stream)
  if (!coop && pdl_enabled()) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    na++;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  cudaError_t e;
  const bool lean = v.ev_lean && lean_allowed();
  if (ev_minb() == 4)
    e = lean ? cudaLaunchKernelEx(&cfg, k_eval_tiles<4, true>, v, zero, ph)
                  : cudaLaunchKernelEx(&cfg, k_eval_tiles<4, false>, v, zero, ph);
  else
    e = lean ? cudaLaunchKernelEx(&cfg, k_eval_tiles<5, true>, v, zero, ph)
                  : cudaLaunchKernelEx(&cfg, k_eval_tiles<5, false>, v, zero, ph);
  count_launch();
  return e;
}

// The three GB passes on the tiles: one cooperative launch when allowed,
// else three launches of the same phases.
cudaError_t launch_eval_tiles(const PackView &v, cudaStream_t st, int zero, bool coop) {
  if (!v.n_sc || v.ev_blocks <= 0) return cudaSuccess;
  if (coop && fused_wanted()) return launch_ev(7, v, st, zero, true);
  cudaError_t e = launch_ev(1, v, st, zero, false);
  if (e == cudaSuccess) e = launch_ev(2, v, st, 0, false);
  if (e == cudaSuccess) e = launch_ev(4, v, st, 0, false);
  return e;
}

cudaError_t launch_born_phase_only(const PackView &v, cudaStream_t st) {
  if (!v.n_sc || v.ev_blocks <= 0) return cudaSuccess;
  return launch_ev(1, v, st, 0, false);
}

// One evaluation (three launches) that counts the tiles each phase
// deferred to its careful form into stats[0..2] (device memory, zeroed by
// the caller).
cudaError_t count_deferred_tiles(const PackView &v, cudaStream_t st, int *stats) {
  if (!v.n_sc || v.ev_blocks <= 0) return cudaSuccess;
  PackView w = v;
  w.defer_stats = stats;
  return launch_eval_tiles(w, st, ZF_PAIRS, false);
}

// Device times of the evaluation: the three phases as three launches
// (ms[0..2]), then the one cooperative launch (ms[3]); averages over reps.
// The forces of the timed evaluations are left in the accumulators.
cudaError_t profile_eval_tiles(const PackView &v, cudaStream_t st, int reps, double *ms) {
  cudaEvent_t ev[5];
  for (int q = 0; q < 5; q++) cudaEventCreate(&ev[q]);
  double acc[4] = {0, 0, 0, 0};
  cudaError_t e = cudaSuccess;
  for (int it = 0; it < reps && e == cudaSuccess; it++) {
    cudaEventRecord(ev[0], st);
    e = launch_ev(1, v, st, ZF_PAIRS, false);
    cudaEventRecord(ev[1], st);
    if (e == cudaSuccess) e = launch_ev(2, v, st, 0, false);
    cudaEventRecord(ev[2], st);
    if (e == cudaSuccess) e = launch_ev(4, v, st, 0, false);
    cudaEventRecord(ev[3], st);
    if (e == cudaSuccess) e = launch_ev(7, v, st, ZF_PAIRS, true);
    cudaEventRecord(ev[4], st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (int q = 0; q < 4 && e == cudaSuccess; q++) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      acc[q] += t;
    }
  }
  for (int q = 0; q < 5; q++) cudaEventDestroy(ev[q]);
  for (int q = 0; q < 4; q++) ms[q] = reps > 0 ? acc[q] / reps : 0.0;
  return e;
}

}  // namespace pdgpu
