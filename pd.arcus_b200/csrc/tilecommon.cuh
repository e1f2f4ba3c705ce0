// Helpers shared by the cluster-pair tile kernels (tiles.cu, evaltiles.cu):
// fixed-point accumulation, tile records and their decoding.
#pragma once
#include "pairmath.cuh"

namespace pdgpu {

__device__ __forceinline__ long long to_fixed_j(float f) {
  // saturate far outside any physical range (clashing trial structures
  // stay well inside: 2^39 kcal/mol/A)
  float s = fminf(fmaxf(f * (float)kJScale, -9.0e18f), 9.0e18f);
  return __float2ll_rn(s);
}
// Add one FP32 partial to a 2^24 fixed-point sum.  A non-finite partial
// (coincident atoms) marks its system, whose potential energy then reads
// NaN as the reference's FP64 sum would.
__device__ __forceinline__ void add_fixed(const PackView &v, long long *p, float x, int s) {
  if (x == 0.f) return;
  if (!(fabsf(x) <= 3.0e38f)) atomicOr(&(v.ebuf ? v.sys_flags_alt : v.sys_flags)[s], SF_NONFINITE);
  atomicAdd((unsigned long long *)p, (unsigned long long)to_fixed_j(x));
}

// A lane's row bits of tile e (bits over the 8 j atoms), and of its
// bond-order rows when the tile has them.
__device__ __forceinline__ unsigned tile_row(const PackView &v, int e, int lane) {
  return reinterpret_cast<const unsigned char *>(v.tile_rows)[32 * (size_t)e + lane];
}
__device__ __forceinline__ unsigned spec_row(const PackView &v, int spec, int which, int lane) {
  return reinterpret_cast<const unsigned char *>(v.spec_rows)[64 * (size_t)spec + 32 * which + lane];
}

// A tile's metadata, decoded.
struct TileInfo {
  int b0, spec, a0, s, na, nb;
};
__device__ __forceinline__ TileInfo tile_info(const int4 m) {
  TileInfo t;
  t.b0 = m.x;
  t.spec = m.y;
  t.a0 = m.z;
  t.s = m.w >> 8;
  t.na = ((m.w >> 3) & 31) + 1;
  t.nb = (m.w & 7) + 1;
  return t;
}

}  // namespace pdgpu
