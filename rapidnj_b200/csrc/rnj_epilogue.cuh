// rnj_epilogue.cuh -- the distance epilogue shared by the counting kernels:
// tile coordinates, the exact per-pair transform, shared-memory staging of a
// 128 x 128 distance tile and its coalesced stores (tile and mirror image).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rnj_device.cuh"
#include "rnj_internal.h"

namespace rnj {

// Dayhoff PAM distances (x100) for p = 0.750 .. 0.930, the table that defines the
// protein Kimura distance above p = 0.75 (rapidNJ KimuraDistance.cpp:30-49).
constexpr int kPamX100[181] = {
    195, 196, 197, 198, 199, 200, 200, 201, 202, 203, 204, 205, 206, 207, 208,
    209, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222,
    223, 224, 226, 227, 228, 229, 230, 231, 232, 233, 234, 236, 237, 238, 239,
    240, 241, 243, 244, 245, 246, 248, 249, 250, 252, 253, 254, 255, 257, 258,
    260, 261, 262, 264, 265, 267, 268, 270, 271, 273, 274, 276, 277, 279, 281,
    282, 284, 285, 287, 289, 291, 292, 294, 296, 298, 299, 301, 303, 305, 307,
    309, 311, 313, 315, 317, 319, 321, 323, 325, 328, 330, 332, 335, 337, 339,
    342, 344, 347, 349, 352, 354, 357, 360, 362, 365, 368, 371, 374, 377, 380,
    383, 386, 389, 393, 396, 399, 403, 407, 410, 414, 418, 422, 426, 430, 434,
    438, 442, 447, 451, 456, 461, 466, 471, 476, 482, 487, 493, 498, 504, 511,
    517, 524, 531, 538, 545, 553, 560, 569, 577, 586, 595, 605, 615, 626, 637,
    649, 661, 675, 688, 703, 719, 736, 754, 775, 796, 819, 845, 874, 907, 945,
    988};

// The table on the device: the integers, and the distances the reference
// returns from them, (float)(PAM / 100.0) (KimuraDistance.cpp:336), rounded at
// compile time (a double division and a float conversion, both correctly
// rounded).  In global memory, read through L1: the lanes of a warp read
// different entries, which the constant cache would serialise.
struct PamTables {
  int x100[181];
  float dist[181];
};
constexpr PamTables pam_tables() {
  PamTables t{};
  for (int k = 0; k < 181; ++k) {
    t.x100[k] = kPamX100[k];
    t.dist[k] = (float)((double)kPamX100[k] / 100.0);
  }
  return t;
}
static __device__ const PamTables c_pam = pam_tables();

// Upper-triangle tile t -> (ti, tj), ti <= tj, row-major over the triangle.
__device__ __forceinline__ void tri_coords(int t, int nt, int &ti, int &tj) {
  const double b = 2.0 * nt + 1.0;
  int r = (int)floor((b - sqrt(b * b - 8.0 * (double)t)) * 0.5);
  auto start = [nt](int x) { return (long long)x * nt - (long long)x * (x - 1) / 2; };
  if (r < 0) r = 0;
  if (r > nt - 1) r = nt - 1;
  while (r > 0 && start(r) > t) --r;
  while (r + 1 < nt && start(r + 1) <= t) ++r;
  ti = r;
  tj = r + (int)(t - start(r));
}

// -1 -> m2 in the rows x 128 block of rows r0 .. and columns c0 .. of the
// matrix (rows and columns below n only; row i is out[(i - row0) * ld]), by
// threads t0, t0 + nthr, ... of a block: consecutive threads take consecutive
// columns, and each thread issues kBatch loads before it tests any (the
// tiles are read at memory latency, not at one load's round trip each).  The
// diagonal holds 0, never -1.  kBatch: loads in flight per thread (fewer where
// registers are short).
template <int kBatch = 16>
__device__ __forceinline__ void fix_block(float *out, size_t ld, int n, int row0, int r0, int c0,
                                          float m2, int t0, int nthr, int rows = kTile) {
  for (int e0 = t0; e0 < rows * kTile; e0 += kBatch * nthr) {
    float v[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const int e = e0 + k * nthr;
      const int i = r0 + (e >> 7), j = c0 + (e & (kTile - 1));
      v[k] = (e < rows * kTile && i < n && j < n) ? out[(size_t)(i - row0) * ld + j] : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      if (v[k] == -1.0f) {
        const int e = e0 + k * nthr;
        out[(size_t)(r0 + (e >> 7) - row0) * ld + c0 + (e & (kTile - 1))] = m2;
      }
    }
  }
}

// The saturation fix-up of one tile (-1 -> m2 = 2 x the alignment's maximum;
// KimuraDistance.cpp:366-395, JCdistance.cpp:201-230), threads t0, t0 + nthr,
// ... of a block: a triangle tile and, off the diagonal, its mirror image (the
// same -1 entries, transposed; each read row by row), or a full-square tile.
// slice / slices: this block's share of the tile's rows (and of its mirror's).
template <int kBatch = 16>
__device__ __forceinline__ void fixup_tile_at(float *out, size_t ld, int n, int row0, bool full,
                                              int ti, int tj, float m2, int t0, int nthr,
                                              int slice = 0, int slices = 1) {
  const int rows = kTile / slices, r = slice * rows;
  fix_block<kBatch>(out, ld, n, row0, ti * kTile + r, tj * kTile, m2, t0, nthr, rows);
  if (!full && ti != tj)
    fix_block<kBatch>(out, ld, n, row0, tj * kTile + r, ti * kTile, m2, t0, nthr, rows);
}

template <int kBatch = 16>
__device__ __forceinline__ void fixup_tile(const AlnDesc &d, int tile, float m2, int t0, int nthr) {
  int ti, tj;
  if (d.full) {
    ti = tile / d.nt;
    tj = tile % d.nt;
  } else {
    tri_coords(tile, d.nt, ti, tj);
  }
  fixup_tile_at<kBatch>(d.out, d.ld, d.n, d.full ? d.row0 : 0, d.full != 0, ti, tj, m2, t0, nthr);
}

// Per-thread pair layout inside a 128 x 128 tile (256 threads = 4 x 2 warps, each
// warp 32 rows x 64 columns, each lane 8 x 8 pairs): rows rbase + {0..3, 16..19},
// columns cbase + {0..3, 32..35}.  The two 4-wide groups keep every 128-bit
// shared load of a quarter warp on distinct banks.
__device__ __forceinline__ int row_of(int rbase, int r) { return rbase + (r < 4 ? r : 12 + r); }
__device__ __forceinline__ int col_of(int cbase, int c) { return cbase + (c < 4 ? c : 28 + c); }

// The exact distance of one pair from its counts.  nr_quotients: the float
// quotients by the valid count come from its Newton-Raphson reciprocal
// (recip_nr, ratio_f32; the same floats) instead of divisions; the wrapping
// valid count of RNJ_COMPAT_PROTEIN_WRAP always divides.
__device__ __forceinline__ float pair_distance(const EpiParams &ep, uint32_t c0, uint32_t c1,
                                               uint32_t valid, bool nr_quotients = false) {
  unsigned long long v = valid;
  double rn = 0.0;
  if (ep.compat_wrap) v = protein_fast_valid(v, ep.L);
  else if (nr_quotients && valid != 0 && valid < (1u << 24)) rn = recip_nr(valid);
  if (ep.model == RNJ_JC) return jc_distance((unsigned long long)c0 + c1, v, ep.jc_b, rn);
  if (ep.type == RNJ_PROTEIN) return kimura_protein_distance(c0, v, c_pam.dist, rn);
  return k2p_distance(c0, c1, v, rn);
}

// Row stride (floats) of the distance tile staged in shared memory: 129 keeps
// both row-wise and column-wise reads on distinct banks.
constexpr int kStageLd = kTile + 1;
constexpr size_t kStageBytes = (size_t)kTile * kStageLd * 4;

// Epilogue, part 1: this thread's distances into the shared tile S (row =
// local i, column = local j), with the running max and saturation flag.  Counts
// come from get(r, c, c0, c1, valid).
template <class Get>
__device__ __forceinline__ void stage_distances(const EpiParams &ep, int ti, int tj, int rbase,
                                                int cbase, float *S, Get get, float &tmax,
                                                bool &sat) {
  const int i0 = ti * kTile, j0 = tj * kTile;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int rl = row_of(rbase, r);
    const int i = i0 + rl;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cl = col_of(cbase, c);
      const int j = j0 + cl;
      const bool ok = ep.full ? (i < ep.n && j < ep.n && i != j) : (i < j && j < ep.n);
      float x = 0.0f;
      if (ok) {
        uint32_t c0, c1, cv;
        get(r, c, c0, c1, cv);
        x = pair_distance(ep, c0, c1, cv);
        if (x > tmax) tmax = x;
        if (x == -1.0f) sat = true;
      }
      S[rl * kStageLd + cl] = x;
    }
  }
}

// Epilogue, part 2 (after a block barrier): coalesced stores of the tile and of
// its mirror image, zero diagonal, block max and saturation flag.
__device__ __forceinline__ void store_distances(const EpiParams &ep, int ti, int tj, int tile_id,
                                                const float *S, float tmax, bool sat, int warp,
                                                int nwarps) {
  const int i0 = ti * kTile, j0 = tj * kTile, n = ep.n;
  const int lane = threadIdx.x & 31;
  // Tile region: row i0 + r, columns j0 + lane + 32 q.
  for (int r = warp; r < kTile; r += nwarps) {
    const int i = i0 + r;
    if (i >= n) break;
    float *row = ep.out + (size_t)(i - ep.row0) * ep.ld + j0;
#pragma unroll
    for (int q = 0; q < kTile / 32; ++q) {
      const int cl = lane + 32 * q;
      const int j = j0 + cl;
      if (j >= n) continue;
      if (ep.full) row[cl] = (i == j) ? 0.0f : S[r * kStageLd + cl];
      else if (i < j) row[cl] = S[r * kStageLd + cl];
      else if (i == j) row[cl] = 0.0f;
    }
  }
  if (!ep.full) {
    // Mirror region: row j0 + c holds column c of S.
    for (int c = warp; c < kTile; c += nwarps) {
      const int j = j0 + c;
      if (j >= n) break;
      float *row = ep.out + (size_t)(j - ep.row0) * ep.ld + i0;
#pragma unroll
      for (int q = 0; q < kTile / 32; ++q) {
        const int rl = lane + 32 * q;
        const int i = i0 + rl;
        if (i < j) row[rl] = S[rl * kStageLd + c];
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, off));
  const bool any_sat = __any_sync(0xffffffffu, sat);
  if (lane == 0) {
    if (tmax > 0.0f) atomicMax(ep.max_bits, __float_as_int(tmax));
    if (any_sat) ep.tile_flags[tile_id] = 1;
  }
}

}  // namespace rnj
