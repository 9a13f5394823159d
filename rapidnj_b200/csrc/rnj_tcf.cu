// rnj_tcf.cu -- the fused tensor-core distance kernel: per-pair counts on the
// tensor cores and the exact transform in the same CTA, straight from tensor
// memory to the distance matrix.
//
// The counting pipeline is the one of rnj_tcgen05.cuh (warp 16 TMA producer,
// warp 17 MMA issuer, three f32 accumulators V, R, T of 128 x 128 in tensor
// memory, a six-stage ring).  Sixteen epilogue warps (0 .. 15, with 112
// registers each after a setmaxnreg split) replace the packed-count round trip
// of the two-kernel form (8 bytes per pair written and read again, then a
// separate transform launch):
//   * warp w reads tensor-memory lane quarter w % 4 (32 tile rows, lane = row)
//     and columns 32 (w / 4) .. + 31 of the three accumulators, 16
//     columns at a time, converts them to integer counts (16 bits each: the
//     fused form takes alignments of at most 65535 columns) and hands tensor
//     memory back to the MMA warp at once;
//   * it then computes the 32 distances of each lane from registers, sixteen
//     pairs at a time (K2P: k2p_decide16, with the logarithm table copied to
//     shared memory; the quotients by the valid count from its Newton-Raphson
//     reciprocal, the same floats as the reference's divisions, ratio_f32)
//     while the tensor cores already count the next tile;
//   * stores: the mirror entries out[j][i] as coalesced 128-byte row segments
//     (lanes are consecutive i), the tile entries out[i][j .. j + 3] as 16-byte
//     vectors, the diagonal as 0; the tile's maximum goes to the alignment's
//     max slot (atomicMax on the float bits) and a saturated pair (-1) sets
//     the tile's flag for the fix-up kernel.  With AlnDesc::full the work items
//     are full-square tiles of a band of rows (out-of-core delivery): every
//     ordered pair is stored in its row of the band buffer, no mirror.
// The transform's instructions overlap the MMAs of the next tile instead of
// following them in a second kernel.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"
#include "rnj_tcgen05.cuh"

namespace rnj {

// Warps 0 .. 15: epilogue (warpgroups 0 .. 3); warp 16: TMA producer; warp 17:
// MMA issuer and tensor-memory owner; warps 18, 19 complete warpgroup 4.
constexpr int kTcfEpiWarps = 16;
constexpr int kTcfThreads = 640;
constexpr int kTcfProducerWarp = 16, kTcfMmaWarp = 17;
// Registers: launched with 640 threads x 96; warpgroup 4 (producer, issuer)
// gives back 64 a thread (setmaxnreg.dec to 32), which lets the 512 epilogue
// threads grow by 16 (setmaxnreg.inc to 112): 128 x 32 + 512 x 112 = 640 x 96,
// so the increase never waits for registers that are not there.
constexpr int kTcfRegsLow = 32, kTcfRegsHigh = 112, kTcfRegsLaunch = 96;
static_assert(128 * kTcfRegsLow + 512 * kTcfRegsHigh <= kTcfThreads * kTcfRegsLaunch,
              "the register split fits the launch's registers");
// A ring of up to six stages (a seventh stage's 32 KB would leave no room; six
// is the default, the tuner may choose fewer) and the logarithm table
// (128 x {-ln F / 4, -1 / (4 F)}, the scaled table of neg_quarter_ln_table_k)
// after the barrier block.
constexpr int kTcfStages = 6;
constexpr size_t kTcfTableBytes = 128 * 2 * sizeof(double);
constexpr size_t kTcfSmemBytes = tc_smem_bytes(kTcfStages, kTcfTableBytes);
static_assert(kTcfSmemBytes <= 232448, "fits the shared memory of one CTA");
constexpr int kTcfGroup = 4;                         // pairs per transform group

// Transform variants of the fused epilogue, one loop each so that only the
// model's own parameters stay in registers (kFusedK2p .. kFusedAny are the
// FusedVariant values of rnj_internal.h).
enum {
  kFusedK2p = FUSED_K2P, kFusedJc = FUSED_JC, kFusedProtein = FUSED_PROTEIN,
  kFusedGeneric = FUSED_GENERIC, kFusedFull = FUSED_FULL, kFusedAny = FUSED_ANY
};

template <int M>
__device__ __forceinline__ float fused_pair(const AlnDesc &d, uint32_t ts, uint32_t tv,
                                            uint32_t vv, double jc_inv_b = 0.0,
                                            const double2 *tab = nullptr) {
  if constexpr (M == kFusedJc || M == kFusedProtein) {
    // the float quotient by the valid count in float arithmetic (quotient16:
    // counts below 2^16 here, the count of differences at most the valid count)
    const float fv = __fsub_rn(__uint_as_float(0x4B000000u | (vv ? vv : 1u)), 8388608.0f);
    const float y = recip16(fv);
    if constexpr (M == kFusedJc)  // jc_inv_b: 1 / d.jc_b, correctly rounded
      return jc_of_q(div_by_b(vv ? (double)quotient16(ts + tv, fv, y) : 0.0, d.jc_b, jc_inv_b),
                     d.jc_b, tab);
    else
      return kimura_protein_of_p(vv ? quotient16(ts, fv, y) : -1.0f, c_pam.dist, tab);
  } else {
    EpiParams ep;
    ep.n = d.n;
    ep.L = d.L;
    ep.model = d.model;
    ep.type = d.type;
    ep.compat_wrap = d.compat;
    ep.jc_b = d.jc_b;
    return pair_distance(ep, ts, tv, vv, true);
  }
}

// k2p_distance out of line: the rare pairs whose one-logarithm value the
// rounding check cannot decide.
static __device__ __noinline__ float k2p_undecided(uint32_t P, uint32_t Q, uint32_t n) {
  return k2p_distance(P, Q, n);
}

// The 32 distances of row i, columns jb .. jb + 31 (counts pq / pv, see the
// epilogue): the mirror entries out[j][i], the row entries out[i][j] for j >= i
// (0 on the diagonal), the running maximum and whether a pair saturated.
// tab: the logarithm table in shared memory, scaled by -1/4.
template <int M>
__device__ __forceinline__ void fused_rows(const AlnDesc &d, int i, int jb, uint32_t (&pq)[32],
                                           uint32_t (&pv)[16], float &tmax, bool &sat,
                                           const double2 *tab) {
  const int n = d.n;
  float *const out = d.out;
  const size_t ld = d.ld;
  const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
  float *const orow = out + (size_t)i * ld;  // dereferenced only for i < n
  const double jc_inv_b = M == kFusedJc ? __ddiv_rn(1.0, d.jc_b) : 0.0;  // once per row
#pragma unroll 1
  for (int g = 0; g < 32 / kTcfGroup; ++g) {
    const int j0 = jb + kTcfGroup * g;
    float x[kTcfGroup];
    {
#pragma unroll
      for (int k = 0; k < kTcfGroup; ++k) {
        const int j = j0 + k;
        x[k] = 0.0f;
        if (i < j && j < n) {
          const uint32_t vv = (pv[k >> 1] >> (16 * (k & 1))) & 0xFFFFu;
          x[k] = fused_pair<M>(d, pq[k] & 0xFFFFu, pq[k] >> 16, vv, jc_inv_b, tab);
          tmax = fmaxf(tmax, x[k]);
          sat |= (x[k] == -1.0f);
          __stcs(out + (size_t)j * ld + i, x[k]);  // mirror: consecutive i across lanes
        }
      }
    }
    // Row i, columns j0 .. j0 + 7 (j >= i; the diagonal is 0).
    if (i < n) {
#pragma unroll
      for (int h = 0; h < kTcfGroup / 4; ++h) {
        const int jj = j0 + 4 * h;
        if (vec && i < jj && jj + 3 < n) {
          __stcs(reinterpret_cast<float4 *>(orow + jj),
                 make_float4(x[4 * h], x[4 * h + 1], x[4 * h + 2], x[4 * h + 3]));
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int j = jj + k;
            if (j < n && i <= j) __stcs(orow + j, (i == j) ? 0.0f : x[4 * h + k]);
          }
        }
      }
    }
    // The next group's counts into registers 0 .. 7.
#pragma unroll
    for (int k = 0; k < 32 - kTcfGroup; ++k) pq[k] = pq[k + kTcfGroup];
#pragma unroll
    for (int k = 0; k < (32 - kTcfGroup) / 2; ++k) pv[k] = pv[k + kTcfGroup / 2];
  }
}

// Kimura-2P rows (the variant of the DNA workloads): the 32 distances of row i,
// columns jb .. jb + 31, in groups of four computed without branches
// (k2p_decide16), the rare undecided pairs out of line; stores as streaming
// stores (.cs), so that the output does not push the logarithm table out of
// L1.  interior: the tile lies above the diagonal and inside the matrix (every
// pair valid, no masks).
constexpr int kK2pGroups = 4;  // groups of four pairs computed per loop iteration

__device__ __forceinline__ void fused_rows_k2p(const AlnDesc &d, int i, int jb, bool interior,
                                               uint32_t (&pq)[32], uint32_t (&pv)[16],
                                               float &tmax, bool &sat, const double2 *tab) {
  const int n = d.n;
  float *const out = d.out;
  const size_t ld = d.ld;
  const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
  float *const orow = out + (size_t)i * ld;  // dereferenced only for i < n
  float *mp = out + (size_t)jb * ld + i;     // out[jb + c][i], one row further per column
  constexpr int U = kK2pGroups;
#pragma unroll 1
  for (int it = 0; it < 8 / U; ++it) {
#pragma unroll
  for (int g = 0; g < U; ++g) {
    float x[4];
    uint32_t undecided = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = 4 * g + k;
      bool slow;
      x[k] = k2p_decide16(pq[c] & 0xFFFFu, pq[c] >> 16, (pv[c >> 1] >> (16 * (c & 1))) & 0xFFFFu,
                          slow, tab);
      undecided |= (uint32_t)slow << k;
    }
    if (undecided) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int c = 4 * g + k;
        if ((undecided >> k) & 1u)
          x[k] = k2p_undecided(pq[c] & 0xFFFFu, pq[c] >> 16,
                               (pv[c >> 1] >> (16 * (c & 1))) & 0xFFFFu);
      }
    }
    const int j0 = jb + 4 * (U * it + g);
    if (interior) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        tmax = fmaxf(tmax, x[k]);
        sat |= (x[k] == -1.0f);
        __stcs(mp, x[k]);  // mirror: consecutive i across lanes
        mp += ld;
      }
      if (vec) {
        __stcs(reinterpret_cast<float4 *>(orow + j0), make_float4(x[0], x[1], x[2], x[3]));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) __stcs(orow + j0 + k, x[k]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = j0 + k;
        const bool in = i < j && j < n;
        x[k] = in ? x[k] : 0.0f;
        tmax = fmaxf(tmax, x[k]);
        sat |= (x[k] == -1.0f);
        if (in) __stcs(mp, x[k]);
        mp += ld;
      }
      if (i < n) {
        if (vec && i < j0 && j0 + 3 < n) {
          __stcs(reinterpret_cast<float4 *>(orow + j0), make_float4(x[0], x[1], x[2], x[3]));
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int j = j0 + k;
            if (j < n && i <= j) __stcs(orow + j, (i == j) ? 0.0f : x[k]);
          }
        }
      }
    }
  }
  // The next iteration's counts into registers 0 .. 4U - 1.
  if constexpr (U < 8) {
#pragma unroll
    for (int k = 0; k < 32 - 4 * U; ++k) pq[k] = pq[k + 4 * U];
#pragma unroll
    for (int k = 0; k < 16 - 2 * U; ++k) pv[k] = pv[k + 2 * U];
  }
  }
}

// Full-rows form (a band of full-square tiles, AlnDesc::full): the 32
// distances of row i, columns jb .. jb + 31, every j != i (0 on the diagonal),
// into row i - row0 of the band buffer; no mirror.
template <int M>
__device__ __forceinline__ void fused_rows_full(const AlnDesc &d, int i, int jb, uint32_t (&pq)[32],
                                                uint32_t (&pv)[16], float &tmax, bool &sat) {
  const int n = d.n;
  if (i >= n) return;
  const size_t ld = d.ld;
  float *const orow = d.out + (size_t)(i - d.row0) * ld;
  const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(d.out) & 15) == 0);
#pragma unroll 1
  for (int g = 0; g < 32 / kTcfGroup; ++g) {
    const int j0 = jb + kTcfGroup * g;
    float x[kTcfGroup];
#pragma unroll
    for (int k = 0; k < kTcfGroup; ++k) {
      const int j = j0 + k;
      x[k] = 0.0f;
      if (j != i && j < n) {
        const uint32_t vv = (pv[k >> 1] >> (16 * (k & 1))) & 0xFFFFu;
        x[k] = fused_pair<M>(d, pq[k] & 0xFFFFu, pq[k] >> 16, vv);
        tmax = fmaxf(tmax, x[k]);
        sat |= (x[k] == -1.0f);
      }
    }
#pragma unroll
    for (int h = 0; h < kTcfGroup / 4; ++h) {
      const int jj = j0 + 4 * h;
      if (vec && jj + 3 < n) {
        __stcs(reinterpret_cast<float4 *>(orow + jj),
               make_float4(x[4 * h], x[4 * h + 1], x[4 * h + 2], x[4 * h + 3]));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (jj + k < n) __stcs(orow + jj + k, x[4 * h + k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 32 - kTcfGroup; ++k) pq[k] = pq[k + kTcfGroup];
#pragma unroll
    for (int k = 0; k < (32 - kTcfGroup) / 2; ++k) pv[k] = pv[k + kTcfGroup / 2];
  }
}

// One tile of the epilogue (every epilogue warp; warp w reads tensor-memory
// lane quarter w % 4 and columns 32 (w / 4) .. + 31): waits for the
// accumulators of the CTA's item number titer, reads them, hands tensor memory
// back, then the transform, the stores, the tile's maximum and saturation
// flag.  False when a wait ran out (the caller sets the abort flag).
template <int V>
__device__ __forceinline__ bool fused_tile(const TcShared &sh, uint32_t tmem, const AlnDesc &d,
                                           int tile, uint32_t titer, int stall, uint64_t limit,
                                           const double2 *tab, int *sat_any = nullptr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3;              // tensor-memory lane quarter
  const int cofs = 32 * (warp >> 2);   // first tile column of this warp
  const int row = 32 * q + lane;       // tile row of this lane
  int ti, tj;
  item_tile(d, tile, ti, tj);
  if ((stall && titer == 0 && !tc_wait(sh.never_bar, 0, sh.abort_flag, limit)) ||
      !tc_wait(sh.acc_full, titer & 1, sh.abort_flag, limit))
    return false;
  tc_fence_after();
  // protein counts (V - M) or DNA (ts, tv): known at compile time for the
  // single-model variants (K2P is DNA, protein Kimura is protein)
  const bool prot = V == kFusedK2p ? false
                                   : (V == kFusedProtein ? true : d.kind == KIND_PROT_TC);
  // Accumulators -> integer counts (DNA: transitions, transversions, valid;
  // protein: mismatches = V - M, 0, valid), 16 columns at a time, 16 bits
  // each (the fused form takes L < 65536): pq[k] = ts | tv << 16, and the
  // valid counts two to a register.
  uint32_t pq[32], pv[16];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t av[16], ar[16], at[16];  // accumulators V, R, T
    const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(cofs + 16 * h);
    tmem_ld16(base, av);
    tmem_ld16(base + kTile, ar);
    tmem_ld16(base + 2 * kTile, at);
    tmem_ld_wait();
    // The sums are exact integers in f32 (below 2^24 in magnitude), and so
    // are P = (V + R - T) / 4 and Q = (V - R) / 2 (DNA) or P = V - M
    // (protein); x + 2^23 holds x in its low mantissa bits (0 <= x < 2^23),
    // from which the 16-bit fields are taken without a conversion.
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float fv = __uint_as_float(av[k]), fr = __uint_as_float(ar[k]);
      const float ft = __uint_as_float(at[k]);
      // DNA: 4P = V + R - T and 2Q = V - R are exact integers, so the scale and
      // the bias fuse into one multiply-add with the same (exact) result.
      const uint32_t bp = __float_as_uint(
          prot ? __fadd_rn(__fsub_rn(fv, fr), 8388608.0f)
               : __fmaf_rn(__fsub_rn(__fadd_rn(fv, fr), ft), 0.25f, 8388608.0f));
      const uint32_t bq = __float_as_uint(
          prot ? 8388608.0f : __fmaf_rn(__fsub_rn(fv, fr), 0.5f, 8388608.0f));
      const uint32_t bv = __float_as_uint(__fadd_rn(fv, 8388608.0f));
      pq[16 * h + k] = __byte_perm(bp, bq, 0x5410);  // P | Q << 16
      if (k & 1) pv[8 * h + (k >> 1)] = __byte_perm(pv[8 * h + (k >> 1)], bv, 0x5410);
      else pv[8 * h + (k >> 1)] = bv;  // high half replaced by the odd column
    }
  }
  // Tensor memory back to the MMA warp: the next tile's MMAs start now.
  tc_fence_before();
  __syncwarp();
  if (lane == 0) mbar_arrive(sh.tmem_empty);

  const int i = ti * kTile + row;
  const int jb = tj * kTile + cofs;
  float tmax = 0.0f;
  bool sat = false;
  if constexpr (V == kFusedFull) {
    // a band of full rows (out-of-core delivery), every model
    fused_rows_full<kFusedGeneric>(d, i, jb, pq, pv, tmax, sat);
  } else if constexpr (V == kFusedK2p) {
    fused_rows_k2p(d, i, jb, ti < tj && (tj + 1) * kTile <= d.n, pq, pv, tmax, sat, tab);
  } else if constexpr (V != kFusedAny) {
    fused_rows<V>(d, i, jb, pq, pv, tmax, sat, tab);
  } else if (d.compat) {
    fused_rows<kFusedGeneric>(d, i, jb, pq, pv, tmax, sat, tab);
  } else if (d.model == RNJ_JC) {
    fused_rows<kFusedJc>(d, i, jb, pq, pv, tmax, sat, tab);
  } else if (d.type == RNJ_PROTEIN) {
    fused_rows<kFusedProtein>(d, i, jb, pq, pv, tmax, sat, tab);
  } else {
    fused_rows_k2p(d, i, jb, ti < tj && (tj + 1) * kTile <= d.n, pq, pv, tmax, sat, tab);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, off));
  const bool any_sat = __any_sync(0xffffffffu, sat);
  if (lane == 0) {
    if (tmax > 0.0f) atomicMax(d.max_bits, __float_as_int(tmax));
    if (any_sat) {
      d.tile_flags[tile] = 1;
      if (sat_any) atomicOr(sat_any, 1);
    }
  }
  return true;
}

// V: the transform variant of every item (kFused*), or kFusedAny to choose per
// item (a work list of alignments with different models).
template <int V>
__global__ void __launch_bounds__(kTcfThreads, 1)
    tc_fused_kernel(const AlnDesc *__restrict__ descs, const WorkItem *__restrict__ items,
                    const int *__restrict__ nitems_ptr, int nitems_direct, int item0, int count,
                    int nst) {
  extern __shared__ uint8_t smem_raw[];
  // A batch's first descriptor may ask for a shallower ring than the launch's
  // shared memory holds (its graph is captured once; batches launch kFusedAny).
  if constexpr (V == kFusedAny)
    if (descs[0].stages > 0) nst = max(kTcMinStages, min(nst, descs[0].stages));
  const TcShared sh = tc_shared(smem_raw, nst, kTcfTableBytes);
  double2 *const tab = reinterpret_cast<double2 *>(tc_extra(sh));
  const uint64_t limit = wait_limit_ns((uint32_t)descs[0].wait_us);
  const int stall = descs[0].stall;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // items [item0, min(nitems, item0 + count))
  const int nitems = (int)min((long long)(nitems_ptr ? *nitems_ptr : nitems_direct),
                              (long long)item0 + count);
  const int it0 = item0 + (int)blockIdx.x;
  if (it0 >= nitems) return;  // no item for this CTA (before any setup)

  for (int e = tid; e < 128; e += kTcfThreads)
    tab[e] = make_double2(-0.25 * c_log_tab[e][0], -0.25 * c_log_tab[e][1]);
  // tmem_empty: one arrival per epilogue warp; the scale factors by warps 0 .. 7
  const uint32_t tmem = tc_setup(sh, kTcfEpiWarps, 0, kTcfMmaWarp);
  uint32_t issued = 0;

  if (warp >= kTcfProducerWarp) {
    // The register split is made inside each role's branch, so that the
    // compiler allocates each role's code within its own limit.
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kTcfRegsLow) : "memory");
    if (warp == kTcfProducerWarp) {
      if (lane == 0) issued = tc_produce(sh, descs, items, it0, nitems, gridDim.x, limit);
    } else if (warp == kTcfMmaWarp) {
      tc_issue(sh, tmem, descs, items, it0, nitems, gridDim.x, limit);
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kTcfRegsHigh) : "memory");
    // ----------------------------------------------------------- epilogue
    uint32_t titer = 0;
    for (int it = it0; it < nitems; it += gridDim.x, ++titer) {
      const WorkItem w = item_at(descs, items, it);
      if (!fused_tile<V>(sh, tmem, descs[w.aln], w.tile, titer, stall, limit, tab)) {
        *sh.abort_flag = 1;
        break;
      }
    }
  }

  tc_teardown(sh, tmem, issued, descs[0].err, kTcfMmaWarp);
}

// ------------------------------------------------------------ live form
//
// The served requests (rnj_server.cu): the roles of tc_fused_kernel over items
// claimed one at a time from a LiveList while the server keeps appending.
// The producer claims an item and hands it to the MMA warp and the epilogue
// warps through a two-slot ring in shared memory (full: the producer's
// arrival; empty: the MMA warp's and the sixteen epilogue warps' arrivals);
// an item with aln < 0 ends every role.  Two kinds of item: a tile to compute
// (loads, MMAs, transform), and a tile to fix up (the epilogue warps only:
// -1 -> 2 x the request's maximum), which the CTA that finished a request's
// last tile appends to the fix-up list, one per flagged tile, so that the
// fix-up of a large saturated request is spread over every CTA.  After each
// item the sixteen epilogue warps meet on an mbarrier (bounded waits, like
// every wait here) and one thread does the item's accounting.

struct LiveRing {
  WorkItem item[2];
  uint64_t full[2], empty[2];
  uint64_t epi;  // the epilogue warps' meeting point after each item
  int last;      // the item just finished completes its request's tiles
  int sat;       // ... and one of them holds a saturated pair
};
constexpr size_t kLiveExtra = kTcfTableBytes + 128;
static_assert(sizeof(LiveRing) <= 128, "the live ring fits its shared-memory slot");
constexpr int kLiveFix = 0x40000000;  // WorkItem::aln bit of a fix-up item in the ring

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_gpu64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Claims index h of a list (head / tail counters) if one is below the tail:
// h, or -1.  A failed compare-and-swap means another CTA took that index.
__device__ __forceinline__ int live_take(unsigned int *head, const unsigned int *tail) {
  for (;;) {
    const unsigned int t = ld_acquire_gpu(tail);
    const unsigned int h = ld_relaxed_gpu(head);
    if (h >= t) return -1;
    if (atomicCAS(head, h, h + 1) == h) return (int)h;
  }
}

// The next item: a fix-up item first (aln | kLiveFix), else a tile to compute;
// aln = -1 when the launch is closing (every CTA idle for idle_ns: the exit
// vote of LiveList), on abort, or when a fix-up item's writer did not complete
// it within the wait limit (err set).  A CTA that voted keeps looking for
// items, and takes its vote back when it finds one, until the vote closes the
// launch (or, as a bound, for the wait limit).
__device__ WorkItem live_claim(const LiveList &L, volatile int *abort_flag, uint64_t idle_ns,
                               uint64_t limit) {
  WorkItem w;
  w.aln = -1;
  w.tile = 0;
  uint64_t t0 = 0;
  bool voted = false;
  for (;;) {
    if (*abort_flag || ld_acquire_gpu(L.closing)) return w;
    int f = live_take(L.fix_head, L.fix_tail);
    if (f >= 0) {
      if (voted) atomicSub(L.idle_ctas, 1u);
      // reserved by atomicAdd before it is written: wait (bounded) for the write
      unsigned long long v = ld_acquire_gpu64(L.fix_items + f);
      const uint64_t s0 = global_timer_ns();
      while (v == 0ull && global_timer_ns() - s0 < limit) {
        __nanosleep(64);
        v = ld_acquire_gpu64(L.fix_items + f);
      }
      if (v == 0ull) {
        atomicOr(L.err, 1);
        *abort_flag = 1;
        return w;
      }
      w.aln = (int)(v & 0xFFFFFFFFull) - 1;
      w.tile = (int)(v >> 32);
      w.aln |= kLiveFix;
      return w;
    }
    f = live_take(L.head, L.tail);
    if (f >= 0) {
      if (voted) atomicSub(L.idle_ctas, 1u);
      return L.items[f];
    }
    const uint64_t now = global_timer_ns();
    if (t0 == 0) t0 = now;
    if (!voted && now - t0 > idle_ns) {
      voted = true;
      if (atomicAdd(L.idle_ctas, 1u) + 1u == gridDim.x) st_release_gpu(L.closing, 1u);
    }
    if (voted && now - t0 > idle_ns + limit) return w;  // bound: leave regardless
    __nanosleep(256);
  }
}

__device__ __forceinline__ long long live_tiles(const AlnDesc &d) {
  return (long long)d.nt * (d.nt + 1) / 2;
}

// One round of the epilogue warps' meeting point: every warp arrives, then
// waits (bounded) for the round to complete.  False when a wait ran out.
__device__ __forceinline__ bool live_epi_sync(const TcShared &sh, LiveRing *lr, uint32_t &phase,
                                              uint64_t limit) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    mbar_arrive(&lr->epi);
    ok = tc_wait(&lr->epi, phase, sh.abort_flag, limit);
  }
  phase ^= 1u;
  ok = __shfl_sync(0xffffffffu, ok, 0);
  __syncwarp();  // the other lanes read what lane 0's wait made visible
  return ok != 0;
}

// The request of slot aln is complete: its maximum, then the flag (thread 0).
__device__ __forceinline__ void live_report(const LiveList &L, const AlnDesc &d, int aln) {
  const int mbits = *reinterpret_cast<volatile int *>(d.max_bits);
  __threadfence_system();
  volatile int2 *slot = L.done + aln;
  slot->y = mbits;
  __threadfence_system();
  slot->x = 1;
}

__global__ void __launch_bounds__(kTcfThreads, 1)
    tc_live_kernel(const AlnDesc *__restrict__ descs, const LiveList live, int nst) {
  extern __shared__ uint8_t smem_raw[];
  const TcShared sh = tc_shared(smem_raw, nst, kLiveExtra);
  double2 *const tab = reinterpret_cast<double2 *>(tc_extra(sh));
  LiveRing *const lr = reinterpret_cast<LiveRing *>(tc_extra(sh) + kTcfTableBytes);
  const uint64_t limit = wait_limit_ns((uint32_t)descs[0].wait_us);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int e = tid; e < 128; e += kTcfThreads)
    tab[e] = make_double2(-0.25 * c_log_tab[e][0], -0.25 * c_log_tab[e][1]);
  if (tid == 0) {
    for (int k = 0; k < 2; ++k) {
      mbar_init(&lr->full[k], 1);
      mbar_init(&lr->empty[k], 1 + kTcfEpiWarps);
    }
    mbar_init(&lr->epi, kTcfEpiWarps);
    lr->last = 0;
    lr->sat = 0;
  }
  // (tc_setup's fence and block barrier publish these barriers too)
  const uint32_t tmem = tc_setup(sh, kTcfEpiWarps, 0, kTcfMmaWarp);
  uint32_t issued = 0;

  if (warp >= kTcfProducerWarp) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kTcfRegsLow) : "memory");
    if (warp == kTcfProducerWarp && lane == 0) {
      // ------------------------------------------------------- producer
      uint32_t gkb = 0, islot = 0, iph = 0, pph = 0;
      int ps = 0;
      const uint64_t idle = (uint64_t)live.idle_us * 1000ull;
      for (;;) {
        WorkItem w = live_claim(live, sh.abort_flag, idle, limit);
        if (w.aln >= 0) {
          const int a = w.aln & ~kLiveFix;
          bool bad = a >= live.cap_aln;
          if (!bad) bad = w.tile < 0 || (long long)w.tile >= live_tiles(descs[a]);
          if (bad) {  // a malformed item ends the launch with an error
            atomicOr(live.err, 1);
            *sh.abort_flag = 1;
            w.aln = -1;
          }
        }
        if (!tc_wait(&lr->empty[islot], iph ^ 1u, sh.abort_flag, limit)) {
          *sh.abort_flag = 1;
          break;
        }
        lr->item[islot] = w;
        mbar_arrive(&lr->full[islot]);
        if (++islot == 2) {
          islot = 0;
          iph ^= 1u;
        }
        if (w.aln < 0) break;
        if (w.aln & kLiveFix) continue;  // the epilogue warps' work only
        if (!tc_produce_item(sh, descs[w.aln], w.tile, gkb, issued, ps, pph, limit)) break;
      }
    } else if (warp == kTcfMmaWarp) {
      // ------------------------------------------------------- MMA issuer
      const uint64_t desc0 = smem_desc_sw128(smem_u32(sh.stages));
      uint32_t titer = 0, islot = 0, iph = 0, ring_ph = 0;  // titer: tiles computed
      int ring = 0;
      for (;;) {
        int ok = 1, aln = -1, tile = 0;
        if (lane == 0) {
          ok = tc_wait(&lr->full[islot], iph, sh.abort_flag, limit);
          if (ok) {
            aln = lr->item[islot].aln;
            tile = lr->item[islot].tile;
            mbar_arrive(&lr->empty[islot]);
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        aln = __shfl_sync(0xffffffffu, aln, 0);
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (++islot == 2) {
          islot = 0;
          iph ^= 1u;
        }
        if (!ok) {
          if (lane == 0) *sh.abort_flag = 1;
          break;
        }
        if (aln < 0) break;
        if (aln & kLiveFix) continue;
        if (!tc_issue_item(sh, tmem, desc0, descs[aln], titer, ring, ring_ph, limit)) break;
        ++titer;
      }
      tc_issue_drain(sh);
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kTcfRegsHigh) : "memory");
    // --------------------------------------------------------- epilogue
    uint32_t titer = 0, islot = 0, iph = 0, ephase = 0;  // titer: tiles computed
    const int nthr = kTcfEpiWarps * 32;
    for (;;) {
      int ok = 1, aln = -1, tile = 0;
      if (lane == 0) {
        ok = tc_wait(&lr->full[islot], iph, sh.abort_flag, limit);
        if (ok) {
          aln = lr->item[islot].aln;
          tile = lr->item[islot].tile;
          mbar_arrive(&lr->empty[islot]);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      aln = __shfl_sync(0xffffffffu, aln, 0);
      tile = __shfl_sync(0xffffffffu, tile, 0);
      if (++islot == 2) {
        islot = 0;
        iph ^= 1u;
      }
      if (!ok) {
        *sh.abort_flag = 1;
        break;
      }
      if (aln < 0) break;
      const bool fix = (aln & kLiveFix) != 0;
      aln &= ~kLiveFix;
      const AlnDesc &d = descs[aln];
      if (fix) {
        // -------------------------------------------- a tile to fix up
        const float m2 = __fmul_rn(__int_as_float(*reinterpret_cast<volatile int *>(d.max_bits)),
                                   2.0f);
        fixup_tile<4>(d, tile, m2, tid, nthr);  // 4 loads in flight: registers are short here
        __threadfence();
        if (!live_epi_sync(sh, lr, ephase, limit)) {
          *sh.abort_flag = 1;
          break;
        }
        if (tid == 0 && atomicSub(&live.fix_pending[aln], 1u) == 1u) {
          __threadfence();
          live_report(live, d, aln);
        }
        continue;
      }
      // ----------------------------------------------- a tile to compute
      if (!fused_tile<kFusedAny>(sh, tmem, d, tile, titer, 0, limit, tab, &live.sat[aln])) {
        *sh.abort_flag = 1;
        break;
      }
      ++titer;
      // The tile's stores, maximum and flags are visible device-wide before the
      // tile is counted; the CTA that counts a request's last tile sees every
      // other tile's (fence, count, fence).
      __threadfence();
      if (!live_epi_sync(sh, lr, ephase, limit)) {
        *sh.abort_flag = 1;
        break;
      }
      if (tid == 0) {
        const unsigned int old = atomicAdd(&live.tiles_done[aln], 1u);
        __threadfence();
        const int last = (long long)old + 1 == live_tiles(d);
        lr->last = last;
        lr->sat = last ? *reinterpret_cast<volatile int *>(&live.sat[aln]) : 0;
        // the appending CTA's hold on the request's completion
        if (last && lr->sat) atomicAdd(&live.fix_pending[aln], 1u);
      }
      if (!live_epi_sync(sh, lr, ephase, limit)) {
        *sh.abort_flag = 1;
        break;
      }
      if (!*reinterpret_cast<volatile int *>(&lr->last)) continue;
      if (!*reinterpret_cast<volatile int *>(&lr->sat)) {
        if (tid == 0) live_report(live, d, aln);
        continue;
      }
      // Saturated pairs: a fix-up item per flagged tile, for any CTA to take.
      const long long nt = live_tiles(d);
      for (long long t = tid; t < nt; t += nthr) {
        if (*reinterpret_cast<volatile int *>(&d.tile_flags[t]) == 0) continue;
        atomicAdd(&live.fix_pending[aln], 1u);
        const unsigned int p = atomicAdd(live.fix_tail, 1u);
        st_release_gpu64(live.fix_items + p,
                         ((unsigned long long)t << 32) | (unsigned long long)(aln + 1));
      }
      __threadfence();
      if (!live_epi_sync(sh, lr, ephase, limit)) {
        *sh.abort_flag = 1;
        break;
      }
      if (tid == 0 && atomicSub(&live.fix_pending[aln], 1u) == 1u) {
        __threadfence();
        live_report(live, d, aln);
      }
    }
  }

  tc_teardown(sh, tmem, issued, live.err, kTcfMmaWarp);
}

// One request into the live list: its slot's scratch cleared (maximum, tile
// count, fix-up count, saturation word, tile flags), then its items, then the
// tail (release).
__global__ void live_publish_kernel(const LiveList live, int aln, int nt, int band,
                                    unsigned int first, unsigned int count, int *max_bits,
                                    int *tile_flags) {
  if (threadIdx.x == 0) {
    *max_bits = 0;
    live.tiles_done[aln] = 0;
    live.fix_pending[aln] = 0;
    live.sat[aln] = 0;
  }
  for (unsigned int k = threadIdx.x; k < count; k += blockDim.x) {
    tile_flags[k] = 0;
    WorkItem w;
    w.aln = aln;
    w.tile = banded_tile((int)k, nt, band);
    live.items[first + k] = w;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) st_release_gpu(live.tail, first + count);
}

cudaError_t launch_tc_live(const AlnDesc *d_descs, const LiveList &live, int grid, int stages,
                           cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  const int nst = tc_ring_depth(stages, kTcfStages, kTcfStages);
  const size_t smem = tc_smem_bytes(nst, kLiveExtra);
  cudaError_t e = cudaFuncSetAttribute(tc_live_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  tc_live_kernel<<<(unsigned)grid, kTcfThreads, smem, s>>>(d_descs, live, nst);
  return cudaGetLastError();
}

cudaError_t launch_live_publish(const LiveList &live, int aln, int nt, int band,
                                unsigned int first, unsigned int count, int *max_bits,
                                int *tile_flags, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  live_publish_kernel<<<1, 1024, 0, s>>>(live, aln, nt, band > 0 ? band : kBand, first, count,
                                         max_bits, tile_flags);
  return cudaGetLastError();
}

template <int V>
static cudaError_t launch_variant(const AlnDesc *d_descs, const WorkItem *d_items,
                                  const int *d_nitems, int nitems, int item0, int count, int grid,
                                  int stages, cudaStream_t s) {
  const int nst = tc_ring_depth(stages, kTcfStages, kTcfStages);
  const size_t smem = tc_smem_bytes(nst, kTcfTableBytes);
  cudaError_t e = cudaFuncSetAttribute(tc_fused_kernel<V>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  tc_fused_kernel<V><<<(unsigned)grid, kTcfThreads, smem, s>>>(d_descs, d_items, d_nitems, nitems,
                                                              item0, count, nst);
  return cudaGetLastError();
}

int fused_variant_for(int model, int type, int compat, int full) {
  if (full) return FUSED_FULL;
  if (compat) return FUSED_GENERIC;
  if (model == RNJ_JC) return FUSED_JC;
  return type == RNJ_PROTEIN ? FUSED_PROTEIN : FUSED_K2P;
}

int fused_ring_depth(int stages) { return tc_ring_depth(stages, kTcfStages, kTcfStages); }

cudaError_t launch_tc_fused(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                            int nitems, int item0, int count, int grid, int variant,
                            cudaStream_t s, int stages) {
  if (grid <= 0) return cudaSuccess;
  using Launch = cudaError_t (*)(const AlnDesc *, const WorkItem *, const int *, int, int, int,
                                 int, int, cudaStream_t);
  // indexed by FusedVariant
  static const Launch kLaunch[] = {launch_variant<kFusedK2p>,     launch_variant<kFusedJc>,
                                   launch_variant<kFusedProtein>, launch_variant<kFusedGeneric>,
                                   launch_variant<kFusedFull>,    launch_variant<kFusedAny>};
  if (variant < FUSED_K2P || variant > FUSED_ANY) return cudaErrorInvalidValue;
  return kLaunch[variant](d_descs, d_items, d_nitems, nitems, item0, count, grid, stages, s);
}

}  // namespace rnj
