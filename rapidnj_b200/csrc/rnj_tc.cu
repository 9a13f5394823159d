// rnj_tc.cu -- DNA pair counting on the 5th-generation tensor cores (tcgen05).
//
// Encoding.  Every valid site of a sequence becomes four signed 8-bit features
// (v, r, t, u): v = 1; r = +1 for a purine (A, G), -1 for a pyrimidine (C, T);
// t = +1 for A and C, -1 for G and T; u = r * t.  A gap is (0, 0, 0, 0).  For
// two sites of a pair the products satisfy
//   identical:     vv' = 1, rr' = 1, tt' + uu' =  2
//   transition:    vv' = 1, rr' = 1, tt' + uu' = -2     (A<->G, C<->T)
//   transversion:  vv' = 1, rr' = -1, tt' + uu' = 0
// so with V = sum vv', R = sum rr', T = sum (tt' + uu') over the columns:
//   valid = V,   transitions = (V + R - T) / 4,   transversions = (V - R) / 2,
// exactly (integers), which are the counts bitDistanceGap.cpp:146-161 produces.
// The three sums are three Gram matrices of the feature matrix F (n x 4L): the
// v block (K = L), the r block (K = L) and the t|u block (K = 2L): 4 int8 MACs
// per pair-column, accumulated in int32 in tensor memory.
//
// Kernel.  One CTA per 128 x 128 tile of the upper triangle, 320 threads:
//   warp 0       TMA producer: 128-row x 128-byte K-blocks of both row tiles,
//                128-byte swizzle, into a 6-stage mbarrier ring
//   warp 1       TMEM owner and MMA issuer: tcgen05.mma.kind::i8, M = N = 128,
//                K = 32 per instruction, three accumulators (V, R, T) of 128
//                columns each; tcgen05.commit releases stages and signals the end
//   warps 2..9   epilogue: tcgen05.ld of the accumulators, the exact transform,
//                shared-memory staging and coalesced stores (tile and mirror)
// Every wait is bounded; on a timeout the CTA records an error, drains what it
// issued, frees its tensor memory and ends.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"

namespace rnj {

constexpr int kTcStages = 6;
constexpr int kTcKBlock = 128;                            // bytes of K per stage
constexpr uint32_t kTcTileBytes = kTile * kTcKBlock;      // 16 KB per operand tile
constexpr uint32_t kTcStageBytes = 2 * kTcTileBytes;      // A + B
constexpr int kTcThreads = 320;
constexpr uint32_t kTmemCols = 512;                       // 3 x 128 used
constexpr size_t kTcSmemBytes = (size_t)kTcStages * kTcStageBytes + 1024 + 256;

// ---------------------------------------------------------------- tcgen05 PTX

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void named_barrier(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, 8-row
// groups 1024 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                   // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;                   // version
  d |= (uint64_t)2u << 61;                   // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::i8: D s32 (bits 4-5 = 2), A and B signed 8-bit
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                              ((uint32_t)(kTile >> 4) << 24);

// A bounded wait that also gives up early once another role has aborted.
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < kWaitIterCap; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u) {
      if (*abort_flag) return false;
      if (global_timer_ns() - t0 > kWaitLimitNs) break;
    }
  }
  return false;
}

// --------------------------------------------------------------- feature pack

// chars (n rows, stride ld) -> F (Np rows, 4 * Lk bytes): [v | r | t | u] blocks
// of Lk bytes each; padding rows and columns are zero.  One thread per
// (sequence, 16-column chunk); writes 4 x 16 bytes.
__global__ void pack_features_kernel(const uint8_t *__restrict__ chars, size_t ld, int n, int L,
                                     int Np, int Lk, int8_t *__restrict__ F) {
  const int chunks = Lk / 16;
  const long long total = (long long)Np * chunks;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / chunks);
    const int c = (int)(t % chunks);
    uint32_t v[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0}, tt[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
    if (i < n) {
      const uint8_t *src = chars + (size_t)i * ld + c * 16;
#pragma unroll
      for (int b = 0; b < 16; ++b) {
        const int k = c * 16 + b;
        if (k >= L) break;
        int vv = 1, rr, ts;
        switch (src[b]) {
          case 'A': case 'a': rr = 1; ts = 1; break;
          case 'G': case 'g': rr = 1; ts = -1; break;
          case 'C': case 'c': rr = -1; ts = 1; break;
          case 'T': case 't': rr = -1; ts = -1; break;
          default: vv = 0; rr = 0; ts = 0; break;
        }
        const int sh = (b & 3) * 8;
        v[b >> 2] |= (uint32_t)(uint8_t)vv << sh;
        r[b >> 2] |= (uint32_t)(uint8_t)(int8_t)rr << sh;
        tt[b >> 2] |= (uint32_t)(uint8_t)(int8_t)ts << sh;
        u[b >> 2] |= (uint32_t)(uint8_t)(int8_t)(rr * ts) << sh;
      }
    }
    int8_t *row = F + (size_t)i * 4 * Lk + c * 16;
    *reinterpret_cast<uint4 *>(row) = make_uint4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<uint4 *>(row + Lk) = make_uint4(r[0], r[1], r[2], r[3]);
    *reinterpret_cast<uint4 *>(row + 2 * (size_t)Lk) = make_uint4(tt[0], tt[1], tt[2], tt[3]);
    *reinterpret_cast<uint4 *>(row + 3 * (size_t)Lk) = make_uint4(u[0], u[1], u[2], u[3]);
  }
}

// ----------------------------------------------------------------- the kernel

template <int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_count_kernel(const __grid_constant__ CUtensorMap fmap, int nt, int Lk, EpiParams ep) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem =
      reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full_bar = reinterpret_cast<uint64_t *>(smem + kTcStages * kTcStageBytes);
  uint64_t *empty_bar = full_bar + kTcStages;
  uint64_t *acc_bar = empty_bar + kTcStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_bar + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int ti, tj;
  const int tile_id = blockIdx.x;
  if (ep.full) {
    ti = tile_id / nt;
    tj = tile_id % nt;
  } else {
    tri_coords(tile_id, nt, ti, tj);
  }
  const int nkb = 4 * Lk / kTcKBlock;   // k-blocks over the whole feature row
  const int seg = Lk / kTcKBlock;       // k-blocks per feature block

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(acc_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
    prefetch_tmap(&fmap);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  int issued = 0;  // k-blocks whose loads the producer issued (thread 0 only)

  if (warp == 0) {
    if (lane == 0) {
      // Producer.
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % kTcStages;
        if (!tc_wait(&empty_bar[s], (uint32_t)(((kb / kTcStages) & 1) ^ 1), abort_flag)) {
          *abort_flag = 1;
          break;
        }
        uint8_t *a = smem + s * kTcStageBytes;
        mbar_arrive_expect_tx(&full_bar[s], kTcStageBytes);
        tma_load_2d(a, &fmap, &full_bar[s], kb * kTcKBlock, ti * kTile);
        tma_load_2d(a + kTcTileBytes, &fmap, &full_bar[s], kb * kTcKBlock, tj * kTile);
        issued = kb + 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer.
      int issued_kb = 0;
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % kTcStages;
        if (!tc_wait(&full_bar[s], (uint32_t)((kb / kTcStages) & 1), abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const int acc = kb < seg ? 0 : (kb < 2 * seg ? 1 : 2);
        const bool first = (kb == 0) || (kb == seg) || (kb == 2 * seg);
        const uint32_t a_addr = smem_u32(smem + s * kTcStageBytes);
        const uint64_t adesc = smem_desc_sw128(a_addr);
        const uint64_t bdesc = smem_desc_sw128(a_addr + kTcTileBytes);
#pragma unroll
        for (int kk = 0; kk < kTcKBlock / 32; ++kk)
          tc_mma_i8(tmem + acc * kTile, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2),
                    kIdescI8, (first && kk == 0) ? 0u : 1u);
        tc_commit(&empty_bar[s]);
        issued_kb = kb + 1;
      }
      // Completion of every MMA issued (also on an abort, so that tensor memory
      // is not freed under a running MMA).
      tc_commit(acc_bar);
      if (issued_kb < nkb) {
        mbar_wait_bounded(acc_bar, 0);
      }
    }
  } else {
    // Epilogue: warps 2..9.  TMEM lane quarter = warp % 4; column half by group.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    float *S = reinterpret_cast<float *>(smem);
    bool ok = tc_wait(acc_bar, 0, abort_flag);
    if (!ok) *abort_flag = 1;
    named_barrier(1, 256);
    ok = (*abort_flag == 0);
    tc_fence_after();
    float tmax = 0.0f;
    bool sat = false;
    if (ok) {
      const int i = ti * kTile + row;
#pragma unroll 1
      for (int cc = 0; cc < 2; ++cc) {
        const int c0 = half * 64 + cc * 32;
        uint32_t V[32], R[32], T[32];
        const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0;
        tmem_ld32(base, V);
        tmem_ld32(base + kTile, R);
        tmem_ld32(base + 2 * kTile, T);
        tmem_ld_wait();
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const int j = tj * kTile + c0 + k;
          const int vv = (int)V[k], rr = (int)R[k], tu = (int)T[k];
          const uint32_t valid = (uint32_t)vv;
          const uint32_t ts = (uint32_t)((vv + rr - tu) >> 2);
          const uint32_t tv = (uint32_t)((vv - rr) >> 1);
          const bool pair_ok = ep.full ? (i < ep.n && j < ep.n && i != j) : (i < j && j < ep.n);
          if constexpr (EPI == EPI_DIST) {
            float x = 0.0f;
            if (pair_ok) {
              x = pair_distance(ep, ep.model == RNJ_JC ? ts + tv : ts, ep.model == RNJ_JC ? 0u : tv,
                                valid);
              if (x > tmax) tmax = x;
              if (x == -1.0f) sat = true;
            }
            S[row * kStageLd + c0 + k] = x;
          } else {
            if (pair_ok || (ep.full && i < ep.n && j < ep.n)) {
              uint32_t *o = ep.counts + ((size_t)i * ep.n + j) * 3;
              o[0] = ts;
              o[1] = tv;
              o[2] = valid;
            }
          }
        }
      }
    }
    tc_fence_before();
    named_barrier(1, 256);
    if constexpr (EPI == EPI_DIST) {
      if (ok) store_distances(ep, ti, tj, tile_id, S, tmax, sat, warp - 2, 8);
    }
    if (!ok && tid == 64) atomicOr(ep.err, 1);
  }
  __syncthreads();
  if (tid == 0 && *abort_flag) {
    // After an abort, loads may still be in flight into stages the MMA never
    // consumed: let the last ring's worth land (bounded) before the shared
    // memory is released.
    for (int kb = issued > kTcStages ? issued - kTcStages : 0; kb < issued; ++kb)
      mbar_wait_bounded(&full_bar[kb % kTcStages], (uint32_t)((kb / kTcStages) & 1));
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ------------------------------------------------------------------ launchers

cudaError_t launch_pack_features(const uint8_t *d_chars, size_t ld, int n, int L, int Np, int Lk,
                                 int8_t *F, cudaStream_t s) {
  const long long work = (long long)Np * (Lk / 16);
  long long g = (work + 255) / 256;
  if (g > 148LL * 64) g = 148LL * 64;
  if (g < 1) g = 1;
  pack_features_kernel<<<(unsigned)g, 256, 0, s>>>(d_chars, ld, n, L, Np, Lk, F);
  return cudaGetLastError();
}

cudaError_t launch_tc_count(const CUtensorMap &fmap, int n, int Lk, int epi_mode, const EpiParams &ep,
                            cudaStream_t s) {
  const int nt = tiles_of(n);
  const long long ntiles = ep.full ? (long long)nt * nt : tri_tiles(nt);
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e;
  if (epi_mode == EPI_DIST) {
    e = cudaFuncSetAttribute(tc_count_kernel<EPI_DIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTcSmemBytes);
    if (e != cudaSuccess) return e;
    tc_count_kernel<EPI_DIST><<<(unsigned)ntiles, kTcThreads, kTcSmemBytes, s>>>(fmap, nt, Lk, ep);
  } else {
    e = cudaFuncSetAttribute(tc_count_kernel<EPI_COUNTS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemBytes);
    if (e != cudaSuccess) return e;
    tc_count_kernel<EPI_COUNTS><<<(unsigned)ntiles, kTcThreads, kTcSmemBytes, s>>>(fmap, nt, Lk, ep);
  }
  return cudaGetLastError();
}

}  // namespace rnj
