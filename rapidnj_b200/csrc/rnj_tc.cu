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
// Kernel.  Persistent, one CTA per SM, over a work list of 128 x 128 triangle
// tiles (of one alignment, or of many in a batch), 320 threads:
//   warp 0       TMA producer: 128-row x 128-byte K-blocks of both row tiles,
//                128-byte swizzle, into a 6-stage mbarrier ring
//   warp 1       TMEM owner and MMA issuer: tcgen05.mma.kind::i8, M = N = 128,
//                K = 32 per instruction, three accumulators (V, R, T) of 128
//                columns each; tcgen05.commit releases stages and signals the end
//   warps 2..9   epilogue: per 32-column chunk, tcgen05.ld of the accumulators,
//                the exact transform and the stores (tile rows as float4, the
//                mirror image with warp-coalesced column stores); then TMEM is
//                handed back to the MMA warp
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

// The reference loader's DNA layout (16 sites per uint32, 2-bit codes A=00 G=01
// T=10 C=11, gap filter 01 per valid site, dataloaderFasta.hpp:147-182) ->
// features.  One thread per (sequence, source word) = 16 sites.
__global__ void pack_features_bits_kernel(const uint32_t *__restrict__ bits,
                                          const uint32_t *__restrict__ gaps, int bs_words, int n,
                                          int L, int Np, int Lk, int8_t *__restrict__ F) {
  const int chunks = Lk / 16;
  const long long total = (long long)Np * chunks;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / chunks);
    const int c = (int)(t % chunks);
    uint32_t v[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0}, tt[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
    if (i < n && c < bs_words) {
      const uint32_t b = bits[(size_t)i * bs_words + c];
      const uint32_t g = gaps[(size_t)i * bs_words + c];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (c * 16 + k >= L || !((g >> (2 * k)) & 1u)) continue;
        const uint32_t code = (b >> (2 * k)) & 3u;  // A=0 G=1 T=2 C=3
        const int rr = (code < 2) ? 1 : -1;
        const int ts = (code == 0 || code == 3) ? 1 : -1;
        const int sh = (k & 3) * 8;
        v[k >> 2] |= 1u << sh;
        r[k >> 2] |= (uint32_t)(uint8_t)(int8_t)rr << sh;
        tt[k >> 2] |= (uint32_t)(uint8_t)(int8_t)ts << sh;
        u[k >> 2] |= (uint32_t)(uint8_t)(int8_t)(rr * ts) << sh;
      }
    }
    int8_t *row = F + (size_t)i * 4 * Lk + c * 16;
    *reinterpret_cast<uint4 *>(row) = make_uint4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<uint4 *>(row + Lk) = make_uint4(r[0], r[1], r[2], r[3]);
    *reinterpret_cast<uint4 *>(row + 2 * (size_t)Lk) = make_uint4(tt[0], tt[1], tt[2], tt[3]);
    *reinterpret_cast<uint4 *>(row + 3 * (size_t)Lk) = make_uint4(u[0], u[1], u[2], u[3]);
  }
}

cudaError_t launch_pack_features_bits(const uint32_t *d_bits, const uint32_t *d_gaps, int bs_words,
                                      int n, int L, int Np, int Lk, int8_t *F, cudaStream_t s) {
  const long long work = (long long)Np * (Lk / 16);
  long long g = (work + 255) / 256;
  if (g > 148LL * 64) g = 148LL * 64;
  if (g < 1) g = 1;
  pack_features_bits_kernel<<<(unsigned)g, 256, 0, s>>>(d_bits, d_gaps, bs_words, n, L, Np, Lk, F);
  return cudaGetLastError();
}

// ----------------------------------------------------------------- the kernel
//
// Persistent over a work list of (alignment, triangle tile) items: CTA b takes
// items b, b + G, b + 2G, ... (the list is ordered by decreasing cost, so this
// round robin balances).  Stage counters run on across items, so the producer
// streams the next tile's operands while the epilogue of the current one runs
// (the epilogue works from tensor memory and registers only, never from the
// stage buffers); the MMA warp waits for the epilogue's hand-back of tensor
// memory before it overwrites the accumulators.

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

__device__ __forceinline__ void item_tile(const AlnDesc &d, int tile, int &ti, int &tj) {
  if (d.full) {
    ti = tile / d.nt;
    tj = tile % d.nt;
  } else {
    tri_coords(tile, d.nt, ti, tj);
  }
}

__device__ __forceinline__ WorkItem item_at(const WorkItem *items, int it) {
  if (items) return items[it];
  WorkItem w;
  w.aln = 0;
  w.tile = it;
  return w;
}

template <int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_batch_kernel(const AlnDesc *__restrict__ descs, const WorkItem *__restrict__ items,
                    const int *__restrict__ nitems_ptr, int nitems_direct) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem =
      reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full_bar = reinterpret_cast<uint64_t *>(smem + kTcStages * kTcStageBytes);
  uint64_t *empty_bar = full_bar + kTcStages;
  uint64_t *acc_full = empty_bar + kTcStages;
  uint64_t *tmem_empty = acc_full + 1;
  uint64_t *drain_bar = tmem_empty + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain_bar + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nitems = nitems_ptr ? *nitems_ptr : nitems_direct;

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(tmem_empty, 256);
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  uint32_t issued = 0;  // producer: k-blocks issued in total (thread 0 only)

  if (warp == 0) {
    if (lane == 0) {
      // ----------------------------------------------------------- producer
      uint32_t gkb = 0;
      for (int it = blockIdx.x; it < nitems && !*abort_flag; it += gridDim.x) {
        const WorkItem w = item_at(items, it);
        const AlnDesc &d = descs[w.aln];
        tensormap_acquire(&d.map);
        int ti, tj;
        item_tile(d, w.tile, ti, tj);
        const int nkb = 4 * d.kdim / kTcKBlock;
        for (int kb = 0; kb < nkb; ++kb, ++gkb) {
          const int s = gkb % kTcStages;
          if (!tc_wait(&empty_bar[s], ((gkb / kTcStages) & 1) ^ 1, abort_flag)) {
            *abort_flag = 1;
            break;
          }
          uint8_t *a = smem + s * kTcStageBytes;
          mbar_arrive_expect_tx(&full_bar[s], kTcStageBytes);
          tma_load_2d(a, &d.map, &full_bar[s], kb * kTcKBlock, ti * kTile);
          tma_load_2d(a + kTcTileBytes, &d.map, &full_bar[s], kb * kTcKBlock, tj * kTile);
          issued = gkb + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // -------------------------------------------------------- MMA issuer
      uint32_t gkb = 0, titer = 0;
      for (int it = blockIdx.x; it < nitems && !*abort_flag; it += gridDim.x, ++titer) {
        const WorkItem w = item_at(items, it);
        const AlnDesc &d = descs[w.aln];
        const int nkb = 4 * d.kdim / kTcKBlock;
        const int seg = d.kdim / kTcKBlock;
        // The epilogue of the previous item must have read the accumulators.
        if (!tc_wait(tmem_empty, (titer & 1) ^ 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb, ++gkb) {
          const int s = gkb % kTcStages;
          if (!tc_wait(&full_bar[s], (gkb / kTcStages) & 1, abort_flag)) {
            ok = false;
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
        }
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        tc_commit(acc_full);
      }
      // Every MMA issued has completed before tensor memory is released.
      tc_commit(drain_bar);
      mbar_wait_bounded(drain_bar, 0);
    }
  } else {
    // ----------------------------------------------------------- epilogue
    // Warps 2..9: TMEM lane quarter = warp % 4 (row block), column half by group.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    uint32_t titer = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x, ++titer) {
      const WorkItem w = item_at(items, it);
      const AlnDesc &d = descs[w.aln];
      int ti, tj;
      item_tile(d, w.tile, ti, tj);
      if (!tc_wait(acc_full, titer & 1, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int n = d.n;
      const int i = ti * kTile + row;
      EpiParams ep;
      ep.n = n;
      ep.L = d.L;
      ep.model = d.model;
      ep.type = d.type;
      ep.compat_wrap = d.compat;
      ep.full = d.full;
      ep.jc_b = d.jc_b;
      float tmax = 0.0f;
      bool sat = false;
      // Per 32-column chunk: accumulators -> counts -> distances -> stores.
#pragma unroll 1
      for (int cc = 0; cc < 2; ++cc) {
        uint32_t V[32], R[32], T[32];
        const int cbase = half * 64 + cc * 32;
        const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)cbase;
        tmem_ld32(base, V);
        tmem_ld32(base + kTile, R);
        tmem_ld32(base + 2 * kTile, T);
        tmem_ld_wait();
        const int jb = tj * kTile + cbase;
        if constexpr (EPI == EPI_DIST) {
          float *orow = d.out + (size_t)i * d.ld;
#pragma unroll
          for (int c4 = 0; c4 < 32; c4 += 4) {
            float x[4];
            bool okc[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int k = c4 + u;
              const int j = jb + k;
              const int vv = (int)V[k], rr = (int)R[k], tu = (int)T[k];
              const uint32_t ts = (uint32_t)((vv + rr - tu) >> 2);
              const uint32_t tv = (uint32_t)((vv - rr) >> 1);
              okc[u] = d.full ? (i < n && j < n && i != j) : (i < j && j < n);
              x[u] = 0.0f;
              if (okc[u]) {
                x[u] = pair_distance(ep, d.model == RNJ_JC ? ts + tv : ts,
                                     d.model == RNJ_JC ? 0u : tv, (uint32_t)vv);
                if (x[u] > tmax) tmax = x[u];
                if (x[u] == -1.0f) sat = true;
              }
              // Mirror (column j of the tile is row j of the matrix): the lanes of
              // a warp hold 32 consecutive rows i, so these stores coalesce.
              if (okc[u] && !d.full) d.out[(size_t)j * d.ld + i] = x[u];
            }
            const int j0 = jb + c4;
            if (okc[0] && okc[1] && okc[2] && okc[3] && ((d.ld & 3) == 0)) {
              *reinterpret_cast<float4 *>(orow + j0) = make_float4(x[0], x[1], x[2], x[3]);
            } else {
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int j = j0 + u;
                if (okc[u]) orow[j] = x[u];
                else if (i == j && i < n) orow[j] = 0.0f;
              }
            }
          }
        } else {
          if (i < n) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
              const int j = jb + k;
              const bool ok = d.full ? (j < n) : (i < j && j < n);
              if (!ok) continue;
              const int vv = (int)V[k], rr = (int)R[k], tu = (int)T[k];
              uint32_t *o = d.counts + ((size_t)i * n + j) * 3;
              o[0] = (uint32_t)((vv + rr - tu) >> 2);
              o[1] = (uint32_t)((vv - rr) >> 1);
              o[2] = (uint32_t)vv;
            }
          }
        }
      }
      // Accumulators read: the MMA warp may start the next item.
      tc_fence_before();
      mbar_arrive(tmem_empty);
      if constexpr (EPI == EPI_DIST) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
          tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, off));
        const bool any_sat = __any_sync(0xffffffffu, sat);
        if (lane == 0) {
          if (tmax > 0.0f) atomicMax(d.max_bits, __float_as_int(tmax));
          if (any_sat) d.tile_flags[w.tile] = 1;
        }
      }
    }
  }

  __syncthreads();
  if (tid == 0 && *abort_flag) {
    // Loads may still be in flight into stages the MMA never consumed: let the
    // last ring's worth land (bounded) before shared memory is released.
    for (uint32_t k = issued > (uint32_t)kTcStages ? issued - kTcStages : 0; k < issued; ++k)
      mbar_wait_bounded(&full_bar[k % kTcStages], (k / kTcStages) & 1);
    atomicOr(descs[0].err, 1);
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

cudaError_t launch_tc_batch(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                            int nitems, int grid, int epi_mode, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  cudaError_t e;
  if (epi_mode == EPI_DIST) {
    e = cudaFuncSetAttribute(tc_batch_kernel<EPI_DIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTcSmemBytes);
    if (e != cudaSuccess) return e;
    tc_batch_kernel<EPI_DIST><<<(unsigned)grid, kTcThreads, kTcSmemBytes, s>>>(d_descs, d_items,
                                                                               d_nitems, nitems);
  } else {
    e = cudaFuncSetAttribute(tc_batch_kernel<EPI_COUNTS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemBytes);
    if (e != cudaSuccess) return e;
    tc_batch_kernel<EPI_COUNTS><<<(unsigned)grid, kTcThreads, kTcSmemBytes, s>>>(d_descs, d_items,
                                                                                 d_nitems, nitems);
  }
  return cudaGetLastError();
}

}  // namespace rnj
