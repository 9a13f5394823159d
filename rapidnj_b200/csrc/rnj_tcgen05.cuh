// rnj_tcgen05.cuh -- tcgen05 (5th-generation tensor core) and TMA building blocks
// shared by the tensor-core counting kernels (rnj_tc.cu, rnj_tcf.cu): tensor
// memory allocation, MMA issue and commit, tensor-memory loads, shared-memory
// descriptors, bounded waits and the work order of a single alignment's
// triangle tiles.  Inline PTX for sm_100a.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"

namespace rnj {

constexpr int kTcStages = 7;  // deepest ring of the two-kernel form (tc_batch_kernel)
constexpr int kTcMinStages = 2;
constexpr int kTcKBlock = 128;                            // bytes of K per stage (256 FP4 columns)
constexpr int kTcKCols = 256;                             // feature columns per stage
constexpr uint32_t kTcTileBytes = kTile * kTcKBlock;      // 16 KB per operand tile
constexpr uint32_t kTcStageBytes = 2 * kTcTileBytes;      // A + B
constexpr int kTcThreads = 320;
constexpr uint32_t kTmemCols = 512;                       // 3 x 128 accumulators + scale factors
constexpr uint32_t kTmemSfa = 384, kTmemSfb = 448;        // scale-factor columns (all 1.0)
// Dynamic shared memory of a counting kernel with an nst-stage ring: 1024
// bytes of alignment slack, the 256-byte barrier block, `extra` bytes after it
// (both padded to 1024), then the ring.  The barriers and the extra bytes sit
// at fixed offsets before the ring, so the ring depth -- a launch parameter,
// the tuner's choice per bucket -- moves nothing but the ring's end, and the
// launch gives the kernel exactly the shared memory of its depth.
__host__ __device__ constexpr size_t tc_head_bytes(size_t extra) { return (256 + extra + 1023) / 1024 * 1024; }
constexpr size_t tc_smem_bytes(int nst, size_t extra = 0) {
  return 1024 + tc_head_bytes(extra) + (size_t)nst * kTcStageBytes;
}
constexpr size_t kTcSmemBytes = tc_smem_bytes(kTcStages);
static_assert(kTcSmemBytes <= 232448, "the deepest two-kernel ring fits the shared memory of one CTA");

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
// D (f32, tensor memory) (+)= A x B^T with FP4 operands from shared memory and
// block scale factors from tensor memory (block of 32 columns), issued by one
// elected lane of a converged warp.  The whole warp runs the issue loop, so the
// descriptor and tensor-memory operands are warp-uniform values; issued from a
// single divergent lane with per-instruction operand arithmetic, the MMA issue
// rate, not the tensor pipe, bounded the kernel (about 150 instead of 64
// cycles per 128 x 128 x 64 instruction).
__device__ __forceinline__ void tc_mma_fp4_elect(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                                 uint32_t idesc, uint32_t sfa_tmem,
                                                 uint32_t sfb_tmem, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "elect.sync _|e, 0xffffffff;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa_tmem),
      "r"(sfb_tmem)
      : "memory");
}
__device__ __forceinline__ void tc_commit_elect(uint64_t *bar) {
  asm volatile(
      "{\n\t.reg .pred e;\n\t"
      "elect.sync _|e, 0xffffffff;\n\t"
      "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}"
      ::"r"(smem_u32(bar))
      : "memory");
}
// 32 lanes x 32 columns of 32-bit words from registers into tensor memory.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, uint32_t x) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1};"
      ::"r"(taddr), "r"(x)
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
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

// Instruction descriptor, kind::mxf4 (block-scaled layout): A and B E2M1
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bits 17-22, scale factors
// UE8M0 (bit 23), M >> 4 at bits 24-28, scale-factor ids 0, dense K = 64.
constexpr uint32_t kIdescFp4 = (1u << 7) | (1u << 10) | ((uint32_t)(kTile >> 3) << 17) | (1u << 23) |
                               ((uint32_t)(kTile >> 4) << 24);

// A bounded wait (limit_ns) that also gives up early once another role has
// aborted.  Between tests the thread sleeps until the phase completes, for at
// most kTcWaitHintNs at a time (the limit and the abort flag are checked every
// 256 tests, at most about 2.6 ms apart).
constexpr uint32_t kTcWaitHintNs = 10000;
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                        uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < kWaitIterCap; ++it) {
    if (mbar_try_wait_hint(bar, parity, kTcWaitHintNs)) return true;
    if ((it & 255u) == 255u) {
      if (*abort_flag) return false;
      if (global_timer_ns() - t0 > limit_ns) break;
    }
  }
  return false;
}

// 32 lanes x 16 columns of 32-bit words from tensor memory into registers.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

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

// Work order of a single alignment's triangle (no explicit work list): bands of
// kBand tile rows, each walked column by column (within a column, its rows of
// the band).  The kernels resident at one time then share about kBand row tiles
// and 148 / kBand column tiles of operands instead of two rows and every
// column, which keeps the operand working set of the running tiles in L2.
// Returns the tile's row-major triangle index (the index of its saturation flag).
constexpr int kBand = 12;  // default band height (the autotuner may choose another)

__host__ __device__ __forceinline__ int banded_tile(int it, int nt, int band) {
  int r0 = 0;
  while (true) {
    const int g = band < nt - r0 ? band : nt - r0;
    const int tri = g * (g + 1) / 2;
    const int count = tri + (nt - r0 - g) * g;
    if (it < count || r0 + g >= nt) {
      int ti, tj;
      if (it < tri) {
        int c = (int)((sqrtf(8.0f * (float)it + 1.0f) - 1.0f) * 0.5f);
        while (c * (c + 1) / 2 > it) --c;
        while ((c + 1) * (c + 2) / 2 <= it) ++c;
        tj = r0 + c;
        ti = r0 + (it - c * (c + 1) / 2);
      } else {
        const int k = it - tri;
        tj = r0 + g + k / g;
        ti = r0 + k % g;
      }
      return ti * nt - ti * (ti - 1) / 2 + (tj - ti);
    }
    it -= count;
    r0 += g;
  }
}

__device__ __forceinline__ WorkItem item_at(const AlnDesc *descs, const WorkItem *items, int it) {
  if (items) return items[it];
  WorkItem w;
  w.aln = 0;
  const int band = descs[0].band > 0 ? descs[0].band : kBand;
  w.tile = descs[0].full ? it : banded_tile(it, descs[0].nt, band);
  return w;
}

// ------------------------------------------------- the counting pipeline
//
// The roles every tensor-core counting kernel shares, over a work list of
// (alignment, triangle tile) items that CTA b walks as b, b + G, b + 2G, ...:
//   warp 0, lane 0   TMA producer: per item, the K blocks of its row tile (A)
//                    and column tile (B) into the stage ring
//   warp 1           MMA issuer: per item, every K block into the accumulators
//                    (DNA blocks v, r, t, u -> V, R, T, T; protein blocks v,
//                    rank 0 .. -> V, M, M, ...), then a commit to acc_full
//   other warps      the kernel's own epilogue, which reads the accumulators,
//                    arrives on tmem_empty and works on from registers
// Stage counters run on across items, so the producer streams the next item's
// operands while the epilogue of the current one runs; the MMA warp waits for
// tmem_empty before it overwrites the accumulators.

// The barrier block at the start of shared memory (before the ring).
struct TcShared {
  uint8_t *stages;            // nst x (A | B), 1024-byte aligned
  uint64_t *full_bar;         // [nst] TMA bytes landed
  uint64_t *empty_bar;        // [nst] MMAs done reading
  uint64_t *acc_full;         // accumulators complete (one per item)
  uint64_t *tmem_empty;       // accumulators read by the epilogue
  uint64_t *drain_bar;        // every issued MMA complete (teardown)
  uint64_t *never_bar;        // nothing completes it: the failure-path test waits here
  uint32_t *tmem_slot;
  volatile int *abort_flag;
  int nst;                    // ring depth, kTcMinStages .. the kernel's maximum
};

// extra: the bytes after the barrier block the kernel asked for in
// tc_smem_bytes (a constant of the kernel).
__device__ __forceinline__ TcShared tc_shared(uint8_t *smem_raw, int nst, size_t extra) {
  TcShared sh;
  sh.nst = nst;
  uint8_t *const base =
      reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  sh.full_bar = reinterpret_cast<uint64_t *>(base);
  sh.empty_bar = sh.full_bar + kTcStages;
  sh.acc_full = sh.empty_bar + kTcStages;
  sh.tmem_empty = sh.acc_full + 1;
  sh.drain_bar = sh.tmem_empty + 1;
  sh.never_bar = sh.drain_bar + 1;
  sh.tmem_slot = reinterpret_cast<uint32_t *>(sh.never_bar + 1);
  sh.abort_flag = reinterpret_cast<volatile int *>(sh.tmem_slot + 1);
  sh.stages = base + tc_head_bytes(extra);
  return sh;
}
static_assert(8 * (2 * kTcStages + 4) + 8 <= 256, "the barrier block fits its 256 bytes");
// The extra bytes after the barrier block.
__device__ __forceinline__ uint8_t *tc_extra(const TcShared &sh) {
  return reinterpret_cast<uint8_t *>(sh.full_bar) + 256;
}
// The ring depth a kernel runs with: `requested` (0: the kernel's default
// `dflt`) within kTcMinStages .. `max_st`.
__host__ __device__ constexpr int tc_ring_depth(int requested, int dflt, int max_st) {
  return requested <= 0 ? dflt
                        : (requested < kTcMinStages ? kTcMinStages
                                                    : (requested > max_st ? max_st : requested));
}

// Barriers, tensor memory and the unit scale factors.  tmem_readers: arrivals
// that release the accumulators (epilogue threads or warps).  epi_warp0 ..
// epi_warp0 + 7: the warps that fill the scale-factor columns (two per lane
// quarter and column half).  alloc_warp allocates tensor memory (and frees it
// in tc_teardown).  Ends with a block barrier; returns the tensor memory base
// address.
__device__ __forceinline__ uint32_t tc_setup(const TcShared &sh, uint32_t tmem_readers,
                                             int epi_warp0, int alloc_warp = 1) {
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < sh.nst; ++s) {
      mbar_init(&sh.full_bar[s], 1);
      mbar_init(&sh.empty_bar[s], 1);
    }
    mbar_init(sh.acc_full, 1);
    mbar_init(sh.tmem_empty, tmem_readers);
    mbar_init(sh.drain_bar, 1);
    mbar_init(sh.never_bar, 1);
    *sh.abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == alloc_warp) {
    tmem_alloc(sh.tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *sh.tmem_slot;
  // Block scale factors: every byte of columns kTmemSfa..511 of all 128 lanes is
  // UE8M0 127 (2^0); the MMAs read theirs from kTmemSfa and kTmemSfb.
  if (warp >= epi_warp0 && warp < epi_warp0 + 8) {
    const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + kTmemSfa +
                          64u * (uint32_t)((warp - epi_warp0) >> 2);
    tmem_st32(base, 0x7F7F7F7Fu);
    tmem_st32(base + 32, 0x7F7F7F7Fu);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return tmem;
}

// The producer's loads of one item: its K blocks of the row tile (A) and the
// column tile (B) into the ring.  ps / pph: the ring stage and parity of the
// next load; gkb / issued: K blocks loaded so far and the count whose loads
// were issued.  False (abort flag set) when a wait ran out.
__device__ __forceinline__ bool tc_produce_item(const TcShared &sh, const AlnDesc &d, int tile,
                                                uint32_t &gkb, uint32_t &issued, int &ps,
                                                uint32_t &pph, uint64_t limit) {
  tensormap_acquire(&d.map);
  int ti, tj;
  item_tile(d, tile, ti, tj);
  const int nkb = d.np * d.kdim / kTcKCols;  // feature blocks x K blocks per block
  for (int kb = 0; kb < nkb; ++kb, ++gkb) {
    const int s = ps;
    if (!tc_wait(&sh.empty_bar[s], pph ^ 1u, sh.abort_flag, limit)) {
      *sh.abort_flag = 1;
      return false;
    }
    uint8_t *a = sh.stages + s * kTcStageBytes;
    mbar_arrive_expect_tx(&sh.full_bar[s], kTcStageBytes);
    tma_load_3d(a, &d.map, &sh.full_bar[s], 0, ti * kTile, kb);
    tma_load_3d(a + kTcTileBytes, &d.map, &sh.full_bar[s], 0, tj * kTile, kb);
    issued = gkb + 1;
    if (++ps == sh.nst) {
      ps = 0;
      pph ^= 1u;
    }
  }
  return true;
}

// The producer (one thread): items it0, it0 + step, ... below nitems.  Returns
// the number of K blocks whose loads it issued.
__device__ __forceinline__ uint32_t tc_produce(const TcShared &sh, const AlnDesc *descs,
                                               const WorkItem *items, int it0, int nitems,
                                               int step, uint64_t limit) {
  uint32_t gkb = 0, issued = 0;
  int ps = 0;           // stage of the next load and the parity of its fill
  uint32_t pph = 0;
  for (int it = it0; it < nitems && !*sh.abort_flag; it += step) {
    const WorkItem w = item_at(descs, items, it);
    if (!tc_produce_item(sh, descs[w.aln], w.tile, gkb, issued, ps, pph, limit)) break;
  }
  return issued;
}

// The MMA issuer's part of one item (the whole warp): waits until the
// epilogue has read the previous item's accumulators (titer: items so far),
// issues every K block into the accumulators (DNA blocks v, r, t, u -> V, R,
// T, T; protein blocks v, rank 0, .. -> V, M, M, ...) and commits to acc_full.
// ring / ring_ph: the stage of the next K block and the parity of its fill.
// Lane 0 waits, the result is broadcast; one elected lane issues each MMA and
// commit.  Descriptors are the stage base descriptors plus constant offsets:
// the 14-bit start-address field (16-byte units) of a shared address below
// 228 KB cannot carry out.  False (abort flag set) when a wait ran out.
__device__ __forceinline__ bool tc_issue_item(const TcShared &sh, uint32_t tmem, uint64_t desc0,
                                              const AlnDesc &d, uint32_t titer, int &ring,
                                              uint32_t &ring_ph, uint64_t limit) {
  const int lane = threadIdx.x & 31;
  constexpr uint64_t kStageStep = kTcStageBytes >> 4, kBStep = kTcTileBytes >> 4;
  const int nkb = d.np * d.kdim / kTcKCols;
  const int seg = d.kdim / kTcKCols;  // K blocks per feature block
  const bool prot = d.kind == KIND_PROT_TC;
  // The epilogue of the previous item must have read the accumulators.
  int ok = 1;
  if (lane == 0) ok = tc_wait(sh.tmem_empty, (titer & 1) ^ 1, sh.abort_flag, limit);
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (!ok) {
    if (lane == 0) *sh.abort_flag = 1;
    return false;
  }
  tc_fence_after();
  // Per K block: every lane tests the stage's full barrier (one warp vote
  // when it is already complete, the common case; otherwise lane 0 waits,
  // bounded); the stage, its parity, the accumulator and whether the block
  // starts that accumulator's sum follow from counters.  Measured: the
  // per-block division, modulo and broadcast cost 15 % of the kernel.
  const int last_acc = prot ? 1 : 2;
  int kin = 0, blk = 0;  // K block within its feature block, feature block
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = ring;
    if (!__all_sync(0xffffffffu, mbar_try_wait(&sh.full_bar[s], ring_ph))) {
      if (lane == 0) ok = tc_wait(&sh.full_bar[s], ring_ph, sh.abort_flag, limit);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
    }
    tc_fence_after();
    const int acc = blk < last_acc ? blk : last_acc;
    const uint32_t first = (kin == 0) && (blk <= last_acc);
    if (++kin == seg) {
      kin = 0;
      ++blk;
    }
    if (++ring == sh.nst) {
      ring = 0;
      ring_ph ^= 1u;
    }
    const uint64_t adesc = desc0 + (uint64_t)s * kStageStep;
    const uint64_t bdesc = adesc + kBStep;
    const uint32_t dt = tmem + (uint32_t)(acc * kTile);
    // 32 bytes = 64 columns per MMA, four per 128-byte stage.
    tc_mma_fp4_elect(dt, adesc, bdesc, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, first ^ 1u);
    tc_mma_fp4_elect(dt, adesc + 2, bdesc + 2, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
    tc_mma_fp4_elect(dt, adesc + 4, bdesc + 4, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
    tc_mma_fp4_elect(dt, adesc + 6, bdesc + 6, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
    tc_commit_elect(&sh.empty_bar[s]);
  }
  if (!ok) {
    if (lane == 0) *sh.abort_flag = 1;
    return false;
  }
  tc_commit_elect(sh.acc_full);
  return true;
}

// Every MMA the warp issued has completed (before tensor memory is released).
__device__ __forceinline__ void tc_issue_drain(const TcShared &sh) {
  tc_commit_elect(sh.drain_bar);
  if ((threadIdx.x & 31) == 0) mbar_wait_bounded(sh.drain_bar, 0);
  __syncwarp();
}

// The MMA issuer (a whole warp): the same items as the producer.  Ends after
// every MMA it issued has completed.
__device__ __forceinline__ void tc_issue(const TcShared &sh, uint32_t tmem, const AlnDesc *descs,
                                         const WorkItem *items, int it0, int nitems, int step,
                                         uint64_t limit) {
  const uint64_t desc0 = smem_desc_sw128(smem_u32(sh.stages));
  uint32_t titer = 0;
  int ring = 0;           // stage of the ring the next K block is in
  uint32_t ring_ph = 0;   // and the parity of its current fill
  for (int it = it0;; it += step, ++titer) {
    int go = it < nitems && !*sh.abort_flag;
    go = __shfl_sync(0xffffffffu, go, 0);
    if (!go) break;
    const WorkItem w = item_at(descs, items, it);
    if (!tc_issue_item(sh, tmem, desc0, descs[w.aln], titer, ring, ring_ph, limit)) break;
  }
  tc_issue_drain(sh);
}

// After every role has finished (call from all threads): when a wait ran out,
// let the loads still in flight land (bounded) before shared memory is
// released and report through err; then free tensor memory.
__device__ __forceinline__ void tc_teardown(const TcShared &sh, uint32_t tmem,
                                            uint32_t issued, int *err, int alloc_warp = 1) {
  const int tid = threadIdx.x, warp = tid >> 5;
  __syncthreads();
  // `issued` is the producer's count; the producer is thread 0 of its warp, so
  // the drain runs on the thread that knows it.
  if (issued > 0 && *sh.abort_flag) {
    const uint32_t nst = (uint32_t)sh.nst;
    for (uint32_t k = issued > nst ? issued - nst : 0; k < issued; ++k)
      mbar_wait_bounded(&sh.full_bar[k % nst], (k / nst) & 1);
  }
  if (tid == 0 && *sh.abort_flag) atomicOr(err, 1);
  __syncthreads();
  if (warp == alloc_warp) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

}  // namespace rnj
