// rnj_kernels.cu -- sm_100a kernels of the distance path.
//
//   pack_chars_kernel       alignment bytes -> bit planes (word-major, sequence fastest)
//   pack_bitstrings_kernel  the reference loader's 2-bit DNA strings -> bit planes
//   count_tiles_kernel      one 128 x 128 tile of sequence pairs per CTA: TMA-staged
//                           plane tiles, LOP3 + POPC counting in registers, fused
//                           exact transform + mirrored store + max + saturation flag
//   transform_counts_kernel the same epilogue from a count buffer (long alignments)
//   fixup_kernel            -1 -> 2 * max on the tiles that hold a saturated pair
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"

namespace rnj {

// ------------------------------------------------------------------- packing

struct Lut256 {
  uint8_t v[256];
};

// Plane words of one 32-site word of one sequence from its bytes.
//   DNA kinds: lut bit0 = code high bit, bit1 = code low bit, bit2 = valid,
//              bit3 = upper-case A/C/G/T (naive rule).
//   MISM kinds: lut = symbol rank, 0xFF = gap.
__device__ __forceinline__ void pack_word(const uint8_t *src, int cnt, int kind,
                                          const uint8_t *s_lut, uint32_t (&p)[8]) {
#pragma unroll
  for (int q = 0; q < 8; ++q) p[q] = 0;
  if (cnt <= 0) return;
  if (kind == KIND_DNA || kind == KIND_NAIVE) {
#pragma unroll 8
    for (int b = 0; b < 32; ++b) {
      const uint32_t x = (b < cnt) ? s_lut[src[b]] : 0u;
      p[0] |= (x & 1u) << b;
      p[1] |= ((x >> 1) & 1u) << b;
      p[2] |= ((x >> 2) & 1u) << b;
      p[3] |= ((x >> 3) & 1u) << b;
    }
  } else {
    const int ncode = (kind == KIND_MISM2) ? 2 : (kind == KIND_MISM5 ? 5 : 7);
#pragma unroll 8
    for (int b = 0; b < 32; ++b) {
      const uint32_t r = (b < cnt) ? s_lut[src[b]] : 0xFFu;
      if (r != 0xFFu) {
        p[ncode] |= 1u << b;
#pragma unroll
        for (int q = 0; q < 7; ++q)
          if (q < ncode) p[q] |= ((r >> q) & 1u) << b;
      }
    }
  }
}

// Bytes -> bit planes, one 32-sequence x 8-word tile per block (256 threads, one
// (sequence, word) each).  Reads: the 8 threads of a sequence cover 256
// contiguous bytes of its row.  The plane words go through shared memory so
// the stores run along the sequence axis (32 consecutive words per warp).  The
// grid covers the padded Np x Wp area, so padding rows and words come out zero.
constexpr int kPackRows = 32, kPackWords = 8;

// One 32-sequence x 8-word tile (i0, w0) of an alignment into its planes;
// s_lut holds the alignment's table.  Called by all 256 threads of a block.
__device__ __forceinline__ void pack_chars_tile(const uint8_t *__restrict__ chars, size_t ld,
                                                int n, int L, int Np, int Wp, int kind,
                                                const uint8_t *s_lut,
                                                uint32_t (*s_words)[kPackWords][kPackRows + 1],
                                                uint32_t *__restrict__ planes, int i0, int w0) {
  const int np = planes_of(kind);
  const size_t plane_stride = (size_t)Np * Wp;
  {
    const int r = threadIdx.x >> 3, ww = threadIdx.x & 7;
    const int i = i0 + r, w = w0 + ww;
    uint32_t p[8];
    const int cnt = (i < n) ? min(32, L - w * 32) : 0;
    pack_word(chars + (size_t)i * ld + (size_t)w * 32, cnt, kind, s_lut, p);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (q < np) s_words[q][ww][r] = p[q];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int pw = warp; pw < np * kPackWords; pw += 8) {
    const int q = pw / kPackWords, ww = pw % kPackWords;
    planes[q * plane_stride + (size_t)(w0 + ww) * Np + i0 + lane] = s_words[q][ww][lane];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) pack_chars_kernel(const uint8_t *__restrict__ chars,
                                                         size_t ld, int n, int L, int Np, int Wp,
                                                         int kind, Lut256 lut,
                                                         uint32_t *__restrict__ planes) {
  __shared__ uint8_t s_lut[256];
  __shared__ uint32_t s_words[8][kPackWords][kPackRows + 1];
  for (int k = threadIdx.x; k < 256; k += blockDim.x) s_lut[k] = lut.v[k];
  __syncthreads();
  const int row_tiles = Np / kPackRows, word_tiles = Wp / kPackWords;
  const long long tiles = (long long)row_tiles * word_tiles;
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    pack_chars_tile(chars, ld, n, L, Np, Wp, kind, s_lut, s_words, planes,
                    (int)(t % row_tiles) * kPackRows, (int)(t / row_tiles) * kPackWords);
}

// The job of work unit u: the last job whose first unit is <= u.
__device__ __forceinline__ int job_of(const PackJob *__restrict__ jobs, int njobs, long long u) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].unit0 <= u) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Planes of many alignments: a block per pack tile of any job (the tiles of
// job j are units jobs[j].unit0 ..), its table loaded when the job changes.
__global__ void __launch_bounds__(256) pack_chars_multi_kernel(const PackJob *__restrict__ jobs,
                                                               int njobs, long long units) {
  __shared__ uint8_t s_lut[256];
  __shared__ uint32_t s_words[8][kPackWords][kPackRows + 1];
  int cur = -1;
  for (long long t = blockIdx.x; t < units; t += gridDim.x) {
    const int j = job_of(jobs, njobs, t);
    const PackJob &jb = jobs[j];
    if (j != cur) {
      __syncthreads();
      for (int k = threadIdx.x; k < 256; k += blockDim.x) s_lut[k] = jb.lut[k];
      __syncthreads();
      cur = j;
    }
    const long long local = t - jb.unit0;
    const int row_tiles = jb.Np / kPackRows;
    pack_chars_tile(jb.chars, jb.ld, jb.n, jb.L, jb.Np, jb.W, jb.kind, s_lut, s_words,
                    (uint32_t *)jb.dst, (int)(local % row_tiles) * kPackRows,
                    (int)(local / row_tiles) * kPackWords);
  }
}

// Byte-presence mask of an alignment (bit c of the 256-bit mask set when byte
// c occurs), used to rank the residue alphabet on the host.  A warp scans row
// segments of kPresenceSeg bytes, 16 bytes a lane from 16-byte aligned blocks
// inside the row (single bytes at the row's unaligned ends, so nothing outside
// the row is read), and marks each byte in its own 256 flags in shared memory
// with a plain store of 1 (any number of lanes may mark the same byte).  The
// flags then become eight mask words, merged into the result with one atomic OR
// per word.
constexpr int kPresenceWarps = 8;  // 256 threads

__device__ __forceinline__ void mark_word(uint8_t *flags, uint32_t w) {
  flags[w & 0xFFu] = 1;
  flags[(w >> 8) & 0xFFu] = 1;
  flags[(w >> 16) & 0xFFu] = 1;
  flags[w >> 24] = 1;
}

// Marks the bytes p[0 .. len) (one warp, len >= 0).
__device__ __forceinline__ void mark_span(const uint8_t *__restrict__ p, int len, uint8_t *flags,
                                          int lane) {
  const int head = min(len, (int)((16u - (uint32_t)(reinterpret_cast<uintptr_t>(p) & 15u)) & 15u));
  if (lane < head) flags[p[lane]] = 1;
  const uint4 *v = reinterpret_cast<const uint4 *>(p + head);
  const int nv = (len - head) >> 4;
#pragma unroll 4
  for (int k = lane; k < nv; k += 32) {
    const uint4 x = __ldg(v + k);
    mark_word(flags, x.x);
    mark_word(flags, x.y);
    mark_word(flags, x.z);
    mark_word(flags, x.w);
  }
  const int tail = head + (nv << 4);
  if (lane < len - tail) flags[p[tail + lane]] = 1;
}

// The warp's flags (one byte per byte value, 0 or 1) -> atomic OR into
// mask[0 .. 8); the flags are cleared.  Lane l reads the flags of bytes 8l ..
// 8l + 7, which are bits 8(l % 4) .. 8(l % 4) + 7 of mask word l / 4.
__device__ __forceinline__ void flush_flags(uint8_t *flags, uint32_t *mask, int lane) {
  __syncwarp();
  uint2 *f2 = reinterpret_cast<uint2 *>(flags);
  const uint2 f = f2[lane];
  uint32_t lo = f.x, hi = f.y;  // a flag in bit 0 of each byte
  lo = (lo | (lo >> 7)) & 0x00030003u;
  lo = (lo | (lo >> 14)) & 0xFu;
  hi = (hi | (hi >> 7)) & 0x00030003u;
  hi = (hi | (hi >> 14)) & 0xFu;
  uint32_t v = (lo | (hi << 4)) << ((lane & 3) * 8);
  v |= __shfl_xor_sync(0xffffffffu, v, 1);
  v |= __shfl_xor_sync(0xffffffffu, v, 2);
  if ((lane & 3) == 0 && v) atomicOr(&mask[lane >> 2], v);
  f2[lane] = make_uint2(0u, 0u);
  __syncwarp();
}

__global__ void __launch_bounds__(256) presence_kernel(const uint8_t *__restrict__ chars,
                                                       size_t ld, int n, int L,
                                                       uint32_t *__restrict__ mask) {
  __shared__ __align__(16) uint8_t s_flags[kPresenceWarps][256];
  const int lane = threadIdx.x & 31;
  uint8_t *flags = s_flags[threadIdx.x >> 5];
  reinterpret_cast<uint2 *>(flags)[lane] = make_uint2(0u, 0u);
  __syncwarp();
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const int segs = (L + kPresenceSeg - 1) / kPresenceSeg;
  const long long units = (long long)n * segs;
  for (long long u = gwarp; u < units; u += nwarps) {
    const int i = (int)(u / segs), s = (int)(u % segs);
    const int k0 = s * kPresenceSeg;
    mark_span(chars + (size_t)i * ld + k0, min(L - k0, kPresenceSeg), flags, lane);
  }
  flush_flags(flags, mask, lane);
}

// Presence masks of many alignments: a warp per row segment of any job, its
// flags merged into the job's 8 words whenever the warp moves on to another job.
__global__ void __launch_bounds__(256) presence_multi_kernel(const PackJob *__restrict__ jobs,
                                                             int njobs, long long units,
                                                             uint32_t *__restrict__ masks) {
  __shared__ __align__(16) uint8_t s_flags[kPresenceWarps][256];
  const int lane = threadIdx.x & 31;
  uint8_t *flags = s_flags[threadIdx.x >> 5];
  reinterpret_cast<uint2 *>(flags)[lane] = make_uint2(0u, 0u);
  __syncwarp();
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  int cur = -1;
  for (long long u = gwarp; u < units; u += nwarps) {
    const int j = job_of(jobs, njobs, u);
    if (j != cur) {
      if (cur >= 0) flush_flags(flags, masks + 8 * cur, lane);
      cur = j;
    }
    const PackJob &jb = jobs[j];
    const int segs = (jb.L + kPresenceSeg - 1) / kPresenceSeg;
    const long long local = u - jb.unit0;
    const int i = (int)(local / segs), sg = (int)(local % segs);
    const int k0 = sg * kPresenceSeg;
    mark_span(jb.chars + (size_t)i * jb.ld + k0, min(jb.L - k0, kPresenceSeg), flags, lane);
  }
  if (cur >= 0) flush_flags(flags, masks + 8 * cur, lane);
}

__device__ __forceinline__ uint32_t compress_even_bits(uint32_t x) {
  x &= 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0f0f0f0fu;
  x = (x | (x >> 4)) & 0x00ff00ffu;
  x = (x | (x >> 8)) & 0x0000ffffu;
  return x;
}

// The reference loader's DNA layout (dataloaderFasta.hpp:147-182): 16 sites per
// uint32, site k in bits 2k..2k+1 holding A=00 G=01 T=10 C=11, and a gap filter
// with 01 in every valid slot.  Two source words make one 32-site plane word.
__global__ void pack_bitstrings_kernel(const uint32_t *__restrict__ bits,
                                       const uint32_t *__restrict__ gaps, int bs_words, int n,
                                       int L, int Np, int Wp, uint32_t *__restrict__ planes) {
  const long long total = (long long)Np * Wp;
  const size_t plane_stride = (size_t)Np * Wp;
  const int W = (L + 31) / 32;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % Np);
    const int w = (int)(t / Np);
    uint32_t hi = 0, lo = 0, v = 0;
    if (i < n && w < W) {
      const uint32_t *b = bits + (size_t)i * bs_words;
      const uint32_t *g = gaps + (size_t)i * bs_words;
      const int k0 = 2 * w, k1 = 2 * w + 1;
      const uint32_t b0 = k0 < bs_words ? b[k0] : 0u, b1 = k1 < bs_words ? b[k1] : 0u;
      const uint32_t g0 = k0 < bs_words ? g[k0] : 0u, g1 = k1 < bs_words ? g[k1] : 0u;
      lo = compress_even_bits(b0) | (compress_even_bits(b1) << 16);
      hi = compress_even_bits(b0 >> 1) | (compress_even_bits(b1 >> 1) << 16);
      v = compress_even_bits(g0) | (compress_even_bits(g1) << 16);
      const int rem = L - 32 * w;  // sites beyond L are padding: mask them out
      if (rem < 32) {
        const uint32_t m = (1u << rem) - 1u;
        hi &= m; lo &= m; v &= m;
      }
    }
    uint32_t *dst = planes + (size_t)w * Np + i;
    dst[0] = hi;
    dst[plane_stride] = lo;
    dst[2 * plane_stride] = v;
  }
}

// ------------------------------------------------------------- tile counting

template <int KIND>
struct KT;
template <>
struct KT<KIND_DNA> { static constexpr int NP = 3, NC = 3, ST = 4; };
template <>
struct KT<KIND_NAIVE> { static constexpr int NP = 4, NC = 3, ST = 4; };
template <>
struct KT<KIND_MISM2> { static constexpr int NP = 3, NC = 2, ST = 4; };
template <>
struct KT<KIND_MISM5> { static constexpr int NP = 6, NC = 2, ST = 3; };
template <>
struct KT<KIND_MISM7> { static constexpr int NP = 8, NC = 2, ST = 3; };
static_assert(8 * (4 + 1) <= 64, "the barriers of count_tiles_kernel (at most 4 + 1) fit its 64 bytes");

// Shared memory of count_tiles_kernel with an nst-stage ring: the stages,
// alignment slack, nst + 1 barriers.
template <int KIND>
constexpr size_t count_smem_bytes(int nst) {
  return (size_t)nst * 2 * KT<KIND>::NP * kKW * kTile * 4 + 1024 + 64;
}
// The ring depths count_tiles_kernel takes: at most its layout's ST, at least
// two and enough stages to hold the distance tile the EPI_DIST epilogue stages
// in the same buffers.
template <int KIND>
__host__ __device__ constexpr int count_min_stages() {
  constexpr size_t stage = 2 * (size_t)KT<KIND>::NP * kKW * kTile * 4;
  return (int)((kStageBytes + stage - 1) / stage) < 2 ? 2 : (int)((kStageBytes + stage - 1) / stage);
}
template <int KIND>
__host__ __device__ constexpr int count_stages(int requested) {
  return requested <= 0 ? KT<KIND>::ST
                        : (requested < count_min_stages<KIND>()
                               ? count_min_stages<KIND>()
                               : (requested > KT<KIND>::ST ? KT<KIND>::ST : requested));
}

template <int KIND>
__device__ __forceinline__ void pair_op(const uint32_t (&a)[KT<KIND>::NP],
                                        const uint32_t (&b)[KT<KIND>::NP], uint32_t &acc0,
                                        uint32_t &acc1) {
  if constexpr (KIND == KIND_DNA) {
    // bitDistanceGap.cpp:146-161: tv = high bit of the code XOR, ts = low bit and
    // not tv, both masked by the shared valid sites.
    const uint32_t v = a[2] & b[2];
    const uint32_t tv = (a[0] ^ b[0]) & v;
    const uint32_t ts = (a[1] ^ b[1]) & (v & ~tv);
    acc0 += __popc(ts) + (__popc(tv) << 16);
    acc1 += __popc(v);
  } else if constexpr (KIND == KIND_NAIVE) {
    // simpleDistanceCalculator.cpp:58-98 over planes: only an upper-case A/C/G/T
    // in the row sequence classifies a difference.
    const uint32_t v = a[2] & b[2];
    const uint32_t xh = a[0] ^ b[0], xl = a[1] ^ b[1];
    const uint32_t ts = a[3] & b[3] & ~xh & xl;
    const uint32_t tv = a[3] & b[2] & (~b[3] | xh);
    acc0 += __popc(ts) + (__popc(tv) << 16);
    acc1 += __popc(v);
  } else {
    // bitDistanceProtein.cpp:77-81: a site differs when any code bit differs;
    // sites with a gap in either sequence are excluded.
    constexpr int P = KT<KIND>::NP - 1;
    uint32_t x = a[0] ^ b[0];
#pragma unroll
    for (int q = 1; q < P; ++q) x |= a[q] ^ b[q];
    const uint32_t v = a[P] & b[P];
    acc0 += __popc(x & v) + (__popc(v) << 16);
  }
}

template <int KIND, int EPI>
__global__ void __launch_bounds__(256, 1)
    count_tiles_kernel(const __grid_constant__ CUtensorMap tmap, int nt, int nk, int kchunk,
                       EpiParams ep) {
  using T = KT<KIND>;
  constexpr int NP = T::NP, NC = T::NC;
  constexpr int TILE_WORDS = NP * kKW * kTile;
  constexpr uint32_t STAGE_BYTES = 2u * TILE_WORDS * 4u;
  static_assert((size_t)count_min_stages<KIND>() * STAGE_BYTES >= kStageBytes,
                "distance tile must fit the stage buffers");
  // ring depth: count_stages() of the launch (the launcher sets ep.stages)
  const int ST = ep.stages;

  extern __shared__ uint8_t smem_raw[];
  uint32_t *smem =
      reinterpret_cast<uint32_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full_bar = reinterpret_cast<uint64_t *>(smem + ST * 2 * TILE_WORDS);

  int ti, tj;
  const int tile_id = ep.tile0 + (int)blockIdx.x;
  if (ep.full) {
    ti = tile_id / nt;
    tj = tile_id % nt;
  } else {
    tri_coords(tile_id, nt, ti, tj);
  }
  const int kc0 = blockIdx.y * kchunk;
  const int nks = min(nk, kc0 + kchunk) - kc0;

  const int tid = threadIdx.x;
  // full_bar[ST]: a barrier that nothing completes, waited on only by the test
  // of the failure path (ep.stall).
  if (tid == 0) {
    for (int s = 0; s <= ST; ++s) mbar_init(&full_bar[s], 1);
    fence_mbar_init();
    prefetch_tmap(&tmap);
  }
  __syncthreads();
  const uint64_t limit = wait_limit_ns(ep.wait_us);

  auto issue = [&](int k) {
    const int s = k % ST;
    uint32_t *a = smem + s * 2 * TILE_WORDS;
    mbar_arrive_expect_tx(&full_bar[s], STAGE_BYTES);
    tma_load_3d(a, &tmap, &full_bar[s], ti * kTile, (kc0 + k) * kKW, 0);
    tma_load_3d(a + TILE_WORDS, &tmap, &full_bar[s], tj * kTile, (kc0 + k) * kKW, 0);
  };
  int issued = 0;
  if (tid == 0) {
    for (; issued < ST - 1 && issued < nks; ++issued) issue(issued);
  }

  const int warp = tid >> 5, lane = tid & 31;
  const int rbase = (warp >> 1) * 32 + (lane >> 3) * 4;
  const int cbase = (warp & 1) * 64 + (lane & 7) * 4;

  uint32_t acc0[8][8], acc1[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      acc0[r][c] = 0;
      acc1[r][c] = 0;
    }

  int kabort = -1;
  for (int k = 0; k < nks; ++k) {
    if (tid == 0 && issued < nks) issue(issued++);
    const int s = k % ST;
    bool ok = !(ep.stall && k == 0) || mbar_wait_bounded(&full_bar[ST], 0, limit);
    if (ok) ok = mbar_wait_bounded(&full_bar[s], (uint32_t)((k / ST) & 1), limit);
    if (ok) {
      const uint32_t *A = smem + s * 2 * TILE_WORDS;
      const uint32_t *B = A + TILE_WORDS;
#pragma unroll 2
      for (int kw = 0; kw < kKW; ++kw) {
        uint32_t bc[8][NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const uint4 x0 = *reinterpret_cast<const uint4 *>(B + (p * kKW + kw) * kTile + cbase);
          const uint4 x1 = *reinterpret_cast<const uint4 *>(B + (p * kKW + kw) * kTile + cbase + 32);
          bc[0][p] = x0.x; bc[1][p] = x0.y; bc[2][p] = x0.z; bc[3][p] = x0.w;
          bc[4][p] = x1.x; bc[5][p] = x1.y; bc[6][p] = x1.z; bc[7][p] = x1.w;
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          uint32_t ar[NP];
          const int row = row_of(rbase, r);
#pragma unroll
          for (int p = 0; p < NP; ++p) ar[p] = A[(p * kKW + kw) * kTile + row];
#pragma unroll
          for (int c = 0; c < 8; ++c) pair_op<KIND>(ar, bc[c], acc0[r][c], acc1[r][c]);
        }
      }
    }
    if (__syncthreads_or(!ok)) {
      kabort = k;
      break;
    }
  }
  if (kabort >= 0) {
    // Let the copies still in flight land before the CTA's shared memory is
    // released, each wait again bounded, then report.
    if (tid == 0) {
      for (int k = kabort; k < issued; ++k)
        mbar_wait_bounded(&full_bar[k % ST], (uint32_t)((k / ST) & 1));
      atomicOr(ep.err, 1);
    }
    return;
  }

  // Per-pair counts from the 16-bit halves of the accumulators.
  auto get = [&](int r, int c, uint32_t &c0, uint32_t &c1, uint32_t &cv) {
    c0 = acc0[r][c] & 0xffffu;
    if constexpr (NC == 3) {
      c1 = acc0[r][c] >> 16;
      cv = acc1[r][c];
    } else {
      c1 = 0;
      cv = acc0[r][c] >> 16;
    }
  };

  if constexpr (EPI == EPI_DIST) {
    // The pipeline buffers are free once every thread is past the last stage
    // (the loop ends on a block barrier); reuse them for the distance tile.
    float *S = reinterpret_cast<float *>(smem);
    float tmax = 0.0f;
    bool sat = false;
    stage_distances(ep, ti, tj, rbase, cbase, S, get, tmax, sat);
    __syncthreads();
    store_distances(ep, ti, tj, tile_id, S, tmax, sat, threadIdx.x >> 5, blockDim.x >> 5);
  } else {
    const int i0 = ti * kTile, j0 = tj * kTile;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + row_of(rbase, r);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int j = j0 + col_of(cbase, c);
        const bool ok = ep.full ? (i < ep.n && j < ep.n) : (i < j && j < ep.n);
        if (!ok) continue;
        uint32_t c0, c1, cv;
        get(r, c, c0, c1, cv);
        uint32_t *o = ep.counts + ((size_t)i * ep.n + j) * 3;
        if constexpr (EPI == EPI_COUNTS) {
          o[0] = c0;
          o[1] = c1;
          o[2] = cv;
        } else {
          atomicAdd(o + 0, c0);
          if (NC == 3) atomicAdd(o + 1, c1);
          atomicAdd(o + 2, cv);
        }
      }
    }
  }
}

// Epilogue over an already complete count buffer (split-K path).
__global__ void __launch_bounds__(256) transform_counts_kernel(int nt, EpiParams ep) {
  extern __shared__ uint8_t smem_raw[];
  float *S = reinterpret_cast<float *>(smem_raw);
  int ti, tj;
  const int tile_id = ep.tile0 + (int)blockIdx.x;
  if (ep.full) {
    ti = tile_id / nt;
    tj = tile_id % nt;
  } else {
    tri_coords(tile_id, nt, ti, tj);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rbase = (warp >> 1) * 32 + (lane >> 3) * 4;
  const int cbase = (warp & 1) * 64 + (lane & 7) * 4;
  const int i0 = ti * kTile, j0 = tj * kTile;
  auto get = [&](int r, int c, uint32_t &c0, uint32_t &c1, uint32_t &cv) {
    const int i = i0 + row_of(rbase, r), j = j0 + col_of(cbase, c);
    const uint32_t *o = ep.counts + ((size_t)i * ep.n + j) * 3;
    c0 = o[0];
    c1 = o[1];
    cv = o[2];
  };
  float tmax = 0.0f;
  bool sat = false;
  stage_distances(ep, ti, tj, rbase, cbase, S, get, tmax, sat);
  __syncthreads();
  store_distances(ep, ti, tj, tile_id, S, tmax, sat, threadIdx.x >> 5, blockDim.x >> 5);
}

// KimuraDistance.cpp:384-386 / JCdistance.cpp:219-221: every -1 becomes
// maxDistance * 2, once the global maximum is known.  Only tiles flagged by the
// epilogue are visited, each by `slices` blocks (a share of its rows each): one
// block per tile when tiles are many (most blocks find no flag and end at
// once; grouping tiles per block serialises the flagged ones and measured
// slower), several when they are few.
__global__ void __launch_bounds__(256, 8) fixup_kernel(int nt, EpiParams ep, int slices) {
  const int tile_id = blockIdx.x / slices, slice = blockIdx.x % slices;
  if (ep.tile_flags[tile_id] == 0) return;
  int ti, tj;
  if (ep.full) {
    ti = tile_id / nt;
    tj = tile_id % nt;
  } else {
    tri_coords(tile_id, nt, ti, tj);
  }
  const float m2 = __fmul_rn(__int_as_float(*ep.max_bits), 2.0f);
  fixup_tile_at<4>(ep.out, ep.ld, ep.n, 0, ep.full != 0, ti, tj, m2, threadIdx.x, blockDim.x,
                   slice, slices);
}

// ------------------------------------------------------- batched popcount path
//
// Persistent over a work list of (alignment, tile) items of any plane layout:
// thread 0 takes the next item with an atomic counter (the list is ordered by
// decreasing cost), the CTA dispatches on the item's kind and runs the same
// TMA-staged counting and epilogue as count_tiles_kernel.  The stage ring is
// sized for the widest layout (8 planes) and its phase counter runs on across
// items.

constexpr int kBatchST = 3;
constexpr uint32_t kBatchStageBytes = 2u * 8 * kKW * kTile * 4;  // 64 KB
constexpr size_t kBatchSmem = (size_t)kBatchST * kBatchStageBytes + 1024 + 64;

__device__ __forceinline__ void tensormap_acquire_pc(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

// One tile of one alignment; returns false (uniformly across the CTA) when a
// bounded wait ran out.  gk: stages consumed so far by this CTA.
template <int KIND, int EPI>
__device__ __forceinline__ bool batch_tile(const AlnDesc &d, int tile, uint32_t *smem,
                                           uint64_t *full_bar, uint32_t &gk) {
  using T = KT<KIND>;
  constexpr int NP = T::NP, NC = T::NC;
  constexpr int TILE_WORDS = NP * kKW * kTile;
  constexpr uint32_t STAGE_BYTES = 2u * TILE_WORDS * 4u;
  constexpr int RING_WORDS = kBatchStageBytes / 4;
  const int tid = threadIdx.x;
  int ti, tj;
  if (d.full) {
    ti = tile / d.nt;
    tj = tile % d.nt;
  } else {
    tri_coords(tile, d.nt, ti, tj);
  }
  const int nks = d.kdim / kKW;
  auto issue = [&](int k) {
    const uint32_t g = gk + (uint32_t)k;
    const int s = g % kBatchST;
    uint32_t *a = smem + s * RING_WORDS;
    mbar_arrive_expect_tx(&full_bar[s], STAGE_BYTES);
    tma_load_3d(a, &d.map, &full_bar[s], ti * kTile, k * kKW, 0);
    tma_load_3d(a + TILE_WORDS, &d.map, &full_bar[s], tj * kTile, k * kKW, 0);
  };
  int issued = 0;
  if (tid == 0) {
    tensormap_acquire_pc(&d.map);
    for (; issued < kBatchST - 1 && issued < nks; ++issued) issue(issued);
  }
  const int warp = tid >> 5, lane = tid & 31;
  const int rbase = (warp >> 1) * 32 + (lane >> 3) * 4;
  const int cbase = (warp & 1) * 64 + (lane & 7) * 4;
  uint32_t acc0[8][8], acc1[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      acc0[r][c] = 0;
      acc1[r][c] = 0;
    }
  int kabort = -1;
  for (int k = 0; k < nks; ++k) {
    if (tid == 0 && issued < nks) issue(issued++);
    const uint32_t g = gk + (uint32_t)k;
    const int s = g % kBatchST;
    const bool ok = mbar_wait_bounded(&full_bar[s], (g / kBatchST) & 1, wait_limit_ns(d.wait_us));
    if (ok) {
      const uint32_t *A = smem + s * RING_WORDS;
      const uint32_t *B = A + TILE_WORDS;
#pragma unroll 2
      for (int kw = 0; kw < kKW; ++kw) {
        uint32_t bc[8][NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const uint4 x0 = *reinterpret_cast<const uint4 *>(B + (p * kKW + kw) * kTile + cbase);
          const uint4 x1 = *reinterpret_cast<const uint4 *>(B + (p * kKW + kw) * kTile + cbase + 32);
          bc[0][p] = x0.x; bc[1][p] = x0.y; bc[2][p] = x0.z; bc[3][p] = x0.w;
          bc[4][p] = x1.x; bc[5][p] = x1.y; bc[6][p] = x1.z; bc[7][p] = x1.w;
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          uint32_t ar[NP];
          const int row = row_of(rbase, r);
#pragma unroll
          for (int p = 0; p < NP; ++p) ar[p] = A[(p * kKW + kw) * kTile + row];
#pragma unroll
          for (int c = 0; c < 8; ++c) pair_op<KIND>(ar, bc[c], acc0[r][c], acc1[r][c]);
        }
      }
    }
    if (__syncthreads_or(!ok)) {
      kabort = k;
      break;
    }
  }
  if (kabort >= 0) {
    if (tid == 0)
      for (int k = kabort; k < issued; ++k) {
        const uint32_t g = gk + (uint32_t)k;
        mbar_wait_bounded(&full_bar[g % kBatchST], (g / kBatchST) & 1);
      }
    return false;
  }
  gk += (uint32_t)nks;

  auto get = [&](int r, int c, uint32_t &c0, uint32_t &c1, uint32_t &cv) {
    c0 = acc0[r][c] & 0xffffu;
    if constexpr (NC == 3) {
      c1 = acc0[r][c] >> 16;
      cv = acc1[r][c];
    } else {
      c1 = 0;
      cv = acc0[r][c] >> 16;
    }
  };
  EpiParams ep;
  ep.n = d.n;
  ep.L = d.L;
  ep.model = d.model;
  ep.type = d.type;
  ep.compat_wrap = d.compat;
  ep.full = d.full;
  ep.jc_b = d.jc_b;
  ep.out = d.out;
  ep.ld = (size_t)d.ld;
  ep.max_bits = d.max_bits;
  ep.tile_flags = d.tile_flags;
  ep.counts = d.counts;
  ep.err = d.err;
  if constexpr (EPI == EPI_DIST) {
    float *S = reinterpret_cast<float *>(smem);
    float tmax = 0.0f;
    bool sat = false;
    stage_distances(ep, ti, tj, rbase, cbase, S, get, tmax, sat);
    __syncthreads();
    store_distances(ep, ti, tj, tile, S, tmax, sat, threadIdx.x >> 5, blockDim.x >> 5);
  } else {
    const int i0 = ti * kTile, j0 = tj * kTile;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + row_of(rbase, r);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int j = j0 + col_of(cbase, c);
        const bool ok = ep.full ? (i < ep.n && j < ep.n) : (i < j && j < ep.n);
        if (!ok) continue;
        uint32_t c0, c1, cv;
        get(r, c, c0, c1, cv);
        uint32_t *o = ep.counts + ((size_t)i * ep.n + j) * 3;
        o[0] = c0;
        o[1] = c1;
        o[2] = cv;
      }
    }
  }
  // The next item's loads reuse the shared memory the epilogue just read.
  __syncthreads();
  return true;
}

template <int EPI>
__global__ void __launch_bounds__(256, 1)
    count_batch_kernel(const AlnDesc *__restrict__ descs, const WorkItem *__restrict__ items,
                       const int *__restrict__ nitems_ptr, int *__restrict__ counter) {
  extern __shared__ uint8_t smem_raw[];
  uint32_t *smem =
      reinterpret_cast<uint32_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full_bar = reinterpret_cast<uint64_t *>(smem + kBatchST * (kBatchStageBytes / 4));
  __shared__ int s_item;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kBatchST; ++s) mbar_init(&full_bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const int nitems = *nitems_ptr;
  uint32_t gk = 0;
  while (true) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const AlnDesc &d = descs[w.aln];
    bool ok = true;
    switch (d.kind) {
      case KIND_DNA: ok = batch_tile<KIND_DNA, EPI>(d, w.tile, smem, full_bar, gk); break;
      case KIND_NAIVE: ok = batch_tile<KIND_NAIVE, EPI>(d, w.tile, smem, full_bar, gk); break;
      case KIND_MISM2: ok = batch_tile<KIND_MISM2, EPI>(d, w.tile, smem, full_bar, gk); break;
      case KIND_MISM5: ok = batch_tile<KIND_MISM5, EPI>(d, w.tile, smem, full_bar, gk); break;
      case KIND_MISM7: ok = batch_tile<KIND_MISM7, EPI>(d, w.tile, smem, full_bar, gk); break;
      default: break;
    }
    if (!ok) {
      if (tid == 0) atomicOr(d.err, 1);
      break;
    }
  }
}

// Saturation fix-up over every item of a batch whose tile holds a -1.
__global__ void __launch_bounds__(256) fixup_batch_kernel(const AlnDesc *__restrict__ descs,
                                                          const WorkItem *__restrict__ items_a,
                                                          const int *__restrict__ n_a,
                                                          const WorkItem *__restrict__ items_b,
                                                          const int *__restrict__ n_b) {
  const int na = *n_a, nb = *n_b;
  for (int it = blockIdx.x; it < na + nb; it += gridDim.x) {
    const WorkItem w = it < na ? items_a[it] : items_b[it - na];
    const AlnDesc &d = descs[w.aln];
    if (d.out == nullptr || d.tile_flags[w.tile] == 0) continue;
    fixup_tile<4>(d, w.tile, __fmul_rn(__int_as_float(*d.max_bits), 2.0f), threadIdx.x, blockDim.x);
  }
}

cudaError_t launch_count_batch(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                               int *d_counter, int grid, int epi_mode, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  cudaError_t e;
  if (epi_mode == EPI_DIST) {
    e = cudaFuncSetAttribute(count_batch_kernel<EPI_DIST>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem);
    if (e != cudaSuccess) return e;
    count_batch_kernel<EPI_DIST><<<grid, 256, kBatchSmem, s>>>(d_descs, d_items, d_nitems, d_counter);
  } else {
    e = cudaFuncSetAttribute(count_batch_kernel<EPI_COUNTS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem);
    if (e != cudaSuccess) return e;
    count_batch_kernel<EPI_COUNTS><<<grid, 256, kBatchSmem, s>>>(d_descs, d_items, d_nitems,
                                                                 d_counter);
  }
  return cudaGetLastError();
}

cudaError_t launch_fixup_batch(const AlnDesc *d_descs, const WorkItem *items_a, const int *n_a,
                               const WorkItem *items_b, const int *n_b, int grid, cudaStream_t s) {
  fixup_batch_kernel<<<grid, 256, 0, s>>>(d_descs, items_a, n_a, items_b, n_b);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers

static int grid_for(long long work, int block) {
  long long g = (work + block - 1) / block;
  if (g > 148LL * 64) g = 148LL * 64;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_pack_chars(const uint8_t *d_chars, size_t ld, const Packed &p,
                              const uint8_t lut[256], cudaStream_t s) {
  Lut256 l;
  for (int k = 0; k < 256; ++k) l.v[k] = lut[k];
  const long long work = (long long)p.Np * p.Wp;
  pack_chars_kernel<<<grid_for(work, 256), 256, 0, s>>>(d_chars, ld, p.n, p.L, p.Np, p.Wp,
                                                        p.kind, l, p.planes);
  return cudaGetLastError();
}

cudaError_t launch_presence(const uint8_t *d_chars, size_t ld, int n, int L, uint32_t *d_mask,
                            cudaStream_t s) {
  const long long units = (long long)n * ((L + kPresenceSeg - 1) / kPresenceSeg);  // a warp each
  presence_kernel<<<grid_for(units * 32, 256), 256, 0, s>>>(d_chars, ld, n, L, d_mask);
  return cudaGetLastError();
}

cudaError_t launch_presence_multi(const PackJob *d_jobs, int njobs, long long units,
                                  uint32_t *d_masks, cudaStream_t s) {
  if (njobs <= 0 || units <= 0) return cudaSuccess;
  presence_multi_kernel<<<grid_for(units * 32, 256), 256, 0, s>>>(d_jobs, njobs, units, d_masks);
  return cudaGetLastError();
}

cudaError_t launch_pack_chars_multi(const PackJob *d_jobs, int njobs, long long units,
                                    cudaStream_t s) {
  if (njobs <= 0 || units <= 0) return cudaSuccess;
  const long long g = std::min<long long>(units, 148LL * 16);
  pack_chars_multi_kernel<<<(unsigned)g, 256, 0, s>>>(d_jobs, njobs, units);
  return cudaGetLastError();
}

cudaError_t launch_pack_bitstrings_dna(const uint32_t *d_bits, const uint32_t *d_gaps,
                                       int bs_words, const Packed &p, cudaStream_t s) {
  const long long work = (long long)p.Np * p.Wp;
  pack_bitstrings_kernel<<<grid_for(work, 256), 256, 0, s>>>(d_bits, d_gaps, bs_words, p.n, p.L,
                                                             p.Np, p.Wp, p.planes);
  return cudaGetLastError();
}

template <int KIND, int EPI>
static cudaError_t launch_one(const Packed &p, const EpiParams &ep, dim3 grid, int nt, int nk,
                              int kchunk, cudaStream_t s) {
  EpiParams e1 = ep;
  e1.stages = count_stages<KIND>(ep.stages);
  const size_t smem = count_smem_bytes<KIND>(e1.stages);
  cudaError_t e = cudaFuncSetAttribute(count_tiles_kernel<KIND, EPI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  count_tiles_kernel<KIND, EPI><<<grid, 256, smem, s>>>(p.tmap, nt, nk, kchunk, e1);
  return cudaGetLastError();
}

template <int EPI>
static cudaError_t launch_kind(int kind, const Packed &p, const EpiParams &ep, dim3 grid, int nt,
                               int nk, int kchunk, cudaStream_t s) {
  switch (kind) {
    case KIND_DNA: return launch_one<KIND_DNA, EPI>(p, ep, grid, nt, nk, kchunk, s);
    case KIND_NAIVE: return launch_one<KIND_NAIVE, EPI>(p, ep, grid, nt, nk, kchunk, s);
    case KIND_MISM2: return launch_one<KIND_MISM2, EPI>(p, ep, grid, nt, nk, kchunk, s);
    case KIND_MISM5: return launch_one<KIND_MISM5, EPI>(p, ep, grid, nt, nk, kchunk, s);
    case KIND_MISM7: return launch_one<KIND_MISM7, EPI>(p, ep, grid, nt, nk, kchunk, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t preload_bitplane_kernels() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, pack_chars_kernel);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, presence_kernel);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, fixup_kernel);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, count_tiles_kernel<KIND_DNA, EPI_DIST>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, count_tiles_kernel<KIND_NAIVE, EPI_DIST>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, count_tiles_kernel<KIND_MISM2, EPI_DIST>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, count_tiles_kernel<KIND_MISM5, EPI_DIST>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, count_tiles_kernel<KIND_MISM7, EPI_DIST>);
  return e;
}

cudaError_t launch_count_tiles(const Packed &p, int count_kind, int epi_mode, const EpiParams &ep,
                               cudaStream_t s, int kchunk_words, long long band_tiles) {
  const int nt = tiles_of(p.n);
  const long long all_tiles = ep.full ? (long long)nt * nt : tri_tiles(nt);
  if (band_tiles > 0 && (epi_mode != EPI_DIST || ep.tile0 < 0 || ep.tile0 + band_tiles > all_tiles))
    return cudaErrorInvalidValue;
  const long long ntiles = band_tiles > 0 ? band_tiles : all_tiles;
  if (ntiles == 0) return cudaSuccess;
  const int nk = p.Wp / kKW;
  const int kmax = kMaxFusedWords / kKW;
  int kchunk = (epi_mode == EPI_ATOMIC) ? kmax : nk;
  if (epi_mode == EPI_ATOMIC && kchunk_words > 0)
    kchunk = std::max(1, std::min(kmax, kchunk_words / kKW));
  const int nsplit = (nk + kchunk - 1) / kchunk;
  dim3 grid((unsigned)ntiles, (unsigned)nsplit);
  switch (epi_mode) {
    case EPI_DIST: return launch_kind<EPI_DIST>(count_kind, p, ep, grid, nt, nk, kchunk, s);
    case EPI_COUNTS: return launch_kind<EPI_COUNTS>(count_kind, p, ep, grid, nt, nk, kchunk, s);
    default: return launch_kind<EPI_ATOMIC>(count_kind, p, ep, grid, nt, nk, kchunk, s);
  }
}

cudaError_t launch_fixup(const EpiParams &ep, int nt, cudaStream_t s) {
  const long long ntiles = ep.full ? (long long)nt * nt : tri_tiles(nt);
  if (ntiles == 0) return cudaSuccess;
  const int slices = ntiles <= 148 ? 16 : (ntiles <= 592 ? 4 : 1);
  fixup_kernel<<<(unsigned)(ntiles * slices), 256, 0, s>>>(nt, ep, slices);
  return cudaGetLastError();
}

cudaError_t launch_transform_counts(const EpiParams &ep, int nt, cudaStream_t s) {
  const long long ntiles = ep.full ? (long long)nt * nt : tri_tiles(nt);
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(transform_counts_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageBytes);
  if (e != cudaSuccess) return e;
  transform_counts_kernel<<<(unsigned)ntiles, 256, kStageBytes, s>>>(nt, ep);
  return cudaGetLastError();
}

}  // namespace rnj
