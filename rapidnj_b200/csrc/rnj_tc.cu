// rnj_tc.cu -- DNA pair counting on the 5th-generation tensor cores (tcgen05).
//
// Encoding.  Every valid site of a sequence becomes four features (v, r, t, u)
// in {-1, 0, +1}: v = 1; r = +1 for a purine (A, G), -1 for a pyrimidine (C, T);
// t = +1 for A and C, -1 for G and T; u = r * t.  A gap is (0, 0, 0, 0).  For
// two sites of a pair the products satisfy
//   identical:     vv' = 1, rr' = 1, tt' + uu' =  2
//   transition:    vv' = 1, rr' = 1, tt' + uu' = -2     (A<->G, C<->T)
//   transversion:  vv' = 1, rr' = -1, tt' + uu' = 0
// so with V = sum vv', R = sum rr', T = sum (tt' + uu') over the columns:
//   valid = V,   transitions = (V + R - T) / 4,   transversions = (V - R) / 2,
// exactly (integers), which are the counts bitDistanceGap.cpp:146-161 produces.
// The three sums are three Gram matrices of the feature matrix F (n x 4L): the
// v block (K = L), the r block (K = L) and the t|u block (K = 2L): 4 MACs per
// pair-column.
//
// Number format.  The features are stored as FP4 (e2m1: +1 = 0x2, -1 = 0xA,
// 0 = 0x0), two per byte, and multiplied by tcgen05.mma.kind::mxf4 with every
// block scale factor 1.0 (UE8M0 127) into f32 accumulators.  Every product is
// -1, 0 or +1 and every partial sum an integer of magnitude <= 2L < 2^24, so
// the f32 sums are exact and convert to the integer counts without rounding.
// FP4 halves the operand bytes per MAC of an 8-bit encoding, and the FP4
// tensor rate is twice the 8-bit one.
//
// Kernel.  Persistent, one CTA per SM, over a work list of 128 x 128 triangle
// tiles (of one alignment, or of many in a batch), 320 threads:
//   warp 0       TMA producer: 128-row x 128-byte (256-column) K-blocks of both
//                row tiles (one contiguous 16 KB run each in the K-blocked
//                layout), 128-byte swizzle, into a 7-stage mbarrier ring
//   warp 1       TMEM owner and MMA issuer: M = N = 128, K = 64 per instruction,
//                three accumulators (V, R, T) of 128 columns each, the scale
//                factors in the last 128 columns; tcgen05.commit releases
//                stages and signals the end of a tile
//   warps 2..9   epilogue: per 32-column chunk, tcgen05.ld of the accumulators,
//                the exact transform and the stores (tile rows as float4, the
//                mirror image with warp-coalesced column stores); then TMEM is
//                handed back to the MMA warp
// Every wait is bounded; on a timeout the CTA records an error, drains what it
// issued, frees its tensor memory and ends.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"
#include "rnj_tcgen05.cuh"

namespace rnj {

// A 256-byte table passed by value to a kernel.
struct Lut8 {
  uint8_t v[256];
};

// --------------------------------------------------------------- feature pack

// FP4 (e2m1) codes of the feature values: +1 = 0x2, -1 = 0xA (sign bit 3), 0 = 0.
__device__ __forceinline__ uint32_t fp4_of(int x) { return x > 0 ? 0x2u : (x < 0 ? 0xAu : 0u); }

// The 32 features of feature block f (0 v, 1 r, 2 t, 3 u) of sequence i,
// columns 32c .. 32c+31 (16 bytes, two per byte, column 32c + k in nibble k of
// the 128-bit word), in the K-blocked layout (see Packed::feat).
__device__ __forceinline__ uint4 *feat_chunk(uint8_t *F, int Np, int Lk, int f, int i, int c) {
  const size_t kb = (size_t)f * (Lk / 256) + (c >> 3);
  return reinterpret_cast<uint4 *>(F + (kb * Np + i) * 128 + (c & 7) * 16);
}

// Accumulates one site's features (k = 0..31 within the chunk).  code: A=0 G=1
// T=2 C=3 (stdinclude.h:25), or -1 for a gap.
__device__ __forceinline__ void add_site(int k, int code, uint32_t (&v)[4], uint32_t (&r)[4],
                                         uint32_t (&t)[4], uint32_t (&u)[4]) {
  if (code < 0) return;
  const int rr = (code < 2) ? 1 : -1;                 // purine A, G
  const int ts = (code == 0 || code == 3) ? 1 : -1;  // A, C
  const int w = k >> 3, sh = (k & 7) * 4;
  v[w] |= fp4_of(1) << sh;
  r[w] |= fp4_of(rr) << sh;
  t[w] |= fp4_of(ts) << sh;
  u[w] |= fp4_of(rr * ts) << sh;
}

__device__ __forceinline__ void store_chunk(uint8_t *F, int Np, int Lk, int i, int c,
                                            const uint32_t (&v)[4], const uint32_t (&r)[4],
                                            const uint32_t (&t)[4], const uint32_t (&u)[4]) {
  *feat_chunk(F, Np, Lk, 0, i, c) = make_uint4(v[0], v[1], v[2], v[3]);
  *feat_chunk(F, Np, Lk, 1, i, c) = make_uint4(r[0], r[1], r[2], r[3]);
  *feat_chunk(F, Np, Lk, 2, i, c) = make_uint4(t[0], t[1], t[2], t[3]);
  *feat_chunk(F, Np, Lk, 3, i, c) = make_uint4(u[0], u[1], u[2], u[3]);
}

// chars (n rows, stride ld) -> F (Np rows of 4 * Lk FP4 features [v | r | t | u],
// K-blocked), rows row0 .. row0 + rows - 1 of F; padding rows and columns are
// zero.  One thread per (sequence, 32-column chunk); writes 4 x 16 bytes.
// Valid sites are A/C/G/T in either case (dataloaderFasta.hpp:155-180).  A
// 256-entry table in shared memory maps each byte to its four FP4 codes
// (v | r << 4 | t << 8 | u << 12).
// The 256-entry byte -> FP4 codes table (v | r << 4 | t << 8 | u << 12) in
// shared memory; thread k fills entry k (256 threads).
__device__ __forceinline__ void fill_feature_lut(uint16_t *lut) {
  const int ch = threadIdx.x;
  int code = -1;
  switch (ch) {
    case 'A': case 'a': code = 0; break;
    case 'G': case 'g': code = 1; break;
    case 'T': case 't': code = 2; break;
    case 'C': case 'c': code = 3; break;
    default: break;
  }
  uint32_t v[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0}, t[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
  add_site(0, code, v, r, t, u);
  lut[ch] = (uint16_t)(v[0] | (r[0] << 4) | (t[0] << 8) | (u[0] << 12));
}

// The 32 bytes of columns 32c .. 32c + 31 of a row as 8 little-endian words;
// returns how many of them are the row's (0 .. 32; the rest are zero).  Each
// 16-byte aligned block that lies inside the row is read with one 16-byte load,
// a block that straddles an end of the row byte by byte within the chunk, and a
// funnel shift brings the chunk's bytes to the start: nothing outside the row is
// read, whatever the row's alignment (rows of stride L are rarely 16-byte
// aligned).
__device__ __forceinline__ int load_chunk(const uint8_t *__restrict__ row, int L, int c,
                                          uint32_t (&q)[8]) {
  const int len = min(32, L - 32 * c);
  if (len <= 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) q[k] = 0u;
    return 0;
  }
  const uintptr_t lo = reinterpret_cast<uintptr_t>(row), hi = lo + (uintptr_t)L;
  const uintptr_t s = lo + (uintptr_t)c * 32u, e = s + (uintptr_t)len;
  const int o = (int)(s & 15u);
  if (o == 0 && len == 32) {
    const uint4 x = __ldg(reinterpret_cast<const uint4 *>(s));
    const uint4 y = __ldg(reinterpret_cast<const uint4 *>(s) + 1);
    q[0] = x.x, q[1] = x.y, q[2] = x.z, q[3] = x.w;
    q[4] = y.x, q[5] = y.y, q[6] = y.z, q[7] = y.w;
    return 32;
  }
  uint32_t w[12];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const uintptr_t blk = s - (uintptr_t)o + 16u * b;
    uint32_t x[4] = {0u, 0u, 0u, 0u};
    if (blk >= lo && blk + 16u <= hi) {
      const uint4 v = __ldg(reinterpret_cast<const uint4 *>(blk));
      x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
    } else if (blk < e) {
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const uintptr_t p = blk + (uintptr_t)m;
        if (p >= s && p < e)
          x[m >> 2] |= (uint32_t)(*reinterpret_cast<const uint8_t *>(p)) << (8 * (m & 3));
      }
    }
    w[4 * b] = x[0], w[4 * b + 1] = x[1], w[4 * b + 2] = x[2], w[4 * b + 3] = x[3];
  }
  // bytes o .. o + 31 of the 48-byte window: whole words first, then the bytes
  const int ow = o >> 2;
  uint32_t u[10], v[9];
#pragma unroll
  for (int k = 0; k < 10; ++k) u[k] = (ow & 2) ? w[k + 2] : w[k];
#pragma unroll
  for (int k = 0; k < 9; ++k) v[k] = (ow & 1) ? u[k + 1] : u[k];
  const uint32_t sh = 8u * (uint32_t)(o & 3);
#pragma unroll
  for (int k = 0; k < 8; ++k) q[k] = __funnelshift_r(v[k], v[k + 1], sh);
  return len;
}

// Row i, 32-column chunk c of the features (zeros for padding rows/columns).
// The table gives each byte its four FP4 codes as two bytes, v | r << 4 and
// t | u << 4 (byte 0, which pads a chunk past the row's end, has none).  Per 8
// sites, byte permutes gather the codes of the even sites and of the odd sites
// into words, whose nibbles interleave into the four feature words.
__device__ __forceinline__ void pack_feature_chunk(const uint8_t *__restrict__ chars, size_t ld,
                                                   int n, int L, int Np, int Lk, int i, int c,
                                                   const uint16_t *lut, uint8_t *__restrict__ F) {
  uint32_t q[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  if (i < n) load_chunk(chars + (size_t)i * ld, L, c, q);
  uint32_t v[4], r[4], tt[4], u[4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const uint32_t a = q[2 * g], b = q[2 * g + 1];
    const uint32_t e0 = lut[a & 0xFFu], e1 = lut[(a >> 8) & 0xFFu];
    const uint32_t e2 = lut[(a >> 16) & 0xFFu], e3 = lut[a >> 24];
    const uint32_t e4 = lut[b & 0xFFu], e5 = lut[(b >> 8) & 0xFFu];
    const uint32_t e6 = lut[(b >> 16) & 0xFFu], e7 = lut[b >> 24];
    // [lo0 lo2 hi0 hi2], [lo4 lo6 hi4 hi6] -> [lo0 lo2 lo4 lo6] and [hi0 hi2 hi4 hi6]
    const uint32_t ea = __byte_perm(e0, e2, 0x5140), eb = __byte_perm(e4, e6, 0x5140);
    const uint32_t oa = __byte_perm(e1, e3, 0x5140), ob = __byte_perm(e5, e7, 0x5140);
    const uint32_t xe = __byte_perm(ea, eb, 0x5410), ze = __byte_perm(ea, eb, 0x7632);
    const uint32_t xo = __byte_perm(oa, ob, 0x5410), zo = __byte_perm(oa, ob, 0x7632);
    v[g] = (xe & 0x0F0F0F0Fu) | ((xo << 4) & 0xF0F0F0F0u);
    r[g] = ((xe >> 4) & 0x0F0F0F0Fu) | (xo & 0xF0F0F0F0u);
    tt[g] = (ze & 0x0F0F0F0Fu) | ((zo << 4) & 0xF0F0F0F0u);
    u[g] = ((ze >> 4) & 0x0F0F0F0Fu) | (zo & 0xF0F0F0F0u);
  }
  store_chunk(F, Np, Lk, i, c, v, r, tt, u);
}

// The per-byte code of the protein feature pack: residue rank r (the host's
// table, 0xFF for a gap) split as (r >> 2) | (r & 3) << 4; a gap as 0x40 (low
// field 4, which no rank has); a rank above 30, which no feature block holds
// (at most kMaxTcRanks + 1 blocks), as rank 31.
__device__ __forceinline__ uint32_t prot_code(uint32_t r) {
  if (r == 0xFFu) return 0x40u;
  if (r > 30u) return 0x37u;
  return (r >> 2) | ((r & 3u) << 4);
}

// Row i, 32-column chunk c of the protein features: block 0 is the valid
// feature (+1 where the residue is not a gap), block 1 + r the one-hot feature
// of residue rank r.  Then for two sites, V = sum v v' counts the columns where
// both are residues and M = sum over the rank blocks counts those where they
// are the same residue: mismatches = V - M, the counts of
// bitDistanceProtein.cpp:31-61.
// Per 8 sites the codes (prot_code) become two nibble words, hw (r >> 2) and lw
// (r & 3, or 4 for a gap).  Site k has rank 4h + l exactly when nibble k of both
// hw ^ h and lw ^ l is zero; adding 7 to every nibble (each is at most 7, so no
// carry crosses nibbles) sets its bit 3 unless it was zero, which tests all
// eight sites of a block word in a few instructions.
__device__ __forceinline__ void pack_prot_chunk(const uint8_t *__restrict__ chars, size_t ld,
                                                int n, int L, int Np, int Lk, int nfb,
                                                const uint8_t *code, int i, int c,
                                                uint8_t *__restrict__ F) {
  uint32_t q[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  const int len = i < n ? load_chunk(chars + (size_t)i * ld, L, c, q) : 0;
  uint32_t hw[4], lw[4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const uint32_t a = q[2 * g], b = q[2 * g + 1];
    const uint32_t c0 = code[a & 0xFFu], c1 = code[(a >> 8) & 0xFFu];
    const uint32_t c2 = code[(a >> 16) & 0xFFu], c3 = code[a >> 24];
    const uint32_t c4 = code[b & 0xFFu], c5 = code[(b >> 8) & 0xFFu];
    const uint32_t c6 = code[(b >> 16) & 0xFFu], c7 = code[b >> 24];
    const uint32_t xe = __byte_perm(__byte_perm(c0, c2, 0x0040), __byte_perm(c4, c6, 0x0040), 0x5410);
    const uint32_t xo = __byte_perm(__byte_perm(c1, c3, 0x0040), __byte_perm(c5, c7, 0x0040), 0x5410);
    hw[g] = (xe & 0x0F0F0F0Fu) | ((xo << 4) & 0xF0F0F0F0u);
    uint32_t l = ((xe >> 4) & 0x0F0F0F0Fu) | (xo & 0xF0F0F0F0u);
    const int m = len - 8 * g;  // sites of this word inside the row
    if (m < 8) {
      const uint32_t keep = m <= 0 ? 0u : (1u << (4 * m)) - 1u;
      l = (l & keep) | (0x44444444u & ~keep);  // the rest are gaps
    }
    lw[g] = l;
  }
  *feat_chunk(F, Np, Lk, 0, i, c) =
      make_uint4((~lw[0] & 0x44444444u) >> 1, (~lw[1] & 0x44444444u) >> 1,
                 (~lw[2] & 0x44444444u) >> 1, (~lw[3] & 0x44444444u) >> 1);
  uint32_t tl[4][4];
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int g = 0; g < 4; ++g) tl[l][g] = (lw[g] ^ (0x11111111u * (uint32_t)l)) + 0x77777777u;
  for (int h = 0; 4 * h + 1 < nfb; ++h) {
    uint32_t th[4];
#pragma unroll
    for (int g = 0; g < 4; ++g) th[g] = (hw[g] ^ (0x11111111u * (uint32_t)h)) + 0x77777777u;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int f = 4 * h + l + 1;
      if (f < nfb)
        *feat_chunk(F, Np, Lk, f, i, c) =
            make_uint4((~(th[0] | tl[l][0]) & 0x88888888u) >> 2,
                       (~(th[1] | tl[l][1]) & 0x88888888u) >> 2,
                       (~(th[2] | tl[l][2]) & 0x88888888u) >> 2,
                       (~(th[3] | tl[l][3]) & 0x88888888u) >> 2);
    }
  }
}

// The (row, chunk) of work unit t of rows x chunks: a 32-bit division below
// 2^32 units (the launchers give one thread per unit, so the loop runs once).
__device__ __forceinline__ void unit_rc(unsigned long long t, int chunks, int &r, int &c) {
  if (t < (1ull << 32)) {
    const uint32_t u = (uint32_t)t, q = u / (uint32_t)chunks;
    r = (int)q;
    c = (int)(u - q * (uint32_t)chunks);
  } else {
    r = (int)(t / (unsigned long long)chunks);
    c = (int)(t % (unsigned long long)chunks);
  }
}

__global__ void __launch_bounds__(256) pack_features_prot_kernel(const uint8_t *__restrict__ chars,
                                                                 size_t ld, int n, int L, int Np,
                                                                 int Lk, int nfb, Lut8 lut_in,
                                                                 int row0, int rows,
                                                                 uint8_t *__restrict__ F) {
  __shared__ uint8_t code[256];
  code[threadIdx.x] = (uint8_t)prot_code(lut_in.v[threadIdx.x]);
  __syncthreads();
  const int chunks = Lk / 32;
  const unsigned long long total = (unsigned long long)rows * chunks;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    int r, c;
    unit_rc(t, chunks, r, c);
    pack_prot_chunk(chars, ld, n, L, Np, Lk, nfb, code, row0 + r, c, F);
  }
}

__global__ void __launch_bounds__(256) pack_features_kernel(const uint8_t *__restrict__ chars,
                                                            size_t ld, int n, int L, int Np, int Lk,
                                                            int row0, int rows,
                                                            uint8_t *__restrict__ F) {
  __shared__ uint16_t lut[256];
  fill_feature_lut(lut);
  __syncthreads();
  const int chunks = Lk / 32;
  const unsigned long long total = (unsigned long long)rows * chunks;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    int r, c;
    unit_rc(t, chunks, r, c);
    pack_feature_chunk(chars, ld, n, L, Np, Lk, row0 + r, c, lut, F);
  }
}

// Features of many alignments: a thread per (row, 32-column chunk) of any job.
// A job's units (Np * Lk / 32, Np a multiple of 128 and Lk of 256) are a
// multiple of 1024, so the 256 units a block takes at a time belong to one job;
// a protein job's rank codes are staged in shared memory when the block moves
// on to it.
__global__ void __launch_bounds__(256) pack_features_multi_kernel(
    const PackJob *__restrict__ jobs, int njobs, long long units) {
  __shared__ uint16_t lut[256];
  __shared__ uint8_t code[256];
  fill_feature_lut(lut);
  __syncthreads();
  int cur = -1;
  for (long long base = (long long)blockIdx.x * 256; base < units;
       base += (long long)gridDim.x * 256) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].unit0 <= base) lo = mid;
      else hi = mid - 1;
    }
    const PackJob &jb = jobs[lo];
    if (lo != cur) {
      if (jb.kind == KIND_PROT_TC) {
        __syncthreads();
        code[threadIdx.x] = (uint8_t)prot_code(jb.lut[threadIdx.x]);
        __syncthreads();
      }
      cur = lo;
    }
    if (base + threadIdx.x >= units) continue;
    const int chunks = jb.W / 32;
    int r, c;
    unit_rc((unsigned long long)(base - jb.unit0 + threadIdx.x), chunks, r, c);
    if (jb.kind == KIND_PROT_TC)
      pack_prot_chunk(jb.chars, jb.ld, jb.n, jb.L, jb.Np, jb.W, jb.nfb, code, r, c,
                      (uint8_t *)jb.dst);
    else
      pack_feature_chunk(jb.chars, jb.ld, jb.n, jb.L, jb.Np, jb.W, r, c, lut, (uint8_t *)jb.dst);
  }
}

// The reference loader's DNA layout (16 sites per uint32, 2-bit codes A=00 G=01
// T=10 C=11, gap filter 01 per valid site, dataloaderFasta.hpp:147-182) ->
// features.  One thread per (sequence, 32 sites) = two source words.
__global__ void pack_features_bits_kernel(const uint32_t *__restrict__ bits,
                                          const uint32_t *__restrict__ gaps, int bs_words, int n,
                                          int L, int Np, int Lk, uint8_t *__restrict__ F) {
  const int chunks = Lk / 32;
  const long long total = (long long)Np * chunks;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / chunks);
    const int c = (int)(t % chunks);
    uint32_t v[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0}, tt[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int wd = 2 * c + h;
      if (i >= n || wd >= bs_words) continue;
      const uint32_t b = bits[(size_t)i * bs_words + wd];
      const uint32_t g = gaps[(size_t)i * bs_words + wd];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const bool ok = wd * 16 + k < L && ((g >> (2 * k)) & 1u);
        add_site(16 * h + k, ok ? (int)((b >> (2 * k)) & 3u) : -1, v, r, tt, u);
      }
    }
    store_chunk(F, Np, Lk, i, c, v, r, tt, u);
  }
}

cudaError_t launch_pack_features_prot(const uint8_t *d_chars, size_t ld, int n, int L, int Np,
                                      int Lk, int nfb, const uint8_t lut[256], uint8_t *F,
                                      cudaStream_t s, int row0, int rows) {
  if (rows < 0) rows = Np - row0;
  if (row0 < 0 || rows < 0 || row0 + rows > Np || nfb < 2 || nfb > kMaxTcRanks + 1)
    return cudaErrorInvalidValue;
  if (rows == 0) return cudaSuccess;
  Lut8 l;
  for (int k = 0; k < 256; ++k) l.v[k] = lut[k];
  const long long work = (long long)rows * (Lk / 32);
  const long long g = std::max(1LL, std::min((work + 255) / 256, 0x7fffffffLL));  // a thread per unit
  pack_features_prot_kernel<<<(unsigned)g, 256, 0, s>>>(d_chars, ld, n, L, Np, Lk, nfb, l, row0,
                                                        rows, F);
  return cudaGetLastError();
}

cudaError_t launch_pack_features_bits(const uint32_t *d_bits, const uint32_t *d_gaps, int bs_words,
                                      int n, int L, int Np, int Lk, uint8_t *F, cudaStream_t s) {
  const long long work = (long long)Np * (Lk / 32);
  long long g = (work + 255) / 256;
  if (g > 148LL * 64) g = 148LL * 64;
  if (g < 1) g = 1;
  pack_features_bits_kernel<<<(unsigned)g, 256, 0, s>>>(d_bits, d_gaps, bs_words, n, L, Np, Lk, F);
  return cudaGetLastError();
}

// ----------------------------------------------------------------- the kernel
//
// The counting pipeline of rnj_tcgen05.cuh (producer, MMA issuer) with an
// epilogue of eight warps that turns the accumulators into integer counts:
// packed per tile for the separate transform kernel (EPI_PACKED), or the
// n x n x 3 count matrix (EPI_COUNTS).  The epilogue works from tensor memory
// and registers only, never from the stage buffers.

// Items [item0, min(nitems, item0 + count)) of the work list.  EPI_PACKED: the
// counts of item it go to packed[(it - item0) * 128 * 128 ...] (see
// pack_counts); EPI_COUNTS: n x n x 3 counts into each alignment's counts.
template <int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_batch_kernel(const AlnDesc *__restrict__ descs, const WorkItem *__restrict__ items,
                    const int *__restrict__ nitems_ptr, int nitems_direct, int item0, int count,
                    uint64_t *__restrict__ packed, int nst) {
  extern __shared__ uint8_t smem_raw[];
  const TcShared sh = tc_shared(smem_raw, nst, 0);
  // The pipeline waits' bound and the failure-path test switch (the same for
  // every alignment of a launch).
  const uint64_t limit = wait_limit_ns((uint32_t)descs[0].wait_us);
  const int stall = descs[0].stall;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nitems = (int)min((long long)(nitems_ptr ? *nitems_ptr : nitems_direct),
                              (long long)item0 + count);
  if (item0 + (int)blockIdx.x >= nitems) return;  // no item for this CTA (before any setup)

  // tmem_empty: one arrival per epilogue thread (warps 2..9)
  const uint32_t tmem = tc_setup(sh, 256, 2);
  uint32_t issued = 0;  // producer: k-blocks issued in total (thread 0 only)

  if (warp == 0) {
    if (lane == 0)
      issued = tc_produce(sh, descs, items, item0 + blockIdx.x, nitems, gridDim.x, limit);
  } else if (warp == 1) {
    tc_issue(sh, tmem, descs, items, item0 + blockIdx.x, nitems, gridDim.x, limit);
  } else {
    // ----------------------------------------------------------- epilogue
    // Warps 2..9: TMEM lane quarter = warp % 4 (row block), column half by group.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    uint32_t titer = 0;
    for (int it = item0 + blockIdx.x; it < nitems; it += gridDim.x, ++titer) {
      const WorkItem w = item_at(descs, items, it);
      const AlnDesc &d = descs[w.aln];
      int ti, tj;
      item_tile(d, w.tile, ti, tj);
      if ((stall && titer == 0 && !tc_wait(sh.never_bar, 0, sh.abort_flag, limit)) ||
          !tc_wait(sh.acc_full, titer & 1, sh.abort_flag, limit)) {
        *sh.abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int n = d.n;
      const int i = ti * kTile + row;
      const bool prot_tile = d.kind == KIND_PROT_TC;
      uint64_t *dst = packed + (size_t)(it - item0) * (kTile * kTile);
      // Per 32-column chunk: accumulators -> integer counts -> stores.  Tensor
      // memory is handed back as soon as the last chunk is in registers.
#pragma unroll 1
      for (int cc = 0; cc < 2; ++cc) {
        uint32_t V[32], R[32], T[32];
        const int cbase = half * 64 + cc * 32;
        const uint32_t base = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)cbase;
        tmem_ld32(base, V);
        tmem_ld32(base + kTile, R);
        tmem_ld32(base + 2 * kTile, T);
        tmem_ld_wait();
        if (cc == 1) {
          tc_fence_before();
          mbar_arrive(sh.tmem_empty);
        }
        const int jb = tj * kTile + cbase;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const int vv = __float2int_rn(__uint_as_float(V[k]));
          const int rr = __float2int_rn(__uint_as_float(R[k]));
          const int tu = __float2int_rn(__uint_as_float(T[k]));
          // DNA: transitions, transversions; protein: mismatches (V - M), 0.
          const uint32_t ts = prot_tile ? (uint32_t)(vv - rr) : (uint32_t)((vv + rr - tu) >> 2);
          const uint32_t tv = prot_tile ? 0u : (uint32_t)((vv - rr) >> 1);
          if constexpr (EPI == EPI_PACKED) {
            // Column-major within the tile: the 32 lanes (consecutive rows)
            // store 256 contiguous bytes.
            dst[(cbase + k) * kTile + row] = pack_counts(ts, tv, (uint32_t)vv);
          } else {
            const int j = jb + k;
            if (i < n && (d.full ? (j < n) : (i < j && j < n))) {
              uint32_t *o = d.counts + ((size_t)i * n + j) * 3;
              o[0] = ts;
              o[1] = tv;
              o[2] = (uint32_t)vv;
            }
          }
        }
      }
    }
  }

  tc_teardown(sh, tmem, issued, descs[0].err);
}

// ------------------------------------------------------------ the transform
//
// Items [item0, min(nitems, item0 + count)): the packed counts of each tile ->
// the exact transform (pair_distance) -> the tile and its mirror image, the
// running maximum and the saturation flag of the tile.  Separate from the
// tensor-core kernel so that the double-precision logarithms run at high
// occupancy instead of on the eight epilogue warps of a tensor-core CTA.
//
// Warp w takes rows 32 (w % 4) .. +31 of the tile (lane = row) and columns
// 64 (w / 4) .. +63 in two 32 x 32 blocks.  For column c the lanes read 32
// consecutive packed counts (the tile's column-major layout) and store the
// mirror entries out[j0 + c][i0 + lane] as one coalesced 128-byte row segment;
// the tile entries out[i0 + row][j0 + c] go through a 32 x 33 per-warp
// transpose buffer and leave as coalesced row segments too.
constexpr int kTransformThreads = 256;
constexpr size_t kTransformSmem = (size_t)(kTransformThreads / 32) * 32 * 33 * sizeof(float);

__global__ void __launch_bounds__(kTransformThreads, kTransformCtasPerSm)
    tc_transform_kernel(const AlnDesc *__restrict__ descs, const WorkItem *__restrict__ items,
                        const int *__restrict__ nitems_ptr, int nitems_direct, int item0, int count,
                        const uint64_t *__restrict__ packed) {
  extern __shared__ uint8_t smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *T = reinterpret_cast<float *>(smem_raw) + warp * (32 * 33);
  const int nitems = (int)min((long long)(nitems_ptr ? *nitems_ptr : nitems_direct),
                              (long long)item0 + count);
  const int rblk = 32 * (warp & 3), chalf = 64 * (warp >> 2);
  for (int it = item0 + blockIdx.x; it < nitems; it += gridDim.x) {
    const WorkItem w = item_at(descs, items, it);
    const AlnDesc &d = descs[w.aln];
    int ti, tj;
    item_tile(d, w.tile, ti, tj);
    EpiParams ep;
    ep.n = d.n;
    ep.L = d.L;
    ep.model = d.model;
    ep.type = d.type;
    ep.compat_wrap = d.compat;
    ep.full = 0;
    ep.jc_b = d.jc_b;
    const int n = d.n;
    const int i0 = ti * kTile, j0 = tj * kTile;
    const int i = i0 + rblk + lane;  // this lane's row
    const uint64_t *src = packed + (size_t)(it - item0) * (kTile * kTile) + rblk + lane;
    float tmax = 0.0f;
    bool sat = false;
#pragma unroll 1
    for (int cb = chalf; cb < chalf + 64; cb += 32) {
#pragma unroll 1
      for (int k0 = 0; k0 < 32; k0 += 4) {
        float x[4];
        // The four packed counts first: the mirror stores below go through a
        // pointer the compiler cannot tell apart from src, so loads written
        // after a store would wait for it.
        uint64_t pk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) pk[u] = src[(size_t)(cb + k0 + u) * kTile];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int c = cb + k0 + u;
          const int j = j0 + c;
          uint32_t ts, tv, vv;
          unpack_counts(pk[u], ts, tv, vv);
          x[u] = 0.0f;
          if (i < j && j < n) {
            x[u] = pair_distance(ep, ts, tv, vv);
            tmax = fmaxf(tmax, x[u]);
            sat |= (x[u] == -1.0f);
            d.out[(size_t)j * d.ld + i] = x[u];  // mirror: consecutive i across lanes
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) T[lane * 33 + k0 + u] = x[u];
      }
      __syncwarp();
      // Tile entries: row i0 + rblk + r, columns j0 + cb + lane.
      const int j = j0 + cb + lane;
#pragma unroll 4
      for (int r = 0; r < 32; ++r) {
        const int ir = i0 + rblk + r;
        if (ir >= n || j >= n || ir > j) continue;
        d.out[(size_t)ir * d.ld + j] = (ir == j) ? 0.0f : T[r * 33 + lane];
      }
      __syncwarp();
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, off));
    const bool any_sat = __any_sync(0xffffffffu, sat);
    if (lane == 0) {
      if (tmax > 0.0f) atomicMax(d.max_bits, __float_as_int(tmax));
      if (any_sat) d.tile_flags[w.tile] = 1;
    }
  }
}

// ------------------------------------------------------------------ launchers

cudaError_t launch_pack_features(const uint8_t *d_chars, size_t ld, int n, int L, int Np, int Lk,
                                 uint8_t *F, cudaStream_t s, int row0, int rows) {
  if (rows < 0) rows = Np - row0;
  if (row0 < 0 || rows < 0 || row0 + rows > Np) return cudaErrorInvalidValue;
  if (rows == 0) return cudaSuccess;
  const long long work = (long long)rows * (Lk / 32);
  const long long g = std::max(1LL, std::min((work + 255) / 256, 0x7fffffffLL));  // a thread per unit
  pack_features_kernel<<<(unsigned)g, 256, 0, s>>>(d_chars, ld, n, L, Np, Lk, row0, rows, F);
  return cudaGetLastError();
}

cudaError_t launch_pack_features_multi(const PackJob *d_jobs, int njobs, long long units,
                                       cudaStream_t s) {
  if (njobs <= 0 || units <= 0) return cudaSuccess;
  long long g = (units + 255) / 256;
  if (g > 148LL * 64) g = 148LL * 64;
  pack_features_multi_kernel<<<(unsigned)g, 256, 0, s>>>(d_jobs, njobs, units);
  return cudaGetLastError();
}

cudaError_t launch_tc_batch(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                            int nitems, int item0, int count, uint64_t *packed, int grid,
                            int epi_mode, cudaStream_t s, int stages) {
  if (grid <= 0) return cudaSuccess;
  const int nst = tc_ring_depth(stages, kTcStages, kTcStages);
  const size_t smem = tc_smem_bytes(nst);
  auto kernel = epi_mode == EPI_PACKED ? tc_batch_kernel<EPI_PACKED> : tc_batch_kernel<EPI_COUNTS>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kernel<<<(unsigned)grid, kTcThreads, smem, s>>>(d_descs, d_items, d_nitems, nitems, item0, count,
                                                  packed, nst);
  return cudaGetLastError();
}

cudaError_t launch_tc_transform(const AlnDesc *d_descs, const WorkItem *d_items,
                                const int *d_nitems, int nitems, int item0, int count,
                                const uint64_t *packed, int grid, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  tc_transform_kernel<<<(unsigned)grid, kTransformThreads, kTransformSmem, s>>>(
      d_descs, d_items, d_nitems, nitems, item0, count, packed);
  return cudaGetLastError();
}

// ------------------------------------------------------ tensor-pipe probe
//
// The FP4 tensor-pipe throughput of the device: one CTA per SM, one thread
// issuing `iters` back-to-back 128 x 128 x 64 kind::mxf4 MMAs into one
// accumulator with loop-invariant descriptors (zero operands in shared
// memory, unit scale factors), then one commit.  The counting kernel's
// roofline is reported against this rate beside the 4 x bf16 GEMM figure.
constexpr int kProbeSmem = 32 * 1024 + 1024;

__global__ void __launch_bounds__(128, 1) tc_peak_probe_kernel(int iters, int *err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem =
      reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ uint64_t bar;
  __shared__ uint32_t slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < 32 * 1024 / 16; i += 128)
    reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(&slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = slot;
  {
    const uint32_t base = tmem + ((uint32_t)(32 * warp) << 16) + kTmemSfa;
    tmem_st32(base, 0x7F7F7F7Fu);
    tmem_st32(base + 32, 0x7F7F7F7Fu);
    tmem_st32(base + 64, 0x7F7F7F7Fu);
    tmem_st32(base + 96, 0x7F7F7F7Fu);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    const uint64_t ad = smem_desc_sw128(smem_u32(smem));
    const uint64_t bd = smem_desc_sw128(smem_u32(smem) + kTcTileBytes);
    for (int i = 0; i < iters; i += 4) {
      tc_mma_fp4_elect(tmem, ad, bd, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, i > 0);
      tc_mma_fp4_elect(tmem, ad + 2, bd + 2, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
      tc_mma_fp4_elect(tmem, ad + 4, bd + 4, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
      tc_mma_fp4_elect(tmem, ad + 6, bd + 6, kIdescFp4, tmem + kTmemSfa, tmem + kTmemSfb, 1u);
    }
    tc_commit_elect(&bar);
    if (tid == 0 && !mbar_wait_bounded(&bar, 0)) atomicOr(err, 1);
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

cudaError_t launch_tc_peak_probe(int grid, int iters, int *err, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(tc_peak_probe_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kProbeSmem);
  if (e != cudaSuccess) return e;
  tc_peak_probe_kernel<<<grid, 128, kProbeSmem, s>>>(iters, err);
  return cudaGetLastError();
}

}  // namespace rnj
