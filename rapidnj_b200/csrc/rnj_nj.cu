// rnj_nj.cu -- the neighbour-joining set-up over a finished distance matrix on
// the device (rnj_nj_init).
//
// rapidNJ, before its first join, makes three O(n^2) passes over the matrix the
// distance step produced (rapidNJ::initialize, rapidNJ.cpp:94-141, and
// rapidNJMem::initialize, rapidNJMem.cpp:92-135):
//   1. the separation sum of every row, summed in float from column 0 on, and
//      from it the separations and the running maximum of the separations;
//   2. redundant rows: for i from n-1 down (rows already marked skipped), every
//      j < i with matrix[i][j] == 0 whose row equals row i in every column is
//      marked and mapped to i (handleRedundancy, rapidNJ.cpp:156-167);
//   3. a sorted row per unmarked row i: the unmarked j < i by distance
//      (buildSortedRow, rapidNJ.cpp:134-154), cut to sortedMatrixSize entries by
//      rapidNJMem (rapidNJMem.cpp:138-153).
//
// On the device:
//   * one pass reads the matrix once: a warp owns 32 rows and streams them in
//     32 x 32 tiles (cp.async into shared memory, eight tiles in its ring), then
//     every lane walks its own row of the tile in column order, so each row is
//     summed exactly in the reference's order; the same walk counts the row's
//     zeros (a second zero besides the diagonal is the zero scan of
//     rdDataInitialiser.cpp:174-189), and the diagonal entry is checked;
//   * with a zero diagonal, row equality is an equivalence whose classes are
//     exactly the reference's redundancy classes (the highest row of a class is
//     its master; a row equal to another has a zero at that row's column), so
//     only rows with a zero off the diagonal are candidates: they are hashed
//     (a warp per row; zero of either sign as +0), each candidate is compared
//     in full with the highest row of its hash group (a warp per pair), and rows
//     that differ (hash collisions, NaN entries) form new groups;
//   * each unmarked row is sorted by a CTA: 64-bit items (the distance's bits
//     made order-preserving, then j) in ascending j, and a stable LSD radix
//     sort on the distance's four bytes (ranking inside each warp by ballots;
//     a pass whose digit is the same for the whole row is skipped) gives the
//     reference's order with equal distances in ascending j; rows of up to
//     8192 items in shared memory, longer ones in the CTA's global scratch rows.
// The O(n) parts (separations, running maximum, the redundancy classes) run on
// the host from the per-row results.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

constexpr int kRowStages = 8;    // 32 x 32 tiles in the ring of a row-pass warp
constexpr int kTileLd = 33;      // padded tile row: lane l reads bank (l + k) % 32
constexpr int kSortBlock = 8192; // entries of a row sorted in shared memory
constexpr int kSortThreads = 1024;

enum : uint32_t { kRowZero = 1u, kRowBadDiag = 4u };

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t bytes = valid ? 4u : 0u;  // 0: nothing read, the word is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Pass 1: per row the float sum in column order, whether it holds a zero off
// the diagonal, and whether its diagonal entry is non-zero.  A CTA (one warp)
// owns rows [32 b, 32 b + 32); lane l sums row 32 b + l.  Tile t holds columns
// [32 t, 32 t + 32) of the 32 rows, in stage t % kRowStages of the ring.  Per
// entry the lane does no more than the sum needs (a load, the add, a zero
// test), so that the pass runs at the rate the matrix streams in.
__global__ void __launch_bounds__(32)
    nj_row_pass_kernel(const float *__restrict__ M, int n, size_t ld, float *__restrict__ sums,
                       uint32_t *__restrict__ flags) {
  extern __shared__ float tiles[];  // [kRowStages][32 * kTileLd]
  const int lane = threadIdx.x;
  const int row0 = blockIdx.x * 32;
  const int ntile = (n + 31) / 32;
  auto issue = [&](int t) {
    if (t < ntile) {
      float *dst = tiles + (t % kRowStages) * (32 * kTileLd);
      const int c = t * 32 + lane;
#pragma unroll 8
      for (int r = 0; r < 32; ++r) {
        const int row = row0 + r;
        const bool ok = row < n && c < n;
        cp_async4(dst + r * kTileLd + lane, ok ? M + (size_t)row * ld + c : M, ok);
      }
    }
    cp_async_commit();  // an empty group past the end keeps the count uniform
  };
#pragma unroll
  for (int t = 0; t < kRowStages - 1; ++t) issue(t);
  const int my_row = row0 + lane;
  float sum = 0.0f;
  int zeros = 0;
  for (int t = 0; t < ntile; ++t) {
    issue(t + kRowStages - 1);
    cp_async_wait<kRowStages - 1>();  // this lane's copies of tile t are done
    __syncwarp();                     // and every lane's are visible
    const float *row = tiles + (t % kRowStages) * (32 * kTileLd) + lane * kTileLd;
    if (t * 32 + 32 <= n) {
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const float v = row[k];
        sum += v;
        zeros += v == 0.0f;
      }
    } else {
      for (int k = 0; k < n - t * 32; ++k) {
        const float v = row[k];
        sum += v;
        zeros += v == 0.0f;
      }
    }
    __syncwarp();  // the stage is refilled by the next iteration's issue
  }
  cp_async_wait<0>();
  if (my_row < n) {
    const float diag = M[(size_t)my_row * ld + my_row];
    sums[my_row] = sum;
    // with a zero diagonal, a second zero is one off the diagonal
    flags[my_row] = (diag == 0.0f ? 0u : kRowBadDiag) | (zeros >= 2 ? kRowZero : 0u);
  }
}

// Pass 1b: a hash of each candidate row (warp p: row cand[p]): two 32-bit sums
// over the columns c of a mix of (entry bits, c), zero of either sign as +0, so
// that rows equal under float == hash equally.
__global__ void __launch_bounds__(256)
    nj_row_hash_kernel(const float *__restrict__ M, int n, size_t ld, const int *__restrict__ cand,
                       int ncand, uint2 *__restrict__ hashes) {
  const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= ncand) return;  // uniform per warp
  const float *row = M + (size_t)cand[p] * ld;
  uint32_t ha = 0, hb = 0;
  for (int c = lane; c < n; c += 32) {
    const float v = row[c];
    const uint32_t u = v == 0.0f ? 0u : __float_as_uint(v);
    const uint32_t z = u ^ ((uint32_t)c * 0x9E3779B9u);
    ha += (z ^ (z >> 15)) * 0x85EBCA6Bu;
    hb += (z ^ (z >> 13)) * 0xC2B2AE35u + z;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ha += __shfl_xor_sync(0xffffffffu, ha, o);
    hb += __shfl_xor_sync(0xffffffffu, hb, o);
  }
  if (lane == 0) hashes[p] = make_uint2(ha, hb);
}

// Pass 2: warp p compares row a = pairs[p].x (the reference's row i) with row
// b = pairs[p].y (its j): equal[p] = matrix[a][b] == 0 and every column equal
// under float ==.  The loop stops for the whole warp at the first difference.
__global__ void __launch_bounds__(256)
    nj_rows_equal_kernel(const float *__restrict__ M, int n, size_t ld,
                         const int2 *__restrict__ pairs, int npairs, int *__restrict__ equal) {
  const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= npairs) return;  // uniform per warp
  const int a = pairs[p].x, b = pairs[p].y;
  const float *ra = M + (size_t)a * ld, *rb = M + (size_t)b * ld;
  bool eq = ra[b] == 0.0f;
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int c = c0 + lane;
    if (c < n && !(ra[c] == rb[c])) eq = false;
    if (!__all_sync(0xffffffffu, eq)) break;
  }
  const bool all = __all_sync(0xffffffffu, eq);
  if (lane == 0) equal[p] = all ? 1 : 0;
}

// Order-preserving 64-bit key of (distance, j): the float's bits with zero of
// either sign as +0 (so that -0 and +0 tie, as under operator<), negative
// values flipped whole, positive ones with the sign bit set; j below.
__device__ __forceinline__ unsigned long long sort_key(float v, int j) {
  uint32_t f = v == 0.0f ? 0u : __float_as_uint(v);
  f = (f & 0x80000000u) ? ~f : (f | 0x80000000u);
  return ((unsigned long long)f << 32) | (uint32_t)j;
}

// Pass 3: a CTA per unmarked row i (rows[], longest first).  The unmarked j < i
// (rank[j] = unmarked rows below j, rank[i] of them in all) become 64-bit items
// (order-preserving distance key << 32 | j) in ascending j, and a stable LSD
// radix sort on the key's four bytes orders them by distance with equal
// distances in ascending j; the first min(rank[i], cap) are written as
// (j, matrix[i][j]).  Each pass, chunk by chunk (8192 items: warp w, slot s,
// lane l holds item w 256 + s 32 + l): a stable rank inside each warp by
// ballots, the per-(digit, warp) offsets from the digit bases, and the scatter.
// The digit bases come from the chunk's own counts when the row is one chunk,
// else from a histogram of the row first; a pass in which one digit holds every
// item is skipped.  Rows of up to 8192 items live in shared memory, longer ones
// in the CTA's scratch rows.
constexpr int kRadixDigits = 256;
constexpr int kWarpsPerSort = kSortThreads / 32;
constexpr int kItems = kSortBlock / kSortThreads;  // per thread and chunk

using u64 = unsigned long long;

// The lanes of the warp holding the same 8-bit digit d as this lane (valid:
// this lane holds an item), from eight ballots: the hardware match instruction
// is far slower than ballots on this part.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, bool valid) {
  uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool bit = (d >> b) & 1u;
    const uint32_t m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

struct SortShared {
  u64 a[kSortBlock];
  u64 b[kSortBlock];
  uint32_t wcnt[kWarpsPerSort * kRadixDigits];  // [warp][digit]
  uint32_t dtot[kRadixDigits];
  uint32_t dbase[kRadixDigits];
  int skip;
};

// Warp 0: the exclusive scan of the digit totals into the digit bases (eight
// digits a lane) and the skip flag (one digit holds every item).
__device__ __forceinline__ void scan_digits(SortShared &S, int cnt, int warp, int lane) {
  if (warp != 0) return;
  uint32_t v[8], s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    v[k] = S.dtot[lane * 8 + k];
    s += v[k];
  }
  uint32_t incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  uint32_t run = incl - s;
  bool one = false;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    S.dbase[lane * 8 + k] = run;
    run += v[k];
    one |= v[k] == (uint32_t)cnt;
  }
  one = __any_sync(0xffffffffu, one);
  if (lane == 0) S.skip = one;
}

__global__ void __launch_bounds__(kSortThreads, 1)
    nj_sort_rows_kernel(const float *__restrict__ M, size_t ld, const int *__restrict__ rank,
                        const uint8_t *__restrict__ keep, const int *__restrict__ rows, int nrows,
                        u64 *__restrict__ scratch, size_t scratch_per_cta,
                        rnj_cluster_pair *__restrict__ out, size_t out_ld, int cap) {
  extern __shared__ __align__(16) unsigned char nj_sort_smem[];
  SortShared &S = *reinterpret_cast<SortShared *>(nj_sort_smem);
  const int th = threadIdx.x, lane = th & 31, warp = th >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    const int cnt = rank[i];
    if (cnt == 0) continue;  // uniform over the CTA
    const float *row = M + (size_t)i * ld;
    u64 *A, *B;
    if (cnt <= kSortBlock) {
      A = S.a;
      B = S.b;
    } else {
      A = scratch + (size_t)blockIdx.x * 2 * scratch_per_cta;
      B = A + scratch_per_cta;
    }
    for (int j = th; j < i; j += blockDim.x)
      if (keep[j]) A[rank[j]] = sort_key(row[j], j);
    __syncthreads();
    for (int pass = 0; pass < 4; ++pass) {
      const int shift = 32 + 8 * pass;
      const bool chunked = cnt > kSortBlock;
      if (chunked) {
        // Histogram of the row's digits (warp-aggregated shared atomics); a row
        // of one chunk takes its totals from the ranking instead.
        for (int d = th; d < kRadixDigits; d += blockDim.x) S.dtot[d] = 0;
        __syncthreads();
        for (int t0 = 0; t0 < cnt; t0 += blockDim.x) {
          const int t = t0 + th;
          const bool ok = t < cnt;
          const uint32_t d = ok ? (uint32_t)((A[t] >> shift) & 255u) : 0u;
          const uint32_t peers = digit_peers(d, ok);
          if (ok && (peers & lt) == 0) atomicAdd(&S.dtot[d], (uint32_t)__popc(peers));
        }
        __syncthreads();
        scan_digits(S, cnt, warp, lane);
        __syncthreads();
        if (S.skip) continue;  // uniform: every item has the same digit
      }
      for (int c0 = 0; c0 < cnt; c0 += kSortBlock) {
        for (int k = th; k < kWarpsPerSort * kRadixDigits; k += blockDim.x) S.wcnt[k] = 0;
        __syncthreads();
        u64 x[kItems];
        uint32_t rk[kItems];
#pragma unroll
        for (int s = 0; s < kItems; ++s) {
          const int t = c0 + warp * (32 * kItems) + s * 32 + lane;
          const bool ok = t < cnt;
          x[s] = ok ? A[t] : 0ull;
          const uint32_t d = ok ? (uint32_t)((x[s] >> shift) & 255u) : 0u;
          const uint32_t peers = digit_peers(d, ok);
          const uint32_t before = ok ? S.wcnt[warp * kRadixDigits + d] : 0u;
          __syncwarp();
          if (ok && (peers & lt) == 0) S.wcnt[warp * kRadixDigits + d] = before + __popc(peers);
          __syncwarp();
          rk[s] = before + __popc(peers & lt);
        }
        __syncthreads();
        if (!chunked) {
          // One chunk: digit totals from the warps' counts, then the bases.
          for (int d = th; d < kRadixDigits; d += blockDim.x) {
            uint32_t t = 0;
            for (int w = 0; w < kWarpsPerSort; ++w) t += S.wcnt[w * kRadixDigits + d];
            S.dtot[d] = t;
          }
          __syncthreads();
          scan_digits(S, cnt, warp, lane);
          __syncthreads();
          if (S.skip) break;  // uniform; the pass leaves the items in place
        }
        // Offsets: digit base, then the warps in order; the base moves on by the
        // chunk's items of that digit.
        for (int d = th; d < kRadixDigits; d += blockDim.x) {
          uint32_t run = S.dbase[d];
          for (int w = 0; w < kWarpsPerSort; ++w) {
            const uint32_t v = S.wcnt[w * kRadixDigits + d];
            S.wcnt[w * kRadixDigits + d] = run;
            run += v;
          }
          S.dbase[d] = run;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < kItems; ++s) {
          const int t = c0 + warp * (32 * kItems) + s * 32 + lane;
          if (t < cnt) {
            const uint32_t d = (uint32_t)((x[s] >> shift) & 255u);
            B[S.wcnt[warp * kRadixDigits + d] + rk[s]] = x[s];
          }
        }
        __syncthreads();
      }
      if (!chunked && S.skip) continue;
      u64 *tmp = A;
      A = B;
      B = tmp;
    }
    const int keepn = cap > 0 ? min(cnt, cap) : cnt;
    rnj_cluster_pair *o = out + (size_t)i * out_ld;
    for (int t = th; t < keepn; t += blockDim.x) {
      const uint32_t id = (uint32_t)A[t];
      rnj_cluster_pair cp;
      cp.id = id;
      cp.distance = row[id];  // the stored value, -0 kept
      o[t] = cp;
    }
    __syncthreads();  // the next row reuses the buffers
  }
}

#define NJ_CUDA(call, what)                          \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

// Device buffers of one call, freed on every return path.
struct NjBuffers {
  cudaStream_t s;
  std::vector<void *> ptrs;
  explicit NjBuffers(cudaStream_t st) : s(st) {}
  template <class T>
  cudaError_t alloc(T **p, size_t bytes) {
    cudaError_t e = cudaMallocAsync((void **)p, std::max<size_t>(bytes, 16), s);
    if (e == cudaSuccess) ptrs.push_back((void *)*p);
    return e;
  }
  ~NjBuffers() {
    for (void *p : ptrs) cudaFreeAsync(p, s);
  }
};

}  // namespace

extern "C" int rnj_nj_init(rnj_ctx *ctx, const float *d_matrix, int n, size_t ld,
                           rnj_nj_data *o) {
  if (!ctx || !o || (!d_matrix && n > 0)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 1 || ld < (size_t)n) return set_error(RNJ_ERR_INVALID, "invalid matrix shape");
  if (n > (1 << 24)) return set_error(RNJ_ERR_INVALID, "more than 2^24 rows");
  const int cap = o->sorted_cap;
  const long long widest = cap > 0 ? std::min(cap, n - 1) : n - 1;
  if (o->sorted && (long long)o->sorted_ld < std::max<long long>(widest, 1))
    return set_error(RNJ_ERR_INVALID, "sorted_ld is smaller than the longest sorted row");
  DeviceGuard guard(ctx->device);
  cudaStream_t st = ctx->stream;
  NjBuffers buf(st);

  // Pass 1.
  float *d_sums = nullptr;
  uint32_t *d_flags = nullptr;
  NJ_CUDA(buf.alloc(&d_sums, (size_t)n * sizeof(float)), "nj buffers");
  NJ_CUDA(buf.alloc(&d_flags, (size_t)n * sizeof(uint32_t)), "nj buffers");
  const int row_smem = kRowStages * 32 * kTileLd * (int)sizeof(float);
  NJ_CUDA(cudaFuncSetAttribute(nj_row_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               row_smem),
          "nj row pass attribute");
  nj_row_pass_kernel<<<(n + 31) / 32, 32, row_smem, st>>>(d_matrix, n, ld, d_sums, d_flags);
  NJ_CUDA(cudaGetLastError(), "nj row pass");
  std::vector<float> sums(n);
  std::vector<uint32_t> flags(n);
  NJ_CUDA(cudaMemcpyAsync(sums.data(), d_sums, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st),
          "nj copy");
  NJ_CUDA(cudaMemcpyAsync(flags.data(), d_flags, (size_t)n * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, st),
          "nj copy");
  NJ_CUDA(cudaStreamSynchronize(st), "nj row pass sync");
  for (int i = 0; i < n; ++i)
    if (flags[i] & kRowBadDiag)
      return set_error(RNJ_ERR_INVALID, "row " + std::to_string(i) +
                                            " has a non-zero diagonal entry (not a distance matrix "
                                            "of this library)");

  // Separations and their running maximum (rapidNJ.cpp:102-118), in float.
  {
    const float div = (float)(n - 2);
    float mx = FLT_MIN;
    for (int i = 0; i < n; ++i) {
      const float sep = sums[i] / div;
      if (o->separation_sums) o->separation_sums[i] = sums[i];
      if (o->separations) o->separations[i] = sep;
      if (o->max_row_separations) o->max_row_separations[i] = mx;
      if (sep > mx) mx = sep;
    }
    if (o->max_separation) *o->max_separation = mx;
    if (o->possible_redundant)
      for (int i = 0; i < n; ++i) o->possible_redundant[i] = (flags[i] & kRowZero) ? 1 : 0;
  }

  // Redundancy classes: candidates grouped by hash, each group's members
  // compared with its highest row; rows that differ form the next round's groups.
  std::vector<int> master(n);
  for (int i = 0; i < n; ++i) master[i] = i;
  {
    // Candidates: rows with a zero off the diagonal (a row equal to another
    // has one, in that row's column).  Their hashes (pass 1b).
    std::vector<int> cand;
    for (int i = 0; i < n; ++i)
      if (flags[i] & kRowZero) cand.push_back(i);
    std::vector<uint2> hash(n, make_uint2(0u, 0u));
    if (cand.size() >= 2) {
      int *d_cand = nullptr;
      uint2 *d_hash = nullptr;
      NJ_CUDA(buf.alloc(&d_cand, cand.size() * sizeof(int)), "nj buffers");
      NJ_CUDA(buf.alloc(&d_hash, cand.size() * sizeof(uint2)), "nj buffers");
      NJ_CUDA(cudaMemcpyAsync(d_cand, cand.data(), cand.size() * sizeof(int), cudaMemcpyHostToDevice,
                              st),
              "nj copy");
      const size_t threads = cand.size() * 32;
      nj_row_hash_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
          d_matrix, n, ld, d_cand, (int)cand.size(), d_hash);
      NJ_CUDA(cudaGetLastError(), "nj row hash");
      std::vector<uint2> h(cand.size());
      NJ_CUDA(cudaMemcpyAsync(h.data(), d_hash, h.size() * sizeof(uint2), cudaMemcpyDeviceToHost, st),
              "nj copy");
      NJ_CUDA(cudaStreamSynchronize(st), "nj row hash sync");
      for (size_t k = 0; k < cand.size(); ++k) hash[cand[k]] = h[k];
    }
    auto same = [&](int a, int b) { return hash[a].x == hash[b].x && hash[a].y == hash[b].y; };
    std::sort(cand.begin(), cand.end(), [&](int a, int b) {
      if (hash[a].x != hash[b].x) return hash[a].x < hash[b].x;
      if (hash[a].y != hash[b].y) return hash[a].y < hash[b].y;
      return a < b;
    });
    std::vector<std::vector<int>> groups;  // members in ascending order
    for (size_t s = 0; s < cand.size();) {
      size_t e = s + 1;
      while (e < cand.size() && same(cand[e], cand[s])) ++e;
      if (e - s >= 2) groups.emplace_back(cand.begin() + s, cand.begin() + e);
      s = e;
    }
    std::vector<int2> pairs;
    std::vector<int> eq;
    int2 *d_pairs = nullptr;
    int *d_eq = nullptr;
    size_t pair_cap = 0;
    while (!groups.empty()) {
      pairs.clear();
      for (const auto &g : groups)
        for (size_t k = 0; k + 1 < g.size(); ++k) pairs.push_back(make_int2(g.back(), g[k]));
      if (pairs.size() > pair_cap) {  // the first round is the largest
        pair_cap = pairs.size();
        NJ_CUDA(buf.alloc(&d_pairs, pair_cap * sizeof(int2)), "nj buffers");
        NJ_CUDA(buf.alloc(&d_eq, pair_cap * sizeof(int)), "nj buffers");
      }
      NJ_CUDA(cudaMemcpyAsync(d_pairs, pairs.data(), pairs.size() * sizeof(int2),
                              cudaMemcpyHostToDevice, st),
              "nj copy");
      const size_t threads = pairs.size() * 32;
      nj_rows_equal_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
          d_matrix, n, ld, d_pairs, (int)pairs.size(), d_eq);
      NJ_CUDA(cudaGetLastError(), "nj row compare");
      eq.resize(pairs.size());
      NJ_CUDA(cudaMemcpyAsync(eq.data(), d_eq, eq.size() * sizeof(int), cudaMemcpyDeviceToHost, st),
              "nj copy");
      NJ_CUDA(cudaStreamSynchronize(st), "nj row compare sync");
      std::vector<std::vector<int>> next;
      size_t p = 0;
      for (const auto &g : groups) {
        std::vector<int> rest;
        for (size_t k = 0; k + 1 < g.size(); ++k, ++p) {
          if (eq[p]) master[g[k]] = g.back();
          else rest.push_back(g[k]);
        }
        if (rest.size() >= 2) next.push_back(std::move(rest));
      }
      groups.swap(next);
    }
  }
  if (o->index_to_id)
    for (int i = 0; i < n; ++i) o->index_to_id[i] = master[i] == i ? i : -1;
  if (o->redundant_to_master) std::copy(master.begin(), master.end(), o->redundant_to_master);
  if (o->redundant_count) {
    std::fill(o->redundant_count, o->redundant_count + n, 1);
    for (int j = 0; j < n; ++j)
      if (master[j] != j) ++o->redundant_count[master[j]];
  }

  // Sorted rows.
  std::vector<int> rank(n);
  std::vector<uint8_t> keep(n);
  std::vector<int> rows;  // unmarked rows with entries, longest first
  {
    int c = 0;
    for (int i = 0; i < n; ++i) {
      rank[i] = c;
      keep[i] = master[i] == i;
      c += keep[i];
    }
    for (int i = n - 1; i >= 0; --i)
      if (keep[i] && rank[i] > 0) rows.push_back(i);
  }
  if (o->row_lengths)
    for (int i = 0; i < n; ++i)
      o->row_lengths[i] = keep[i] ? (cap > 0 ? std::min(rank[i], cap) : rank[i]) : 0;
  if (o->sorted && !rows.empty()) {
    int *d_rank = nullptr, *d_rows = nullptr;
    uint8_t *d_keep = nullptr;
    NJ_CUDA(buf.alloc(&d_rank, (size_t)n * sizeof(int)), "nj buffers");
    NJ_CUDA(buf.alloc(&d_keep, (size_t)n), "nj buffers");
    NJ_CUDA(buf.alloc(&d_rows, rows.size() * sizeof(int)), "nj buffers");
    NJ_CUDA(cudaMemcpyAsync(d_rank, rank.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st),
            "nj copy");
    NJ_CUDA(cudaMemcpyAsync(d_keep, keep.data(), (size_t)n, cudaMemcpyHostToDevice, st), "nj copy");
    NJ_CUDA(cudaMemcpyAsync(d_rows, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice,
                            st),
            "nj copy");
    const int smem = (int)sizeof(SortShared);
    NJ_CUDA(cudaFuncSetAttribute(nj_sort_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem),
            "nj sort attribute");
    int per_sm = 1;
    NJ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nj_sort_rows_kernel, kSortThreads,
                                                          smem),
            "nj sort occupancy");
    const int grid =
        (int)std::min<size_t>(rows.size(), (size_t)std::max(1, per_sm) * ctx->num_sms);
    // Rows of more than kSortBlock items: two scratch rows per CTA.
    const size_t longest = (size_t)rank[rows[0]];
    u64 *d_scratch = nullptr;
    size_t per_cta = 0;
    if (longest > (size_t)kSortBlock) {
      per_cta = longest;
      NJ_CUDA(buf.alloc(&d_scratch, (size_t)grid * 2 * per_cta * sizeof(u64)),
              "nj sort scratch");
    }
    nj_sort_rows_kernel<<<grid, kSortThreads, smem, st>>>(d_matrix, ld, d_rank, d_keep, d_rows,
                                                         (int)rows.size(), d_scratch, per_cta,
                                                         o->sorted, o->sorted_ld, cap);
    NJ_CUDA(cudaGetLastError(), "nj sort");
  }
  NJ_CUDA(cudaStreamSynchronize(st), "nj sync");
  return RNJ_OK;
}
