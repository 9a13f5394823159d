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
//     32 x 32 tiles (cp.async into shared memory, four tiles in flight), then
//     every lane walks its own row of the tile in column order, so each row is
//     summed exactly in the reference's order; the same walk hashes the row
//     (zero of either sign hashed as +0), and flags a zero off the diagonal
//     (rdDataInitialiser.cpp:174-189), a NaN and a non-zero diagonal;
//   * with a zero diagonal, row equality is an equivalence whose classes are
//     exactly the reference's redundancy classes (the highest row of a class is
//     its master; a row equal to another has a zero at that row's column), so
//     only rows with a zero and no NaN and with an equal hash are candidates:
//     each candidate is compared in full with the highest row of its hash group
//     (a warp per pair), and rows that differ (hash collisions) form new groups;
//   * each unmarked row is sorted by a CTA: 64-bit keys (the distance's bits
//     made order-preserving, then j), unique, so a bitonic network gives the
//     reference's order with equal distances in ascending j; rows of up to 8192
//     entries are sorted in shared memory, longer ones in a global scratch row
//     with the short strides done in shared memory.
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

constexpr int kRowWarps = 2;     // warps per CTA of the row pass
constexpr int kRowStages = 4;    // 32 x 32 tiles in flight per warp
constexpr int kTileLd = 33;      // padded tile row: lane l reads bank (l + k) % 32
constexpr int kSortBlock = 8192; // entries of a row sorted in shared memory
constexpr int kSortThreads = 1024;

enum : uint32_t { kRowZero = 1u, kRowNan = 2u, kRowBadDiag = 4u };

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

// Pass 1: per row the float sum in column order, two 32-bit hashes and flags.
// Warp w of CTA b owns rows [32 (b kRowWarps + w), +32); lane l sums row
// row0 + l.  Tile t holds columns [32 t, 32 t + 32) of the 32 rows; stage
// t % kRowStages of the warp's ring.
__global__ void __launch_bounds__(32 * kRowWarps)
    nj_row_pass_kernel(const float *__restrict__ M, int n, size_t ld, float *__restrict__ sums,
                       uint2 *__restrict__ hashes, uint32_t *__restrict__ flags) {
  __shared__ float tiles[kRowWarps][kRowStages][32 * kTileLd];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = (blockIdx.x * kRowWarps + warp) * 32;
  if (row0 >= n) return;  // the whole warp; the kernel has no CTA-wide barrier
  const int ntile = (n + 31) / 32;
  auto issue = [&](int t) {
    if (t < ntile) {
      float *dst = tiles[warp][t % kRowStages];
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
  uint32_t h1 = 2166136261u, h2 = 0x9E3779B9u, fl = 0;
  for (int t = 0; t < ntile; ++t) {
    issue(t + kRowStages - 1);
    cp_async_wait<kRowStages - 1>();  // this lane's copies of tile t are done
    __syncwarp();                     // and every lane's are visible
    const float *row = tiles[warp][t % kRowStages] + lane * kTileLd;
    const int c0 = t * 32;
    const int kmax = min(32, n - c0);
    if (my_row < n) {
      for (int k = 0; k < kmax; ++k) {
        const float v = row[k];
        sum += v;
        const uint32_t u = v == 0.0f ? 0u : __float_as_uint(v);
        h1 = (h1 ^ u) * 16777619u;
        h2 = h2 * 0x9E3779B1u + (u ^ (u >> 15));
        if (c0 + k == my_row) {
          if (!(v == 0.0f)) fl |= kRowBadDiag;
        } else if (v == 0.0f) {
          fl |= kRowZero;
        }
        if (v != v) fl |= kRowNan;
      }
    }
    __syncwarp();  // the stage is refilled by the next iteration's issue
  }
  cp_async_wait<0>();
  if (my_row < n) {
    sums[my_row] = sum;
    hashes[my_row] = make_uint2(h1, h2);
    flags[my_row] = fl;
  }
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

// Compare-exchange stages of the bitonic network over a[0, len) (shared memory,
// or a global row only this CTA touches) for merge size k, strides j0, j0/2,
// .., jend.  Element t of a is element base + t of the whole row: the direction
// of its pair is ascending when bit k of that index is clear.
__device__ __forceinline__ void bitonic_stages(unsigned long long *a, int len, long long base,
                                               long long k, int j0, int jend) {
  for (int j = j0; j >= jend; j >>= 1) {
    for (int q = threadIdx.x; q < (len >> 1); q += blockDim.x) {
      const int t = ((q & ~(j - 1)) << 1) | (q & (j - 1));  // bit j clear; partner t + j
      const bool asc = ((base + t) & k) == 0;
      const unsigned long long x = a[t], y = a[t + j];
      if ((x > y) == asc) {
        a[t] = y;
        a[t + j] = x;
      }
    }
    __syncthreads();
  }
}

// Pass 3: a CTA per unmarked row i (rows[], longest first): the unmarked j < i
// (rank[j] = unmarked rows below j, rank[i] of them in all) as keys, sorted, and
// the first min(rank[i], cap) written as (j, matrix[i][j]).  Rows longer than
// kSortBlock entries are sorted in this CTA's scratch row (P entries, P the
// next power of two): blocks of kSortBlock in shared memory first, then each
// merge's long strides in global memory and its short ones block by block.
__global__ void __launch_bounds__(kSortThreads)
    nj_sort_rows_kernel(const float *__restrict__ M, size_t ld, const int *__restrict__ rank,
                        const uint8_t *__restrict__ keep, const int *__restrict__ rows, int nrows,
                        unsigned long long *__restrict__ scratch, size_t scratch_per_cta,
                        rnj_cluster_pair *__restrict__ out, size_t out_ld, int cap) {
  extern __shared__ unsigned long long sk[];
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    const int cnt = rank[i];
    if (cnt == 0) continue;  // uniform over the CTA
    int P = 1;
    while (P < cnt) P <<= 1;
    const float *row = M + (size_t)i * ld;
    unsigned long long *a = P <= kSortBlock ? sk : scratch + (size_t)blockIdx.x * scratch_per_cta;
    for (int t = cnt + threadIdx.x; t < P; t += blockDim.x) a[t] = ~0ull;
    for (int j = threadIdx.x; j < i; j += blockDim.x)
      if (keep[j]) a[rank[j]] = sort_key(row[j], j);
    __syncthreads();
    if (P <= kSortBlock) {
      for (int k = 2; k <= P; k <<= 1) bitonic_stages(sk, P, 0, k, k >> 1, 1);
    } else {
      for (int b0 = 0; b0 < P; b0 += kSortBlock) {
        for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) sk[t] = a[b0 + t];
        __syncthreads();
        for (int k = 2; k <= kSortBlock; k <<= 1) bitonic_stages(sk, kSortBlock, b0, k, k >> 1, 1);
        for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) a[b0 + t] = sk[t];
        __syncthreads();
      }
      for (long long k = 2LL * kSortBlock; k <= P; k <<= 1) {
        for (int j = (int)(k >> 1); j >= kSortBlock; j >>= 1) bitonic_stages(a, P, 0, k, j, j);
        for (int b0 = 0; b0 < P; b0 += kSortBlock) {
          for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) sk[t] = a[b0 + t];
          __syncthreads();
          bitonic_stages(sk, kSortBlock, b0, k, kSortBlock >> 1, 1);
          for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) a[b0 + t] = sk[t];
          __syncthreads();
        }
      }
    }
    const int keepn = cap > 0 ? min(cnt, cap) : cnt;
    rnj_cluster_pair *o = out + (size_t)i * out_ld;
    for (int t = threadIdx.x; t < keepn; t += blockDim.x) {
      const uint32_t id = (uint32_t)a[t];
      rnj_cluster_pair cp;
      cp.id = id;
      cp.distance = row[id];  // the stored value, -0 kept
      o[t] = cp;
    }
    __syncthreads();  // the next row reuses the keys
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
  uint2 *d_hash = nullptr;
  uint32_t *d_flags = nullptr;
  NJ_CUDA(buf.alloc(&d_sums, (size_t)n * sizeof(float)), "nj buffers");
  NJ_CUDA(buf.alloc(&d_hash, (size_t)n * sizeof(uint2)), "nj buffers");
  NJ_CUDA(buf.alloc(&d_flags, (size_t)n * sizeof(uint32_t)), "nj buffers");
  const int warps = (n + 31) / 32;
  nj_row_pass_kernel<<<(warps + kRowWarps - 1) / kRowWarps, 32 * kRowWarps, 0, st>>>(
      d_matrix, n, ld, d_sums, d_hash, d_flags);
  NJ_CUDA(cudaGetLastError(), "nj row pass");
  std::vector<float> sums(n);
  std::vector<uint2> hash(n);
  std::vector<uint32_t> flags(n);
  NJ_CUDA(cudaMemcpyAsync(sums.data(), d_sums, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st),
          "nj copy");
  NJ_CUDA(cudaMemcpyAsync(hash.data(), d_hash, (size_t)n * sizeof(uint2), cudaMemcpyDeviceToHost, st),
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
    std::vector<int> cand;
    for (int i = 0; i < n; ++i)
      if ((flags[i] & kRowZero) && !(flags[i] & kRowNan)) cand.push_back(i);
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
    const int grid = (int)std::min<size_t>(rows.size(), (size_t)2 * ctx->num_sms);
    size_t pmax = 1;
    while (pmax < (size_t)rank[rows[0]]) pmax <<= 1;
    unsigned long long *d_scratch = nullptr;
    size_t per_cta = 0;
    if (pmax > (size_t)kSortBlock) {
      per_cta = pmax;
      NJ_CUDA(buf.alloc(&d_scratch, (size_t)grid * per_cta * sizeof(unsigned long long)),
              "nj sort scratch");
    }
    const int smem = kSortBlock * (int)sizeof(unsigned long long);
    NJ_CUDA(cudaFuncSetAttribute(nj_sort_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem),
            "nj sort attribute");
    nj_sort_rows_kernel<<<grid, kSortThreads, smem, st>>>(d_matrix, ld, d_rank, d_keep, d_rows,
                                                         (int)rows.size(), d_scratch, per_cta,
                                                         o->sorted, o->sorted_ld, cap);
    NJ_CUDA(cudaGetLastError(), "nj sort");
  }
  NJ_CUDA(cudaStreamSynchronize(st), "nj sync");
  return RNJ_OK;
}
