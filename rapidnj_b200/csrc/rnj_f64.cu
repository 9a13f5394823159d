// rnj_f64.cu -- the distance matrix in double precision: each pair's value is
// the reference's double expression before its cast to distType (float), so
// that the transform can be compared with the reference's doubles (and a
// caller can keep the extra precision).
//
// The counts come from the counting kernels (rnj_counts_into: tensor cores or
// bit planes, exact integers); a pair kernel evaluates the reference's
// arithmetic operation by operation in double with explicitly rounded
// intrinsics (no contraction; the reference's x86-64 build has none) and CUDA's
// double log (within one ulp of glibc's); then the post-process of
// KimuraDistance.cpp:366-395 / JCdistance.cpp:201-230 in double: the maximum
// over the doubles, saturated pairs (-1) set to twice it, the lower triangle
// mirrored (unless the alignment asked for full rows), the diagonal 0.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "rnj.h"
#include "rnj_device.cuh"
#include "rnj_epilogue.cuh"
#include "rnj_internal.h"
#include "rnj_objects.h"

namespace rnj {
namespace {

// JCdistance.cpp:171-183: p = (float) total / (float) valid (0 when valid is
// 0); -1 when p / b >= 1; else -b log(1 - p / b), all in double.
__device__ double jc_double(unsigned long long total, unsigned long long valid, double b) {
  const float p = valid == 0 ? 0.0f
                             : __fdiv_rn(__ll2float_rn((long long)total), __ull2float_rn(valid));
  const double q = __ddiv_rn((double)p, b);
  if (q >= 1.0) return -1.0;
  return __dmul_rn(-b, log(__dsub_rn(1.0, q)));
}

// KimuraDistance.cpp:339-349: -1 when valid is 0 or 1 - 2 ts - tv or 1 - 2 tv
// (as floats) is not positive; else -0.5 log(1 - 2 ts - tv) - 0.25 log(1 - 2 tv)
// in double from the float quotients.
__device__ double k2p_double(unsigned long long P, unsigned long long Q,
                             unsigned long long valid) {
  if (valid == 0) return -1.0;
  const float ts = __double2float_rn(__ddiv_rn((double)P, (double)valid));
  const float tv = __double2float_rn(__ddiv_rn((double)Q, (double)valid));
  const double a = __dsub_rn(__dsub_rn(1.0, __dmul_rn(2.0, (double)ts)), (double)tv);
  const double b = __dsub_rn(1.0, __dmul_rn(2.0, (double)tv));
  if (__double2float_rn(a) <= 0.0f || __double2float_rn(b) <= 0.0f) return -1.0;
  return __dsub_rn(__dmul_rn(-0.5, log(a)), __dmul_rn(0.25, log(b)));
}

// KimuraDistance.cpp:322-338 with the Dayhoff table of KimuraDistance.cpp:30-49.
__device__ double kimura_protein_double(unsigned long long mism, unsigned long long valid) {
  float p = -1.0f;
  if (valid != 0) p = __fdiv_rn(__ll2float_rn((long long)mism), __ull2float_rn(valid));
  const double dp = (double)p;
  if (dp < 0.75) {
    if (dp > 0.0) {
      const double sq = (double)__fmul_rn(p, p);
      return -log(__dsub_rn(__dsub_rn(1.0, dp), __dmul_rn(sq, 0.20)));
    }
    return dp;  // 0, or -1 (no valid site)
  }
  if (dp > 0.930) return 10.0;
  const int idx = (int)__dsub_rn(__dmul_rn(dp, 1000.0), 750.0);
  return __ddiv_rn((double)c_pam.x100[idx], 100.0);
}

struct F64Params {
  const uint32_t *counts;  // n x n x 3
  double *out;
  size_t ld;
  int n, L, model, type, compat, full;
  double jc_b;
  unsigned long long *max_bits;  // the maximum (non-negative doubles order as their bits)
  int *saturated;
};

__device__ double pair_double(const F64Params &f, const uint32_t *c) {
  unsigned long long valid = c[2];
  if (f.compat) valid = protein_fast_valid(valid, f.L);
  if (f.model == RNJ_JC) return jc_double((unsigned long long)c[0] + c[1], valid, f.jc_b);
  if (f.type == RNJ_PROTEIN) return kimura_protein_double(c[0], valid);
  return k2p_double(c[0], c[1], valid);
}

// One thread per (i, j), j > i (every j != i with full rows): the raw value
// into out[i][j] and, unless full, out[j][i]; the diagonal 0.
__global__ void __launch_bounds__(256) f64_pairs_kernel(F64Params f) {
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (i >= f.n || j >= f.n) return;
  if (i == j) {
    f.out[(size_t)i * f.ld + j] = 0.0;
    return;
  }
  if (!f.full && j < i) return;
  const double d = pair_double(f, f.counts + ((size_t)i * f.n + j) * 3);
  if (d > 0.0) atomicMax(f.max_bits, (unsigned long long)__double_as_longlong(d));
  if (d == -1.0) *f.saturated = 1;
  f.out[(size_t)i * f.ld + j] = d;
  if (!f.full) f.out[(size_t)j * f.ld + i] = d;
}

// -1 -> 2 x the maximum (only launched when a pair saturated).
__global__ void __launch_bounds__(256) f64_fixup_kernel(F64Params f) {
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (i >= f.n || j >= f.n || i == j) return;
  double *o = f.out + (size_t)i * f.ld + j;
  if (*o == -1.0) *o = 2.0 * __longlong_as_double((long long)*f.max_bits);
}

}  // namespace
}  // namespace rnj

using namespace rnj;

#define RNJ_CUDA(call, what)                            \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

extern "C" int rnj_distance_f64(rnj_ctx *ctx, rnj_aln *aln, int model, double *d_out, size_t ld,
                                double *max_out) {
  if (!ctx || !aln || (!d_out && aln->p.n > 0)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  const Packed &p = aln->p;
  if (ld < (size_t)p.n) return set_error(RNJ_ERR_INVALID, "ld smaller than n");
  if (max_out) *max_out = 0.0;
  if (p.n == 0) return RNJ_OK;
  DeviceGuard g(ctx->device);
  const size_t nc = (size_t)p.n * p.n * 3;
  uint32_t *counts = nullptr;
  unsigned long long *words = nullptr;  // [0] max bits, [1] saturated
  RNJ_CUDA(cudaMallocAsync((void **)&counts, nc * sizeof(uint32_t), ctx->stream), "count buffer");
  cudaError_t e = cudaMallocAsync((void **)&words, 2 * sizeof(unsigned long long), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(words, 0, 2 * sizeof(unsigned long long), ctx->stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(counts, ctx->stream);
    return cuda_error(e, "f64 scratch");
  }
  auto release = [&]() {
    cudaFreeAsync(counts, ctx->stream);
    cudaFreeAsync(words, ctx->stream);
  };
  int rc = rnj_counts_into(ctx, aln, counts);
  if (rc != RNJ_OK) {
    release();
    return rc;
  }
  const EpiParams ep = epi_params_for(p, model);
  F64Params f;
  f.counts = counts;
  f.out = d_out;
  f.ld = ld;
  f.n = p.n;
  f.L = p.L;
  f.model = model;
  f.type = p.type;
  f.compat = ep.compat_wrap;
  f.full = (p.flags & RNJ_FULL_ROWS) ? 1 : 0;
  f.jc_b = ep.jc_b;
  f.max_bits = words;
  f.saturated = reinterpret_cast<int *>(words + 1);
  const dim3 grid((unsigned)((p.n + 31) / 32), (unsigned)((p.n + 7) / 8));
  f64_pairs_kernel<<<grid, 256, 0, ctx->stream>>>(f);
  e = cudaGetLastError();
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, words, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && h[1]) {
    f64_fixup_kernel<<<grid, 256, 0, ctx->stream>>>(f);
    e = cudaGetLastError();
  }
  release();
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "f64 distance kernels");
  if (max_out) {
    const long long bits = (long long)h[0];
    memcpy(max_out, &bits, sizeof(double));
  }
  return RNJ_OK;
}
