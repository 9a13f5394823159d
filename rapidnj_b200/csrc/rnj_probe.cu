// rnj_probe.cu -- microbenchmark of the integer pipes the counting kernels are
// bound by: POPC (population count) and LOP3 (three-input logic) throughput of
// the whole device, in operations per second.  The distance kernels report their
// achieved rates against these measured peaks.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "rnj.h"
#include "rnj_device.cuh"
#include "rnj_internal.h"

namespace rnj {

constexpr int kProbeIters = 4096;

// 8 independent chains per thread; every op is a real popc.b32 whose result
// feeds the next, and the final values are stored so nothing is dead code.
__global__ void __launch_bounds__(256) probe_popc_kernel(uint32_t seed, uint32_t *out) {
  uint32_t x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = seed ^ (threadIdx.x * 2654435761u + k * 40503u + blockIdx.x);
  for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      uint32_t p;
      asm volatile("popc.b32 %0, %1;" : "=r"(p) : "r"(x[k]));
      x[k] ^= p;
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) probe_lop3_kernel(uint32_t seed, uint32_t *out) {
  uint32_t x[8], y = seed * 747796405u + threadIdx.x, z = seed ^ 0x9e3779b9u ^ blockIdx.x;
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = seed ^ (threadIdx.x * 2654435761u + k * 40503u);
  for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[k]) : "r"(y), "r"(z));
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace rnj

using namespace rnj;

extern "C" int rnj_probe_int_peaks(rnj_ctx *ctx, double *popc_per_s, double *lop3_per_s) {
  if (!ctx) return set_error(RNJ_ERR_INVALID, "null context");
  void *sv = nullptr;
  int rc = rnj_ctx_stream(ctx, &sv);
  if (rc != RNJ_OK) return rc;
  cudaStream_t s = (cudaStream_t)sv;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256;
  uint32_t *out = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&out, (size_t)blocks * threads * 4, s);
  if (e != cudaSuccess) return cuda_error(e, "probe buffer");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const double ops = (double)blocks * threads * 8.0 * kProbeIters;
  double best[2] = {0, 0};
  for (int which = 0; which < 2; ++which) {
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(a, s);
      if (which == 0) probe_popc_kernel<<<blocks, threads, 0, s>>>(rep + 1, out);
      else probe_lop3_kernel<<<blocks, threads, 0, s>>>(rep + 1, out);
      cudaEventRecord(b, s);
      e = cudaEventSynchronize(b);
      if (e != cudaSuccess) break;
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0 && ms > 0) best[which] = std::max(best[which], ops / (ms * 1e-3));
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(out, s);
  if (e != cudaSuccess) return cuda_error(e, "probe kernels");
  if (popc_per_s) *popc_per_s = best[0];
  if (lop3_per_s) *lop3_per_s = best[1];
  return RNJ_OK;
}

// FP4 tensor-pipe peak: every SM issues back-to-back 128 x 128 x 64 kind::mxf4
// MMAs (2 * 128 * 128 * 64 flops each); best of three launches.
extern "C" int rnj_probe_tc_peak(rnj_ctx *ctx, double *fp4_flops_per_s) {
  if (!ctx || !fp4_flops_per_s) return set_error(RNJ_ERR_INVALID, "null argument");
  void *sv = nullptr;
  int rc = rnj_ctx_stream(ctx, &sv);
  if (rc != RNJ_OK) return rc;
  cudaStream_t s = (cudaStream_t)sv;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int iters = 16384;
  int *err = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&err, sizeof(int), s);
  if (e != cudaSuccess) return cuda_error(e, "probe flag");
  e = cudaMemsetAsync(err, 0, sizeof(int), s);
  cudaEvent_t a = nullptr, b = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  double best = 0.0;
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    cudaEventRecord(a, s);
    e = launch_tc_peak_probe(sms, iters, err, s);
    cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.0f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
    if (rep > 0 && ms > 0.0f)
      best = std::max(best, (double)sms * iters * 2.0 * 128 * 128 * 64 / (ms * 1e-3));
  }
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFreeAsync(err, s);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_error(e, "tensor-pipe probe");
  if (h_err) return set_error(RNJ_ERR_TIMEOUT, "tensor-pipe probe: a bounded wait ran out");
  *fp4_flops_per_s = best;
  return RNJ_OK;
}

namespace rnj {

// Every (num, d) with 1 <= d < 2^16 and 0 <= num <= d (block d, threads over
// num): quotient16 against the correctly rounded float division and against
// the reference's double division rounded to float; mismatches counted.
__global__ void __launch_bounds__(256) quotient16_check_kernel(unsigned long long *mismatches) {
  const uint32_t d = blockIdx.x + 1;
  const float fd = (float)d, y = recip16(fd);
  unsigned long long bad = 0;
  for (uint32_t num = threadIdx.x; num <= d; num += blockDim.x) {
    const float q = quotient16(num, fd, y);
    const float f = __fdiv_rn((float)num, fd);
    const float g = __double2float_rn(__ddiv_rn((double)num, (double)d));
    bad += (__float_as_uint(q) != __float_as_uint(f)) + (__float_as_uint(q) != __float_as_uint(g));
  }
  if (bad) atomicAdd(mismatches, bad);
}

// Every float p in [0, 1] (2^30 + 1 values; thread t of the grid takes the
// floats with bit patterns t, t + stride, ...): div_by_b against the correctly
// rounded double division for b = 3/4 and b = 19/20, the two JC constants.
__global__ void __launch_bounds__(256) jc_quotient_check_kernel(unsigned long long *mismatches) {
  const double b4 = (4.0 - 1) / 4.0, b20 = (20.0 - 1) / 20.0;
  const double y4 = __ddiv_rn(1.0, b4), y20 = __ddiv_rn(1.0, b20);
  unsigned long long bad = 0;
  const uint32_t one = 0x3F800000u;  // the bits of 1.0f: floats in [0, 1] are 0 .. one
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= one;
       u += gridDim.x * blockDim.x) {
    const double p = (double)__uint_as_float(u);
    bad += __double_as_longlong(div_by_b(p, b4, y4)) != __double_as_longlong(__ddiv_rn(p, b4));
    bad += __double_as_longlong(div_by_b(p, b20, y20)) != __double_as_longlong(__ddiv_rn(p, b20));
  }
  if (bad) atomicAdd(mismatches, bad);
}

}  // namespace rnj

// The fused epilogue's quotients over their whole domain: the float quotients
// (quotient16) and the JC double quotients (div_by_b).
extern "C" int rnj_check_quotient16(rnj_ctx *ctx, unsigned long long *mismatches) {
  if (!ctx || !mismatches) return set_error(RNJ_ERR_INVALID, "null argument");
  void *sv = nullptr;
  int rc = rnj_ctx_stream(ctx, &sv);
  if (rc != RNJ_OK) return rc;
  cudaStream_t s = (cudaStream_t)sv;
  unsigned long long *d_bad = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&d_bad, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_error(e, "check counter");
  e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) {
    rnj::quotient16_check_kernel<<<(1u << 16) - 1, 256, 0, s>>>(d_bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    rnj::jc_quotient_check_kernel<<<148 * 16, 256, 0, s>>>(d_bad);
    e = cudaGetLastError();
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_bad, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(d_bad, s);
  if (e != cudaSuccess) return cuda_error(e, "quotient check");
  *mismatches = h;
  return RNJ_OK;
}
