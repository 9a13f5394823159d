// rnj_text.cu -- the "-o m" text matrix formatted on the device
// (rnj_write_matrix_text_device).
//
// rapidNJ prints the matrix as "\t<n>\n", then per row the name, a tab and the n
// distances, each with six fixed decimals followed by a space, and a newline
// (printDistanceMatrix, main.cpp:212-221; iostream setprecision(6) << fixed, the
// same digits as printf("%.6f")).  For a float v the decimal digits are exact to
// compute: v * 10^6 = m * 15625 * 2^(e+6) with a 24-bit m needs at most 38
// significant bits, so the product in double is exact, and rounding it to an
// integer with ties to even (rint) is the correctly rounded 6-decimal value the C
// library prints; the sign is v's sign bit ("-0.000000" for -0 and for negative
// values that round to zero).  Values whose integer part needs more than ten
// digits (|v| >= 8e9), infinities and NaNs are printed by the host with
// snprintf, row by row.
//
// Pass 1 gives every row its length (a warp per row); the host turns the lengths
// into file offsets and cuts the rows into bands of at most 64 MB of text; per
// band a warp per row writes the name, the tab, the values (a warp scan of the
// values' lengths places them) and the newline; the band comes down into one of
// two page-locked buffers while the next band is formatted, and is written to
// the file in one call.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

constexpr size_t kBandBytes = (size_t)64 << 20;  // text per band (at most; a row may exceed it)
constexpr float kHostValue = 8e9f;               // |v| from here on: printed by the host

__device__ __forceinline__ bool device_value(float v) { return isfinite(v) && fabsf(v) < kHostValue; }

// The rounded value |v| * 10^6 as an integer (exact, see the file comment).
__device__ __forceinline__ uint64_t scaled(float v) {
  return (uint64_t)rint(fabs((double)v * 1e6));
}

__device__ __forceinline__ int int_digits(uint64_t ip) {
  int d = 1;
  while (ip >= 10) {
    ip /= 10;
    ++d;
  }
  return d;
}

// Characters of "%.6f " for a device value.
__device__ __forceinline__ int value_len(float v) {
  return (signbit(v) ? 1 : 0) + int_digits(scaled(v) / 1000000u) + 8;
}

__device__ __forceinline__ void value_write(char *o, float v) {
  const uint64_t u = scaled(v);
  uint64_t ip = u / 1000000u;
  uint32_t fp = (uint32_t)(u % 1000000u);
  int k = 0;
  if (signbit(v)) o[k++] = '-';
  const int nd = int_digits(ip);
  for (int d = nd - 1; d >= 0; --d) {
    o[k + d] = (char)('0' + ip % 10);
    ip /= 10;
  }
  k += nd;
  o[k++] = '.';
  for (int d = 5; d >= 0; --d) {
    o[k + d] = (char)('0' + fp % 10);
    fp /= 10;
  }
  k += 6;
  o[k] = ' ';
}

// Pass 1: a warp per row: the row's text length (name, tab, values, newline)
// and whether the host must print it.
__global__ void __launch_bounds__(256)
    text_lengths_kernel(const float *__restrict__ M, size_t ld, int n,
                        const int *__restrict__ name_off, int64_t *__restrict__ len,
                        uint8_t *__restrict__ host_row) {
  const int lane = threadIdx.x & 31;
  const int stride = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += stride) {
    const float *row = M + (size_t)r * ld;
    int64_t s = 0;
    bool host = false;
    for (int j = lane; j < n; j += 32) {
      const float v = row[j];
      if (device_value(v)) s += value_len(v);
      else host = true;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    host = __any_sync(0xffffffffu, host);
    if (lane == 0) {
      len[r] = (int64_t)(name_off[r + 1] - name_off[r]) + 1 + s + 1;
      host_row[r] = host ? 1 : 0;
    }
  }
}

// Pass 2: rows [r0, r1) into out (row r at off[r] - off[r0]); host rows skipped.
__global__ void __launch_bounds__(256)
    text_rows_kernel(const float *__restrict__ M, size_t ld, int n, int r0, int r1,
                     const char *__restrict__ names, const int *__restrict__ name_off,
                     const int64_t *__restrict__ off, const uint8_t *__restrict__ host_row,
                     char *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int stride = (gridDim.x * blockDim.x) >> 5;
  for (int r = r0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < r1; r += stride) {
    if (host_row[r]) continue;  // uniform per warp
    char *o = out + (off[r] - off[r0]);
    const int nl = name_off[r + 1] - name_off[r];
    for (int k = lane; k < nl; k += 32) o[k] = names[name_off[r] + k];
    if (lane == 0) o[nl] = '\t';
    int64_t base = nl + 1;
    const float *row = M + (size_t)r * ld;
    for (int j0 = 0; j0 < n; j0 += 32) {
      const int j = j0 + lane;
      const float v = j < n ? row[j] : 0.0f;
      const int l = j < n ? value_len(v) : 0;
      int incl = l;
#pragma unroll
      for (int s = 1; s < 32; s <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, s);
        if (lane >= s) incl += y;
      }
      if (j < n) value_write(o + base + (incl - l), v);
      base += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) o[base] = '\n';
  }
}

// "%.6f " of one value by the C library, as the host writer prints it.
inline int host_value(char *out, float v) { return snprintf(out, 64, "%.6f ", (double)v); }

#define TEXT_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_error(e_, what);  \
  } while (0)

struct TextBuffers {
  cudaStream_t s;
  std::vector<void *> dev;
  explicit TextBuffers(cudaStream_t st) : s(st) {}
  template <class T>
  cudaError_t alloc(T **p, size_t bytes) {
    cudaError_t e = cudaMallocAsync((void **)p, std::max<size_t>(bytes, 16), s);
    if (e == cudaSuccess) dev.push_back((void *)*p);
    return e;
  }
  ~TextBuffers() {
    cudaStreamSynchronize(s);
    for (void *p : dev) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  }
};

int write_all(FILE *f, const char *p, size_t k) {
  if (k && fwrite(p, 1, k, f) != k) return set_error(RNJ_ERR_IO, "write to the output file failed");
  return RNJ_OK;
}

}  // namespace

extern "C" int rnj_write_matrix_text_device(rnj_ctx *ctx, const char *path,
                                            const char *const *names, const float *d_matrix,
                                            size_t ld, int n) {
  if (!ctx || n < 0 || (n > 0 && (!names || !d_matrix)))
    return set_error(RNJ_ERR_INVALID, "null argument");
  if (n > 0 && ld < (size_t)n) return set_error(RNJ_ERR_INVALID, "ld < n");
  DeviceGuard guard(ctx->device);
  cudaStream_t st = ctx->stream;
  FILE *f = path ? fopen(path, "wb") : stdout;
  if (!f) return set_error(RNJ_ERR_IO, std::string("Could not open the output file \"") + path + "\"");
  struct Closer {
    FILE *f;
    bool own;
    ~Closer() {
      if (own) fclose(f);
      else fflush(f);
    }
  } closer{f, path != nullptr};
  char head[32];
  int rc = write_all(f, head, (size_t)snprintf(head, sizeof head, "\t%d\n", n));
  if (rc != RNJ_OK || n == 0) return rc;

  TextBuffers buf(st);
  // Names: concatenated bytes and offsets.
  std::vector<int> name_off(n + 1, 0);
  for (int i = 0; i < n; ++i) name_off[i + 1] = name_off[i] + (int)strlen(names[i] ? names[i] : "");
  std::vector<char> name_bytes((size_t)name_off[n] + 1);
  for (int i = 0; i < n; ++i)
    if (names[i]) memcpy(name_bytes.data() + name_off[i], names[i], name_off[i + 1] - name_off[i]);
  char *d_names = nullptr;
  int *d_name_off = nullptr;
  int64_t *d_len = nullptr;
  uint8_t *d_host = nullptr;
  TEXT_CUDA(buf.alloc(&d_names, name_bytes.size()), "text buffers");
  TEXT_CUDA(buf.alloc(&d_name_off, (size_t)(n + 1) * sizeof(int)), "text buffers");
  TEXT_CUDA(buf.alloc(&d_len, (size_t)(n + 1) * sizeof(int64_t)), "text buffers");
  TEXT_CUDA(buf.alloc(&d_host, (size_t)n), "text buffers");
  TEXT_CUDA(cudaMemcpyAsync(d_names, name_bytes.data(), name_bytes.size(), cudaMemcpyHostToDevice, st),
            "names upload");
  TEXT_CUDA(cudaMemcpyAsync(d_name_off, name_off.data(), (size_t)(n + 1) * sizeof(int),
                            cudaMemcpyHostToDevice, st),
            "names upload");
  const unsigned grid = (unsigned)std::min<long long>(((long long)n * 32 + 255) / 256,
                                                      (long long)ctx->num_sms * 16);
  text_lengths_kernel<<<grid, 256, 0, st>>>(d_matrix, ld, n, d_name_off, d_len, d_host);
  TEXT_CUDA(cudaGetLastError(), "text lengths");
  std::vector<int64_t> off(n + 1);
  std::vector<uint8_t> host_row(n);
  TEXT_CUDA(cudaMemcpyAsync(off.data(), d_len, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, st),
            "text copy");
  TEXT_CUDA(cudaMemcpyAsync(host_row.data(), d_host, (size_t)n, cudaMemcpyDeviceToHost, st), "text copy");
  TEXT_CUDA(cudaStreamSynchronize(st), "text lengths sync");
  // Rows the host prints: their text now, their true lengths into the offsets.
  std::vector<std::string> host_text(n);
  {
    std::vector<float> row;
    char tmp[64];
    for (int r = 0; r < n; ++r) {
      if (!host_row[r]) continue;
      row.resize(n);
      TEXT_CUDA(cudaMemcpy(row.data(), d_matrix + (size_t)r * ld, (size_t)n * sizeof(float),
                           cudaMemcpyDeviceToHost),
                "row copy");
      std::string &s = host_text[r];
      s.append(names[r] ? names[r] : "");
      s.push_back('\t');
      for (int j = 0; j < n; ++j) s.append(tmp, host_value(tmp, row[j]));
      s.push_back('\n');
      off[r] = (int64_t)s.size();
    }
  }
  int64_t run = 0;  // lengths -> offsets
  for (int r = 0; r < n; ++r) {
    const int64_t l = off[r];
    off[r] = run;
    run += l;
  }
  off[n] = run;
  TEXT_CUDA(cudaMemcpyAsync(d_len, off.data(), (size_t)(n + 1) * sizeof(int64_t),
                            cudaMemcpyHostToDevice, st),
            "offsets upload");
  // Bands of rows with at most kBandBytes of text (one row at least).
  std::vector<int> band{0};
  size_t cap = 0;
  while (band.back() < n) {
    const int r0 = band.back();
    int r1 = r0 + 1;
    while (r1 < n && (size_t)(off[r1 + 1] - off[r0]) <= kBandBytes) ++r1;
    cap = std::max(cap, (size_t)(off[r1] - off[r0]));
    band.push_back(r1);
  }
  const int nb = (int)band.size() - 1;
  // Two page-locked band buffers: the context's staging buffer (shared with
  // rnj_msa_read_device), grown when needed.
  if (ctx->h_file_cap < 2 * cap) {
    if (ctx->h_file) cudaFreeHost(ctx->h_file);
    ctx->h_file = nullptr;
    ctx->h_file_cap = 0;
    TEXT_CUDA(cudaMallocHost((void **)&ctx->h_file, 2 * cap), "page-locked text buffers");
    ctx->h_file_cap = 2 * cap;
  }
  char *d_text[2] = {nullptr, nullptr}, *h_text[2] = {ctx->h_file, ctx->h_file + cap};
  cudaEvent_t done[2] = {nullptr, nullptr};
  for (int k = 0; k < 2 && k < nb; ++k) {
    TEXT_CUDA(buf.alloc(&d_text[k], cap), "text buffers");
    TEXT_CUDA(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming), "event");
  }
  struct Events {
    cudaEvent_t *e;
    ~Events() {
      for (int k = 0; k < 2; ++k)
        if (e[k]) cudaEventDestroy(e[k]);
    }
  } events{done};
  auto enqueue = [&](int b) -> int {
    const int k = b & 1;
    const int r0 = band[b], r1 = band[b + 1];
    const unsigned g = (unsigned)std::min<long long>(((long long)(r1 - r0) * 32 + 255) / 256,
                                                     (long long)ctx->num_sms * 16);
    text_rows_kernel<<<g, 256, 0, st>>>(d_matrix, ld, n, r0, r1, d_names, d_name_off, d_len, d_host,
                                        d_text[k]);
    TEXT_CUDA(cudaGetLastError(), "text rows");
    TEXT_CUDA(cudaMemcpyAsync(h_text[k], d_text[k], (size_t)(off[r1] - off[r0]),
                              cudaMemcpyDeviceToHost, st),
              "text copy");
    TEXT_CUDA(cudaEventRecord(done[k], st), "event");
    return RNJ_OK;
  };
  rc = enqueue(0);
  if (rc != RNJ_OK) return rc;
  for (int b = 0; b < nb; ++b) {
    // The next band is formatted and copied while this one is written.  Its
    // buffer (b + 1) & 1 held band b - 1, which was written before this turn.
    if (b + 1 < nb) {
      rc = enqueue(b + 1);
      if (rc != RNJ_OK) return rc;
    }
    const int k = b & 1;
    TEXT_CUDA(cudaEventSynchronize(done[k]), "text band sync");
    const int r0 = band[b], r1 = band[b + 1];
    for (int r = r0; r < r1; ++r)
      if (host_row[r]) memcpy(h_text[k] + (off[r] - off[r0]), host_text[r].data(), host_text[r].size());
    rc = write_all(f, h_text[k], (size_t)(off[r1] - off[r0]));
    if (rc != RNJ_OK) return rc;
  }
  return RNJ_OK;
}
