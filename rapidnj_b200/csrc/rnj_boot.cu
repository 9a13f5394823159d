// rnj_boot.cu -- bootstrap replicates on the device.
//
// rapidNJ's bootstrap (main.cpp:519-532) re-runs the whole distance computation
// once per replicate on an alignment whose column k is column rand() % L of the
// original (dataloader::sample_fast_dist, dataloader.cpp:16-58).  Here the
// original bytes stay on the device: a gather kernel writes the replicates'
// bytes (column k of replicate r = column cols[r * L + k]), and the replicates
// of a chunk are packed and counted together as one batch (one presence scan,
// one pack launch per layout, one persistent launch per kernel family).  The
// caller draws the columns, so the replicates are exactly rapidNJ's when it
// draws them with the same rand() sequence.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

// out[r][i][k] = chars[i][cols[r][k]] for replicates r0 .. r0 + nr - 1: a
// thread per (replicate, row, 4 columns); the column indices are read once per
// row from L1/L2, the source row is gathered byte by byte, the output written
// as 32-bit words when L allows it.
__global__ void __launch_bounds__(256) gather_columns_kernel(const uint8_t *__restrict__ chars,
                                                             size_t ld, int n, int L,
                                                             const int *__restrict__ cols,
                                                             int nr, uint8_t *__restrict__ out) {
  const int q = (L + 3) / 4;
  const long long total = (long long)nr * n * q;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k4 = (int)(t % q);
    const long long ri = t / q;
    const int i = (int)(ri % n), r = (int)(ri / n);
    const uint8_t *src = chars + (size_t)i * ld;
    const int *c = cols + (size_t)r * L;
    uint8_t *dst = out + ((size_t)r * n + i) * L;
    const int k0 = 4 * k4;
    if ((L & 3) == 0) {
      const uint32_t w = (uint32_t)src[c[k0]] | ((uint32_t)src[c[k0 + 1]] << 8) |
                         ((uint32_t)src[c[k0 + 2]] << 16) | ((uint32_t)src[c[k0 + 3]] << 24);
      *reinterpret_cast<uint32_t *>(dst + k0) = w;
    } else {
      for (int k = k0; k < min(L, k0 + 4); ++k) dst[k] = src[c[k]];
    }
  }
}

}  // namespace

extern "C" int rnj_bootstrap(rnj_ctx *ctx, const void *d_chars, int n, int L, size_t ld, int type,
                             int model, int flags, int R, const int *cols, float *const *d_out,
                             size_t ld_out, float *max_out) {
  if (!ctx || (!d_chars && n > 0 && L > 0) || (!cols && R > 0 && L > 0) || (!d_out && R > 0))
    return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 1 || L < 1 || R < 0 || ld < (size_t)L || ld_out < (size_t)n)
    return set_error(RNJ_ERR_INVALID, "invalid bootstrap shape");
  if (type != RNJ_DNA && type != RNJ_PROTEIN)
    return set_error(RNJ_ERR_INVALID, "type must be RNJ_DNA or RNJ_PROTEIN");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  for (long long k = 0; k < (long long)R * L; ++k)
    if (cols[k] < 0 || cols[k] >= L) return set_error(RNJ_ERR_INVALID, "column index out of range");
  for (int r = 0; r < R; ++r)
    if (!d_out[r]) return set_error(RNJ_ERR_INVALID, "null output matrix");
  if (R == 0) return RNJ_OK;
  if (tri_tiles(tiles_of(n)) > 8LL * kTcChunkTiles)
    return set_error(RNJ_ERR_INVALID, "bootstrap replicates of more than " +
                                          std::to_string(kTile * 255) +
                                          " sequences are not batched; use rnj_distance per replicate");
  DeviceGuard guard(ctx->device);
  // Replicates per chunk: gathered bytes up to 1 GiB, tiles within one batch.
  const long long rep_bytes = (long long)n * L;
  const long long rep_tiles = tri_tiles(tiles_of(n));
  int chunk = (int)std::max<long long>(1, std::min<long long>(R, (1LL << 30) / rep_bytes));
  chunk = (int)std::min<long long>(chunk, std::max<long long>(1, (8LL * kTcChunkTiles) / rep_tiles));
  // The context keeps the batch (its graph and buffers) for later calls of the
  // same or a smaller size.
  int rc = RNJ_OK;
  if (!ctx->boot || ctx->boot_aln < chunk || ctx->boot_tiles < (long long)chunk * rep_tiles) {
    if (ctx->boot) rnj_batch_destroy(ctx->boot);
    ctx->boot = nullptr;
    rc = rnj_batch_create(ctx, chunk, (long long)chunk * rep_tiles, &ctx->boot);
    if (rc != RNJ_OK) return rc;
    ctx->boot_aln = chunk;
    ctx->boot_tiles = (long long)chunk * rep_tiles;
  }
  rnj_batch *b = ctx->boot;
  uint8_t *d_rep = nullptr;
  int *d_cols = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&d_rep, (size_t)chunk * rep_bytes, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMallocAsync((void **)&d_cols, (size_t)chunk * L * sizeof(int), ctx->stream);
  std::vector<const void *> ptrs(chunk);
  std::vector<int> ns(chunk, n), Ls(chunk, L), types(chunk, type), models(chunk, model);
  std::vector<size_t> lds(chunk, (size_t)L), ldo(chunk, ld_out);
  std::vector<int> slots(chunk);
  for (int r0 = 0; r0 < R && e == cudaSuccess && rc == RNJ_OK; r0 += chunk) {
    const int nr = std::min(chunk, R - r0);
    e = cudaMemcpyAsync(d_cols, cols + (size_t)r0 * L, (size_t)nr * L * sizeof(int),
                        cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) break;
    const long long work = (long long)nr * n * ((L + 3) / 4);
    long long g = std::min<long long>((work + 255) / 256, 148LL * 32);
    gather_columns_kernel<<<(unsigned)std::max<long long>(g, 1), 256, 0, ctx->stream>>>(
        (const uint8_t *)d_chars, ld, n, L, d_cols, nr, d_rep);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    for (int k = 0; k < nr; ++k) ptrs[k] = d_rep + (size_t)k * rep_bytes;
    rc = rnj_batch_add_many(b, nr, ptrs.data(), ns.data(), Ls.data(), lds.data(), types.data(),
                            models.data(), flags, d_out + r0, ldo.data(),
                            slots.data());
    if (rc == RNJ_OK) rc = rnj_batch_run(b);
    if (rc == RNJ_OK) rc = rnj_batch_synchronize(b);
    for (int k = 0; k < nr && rc == RNJ_OK; ++k)
      rc = rnj_batch_output(b, slots[k], nullptr, nullptr, max_out ? max_out + r0 + k : nullptr);
    if (rc == RNJ_OK) rc = rnj_batch_clear(b);
  }
  if (d_rep) cudaFreeAsync(d_rep, ctx->stream);
  if (d_cols) cudaFreeAsync(d_cols, ctx->stream);
  const cudaError_t es = cudaStreamSynchronize(ctx->stream);
  if (rc != RNJ_OK) rnj_batch_clear(b);
  if (rc != RNJ_OK) return rc;
  if (e != cudaSuccess) return cuda_error(e, "bootstrap");
  if (es != cudaSuccess) return cuda_error(es, "bootstrap sync");
  return RNJ_OK;
}
