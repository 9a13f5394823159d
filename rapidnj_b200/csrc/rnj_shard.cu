// rnj_shard.cu -- one alignment split over several GPUs by triangle tiles.
//
// Pairs are independent, so the only step that couples GPUs is the saturation
// cap of the post-process (KimuraDistance.cpp:366-395, JCdistance.cpp:201-230):
// every -1 becomes twice the maximum over the WHOLE matrix.  A shard therefore
// runs its contiguous range of tiles through the persistent work-list kernels
// (the same kernels the batched form uses, with a work list of this shard's
// tiles), reports its local maximum, and after the caller's one-float max
// exchange rewrites its flagged tiles with the global cap.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

#define RNJ_CUDA(call, what)                            \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

struct rnj_shard {
  rnj_ctx *ctx = nullptr;
  rnj_aln *aln = nullptr;
  int model = RNJ_KIMURA;
  int full = 0;
  long long t0 = 0, t1 = 0, ntiles = 0;
  float *out = nullptr;
  size_t ld = 0;
  bool owns_out = false;
  AlnDesc *d_desc = nullptr;
  WorkItem *d_items = nullptr;
  int *d_ints = nullptr;   // [0] items of this shard, [1] item counter, [2] zero
  int *d_words = nullptr;  // [0] max bits, [1] error word, [2..] tile flags of every tile
};

namespace {

long long tiles_for(int n, int full) {
  const int nt = tiles_of(n);
  return full ? (long long)nt * nt : tri_tiles(nt);
}

// Start of tile row r in the row-major upper triangle of nt x nt tiles.
long long row_start(int nt, int r) { return (long long)r * nt - (long long)r * (r - 1) / 2; }

void coords(int nt, int full, long long t, int &ti, int &tj) {
  if (full) {
    ti = (int)(t / nt);
    tj = (int)(t % nt);
    return;
  }
  int lo = 0, hi = nt - 1;  // last row whose start is <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (row_start(nt, mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  ti = lo;
  tj = lo + (int)(t - row_start(nt, lo));
}

void free_shard(rnj_shard *s) {
  if (!s) return;
  cudaStream_t st = s->ctx->stream;
  cudaStreamSynchronize(st);
  if (s->owns_out && s->out) cudaFreeAsync(s->out, st);
  if (s->d_desc) cudaFreeAsync(s->d_desc, st);
  if (s->d_items) cudaFreeAsync(s->d_items, st);
  if (s->d_ints) cudaFreeAsync(s->d_ints, st);
  if (s->d_words) cudaFreeAsync(s->d_words, st);
  delete s;
}

int read_words(rnj_shard *s, float *max_out) {
  rnj_ctx *ctx = s->ctx;
  RNJ_CUDA(cudaMemcpyAsync(ctx->h_max, s->d_words, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "shard words copy");
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "shard sync");
  if (ctx->h_max[1] != 0)
    return set_error(RNJ_ERR_TIMEOUT, "a bounded device wait ran out (pipeline stage lost)");
  if (max_out) memcpy(max_out, ctx->h_max, sizeof(float));
  return RNJ_OK;
}

}  // namespace

extern "C" {

int rnj_shard_tiles(int n, int full_rows, int shard, int nshards, long long *tile0,
                    long long *tile1, long long *ntiles) {
  if (n < 0 || nshards < 1 || shard < 0 || shard >= nshards)
    return set_error(RNJ_ERR_INVALID, "invalid shard (need 0 <= shard < nshards, n >= 0)");
  const long long nt = tiles_for(n, full_rows ? 1 : 0);
  if (tile0) *tile0 = nt * shard / nshards;
  if (tile1) *tile1 = nt * (shard + 1) / nshards;
  if (ntiles) *ntiles = nt;
  return RNJ_OK;
}

int rnj_tile_coords(int n, int full_rows, long long tile, int *tile_row, int *tile_col) {
  if (n < 0 || tile < 0 || tile >= tiles_for(n, full_rows ? 1 : 0) || !tile_row || !tile_col)
    return set_error(RNJ_ERR_INVALID, "tile index out of range");
  coords(tiles_of(n), full_rows ? 1 : 0, tile, *tile_row, *tile_col);
  return RNJ_OK;
}

int rnj_shard_create(rnj_ctx *ctx, rnj_aln *aln, int model, int shard, int nshards, float *d_out,
                     size_t ld, rnj_shard **out) {
  if (!ctx || !aln || !out) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (aln->ctx != ctx) return set_error(RNJ_ERR_INVALID, "alignment from another context");
  const Packed &p = aln->p;
  if (p.n < 1) return set_error(RNJ_ERR_INVALID, "empty alignment");
  if (d_out && ld < (size_t)p.n) return set_error(RNJ_ERR_INVALID, "ld < n");
  if (!is_tc_kind(p.kind) && p.Wp / kKW > kMaxFusedWords / kKW)
    return set_error(RNJ_ERR_UNSUPPORTED, "alignments longer than 65280 columns on the bit-plane "
                                          "kernels are not sharded; use rnj_distance");
  const int full = (p.kind == KIND_NAIVE && (p.flags & RNJ_FULL_ROWS)) ? 1 : 0;
  long long t0, t1, nt;
  int rc = rnj_shard_tiles(p.n, full, shard, nshards, &t0, &t1, &nt);
  if (rc != RNJ_OK) return rc;
  DeviceGuard g(ctx->device);
  rnj_shard *s = new rnj_shard();
  s->ctx = ctx;
  s->aln = aln;
  s->model = model;
  s->full = full;
  s->t0 = t0;
  s->t1 = t1;
  s->ntiles = nt;
  s->owns_out = (d_out == nullptr);
  s->ld = d_out ? ld : (size_t)std::max(4, (p.n + 3) / 4 * 4);
  s->out = d_out;
  const long long nitems = t1 - t0;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (!d_out) e = cudaMallocAsync((void **)&s->out, s->ld * p.n * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&s->d_desc, sizeof(AlnDesc), st);
  if (e == cudaSuccess)
    e = cudaMallocAsync((void **)&s->d_items, sizeof(WorkItem) * std::max(nitems, 1LL), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&s->d_ints, 4 * sizeof(int), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&s->d_words, (nt + 2) * sizeof(int), st);
  if (e != cudaSuccess) {
    free_shard(s);
    return cuda_error(e, "shard allocation");
  }
  std::vector<WorkItem> items((size_t)nitems);
  for (long long k = 0; k < nitems; ++k) items[(size_t)k] = WorkItem{0, (int)(t0 + k)};
  const int ints[4] = {(int)nitems, 0, 0, 0};
  EpiParams ep = epi_params_for(p, model);
  ep.out = s->out;
  ep.ld = s->ld;
  ep.max_bits = s->d_words;
  ep.err = s->d_words + 1;
  ep.tile_flags = s->d_words + 2;
  const AlnDesc d = desc_for(p, ep);
  // Pageable sources: each copy has consumed its source when the call returns.
  e = cudaMemcpyAsync(s->d_desc, &d, sizeof(d), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nitems)
    e = cudaMemcpyAsync(s->d_items, items.data(), sizeof(WorkItem) * nitems,
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_ints, ints, sizeof(ints), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    free_shard(s);
    return cuda_error(e, "shard upload");
  }
  *out = s;
  return RNJ_OK;
}

int rnj_shard_run(rnj_shard *s, float *local_max) {
  if (!s) return set_error(RNJ_ERR_INVALID, "null argument");
  rnj_ctx *ctx = s->ctx;
  DeviceGuard g(ctx->device);
  cudaStream_t st = ctx->stream;
  const Packed &p = s->aln->p;
  const long long nitems = s->t1 - s->t0;
  RNJ_CUDA(cudaMemsetAsync(s->d_words, 0, (s->ntiles + 2) * sizeof(int), st), "shard scratch clear");
  RNJ_CUDA(cudaMemsetAsync(s->d_ints + 1, 0, sizeof(int), st), "shard counter clear");
  if (p.n == 1 && nitems > 0)
    RNJ_CUDA(cudaMemsetAsync(s->out, 0, sizeof(float), st), "diagonal");
  if (nitems > 0) {
    const int grid = (int)std::min<long long>(nitems, ctx->num_sms);
    if (is_tc_kind(p.kind)) {
      // Marks stage 1 around the counting kernels.
      const int rc = run_tc_distances(ctx, p, epi_params_for(p, s->model), s->d_desc, s->d_items,
                                      nitems, st, tune_lookup(p.n, p.L, p.type, p.flags));
      if (rc != RNJ_OK) return rc;
    } else {
      ctx_mark(ctx, 1, 0);
      RNJ_CUDA(launch_count_batch(s->d_desc, s->d_items, s->d_ints, s->d_ints + 1, grid, EPI_DIST,
                                  st),
               "count kernel");
      ctx_mark(ctx, 1, 1);
    }
  }
  return read_words(s, local_max);
}

int rnj_shard_finish(rnj_shard *s, float global_max) {
  if (!s) return set_error(RNJ_ERR_INVALID, "null argument");
  rnj_ctx *ctx = s->ctx;
  DeviceGuard g(ctx->device);
  cudaStream_t st = ctx->stream;
  const long long nitems = s->t1 - s->t0;
  if (nitems == 0) return RNJ_OK;
  memcpy(ctx->h_max, &global_max, sizeof(float));
  RNJ_CUDA(cudaMemcpyAsync(s->d_words, ctx->h_max, sizeof(int), cudaMemcpyHostToDevice, st),
           "global max upload");
  const int grid = (int)std::min<long long>(nitems, 4LL * ctx->num_sms);
  ctx_mark(ctx, 2, 0);
  RNJ_CUDA(launch_fixup_batch(s->d_desc, s->d_items, s->d_ints, s->d_items, s->d_ints + 2, grid, st),
           "fix-up kernel");
  ctx_mark(ctx, 2, 1);
  return read_words(s, nullptr);
}

int rnj_shard_output(rnj_shard *s, float **d_out, size_t *ld) {
  if (!s) return set_error(RNJ_ERR_INVALID, "null argument");
  if (d_out) *d_out = s->out;
  if (ld) *ld = s->ld;
  return RNJ_OK;
}

int rnj_shard_copy_tiles(rnj_shard *s, float *host, size_t host_ld, size_t *bytes) {
  if (!s || !host) return set_error(RNJ_ERR_INVALID, "null argument");
  const int n = s->aln->p.n;
  if (host_ld < (size_t)n) return set_error(RNJ_ERR_INVALID, "host_ld < n");
  rnj_ctx *ctx = s->ctx;
  DeviceGuard g(ctx->device);
  const int nt = tiles_of(n);
  size_t total = 0;
  long long t = s->t0;
  while (t < s->t1) {
    int ti, tj;
    coords(nt, s->full, t, ti, tj);
    // This tile row's run of the shard's tiles: columns tj .. tj + run - 1.
    const long long row_end = s->full ? (long long)(ti + 1) * nt : row_start(nt, ti + 1);
    const long long run = std::min(s->t1, row_end) - t;
    const int r0 = ti * kTile, r1 = std::min(n, r0 + kTile);
    const int c0 = tj * kTile, c1 = std::min(n, (int)((tj + run) * kTile));
    const size_t w = (size_t)(c1 - c0) * sizeof(float);
    RNJ_CUDA(cudaMemcpy2DAsync(host + (size_t)r0 * host_ld + c0, host_ld * sizeof(float),
                               s->out + (size_t)r0 * s->ld + c0, s->ld * sizeof(float), w,
                               (size_t)(r1 - r0), cudaMemcpyDeviceToHost, ctx->stream),
             "shard tile copy");
    total += w * (size_t)(r1 - r0);
    t += run;
  }
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "shard copy sync");
  if (bytes) *bytes = total;
  return RNJ_OK;
}

int rnj_shard_destroy(rnj_shard *s) {
  if (!s) return RNJ_OK;
  DeviceGuard g(s->ctx->device);
  free_shard(s);
  return RNJ_OK;
}

}  // extern "C"
