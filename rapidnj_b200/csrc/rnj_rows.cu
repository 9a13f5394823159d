// rnj_rows.cu -- distance matrices larger than device memory, delivered in bands
// of full rows (rnj_distance_rows).
//
// rapidNJ keeps a matrix that does not fit in RAM in a disk matrix
// (main.cpp:702-723): its distance drivers then compute every row in full,
// j = 0 .. n - 1 (KimuraDistance.cpp:308-354 and JCdistance.cpp:160-195 with
// dm != NULL), hand each finished row to diskMatrix::writeArray
// (diskMatrix.cpp:96-117), and once the maximum is known rewrite every row
// through readArray / writeArray with the diagonal 0 and every -1 replaced by
// twice the maximum (KimuraDistance.cpp:366-395, JCdistance.cpp:201-230).
//
// Here only the packed alignment and two bands of rows live on the device:
//   * band k = rows [r0, r1) (a multiple of the 128-row tile), computed as the
//     full-square tiles (ti, tj) with ti in the band and every tj, each ordered
//     pair once (the counts of the -f estimator are not symmetric), into a
//     band buffer of (r1 - r0) x n floats (the fused tensor-core kernel, or the
//     bit-plane kernel, in their full-rows forms);
//   * the band is copied to page-locked host memory on a second stream while
//     the next band computes, and handed to the caller's callback row block by
//     row block, in row order: the rows as the reference's drivers write them
//     (diagonal 0, saturated pairs -1);
//   * the global maximum and whether any pair saturated are returned at the
//     end; the caller's post-process (-1 -> 2 * max) follows, as in the
//     reference.
// Device memory: the packed alignment, two band buffers and one saturation flag
// per full-square tile; host memory: two page-locked band buffers.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

struct RowBuffers {
  rnj_ctx *ctx;
  float *d_band[2] = {nullptr, nullptr};
  float *h_band[2] = {nullptr, nullptr};
  int *h_flags[2] = {nullptr, nullptr};
  AlnDesc *d_desc[2] = {nullptr, nullptr};
  cudaEvent_t ev_comp[2] = {nullptr, nullptr}, ev_down[2] = {nullptr, nullptr};
  explicit RowBuffers(rnj_ctx *c) : ctx(c) {}
  ~RowBuffers() {
    cudaStreamSynchronize(ctx->s_down);
    cudaStreamSynchronize(ctx->stream);
    for (int b = 0; b < 2; ++b) {
      if (d_band[b]) cudaFreeAsync(d_band[b], ctx->stream);
      if (d_desc[b]) cudaFreeAsync(d_desc[b], ctx->stream);
      if (h_band[b]) cudaFreeHost(h_band[b]);
      if (h_flags[b]) cudaFreeHost(h_flags[b]);
      if (ev_comp[b]) cudaEventDestroy(ev_comp[b]);
      if (ev_down[b]) cudaEventDestroy(ev_down[b]);
    }
    cudaStreamSynchronize(ctx->stream);
  }
};

#define RNJ_TRY(call, what)                      \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

}  // namespace

extern "C" int rnj_distance_rows(rnj_ctx *ctx, rnj_aln *aln, int model, int band_rows,
                                 rnj_rows_fn fn, void *user, float *max_out,
                                 int *saturated_out) {
  if (!ctx || !aln || !fn) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (aln->ctx != ctx) return set_error(RNJ_ERR_INVALID, "alignment from another context");
  if (band_rows < 0) return set_error(RNJ_ERR_INVALID, "negative band height");
  const Packed &p = aln->p;
  const int n = p.n;
  if (max_out) *max_out = 0.0f;
  if (saturated_out) *saturated_out = 0;
  if (n == 0) return RNJ_OK;
  const bool tc = is_tc_kind(p.kind);
  if (tc && p.L > kMaxFusedColumns)
    return set_error(RNJ_ERR_UNSUPPORTED,
                     "row bands of tensor-core alignments take at most 65535 columns (pack "
                     "longer ones with RNJ_POPCOUNT)");
  if (!tc && p.Wp / kKW > kMaxFusedWords / kKW)
    return set_error(RNJ_ERR_UNSUPPORTED, "row bands take alignments of at most 65280 columns");
  DeviceGuard guard(ctx->device);
  int rc = ensure_side_streams(ctx);
  if (rc != RNJ_OK) return rc;

  const int nt = tiles_of(n);
  // Band height: a multiple of the tile; by default two band buffers of at most
  // 512 MiB together.
  int band = band_rows > 0 ? band_rows : (int)std::min<long long>(
                                             (long long)n, ((256LL << 20) / 4) / std::max(1, n));
  band = std::max(kTile, (band + kTile - 1) / kTile * kTile);
  band = std::min(band, nt * kTile);
  const int band_tiles_rows = band / kTile;
  const int nbands = (nt + band_tiles_rows - 1) / band_tiles_rows;
  const long long all_tiles = (long long)nt * nt;

  rc = ctx_scratch(ctx, (size_t)all_tiles + 2);
  if (rc != RNJ_OK) return rc;
  RNJ_TRY(cudaMemsetAsync(ctx->scratch.words, 0, ((size_t)all_tiles + 2) * sizeof(int), ctx->stream),
          "scratch clear");
  EpiParams ep = ctx_epi(ctx, p, model);
  ep.full = 1;
  ep.ld = (size_t)n;
  const TuneParams tp = tune_lookup(p.n, p.L, p.type, p.flags);
  ep.stages = tp.pop_stages;

  RowBuffers buf(ctx);
  const size_t band_floats = (size_t)band * n;
  const size_t band_flags = (size_t)band_tiles_rows * nt;
  for (int b = 0; b < 2 && b < nbands; ++b) {
    RNJ_TRY(cudaMallocAsync((void **)&buf.d_band[b], band_floats * sizeof(float), ctx->stream),
            "band buffer");
    RNJ_TRY(cudaMallocHost((void **)&buf.h_band[b], band_floats * sizeof(float)),
            "page-locked band buffer");
    RNJ_TRY(cudaMallocHost((void **)&buf.h_flags[b], band_flags * sizeof(int)),
            "page-locked band flags");
    RNJ_TRY(cudaEventCreateWithFlags(&buf.ev_comp[b], cudaEventDisableTiming), "event");
    RNJ_TRY(cudaEventCreateWithFlags(&buf.ev_down[b], cudaEventDisableTiming), "event");
    if (tc)
      RNJ_TRY(cudaMallocAsync((void **)&buf.d_desc[b], sizeof(AlnDesc), ctx->stream),
              "band descriptor");
  }

  // Hands band k (in buffer k % 2, downloaded) to the caller.
  bool any_sat = false;
  auto deliver = [&](int k) -> int {
    const int b = k % 2;
    const int r0 = k * band, r1 = std::min(n, (k + 1) * band);
    RNJ_TRY(cudaEventSynchronize(buf.ev_down[b]), "band download");
    const int t0 = k * band_tiles_rows, t1 = std::min(nt, (k + 1) * band_tiles_rows);
    for (size_t f = 0; f < (size_t)(t1 - t0) * nt; ++f) any_sat |= buf.h_flags[b][f] != 0;
    if (fn(user, r0, r1 - r0, buf.h_band[b], (size_t)n) != 0)
      return set_error(RNJ_ERR_INVALID, "the row callback stopped the computation");
    return RNJ_OK;
  };

  for (int k = 0; k < nbands; ++k) {
    const int b = k % 2;
    const int t0 = k * band_tiles_rows, t1 = std::min(nt, (k + 1) * band_tiles_rows);
    const int r0 = t0 * kTile, r1 = std::min(n, t1 * kTile);
    const long long tile0 = (long long)t0 * nt, btiles = (long long)(t1 - t0) * nt;
    // The buffer's previous band must be on the host before it is overwritten.
    if (k >= 2) RNJ_TRY(cudaStreamWaitEvent(ctx->stream, buf.ev_down[b], 0), "band reuse");
    EpiParams eb = ep;
    eb.out = buf.d_band[b];
    eb.row0 = r0;
    eb.tile0 = (int)tile0;
    if (tc) {
      AlnDesc d = desc_for(p, eb);
      d.full = 1;
      RNJ_TRY(cudaMemcpyAsync(buf.d_desc[b], &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream),
              "band descriptor upload");
      RNJ_TRY(launch_tc_fused(buf.d_desc[b], nullptr, nullptr, (int)all_tiles, (int)tile0,
                              (int)btiles, (int)std::min<long long>(btiles, ctx->num_sms),
                              FUSED_FULL, ctx->stream, tp.tc_stages),
              "fused tensor-core kernel (row band)");
    } else {
      const int ckind = (p.kind == KIND_DNA && model == RNJ_JC) ? KIND_MISM2 : p.kind;
      RNJ_TRY(launch_count_tiles(p, ckind, EPI_DIST, eb, ctx->stream, 0, btiles),
              "count kernel (row band)");
    }
    RNJ_TRY(cudaEventRecord(buf.ev_comp[b], ctx->stream), "event");
    RNJ_TRY(cudaStreamWaitEvent(ctx->s_down, buf.ev_comp[b], 0), "download wait");
    RNJ_TRY(cudaMemcpyAsync(buf.h_band[b], buf.d_band[b], (size_t)(r1 - r0) * n * sizeof(float),
                            cudaMemcpyDeviceToHost, ctx->s_down),
            "band download");
    RNJ_TRY(cudaMemcpyAsync(buf.h_flags[b], ctx->scratch.words + 2 + tile0,
                            (size_t)btiles * sizeof(int), cudaMemcpyDeviceToHost, ctx->s_down),
            "band flags download");
    RNJ_TRY(cudaEventRecord(buf.ev_down[b], ctx->s_down), "event");
    // While band k computes and downloads, the caller takes band k - 1.
    if (k >= 1 && (rc = deliver(k - 1)) != RNJ_OK) return rc;
  }
  if ((rc = deliver(nbands - 1)) != RNJ_OK) return rc;
  RNJ_TRY(cudaMemcpyAsync(ctx->h_max, ctx->scratch.words, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream),
          "max copy");
  rc = ctx_check_error(ctx);  // synchronises; reports a device timeout
  if (rc != RNJ_OK) return rc;
  if (max_out) memcpy(max_out, ctx->h_max, sizeof(float));
  if (saturated_out) *saturated_out = any_sat ? 1 : 0;
  return RNJ_OK;
}
