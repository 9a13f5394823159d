// rnj_stream.cu -- the host-to-host distance call (rnj_distance_matrix_host) of
// the tensor-core path (DNA and protein), streamed.
//
// The n x n float matrix is 16x the bytes of the alignment, so a host-in /
// host-out call is bound by the device-to-host copy, not by the kernels.  This
// path overlaps the three: the triangle is cut into bands of tile rows and the
// bands run LAST FIRST.  Band b (rows r0 .. r1-1, tiles (ti, tj) with ti in
// the band and tj >= ti) needs only sequences r0 .. n-1, which the previous
// bands have already uploaded and packed, plus its own rows.  When band b is
// done, every cell (i, j) with min(i, j) >= r0 is final, and the newly final
// cells are two rectangles of the output:
//   rows r0 .. r1-1,  columns r0 .. n-1      (band rows, right of the band start)
//   rows r1 .. n-1,   columns r0 .. r1-1     (the band's mirror image below it)
// Each leaves as one 2-D copy into the caller's page-locked matrix while the
// next bands are computed; every band's upload is enqueued at the start, on its
// own copy engine.  Saturated pairs
// (-1) can only take their final value, 2 x the global maximum, at the end:
// their tiles are fixed on the device after the last band and copied again.
// When the first band shows saturation in more than a quarter of its tiles,
// the call defers every download to one copy after the fix-up instead.
//
// Streams: uploads on ctx->s_up, kernels on ctx->stream, downloads on
// ctx->s_down, ordered by events (upload k -> kernels k -> download k).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

#define RNJ_TRY(call, what)                      \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

// Default band height in tile rows: about five bands, 4 to 32 tile rows (the
// mirror rectangle's rows are then 2 to 16 KB wide, which the copy engines move
// at full rate), and no band larger than one packed-count pass.  Measured on
// 10,000 x 10,000: 16 tile rows beat 8 and 4 (fewer, larger copies).
// The library streams a host call from this many tile rows on (band_tiles 0).
constexpr int kStreamMinTiles = 12;

int default_band_tiles(int nt) {
  const int g = std::max(4, std::min(32, (nt + 4) / 5));
  return std::max(1, std::min(g, kTcChunkTiles / std::max(1, nt)));
}

// Tile-row boundaries of the bands, first band (the last rows) first.
// bounds[k] .. bounds[k + 1] - 1 are the tile rows of band k in processing
// order, counted from the top (bounds decrease).  A band's download is about its
// height times the rows below it and its upload its height times L, so the
// bottom bands have little to download and the download engine waits for their
// uploads: with `ramp` the first bands are short and grow (1/8, 1/4, 3/8, 1/2,
// 3/4 of g, at least one tile row each) so that downloads start early, then
// bands of g.  Without it (an alignment uploaded whole before the bands) only
// the first band is short (g/4), for an early first download and the
// saturation sample.
std::vector<int> band_bounds(int nt, int g, bool ramp) {
  static const int grow[5][2] = {{1, 8}, {1, 4}, {3, 8}, {1, 2}, {3, 4}};
  std::vector<int> b{nt};
  int top = nt;
  for (int k = 0; top > 0; ++k) {
    int h = g;
    if (ramp && k < 5) h = std::max(1, g * grow[k][0] / grow[k][1]);
    else if (k == 0) h = std::max(1, g / 4);
    top = std::max(0, top - h);
    b.push_back(top);
  }
  return b;
}

struct Events {
  std::vector<cudaEvent_t> ev;
  ~Events() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  cudaError_t make(size_t k) {
    ev.assign(k, nullptr);
    for (auto &e : ev) {
      cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  }
};

// Device buffers of one call, released on the context stream once every
// stream of the call has been synchronised.
struct CallBuffers {
  rnj_ctx *ctx;
  uint8_t *chars = nullptr, *feat = nullptr;
  float *out = nullptr;
  WorkItem *items = nullptr;
  explicit CallBuffers(rnj_ctx *c) : ctx(c) {}
  ~CallBuffers() {
    cudaStreamSynchronize(ctx->s_up);
    cudaStreamSynchronize(ctx->s_down);
    if (chars) cudaFreeAsync(chars, ctx->stream);
    if (feat) cudaFreeAsync(feat, ctx->stream);
    if (out) cudaFreeAsync(out, ctx->stream);
    if (items) cudaFreeAsync(items, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  }
};


int ensure_host_words(rnj_ctx *ctx, size_t words) {
  if (ctx->h_words_cap >= words) return RNJ_OK;
  if (ctx->h_words) cudaFreeHost(ctx->h_words);
  ctx->h_words = nullptr;
  ctx->h_words_cap = 0;
  RNJ_TRY(cudaMallocHost((void **)&ctx->h_words, words * sizeof(int)), "pinned flag words");
  ctx->h_words_cap = words;
  return RNJ_OK;
}

// Rows [r0, r1) x columns [c0, c1) of the device matrix (ld floats per row)
// into the same cells of the host matrix (n floats per row).
cudaError_t copy_block(float *h, const float *d, size_t ld, int n, int r0, int r1, int c0, int c1,
                       cudaStream_t s) {
  if (r1 <= r0 || c1 <= c0) return cudaSuccess;
  return cudaMemcpy2DAsync(h + (size_t)r0 * n + c0, (size_t)n * sizeof(float),
                           d + (size_t)r0 * ld + c0, ld * sizeof(float),
                           (size_t)(c1 - c0) * sizeof(float), (size_t)(r1 - r0),
                           cudaMemcpyDeviceToHost, s);
}

}  // namespace

int ensure_side_streams(rnj_ctx *ctx) {
  if (!ctx->s_up) RNJ_TRY(cudaStreamCreateWithFlags(&ctx->s_up, cudaStreamNonBlocking), "upload stream");
  if (!ctx->s_down)
    RNJ_TRY(cudaStreamCreateWithFlags(&ctx->s_down, cudaStreamNonBlocking), "download stream");
  return RNJ_OK;
}

int distance_host_streamed(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld, int type,
                           int model, int flags, int band_tiles, float *out, float *max_out) {
  // Eligibility: DNA with the fast rules, or protein, on the tensor-core
  // kernel, a page-locked output and at least two bands.
  const bool prot = type == RNJ_PROTEIN;
  if (n < 2 || L < 1 || (type != RNJ_DNA && !prot) || (flags & RNJ_POPCOUNT) ||
      (!prot && (!(flags & RNJ_FASTDIST) || (flags & RNJ_FULL_ROWS))) || L > kMaxTcColumns ||
      (model != RNJ_JC && model != RNJ_KIMURA))
    return RNJ_ERR_UNSUPPORTED;
  const int nt = tiles_of(n);
  // Small matrices: one upload, one launch sequence and one download beat the
  // bands' extra launches, events and copies (measured host-to-host, DNA
  // 1024 x 2000 0.31 against 0.35 ms, 2048 x 2000 0.67 against 0.58 ms).
  if (band_tiles == 0 && nt < kStreamMinTiles) return RNJ_ERR_UNSUPPORTED;
  const TuneParams tp = tune_lookup(n, L, type, flags);
  if (tp.dna_kernel != 0) return RNJ_ERR_UNSUPPORTED;  // this bucket counts on the bit planes
  const int g = band_tiles > 0 ? band_tiles
                               : (tp.stream_band > 0 ? tp.stream_band : default_band_tiles(nt));
  // DNA uploads band by band (the ramp pays); protein is uploaded whole first.
  const std::vector<int> bounds = band_bounds(nt, g, !prot);
  const int nbands = (int)bounds.size() - 1;
  if (nbands < 2) return RNJ_ERR_UNSUPPORTED;
  const long long ntiles = tri_tiles(nt);
  // Every band must fit one packed-count pass.
  long long max_band_tiles = 0;
  for (int k = 0; k < nbands; ++k) {
    const long long t0 = bounds[k + 1], h = bounds[k] - bounds[k + 1];
    max_band_tiles = std::max(max_band_tiles, h * (nt - t0) - h * (h - 1) / 2);
  }
  // Counts and transform in one kernel (rnj_tcf.cu), or through the packed
  // counts (one pass per band) and the transform kernel.
  const bool fused = tp.tc_epilogue == 0 && L <= kMaxFusedColumns;
  if (!fused && max_band_tiles > kTcChunkTiles) return RNJ_ERR_UNSUPPORTED;
  if (!ctx_block_pinned(out, (size_t)n * n * sizeof(float))) return RNJ_ERR_UNSUPPORTED;

  DeviceGuard guard(ctx->device);
  int rc = ensure_side_streams(ctx);
  if (rc != RNJ_OK) return rc;
  rc = ensure_host_words(ctx, (size_t)ntiles + 2);
  if (rc != RNJ_OK) return rc;
  if (!fused) {
    rc = ensure_packed(ctx, max_band_tiles);
    if (rc != RNJ_OK) return rc;
  }
  rc = ctx_scratch(ctx, (size_t)ntiles + 2);
  if (rc != RNJ_OK) return rc;

  // Packed layout of the alignment (as pack_prepared lays it out).
  Packed p;
  p.n = n;
  p.L = L;
  p.type = type;
  p.flags = flags;
  p.kind = prot ? KIND_PROT_TC : KIND_DNA_TC;
  p.W = (L + 31) / 32;
  p.Wp = std::max(kKW, (p.W + kKW - 1) / kKW * kKW);
  p.Np = nt * kTile;
  p.NP = 0;
  p.Lk = std::max(256, (L + 255) / 256 * 256);

  const int transform_ctas = tp.transform_ctas > 0
                                 ? std::min(tp.transform_ctas, kTransformCtasPerSm)
                                 : kTransformCtasPerSm;

  // Work items, band by band, last band first; within a band column by
  // column, so that the CTAs running at one time share the band's row tiles.
  std::vector<WorkItem> items;
  items.reserve((size_t)ntiles);
  std::vector<long long> band_off(nbands + 1, 0);
  for (int k = 0; k < nbands; ++k) {
    const int t0 = bounds[k + 1], t1 = bounds[k];
    band_off[k] = (long long)items.size();
    for (int tj = t0; tj < nt; ++tj)
      for (int ti = t0; ti < t1 && ti <= tj; ++ti) {
        WorkItem w;
        w.aln = 0;
        w.tile = (int)((long long)ti * nt - (long long)ti * (ti - 1) / 2 + (tj - ti));
        items.push_back(w);
      }
  }
  band_off[nbands] = (long long)items.size();

  CallBuffers buf(ctx);
  RNJ_TRY(cudaMallocAsync((void **)&buf.chars, (size_t)n * L, ctx->stream), "upload buffer");
  // Protein: the residue ranks come from the whole alignment, so its bytes
  // (small next to the n x n matrix) are uploaded at once and scanned first.
  uint8_t lut[256];
  if (prot) {
    if (ld == (size_t)L)
      RNJ_TRY(cudaMemcpyAsync(buf.chars, chars, (size_t)n * L, cudaMemcpyHostToDevice, ctx->stream),
              "alignment upload");
    else
      RNJ_TRY(cudaMemcpy2DAsync(buf.chars, (size_t)L, chars, ld, (size_t)L, (size_t)n,
                                cudaMemcpyHostToDevice, ctx->stream),
              "alignment upload");
    RNJ_TRY(cudaMemsetAsync(ctx->d_mask, 0, 8 * sizeof(uint32_t), ctx->stream), "mask clear");
    RNJ_TRY(launch_presence(buf.chars, (size_t)L, n, L, ctx->d_mask, ctx->stream), "presence kernel");
    RNJ_TRY(cudaMemcpyAsync(ctx->h_mask, ctx->d_mask, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            ctx->stream),
            "mask copy");
    RNJ_TRY(cudaStreamSynchronize(ctx->stream), "mask sync");
    int kind = 0;
    lut_for(RNJ_PROTEIN, flags, ctx->h_mask, lut, &kind);
    int ranks = 0;
    for (int c = 0; c < 256; ++c)
      if (lut[c] != 0xFF) ranks = std::max(ranks, lut[c] + 1);
    if (ranks < 1 || ranks > kMaxTcRanks) return RNJ_ERR_UNSUPPORTED;
    p.nfb = 1 + ranks;
  }
  const size_t fbytes = (size_t)p.Np * p.nfb * (p.Lk / 2);
  RNJ_TRY(cudaMallocAsync((void **)&buf.feat, fbytes, ctx->stream), "feature allocation");
  RNJ_TRY(cudaMallocAsync((void **)&buf.out, (size_t)n * n * sizeof(float), ctx->stream),
          "matrix allocation");
  RNJ_TRY(cudaMallocAsync((void **)&buf.items, items.size() * sizeof(WorkItem), ctx->stream),
          "work list allocation");
  RNJ_TRY(cudaMemcpyAsync(buf.items, items.data(), items.size() * sizeof(WorkItem),
                          cudaMemcpyHostToDevice, ctx->stream),
          "work list upload");
  RNJ_TRY(cudaMemsetAsync(ctx->scratch.words, 0, ((size_t)ntiles + 2) * sizeof(int), ctx->stream),
          "scratch clear");
  p.feat = buf.feat;
  rc = encode_features_map(p);
  if (rc != RNJ_OK) return rc;
  EpiParams ep = ctx_epi(ctx, p, model);
  ep.out = buf.out;
  ep.ld = (size_t)n;
  AlnDesc desc = desc_for(p, ep);
  RNJ_TRY(cudaMemcpyAsync(ctx->d_desc, &desc, sizeof(desc), cudaMemcpyHostToDevice, ctx->stream),
          "descriptor upload");

  // Events: [0] allocations done, then per band k: 1 + 2k upload done,
  // 2 + 2k band computed; last: every download enqueued has been issued.
  Events ev;
  RNJ_TRY(ev.make(2 + 2 * (size_t)nbands), "events");
  cudaEvent_t ev_alloc = ev.ev[0], ev_down_end = ev.ev[1 + 2 * nbands];
  RNJ_TRY(cudaEventRecord(ev_alloc, ctx->stream), "event");
  RNJ_TRY(cudaStreamWaitEvent(ctx->s_up, ev_alloc, 0), "upload wait");

  // The uploads of every band, in band order, back to back on their own
  // stream: none depends on a band's results, so they run ahead of the kernels
  // and of the first band's saturation check.  One contiguous copy per band when
  // the host rows are packed.  (Protein: uploaded above.)
  for (int k = 0; k < nbands; ++k) {
    const int r0 = bounds[k + 1] * kTile, rn1 = std::min(bounds[k] * kTile, n);
    if (prot) {
    } else if (ld == (size_t)L)
      RNJ_TRY(cudaMemcpyAsync(buf.chars + (size_t)r0 * L, chars + (size_t)r0 * L,
                              (size_t)(rn1 - r0) * L, cudaMemcpyHostToDevice, ctx->s_up),
              "alignment upload");
    else
      RNJ_TRY(cudaMemcpy2DAsync(buf.chars + (size_t)r0 * L, (size_t)L, chars + (size_t)r0 * ld, ld,
                                (size_t)L, (size_t)(rn1 - r0), cudaMemcpyHostToDevice, ctx->s_up),
              "alignment upload");
    RNJ_TRY(cudaEventRecord(ev.ev[1 + 2 * k], ctx->s_up), "event");
  }

  // Band k: once its sequences are up, pack them, count and transform its
  // tiles, then (unless deferred) download what it finished.
  bool deferred = false;
  auto run_band = [&](int k) -> int {
    const int r0 = bounds[k + 1] * kTile;
    const int r1 = bounds[k] * kTile;                // packed rows (with padding)
    const int rn1 = std::min(r1, n);                 // output rows
    cudaEvent_t ev_up = ev.ev[1 + 2 * k], ev_done = ev.ev[2 + 2 * k];
    RNJ_TRY(cudaStreamWaitEvent(ctx->stream, ev_up, 0), "kernel wait");
    RNJ_TRY(prot ? launch_pack_features_prot(buf.chars, (size_t)L, n, L, p.Np, p.Lk, p.nfb, lut,
                                             p.feat, ctx->stream, r0, r1 - r0)
                 : launch_pack_features(buf.chars, (size_t)L, n, L, p.Np, p.Lk, p.feat,
                                        ctx->stream, r0, r1 - r0),
            "feature pack kernel");
    const long long i0 = band_off[k], cnt = band_off[k + 1] - band_off[k];
    if (fused) {
      RNJ_TRY(launch_tc_fused(ctx->d_desc, buf.items, nullptr, (int)items.size(), (int)i0,
                              (int)cnt, (int)std::min<long long>(cnt, ctx->num_sms),
                              fused_variant_for(ep.model, ep.type, ep.compat_wrap, 0),
                              ctx->stream, tp.tc_stages),
              "fused tensor-core kernel");
    } else {
      RNJ_TRY(launch_tc_batch(ctx->d_desc, buf.items, nullptr, (int)items.size(), (int)i0,
                              (int)cnt, ctx->d_packed, (int)std::min<long long>(cnt, ctx->num_sms),
                              EPI_PACKED, ctx->stream, tp.tc_stages),
              "tensor-core kernel");
      RNJ_TRY(launch_tc_transform(ctx->d_desc, buf.items, nullptr, (int)items.size(), (int)i0,
                                  (int)cnt, ctx->d_packed,
                                  (int)std::min<long long>(cnt, (long long)transform_ctas *
                                                                    ctx->num_sms),
                                  ctx->stream),
              "transform kernel");
    }
    RNJ_TRY(cudaEventRecord(ev_done, ctx->stream), "event");
    if (deferred) return RNJ_OK;
    RNJ_TRY(cudaStreamWaitEvent(ctx->s_down, ev_done, 0), "download wait");
    RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, r0, rn1, r0, n, ctx->s_down), "row copy");
    RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, rn1, n, r0, rn1, ctx->s_down), "column copy");
    return RNJ_OK;
  };

  rc = run_band(0);
  if (rc != RNJ_OK) return rc;
  // A sample of the saturation: when more than a quarter of the first band's
  // tiles hold saturated pairs (unrelated sequences), most of the matrix would
  // have to be fixed and downloaded twice.  Such inputs take the deferred
  // order instead: every band computed, the fix-up, then one download.
  RNJ_TRY(cudaMemcpyAsync(ctx->h_words, ctx->scratch.words, ((size_t)ntiles + 2) * sizeof(int),
                          cudaMemcpyDeviceToHost, ctx->stream),
          "flag copy");
  RNJ_TRY(cudaStreamSynchronize(ctx->stream), "first band sync");
  {
    long long sat = 0;
    for (long long it = band_off[0]; it < band_off[1]; ++it) sat += ctx->h_words[2 + items[it].tile] != 0;
    deferred = sat * 4 > band_off[1] - band_off[0];
  }
  for (int k = 1; k < nbands; ++k) {
    rc = run_band(k);
    if (rc != RNJ_OK) return rc;
  }
  RNJ_TRY(cudaEventRecord(ev_down_end, ctx->s_down), "event");

  if (deferred) {
    RNJ_TRY(cudaStreamWaitEvent(ctx->stream, ev_down_end, 0), "fix-up wait");
    RNJ_TRY(launch_fixup(ep, nt, ctx->stream), "fix-up kernel");
    RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, 0, n, 0, n, ctx->stream), "matrix copy");
  }
  // Max, error word and saturation flags, while the downloads run.
  RNJ_TRY(cudaMemcpyAsync(ctx->h_words, ctx->scratch.words, ((size_t)ntiles + 2) * sizeof(int),
                          cudaMemcpyDeviceToHost, ctx->stream),
          "flag copy");
  RNJ_TRY(cudaMemcpyAsync(ctx->h_max + 1, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream),
          "error word copy");
  RNJ_TRY(cudaStreamSynchronize(ctx->stream), "band sync");
  rc = take_device_error(ctx);
  if (rc != RNJ_OK) return rc;
  std::vector<int> flagged;
  if (!deferred)
    for (long long t = 0; t < ntiles; ++t)
      if (ctx->h_words[2 + t]) flagged.push_back((int)t);
  float mx;
  memcpy(&mx, &ctx->h_words[0], sizeof(float));
  if (!flagged.empty()) {
    // -1 -> 2 x max on the flagged tiles once their first copies have left,
    // then those tiles (and their mirror images) again.
    RNJ_TRY(cudaStreamWaitEvent(ctx->stream, ev_down_end, 0), "fix-up wait");
    RNJ_TRY(launch_fixup(ep, nt, ctx->stream), "fix-up kernel");
    if ((long long)flagged.size() * 4 > ntiles) {
      RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, 0, n, 0, n, ctx->stream), "matrix copy");
    } else {
      for (int t : flagged) {
        int ti = 0, tj = 0;
        {
          // Row-major triangle index -> (ti, tj).
          long long rem = t;
          while (rem >= nt - ti) {
            rem -= nt - ti;
            ++ti;
          }
          tj = ti + (int)rem;
        }
        const int a0 = ti * kTile, a1 = std::min(n, a0 + kTile);
        const int c0 = tj * kTile, c1 = std::min(n, c0 + kTile);
        RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, a0, a1, c0, c1, ctx->stream), "tile copy");
        if (ti != tj)
          RNJ_TRY(copy_block(out, buf.out, (size_t)n, n, c0, c1, a0, a1, ctx->stream),
                  "mirror copy");
      }
    }
  }
  RNJ_TRY(cudaStreamSynchronize(ctx->s_down), "download sync");
  RNJ_TRY(cudaStreamSynchronize(ctx->stream), "fix-up sync");
  if (max_out) *max_out = mx;
  return RNJ_OK;
}
