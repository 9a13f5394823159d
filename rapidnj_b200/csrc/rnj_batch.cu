// rnj_batch.cu -- many alignments in one pass: a device work list of the
// triangle tiles of every alignment in the batch, ordered by decreasing cost,
// consumed by one persistent launch per kernel family (the tcgen05 kernel for
// DNA, the bit-plane kernel for protein and -f alignments) and a fix-up over the
// flagged tiles.  The launch sequence is captured once in a CUDA graph; a run
// only uploads the descriptors and work lists the graph's kernels read.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"
#include "rnj_tcgen05.cuh"

using namespace rnj;

namespace {

#define RNJ_CUDA(call, what)                                \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_error(e_, what);     \
  } while (0)

struct Entry {
  rnj_aln *aln;
  int model;
  float *out;
  size_t ld;
  bool owned;
  long long flag_off;  // offset of this alignment's tile flags
  long long ntiles;
  bool owns_aln;       // packed by rnj_batch_add_many: freed with the entry
};

}  // namespace

struct rnj_batch {
  rnj_ctx *ctx = nullptr;
  int cap_aln = 0;
  long long cap_tiles = 0;
  cudaStream_t stream = nullptr;  // capture / launch stream (non-blocking)
  cudaEvent_t ev_ready = nullptr, ev_uploaded = nullptr, ev_done = nullptr;
  bool uploaded_pending = false;
  // device
  AlnDesc *d_descs = nullptr;
  WorkItem *d_items_tc = nullptr, *d_items_pc = nullptr;
  int *d_ints = nullptr;  // [0] tensor-core items, [1] popcount items, [2] item counter, [3] error
  int *d_max = nullptr;   // per-alignment max bits
  int *d_flags = nullptr; // per-tile saturation flags of all alignments
  // pinned host staging of the uploads
  AlnDesc *h_descs = nullptr;
  WorkItem *h_items_tc = nullptr, *h_items_pc = nullptr;
  int *h_ints = nullptr;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<Entry> entries;
  long long tiles_used = 0;
  bool join = true;  // make the context stream wait for each run's completion
  std::vector<void *> arenas;  // packed alignments of rnj_batch_add_many, freed by clear
  std::vector<int> host_max;  // maxima of the last run, read once per run
  bool host_max_valid = false;
  // Launch shape from the tuner: the fused kernel's ring depth of the last run
  // (that of the bucket holding most of its work; 0 = the default) and how
  // many of its alignments had a tuned entry (their tile-order band comes
  // from it).
  int tc_stages = 0;
  int tuned_alns = 0;
};

void batch_set_join(rnj_batch *b, bool join) { b->join = join; }

namespace {

void free_batch(rnj_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &e : b->entries)
  {
    if (e.owned && e.out) cudaFreeAsync(e.out, b->ctx->stream);
    if (e.owns_aln) rnj_aln_destroy(e.aln);
  }
  for (void *a : b->arenas) cudaFreeAsync(a, b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_descs);
  cudaFree(b->d_items_tc);
  cudaFree(b->d_items_pc);
  cudaFree(b->d_ints);
  cudaFree(b->d_max);
  cudaFree(b->d_flags);
  cudaFreeHost(b->h_descs);
  cudaFreeHost(b->h_items_tc);
  cudaFreeHost(b->h_items_pc);
  cudaFreeHost(b->h_ints);
  if (b->ev_ready) cudaEventDestroy(b->ev_ready);
  if (b->ev_uploaded) cudaEventDestroy(b->ev_uploaded);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// Captures: clear scratch -> the fused tensor-core kernel over every
// tensor-core item (counts and transform, per-item model) -> popcount kernel ->
// fix-up.
int capture_graph(rnj_batch *b) {
  const int sms = b->ctx->num_sms;
  RNJ_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaMemsetAsync(b->d_max, 0, sizeof(int) * b->cap_aln, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_flags, 0, sizeof(int) * b->cap_tiles, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_ints + 2, 0, 2 * sizeof(int), b->stream);
  if (e == cudaSuccess)
    e = launch_tc_fused(b->d_descs, b->d_items_tc, b->d_ints + 0, 0, 0, (int)b->cap_tiles, sms,
                        FUSED_ANY, b->stream);
  if (e == cudaSuccess)
    e = launch_count_batch(b->d_descs, b->d_items_pc, b->d_ints + 1, b->d_ints + 2, sms, EPI_DIST,
                           b->stream);
  if (e == cudaSuccess)
    e = launch_fixup_batch(b->d_descs, b->d_items_tc, b->d_ints + 0, b->d_items_pc, b->d_ints + 1,
                           sms * 4, b->stream);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_error(e, "batch graph capture");
  }
  if (e2 != cudaSuccess) return cuda_error(e2, "end capture");
  b->graph = g;
  RNJ_CUDA(cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
  return RNJ_OK;
}

}  // namespace

extern "C" {

int rnj_batch_create(rnj_ctx *ctx, int max_alignments, long long max_tiles, rnj_batch **out) {
  if (!ctx || !out || max_alignments <= 0 || max_tiles <= 0)
    return set_error(RNJ_ERR_INVALID, "invalid batch capacity");
  DeviceGuard g(ctx->device);
  rnj_batch *b = new rnj_batch();
  b->ctx = ctx;
  b->cap_aln = max_alignments;
  b->cap_tiles = max_tiles;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_uploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_descs, sizeof(AlnDesc) * max_alignments);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_items_tc, sizeof(WorkItem) * max_tiles);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_items_pc, sizeof(WorkItem) * max_tiles);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_ints, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_max, sizeof(int) * max_alignments);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_flags, sizeof(int) * max_tiles);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_descs, sizeof(AlnDesc) * max_alignments);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_items_tc, sizeof(WorkItem) * max_tiles);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_items_pc, sizeof(WorkItem) * max_tiles);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_ints, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_ints, 0, 4 * sizeof(int));
  if (e != cudaSuccess) {
    free_batch(b);
    return cuda_error(e, "batch allocation");
  }
  int rc = capture_graph(b);
  if (rc != RNJ_OK) {
    free_batch(b);
    return rc;
  }
  *out = b;
  return RNJ_OK;
}

int rnj_batch_add(rnj_batch *b, rnj_aln *aln, int model, float *d_out, size_t ld, int *slot) {
  if (!b || !aln) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (aln->ctx != b->ctx) return set_error(RNJ_ERR_INVALID, "alignment from another context");
  const Packed &p = aln->p;
  if (p.n < 1) return set_error(RNJ_ERR_INVALID, "empty alignment");
  if (!is_tc_kind(p.kind) && p.Wp / kKW > kMaxFusedWords / kKW)
    return set_error(RNJ_ERR_INVALID, "alignments longer than 65280 columns on the bit-plane "
                                      "kernels are not batched; use rnj_distance");
  if (is_tc_kind(p.kind) && p.L > kMaxFusedColumns)
    return set_error(RNJ_ERR_INVALID, "alignments longer than 65535 columns on the tensor "
                                      "cores are not batched; use rnj_distance");
  if ((int)b->entries.size() >= b->cap_aln)
    return set_error(RNJ_ERR_BUSY, "batch is full (alignments)");
  const int nt = tiles_of(p.n);
  const long long ntiles = (p.kind == KIND_NAIVE && (p.flags & RNJ_FULL_ROWS))
                               ? (long long)nt * nt
                               : tri_tiles(nt);
  if (b->tiles_used + ntiles > b->cap_tiles) return set_error(RNJ_ERR_BUSY, "batch is full (tiles)");
  DeviceGuard g(b->ctx->device);
  Entry en;
  en.aln = aln;
  en.model = model;
  en.owned = (d_out == nullptr);
  en.ld = d_out ? ld : (size_t)std::max(4, (p.n + 3) / 4 * 4);
  en.out = d_out;
  if (d_out && ld < (size_t)p.n) return set_error(RNJ_ERR_INVALID, "ld < n");
  if (!d_out) {
    cudaError_t e = cudaMallocAsync((void **)&en.out, en.ld * p.n * sizeof(float), b->ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "batch output allocation");
  }
  en.owns_aln = false;
  en.flag_off = b->tiles_used;
  en.ntiles = ntiles;
  b->tiles_used += ntiles;
  b->entries.push_back(en);
  if (slot) *slot = (int)b->entries.size() - 1;
  return RNJ_OK;
}

int rnj_batch_add_many(rnj_batch *b, int count, const void *const *d_chars, const int *n,
                       const int *L, const size_t *ld, const int *type, const int *model, int flags,
                       float *const *d_out, const size_t *ld_out, int *slots) {
  if (!b || count < 0 || (count > 0 && (!d_chars || !n || !L || !ld || !type || !model)))
    return set_error(RNJ_ERR_INVALID, "null argument");
  rnj_ctx *ctx = b->ctx;
  DeviceGuard g(ctx->device);
  for (int k = 0; k < count; ++k) {
    if (type[k] != RNJ_DNA && type[k] != RNJ_PROTEIN)
      return set_error(RNJ_ERR_INVALID, "types must be resolved (RNJ_DNA or RNJ_PROTEIN)");
    if (n[k] < 1 || L[k] < 0 || ld[k] < (size_t)L[k])
      return set_error(RNJ_ERR_INVALID, "invalid alignment shape");
  }
  // Residue alphabets of every protein alignment: one presence launch over all
  // of them, one copy and one synchronisation.
  std::vector<int> pidx(count, -1);
  std::vector<PackJob> pres;
  long long pres_units = 0;
  for (int k = 0; k < count; ++k) {
    if (type[k] != RNJ_PROTEIN) continue;
    pidx[k] = (int)pres.size();
    PackJob j;
    memset(&j, 0, sizeof j);
    j.chars = (const uint8_t *)d_chars[k];
    j.ld = ld[k];
    j.n = n[k];
    j.L = L[k];
    j.unit0 = pres_units;
    pres_units += (long long)n[k] * ((L[k] + kPresenceSeg - 1) / kPresenceSeg);
    pres.push_back(j);
  }
  const int np = (int)pres.size();
  std::vector<uint32_t> masks((size_t)np * 8, 0);
  if (np > 0) {
    uint8_t *d_buf = nullptr;
    const size_t jbytes = pres.size() * sizeof(PackJob);
    RNJ_CUDA(cudaMallocAsync((void **)&d_buf, jbytes + masks.size() * sizeof(uint32_t), ctx->stream),
             "mask buffer");
    PackJob *d_jobs = (PackJob *)d_buf;
    uint32_t *d_masks = (uint32_t *)(d_buf + jbytes);
    cudaError_t e = cudaMemcpyAsync(d_jobs, pres.data(), jbytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_masks, 0, masks.size() * sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = launch_presence_multi(d_jobs, np, pres_units, d_masks, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(masks.data(), d_masks, masks.size() * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(d_buf, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "residue presence");
  }
  // Layouts of all alignments in one device arena; one pack launch for the bit
  // planes of all of them and one for the tensor-core features.
  std::vector<rnj_aln *> alns(count, nullptr);
  std::vector<size_t> offs(count, 0);
  std::vector<PackJob> planes, feats;
  long long plane_units = 0, feat_units = 0;
  size_t total = 0;
  for (int k = 0; k < count; ++k) {
    uint8_t lut[256];
    int kind;
    lut_for(type[k], flags, pidx[k] >= 0 ? masks.data() + 8 * pidx[k] : nullptr, lut, &kind);
    rnj_aln *a = new rnj_aln();
    a->ctx = ctx;
    a->owns_mem = false;
    const size_t bytes = packed_layout(a->p, n[k], L[k], type[k], flags, kind, lut, false);
    alns[k] = a;
    offs[k] = total;
    total += (bytes + 255) / 256 * 256;
    PackJob j;
    memset(&j, 0, sizeof j);
    j.chars = (const uint8_t *)d_chars[k];
    j.ld = ld[k];
    j.n = n[k];
    j.L = L[k];
    j.Np = a->p.Np;
    j.kind = a->p.kind;
    if (is_tc_kind(a->p.kind)) {
      j.W = a->p.Lk;
      j.nfb = a->p.nfb;
      memcpy(j.lut, lut, 256);
      j.unit0 = feat_units;
      feat_units += (long long)a->p.Np * (a->p.Lk / 32);
      if (feat_units % 256 != 0) {  // Np is a multiple of 128 and Lk of 256
        for (rnj_aln *x : alns) delete x;
        return set_error(RNJ_ERR_UNSUPPORTED, "feature pack units not a multiple of 256");
      }
      feats.push_back(j);
    } else {
      j.W = a->p.Wp;
      memcpy(j.lut, lut, 256);
      j.unit0 = plane_units;
      plane_units += (long long)(a->p.Np / 32) * (a->p.Wp / 8);
      planes.push_back(j);
    }
  }
  auto drop = [&](uint8_t *arena) {
    for (rnj_aln *a : alns) delete a;
    if (arena) cudaFreeAsync(arena, ctx->stream);
  };
  uint8_t *arena = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&arena, std::max<size_t>(total, 256), ctx->stream);
  if (e != cudaSuccess) {
    drop(nullptr);
    return cuda_error(e, "batch pack arena");
  }
  {
    size_t pi = 0, fi = 0;
    for (int k = 0; k < count; ++k) {
      Packed &p = alns[k]->p;
      if (is_tc_kind(p.kind)) {
        p.feat = arena + offs[k];
        feats[fi++].dst = p.feat;
      } else {
        p.planes = (uint32_t *)(arena + offs[k]);
        planes[pi++].dst = p.planes;
      }
    }
  }
  {
    const size_t pb = planes.size() * sizeof(PackJob), fb = feats.size() * sizeof(PackJob);
    uint8_t *d_jobs = nullptr;
    e = cudaMallocAsync((void **)&d_jobs, std::max<size_t>(pb + fb, 16), ctx->stream);
    if (e == cudaSuccess && pb)
      e = cudaMemcpyAsync(d_jobs, planes.data(), pb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && fb)
      e = cudaMemcpyAsync(d_jobs + pb, feats.data(), fb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = launch_pack_chars_multi((const PackJob *)d_jobs, (int)planes.size(), plane_units,
                                  ctx->stream);
    if (e == cudaSuccess)
      e = launch_pack_features_multi((const PackJob *)(d_jobs + pb), (int)feats.size(), feat_units,
                                     ctx->stream);
    if (d_jobs) cudaFreeAsync(d_jobs, ctx->stream);
    if (e != cudaSuccess) {
      drop(arena);
      return cuda_error(e, "batch pack kernels");
    }
  }
  for (int k = 0; k < count; ++k) {
    const int rc = is_tc_kind(alns[k]->p.kind) ? encode_features_map(alns[k]->p)
                                                   : encode_planes_map(alns[k]->p);
    if (rc != RNJ_OK) {
      drop(arena);
      return rc;
    }
  }
  b->arenas.push_back(arena);
  for (int k = 0; k < count; ++k) {
    int slot = -1;
    const int rc = rnj_batch_add(b, alns[k], model[k], d_out ? d_out[k] : nullptr,
                                 ld_out ? ld_out[k] : 0, &slot);
    if (rc != RNJ_OK) {
      // Alignments already added stay in the batch (its arena is the batch's);
      // the rest are released here.
      for (int r = k; r < count; ++r) delete alns[r];
      return rc;
    }
    b->entries[slot].owns_aln = true;
    if (slots) slots[k] = slot;
  }
  return RNJ_OK;
}

int rnj_batch_run(rnj_batch *b) {
  if (!b) return set_error(RNJ_ERR_INVALID, "null batch");
  rnj_ctx *ctx = b->ctx;
  DeviceGuard g(ctx->device);
  // The pinned upload buffers of the previous run must have been read.
  if (b->uploaded_pending) RNJ_CUDA(cudaEventSynchronize(b->ev_uploaded), "previous upload");
  const int na = (int)b->entries.size();
  long long ntc = 0, npc = 0;
  std::vector<int> order(na);
  for (int a = 0; a < na; ++a) order[a] = a;
  // Cost per tile grows with the columns; longest first.
  // (tensor cores: feature blocks x columns; bit planes: planes x words).
  auto cost = [&](int a) {
    const Packed &p = b->entries[a].aln->p;
    return is_tc_kind(p.kind) ? (long long)p.nfb * p.Lk : (long long)p.NP * p.Wp * 32;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
  for (int a = 0; a < na; ++a) {
    const Entry &en = b->entries[a];
    const Packed &p = en.aln->p;
    EpiParams ep = epi_params_for(p, en.model);
    ep.out = en.out;
    ep.ld = en.ld;
    ep.max_bits = b->d_max + a;
    ep.tile_flags = b->d_flags + en.flag_off;
    ep.err = b->d_ints + 3;
    b->h_descs[a] = desc_for(p, ep);
  }
  // Tuned launch shape: each alignment's tile-order band from its bucket, the
  // ring depth from the bucket of the tensor-core alignment with the most
  // work (tiles x K).
  std::vector<int> bands(na, 0);
  {
    int tuned = 0, depth = 0;
    long long top = -1;
    for (int a = 0; a < na; ++a) {
      const Packed &p = b->entries[a].aln->p;
      bool found = false;
      const TuneParams tp = tune_lookup(p.n, p.L, p.type, p.flags, &found);
      tuned += found ? 1 : 0;
      bands[a] = tp.tile_band > 0 ? tp.tile_band : kBand;
      const long long work = b->entries[a].ntiles * cost(a);
      if (is_tc_kind(p.kind) && work > top) {
        top = work;
        depth = tp.tc_stages;
      }
    }
    b->tuned_alns = tuned;
    // The graph's launch holds the deepest ring; the run's depth travels in
    // the first descriptor (no re-capture).
    b->tc_stages = depth;
    if (na > 0) b->h_descs[0].stages = depth;
  }
  for (int oi = 0; oi < na; ++oi) {
    const int a = order[oi];
    const Entry &en = b->entries[a];
    const bool tc = is_tc_kind(en.aln->p.kind);
    // tensor-core triangles in the banded order of their bucket's band
    // height (consecutive items go to consecutive CTAs, which then share row
    // tiles in L2); full-square and bit-plane items in row-major order
    const bool banded = tc && !b->h_descs[a].full;
    const int nt = b->h_descs[a].nt;
    for (long long t = 0; t < en.ntiles; ++t) {
      WorkItem w;
      w.aln = a;
      w.tile = banded ? banded_tile((int)t, nt, bands[a]) : (int)t;
      if (tc) b->h_items_tc[ntc++] = w;
      else b->h_items_pc[npc++] = w;
    }
  }
  b->h_ints[0] = (int)ntc;
  b->h_ints[1] = (int)npc;
  // Order after the packing work queued on the context stream.
  RNJ_CUDA(cudaEventRecord(b->ev_ready, ctx->stream), "ready event");
  RNJ_CUDA(cudaStreamWaitEvent(b->stream, b->ev_ready, 0), "wait ready");
  if (na > 0)
    RNJ_CUDA(cudaMemcpyAsync(b->d_descs, b->h_descs, sizeof(AlnDesc) * na, cudaMemcpyHostToDevice,
                             b->stream),
             "descriptor upload");
  if (ntc > 0)
    RNJ_CUDA(cudaMemcpyAsync(b->d_items_tc, b->h_items_tc, sizeof(WorkItem) * ntc,
                             cudaMemcpyHostToDevice, b->stream),
             "work list upload");
  if (npc > 0)
    RNJ_CUDA(cudaMemcpyAsync(b->d_items_pc, b->h_items_pc, sizeof(WorkItem) * npc,
                             cudaMemcpyHostToDevice, b->stream),
             "work list upload");
  RNJ_CUDA(cudaMemcpyAsync(b->d_ints, b->h_ints, 2 * sizeof(int), cudaMemcpyHostToDevice, b->stream),
           "count upload");
  RNJ_CUDA(cudaMemsetAsync(b->d_ints + 3, 0, sizeof(int), b->stream), "error clear");
  RNJ_CUDA(cudaEventRecord(b->ev_uploaded, b->stream), "upload event");
  b->uploaded_pending = true;
  b->host_max_valid = false;
  RNJ_CUDA(cudaGraphLaunch(b->exec, b->stream), "graph launch");
  RNJ_CUDA(cudaEventRecord(b->ev_done, b->stream), "done event");
  // Later work on the context stream (copies, new packs) sees the results.
  if (b->join) RNJ_CUDA(cudaStreamWaitEvent(ctx->stream, b->ev_done, 0), "join");
  return RNJ_OK;
}

int rnj_batch_poll(rnj_batch *b, int *done) {
  if (!b || !done) return set_error(RNJ_ERR_INVALID, "null argument");
  DeviceGuard g(b->ctx->device);
  const cudaError_t e = cudaEventQuery(b->ev_done);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return RNJ_OK;
  }
  if (e != cudaSuccess) return cuda_error(e, "batch poll");
  *done = 1;
  return RNJ_OK;
}

int rnj_batch_synchronize(rnj_batch *b) {
  if (!b) return set_error(RNJ_ERR_INVALID, "null batch");
  DeviceGuard g(b->ctx->device);
  RNJ_CUDA(cudaEventSynchronize(b->ev_done), "batch sync");
  int err = 0;
  RNJ_CUDA(cudaMemcpyAsync(&err, b->d_ints + 3, sizeof(int), cudaMemcpyDeviceToHost, b->stream),
           "error word");
  RNJ_CUDA(cudaStreamSynchronize(b->stream), "error word");
  if (err) return set_error(RNJ_ERR_TIMEOUT, "a bounded device wait ran out in the batch");
  return RNJ_OK;
}

int rnj_batch_output(rnj_batch *b, int slot, float **d_out, size_t *ld, float *max_out) {
  if (!b || slot < 0 || slot >= (int)b->entries.size())
    return set_error(RNJ_ERR_INVALID, "no such batch slot");
  const Entry &en = b->entries[slot];
  if (d_out) *d_out = en.out;
  if (ld) *ld = en.ld;
  if (max_out) {
    // The maxima of all slots are read once per run (one copy, one wait).
    DeviceGuard g(b->ctx->device);
    RNJ_CUDA(cudaEventSynchronize(b->ev_done), "batch sync");
    if (!b->host_max_valid) {
      b->host_max.assign(b->entries.size(), 0);
      RNJ_CUDA(cudaMemcpyAsync(b->host_max.data(), b->d_max, sizeof(int) * b->entries.size(),
                               cudaMemcpyDeviceToHost, b->stream),
               "max copy");
      RNJ_CUDA(cudaStreamSynchronize(b->stream), "max copy");
      b->host_max_valid = true;
    }
    memcpy(max_out, &b->host_max[slot], sizeof(float));
  }
  return RNJ_OK;
}

int rnj_batch_take(rnj_batch *b, int slot, rnj_mat **out) {
  if (!b || !out || slot < 0 || slot >= (int)b->entries.size())
    return set_error(RNJ_ERR_INVALID, "no such batch slot");
  Entry &en = b->entries[slot];
  if (!en.owned || !en.out) return set_error(RNJ_ERR_INVALID, "slot output is not owned by the batch");
  DeviceGuard g(b->ctx->device);
  RNJ_CUDA(cudaEventSynchronize(b->ev_done), "batch sync");
  if (!b->host_max_valid) {
    b->host_max.assign(b->entries.size(), 0);
    RNJ_CUDA(cudaMemcpyAsync(b->host_max.data(), b->d_max, sizeof(int) * b->entries.size(),
                             cudaMemcpyDeviceToHost, b->stream),
             "max copy");
    RNJ_CUDA(cudaStreamSynchronize(b->stream), "max copy");
    b->host_max_valid = true;
  }
  const int bits = b->host_max[slot];
  rnj_mat *m = new rnj_mat();
  m->ctx = b->ctx;
  m->d = en.out;
  m->n = en.aln->p.n;
  m->ld = en.ld;
  m->owns = true;  // the matrix now owns the output buffer
  m->has_host_max = true;
  memcpy(&m->host_max, &bits, sizeof(float));
  en.owned = false;
  en.out = nullptr;
  *out = m;
  return RNJ_OK;
}

int rnj_batch_tuning(rnj_batch *b, int *ring_depth, int *tuned_alignments) {
  if (!b) return set_error(RNJ_ERR_INVALID, "null batch");
  if (ring_depth) *ring_depth = fused_ring_depth(b->tc_stages);
  if (tuned_alignments) *tuned_alignments = b->tuned_alns;
  return RNJ_OK;
}

int rnj_batch_size(rnj_batch *b, int *alignments, long long *tiles) {
  if (!b) return set_error(RNJ_ERR_INVALID, "null batch");
  if (alignments) *alignments = (int)b->entries.size();
  if (tiles) *tiles = b->tiles_used;
  return RNJ_OK;
}

int rnj_batch_clear(rnj_batch *b) {
  if (!b) return set_error(RNJ_ERR_INVALID, "null batch");
  DeviceGuard g(b->ctx->device);
  RNJ_CUDA(cudaStreamSynchronize(b->stream), "batch sync");
  for (auto &e : b->entries)
  {
    if (e.owned && e.out) cudaFreeAsync(e.out, b->ctx->stream);
    if (e.owns_aln) rnj_aln_destroy(e.aln);
  }
  for (void *a : b->arenas) cudaFreeAsync(a, b->ctx->stream);
  b->arenas.clear();
  b->entries.clear();
  b->tiles_used = 0;
  b->host_max_valid = false;
  return RNJ_OK;
}

int rnj_batch_destroy(rnj_batch *b) {
  if (!b) return RNJ_OK;
  DeviceGuard g(b->ctx->device);
  free_batch(b);
  return RNJ_OK;
}

}  // extern "C"
