// rnj_api.cu -- the C ABI of librnjgpu.so (declared in include/rnj.h): context,
// alignment upload and packing, distance orchestration, copy-out into host rows.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

namespace rnj {

static thread_local std::string g_error;

int set_error(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char *what) {
  const int code = (e == cudaErrorMemoryAllocation) ? RNJ_ERR_NOMEM : RNJ_ERR_CUDA;
  return set_error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RNJ_CUDA(call, what)                       \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_error(e_, what); \
  } while (0)

// cuTensorMapEncodeTiled, resolved through the runtime so the library loads on
// hosts without a driver (the symbol is only needed once a device is in use).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

int encode_planes_map(Packed &p) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(RNJ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  cuuint64_t dims[3] = {(cuuint64_t)p.Np, (cuuint64_t)p.Wp, (cuuint64_t)p.NP};
  cuuint64_t strides[2] = {(cuuint64_t)p.Np * 4, (cuuint64_t)p.Np * p.Wp * 4};
  cuuint32_t box[3] = {(cuuint32_t)kTile, (cuuint32_t)kKW, (cuuint32_t)p.NP};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&p.tmap, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, p.planes, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(RNJ_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return RNJ_OK;
}

// 3-D map over the K-blocked FP4 features: (128 bytes, Np rows, 4 * Lk / 256
// blocks), box 128 x 128 x 1 = one contiguous 16 KB run, 128-byte swizzle (the
// layout the tcgen05 shared-memory descriptors expect).
int encode_features_map(Packed &p) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(RNJ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  cuuint64_t dims[3] = {128, (cuuint64_t)p.Np, (cuuint64_t)p.nfb * (p.Lk / 256)};
  cuuint64_t strides[2] = {128, (cuuint64_t)p.Np * 128};
  cuuint32_t box[3] = {128, (cuuint32_t)kTile, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&p.fmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, p.feat, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(RNJ_ERR_CUDA, "cuTensorMapEncodeTiled (features) failed (" +
                                       std::to_string((int)r) + ")");
  return RNJ_OK;
}

// resolveChar of the loaders (dataloaderFasta.hpp:184-199).
char resolve_char(char c, int type) {
  if (type == RNJ_DNA) {
    if (!(c == 'a' || c == 'A' || c == 'c' || c == 'C' || c == 'g' || c == 'G' || c == 't' ||
          c == 'T' || c == 'u' || c == 'U'))
      return '-';
    return c;
  }
  if (c == '-' || c == '.' || c == 'X' || c == 'x' || c == 'z' || c == 'Z' || c == 'b' ||
      c == 'B' || c == 'J' || c == 'j' || c == '?')
    return '-';
  return c;
}

// Per-byte plane bits for DNA (bit0 code high, bit1 code low, bit2 valid, bit3
// upper-case A/C/G/T).  Fast rule (dataloaderFasta.hpp:155-180): only A/C/G/T in
// either case are valid.  Naive rule (simpleDistanceCalculator.cpp with
// resolveChar): A/C/G/T/U in either case are valid.
void dna_lut(bool naive, uint8_t lut[256]) {
  memset(lut, 0, 256);
  struct { char c; int code; } letters[] = {{'A', 0}, {'G', 1}, {'T', 2}, {'C', 3}};
  for (auto &l : letters) {
    const uint8_t bits = (uint8_t)(((l.code >> 1) & 1) | ((l.code & 1) << 1) | 4);
    lut[(uint8_t)l.c] = bits | 8;
    lut[(uint8_t)(l.c - 'A' + 'a')] = bits;
  }
  if (naive) {
    lut[(uint8_t)'U'] = 4;
    lut[(uint8_t)'u'] = 4;
  }
}

// Transform parameters of a packed alignment (scratch pointers left null).
namespace {
std::atomic<uint32_t> g_wait_us{0};
std::atomic<int> g_wait_stall{0};
}  // namespace

void apply_wait_settings(EpiParams &ep) {
  ep.wait_us = g_wait_us.load(std::memory_order_relaxed);
  ep.stall = g_wait_stall.load(std::memory_order_relaxed);
}

EpiParams epi_params_for(const Packed &p, int model) {
  EpiParams ep;
  apply_wait_settings(ep);
  ep.n = p.n;
  ep.L = p.L;
  ep.model = model;
  ep.type = p.type;
  ep.compat_wrap = (p.type == RNJ_PROTEIN && (p.flags & RNJ_FASTDIST) &&
                    (p.flags & RNJ_COMPAT_PROTEIN_WRAP)) ? 1 : 0;
  ep.full = (p.kind == KIND_NAIVE && (p.flags & RNJ_FULL_ROWS)) ? 1 : 0;
  ep.jc_b = (p.type == RNJ_PROTEIN) ? (20.0 - 1) / 20.0 : (4.0 - 1) / 4.0;
  return ep;
}

// Work-list descriptor of one packed alignment for the persistent kernels.
AlnDesc desc_for(const Packed &p, const EpiParams &ep) {
  AlnDesc d;
  memset(&d, 0, sizeof(d));
  d.map = is_tc_kind(p.kind) ? p.fmap : p.tmap;
  d.out = ep.out;
  d.counts = ep.counts;
  d.ld = ep.ld;
  d.max_bits = ep.max_bits;
  d.tile_flags = ep.tile_flags;
  d.err = ep.err;
  d.n = p.n;
  d.L = p.L;
  d.nt = tiles_of(p.n);
  d.kdim = is_tc_kind(p.kind) ? p.Lk : p.Wp;
  d.model = ep.model;
  d.type = ep.type;
  d.compat = ep.compat_wrap;
  d.full = ep.full;
  d.kind = p.kind;
  d.np = is_tc_kind(p.kind) ? p.nfb : p.NP;
  d.wait_us = (int)ep.wait_us;
  d.stall = ep.stall;
  d.row0 = ep.row0;
  d.jc_b = ep.jc_b;
  return d;
}

}  // namespace rnj

using namespace rnj;

namespace {

void mark(rnj_ctx *ctx, int stage, int end) {
  if (!ctx->profiling) return;
  cudaEventRecord(ctx->ev[2 * stage + end], ctx->stream);
  if (end) ctx->ev_used[stage] = true;
}

int ensure_scratch_words(rnj_ctx *ctx, size_t words) {
  Scratch &s = ctx->scratch;
  if (s.words_cap >= words) return RNJ_OK;
  if (s.words) cudaFreeAsync(s.words, ctx->stream);
  s.words = nullptr;
  s.words_cap = 0;
  RNJ_CUDA(cudaMallocAsync((void **)&s.words, words * sizeof(int), ctx->stream), "scratch");
  s.words_cap = words;
  return RNJ_OK;
}

int ensure_stage(rnj_ctx *ctx, size_t bytes) {
  if (ctx->stage_cap >= bytes) return RNJ_OK;
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "staging sync");
  for (int b = 0; b < 2; ++b) {
    if (ctx->h_stage[b]) cudaFreeHost(ctx->h_stage[b]);
    ctx->h_stage[b] = nullptr;
  }
  ctx->stage_cap = 0;
  for (int b = 0; b < 2; ++b)
    RNJ_CUDA(cudaMallocHost(&ctx->h_stage[b], bytes), "pinned staging");
  ctx->stage_cap = bytes;
  return RNJ_OK;
}

int host_threads(int threads) {
  if (threads > 0) return threads;
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)std::min<long>(n, 64) : 1;
}

// True when rows[0..nrows) are one contiguous block of n-float rows in
// page-locked (pinned or registered) host memory: the device can write it
// directly, without the staging buffers.
bool rows_pinned_block(float *const *rows, int nrows, int n) {
  for (int r = 1; r < nrows; ++r)
    if (rows[r] != rows[0] + (size_t)r * n) return false;
  cudaPointerAttributes a0, a1;
  if (cudaPointerGetAttributes(&a0, rows[0]) != cudaSuccess ||
      cudaPointerGetAttributes(&a1, rows[0] + (size_t)nrows * n - 1) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of a failed query
    return false;
  }
  return a0.type == cudaMemoryTypeHost && a1.type == cudaMemoryTypeHost;
}

// Parallel row copy: dst[r] (n floats) <- src + r * n.
void scatter_rows(const float *src, float **dst, int nrows, int n, int threads) {
  const size_t bytes = (size_t)nrows * n * sizeof(float);
  int t = std::max(1, std::min(threads, (int)(bytes / (1 << 20)) + 1));
  t = std::min(t, nrows);
  if (t <= 1) {
    for (int r = 0; r < nrows; ++r) memcpy(dst[r], src + (size_t)r * n, (size_t)n * sizeof(float));
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 0; k < t; ++k) {
    pool.emplace_back([=] {
      for (int r = k; r < nrows; r += t)
        memcpy(dst[r], src + (size_t)r * n, (size_t)n * sizeof(float));
    });
  }
  for (auto &th : pool) th.join();
}

// Upload raw bytes already on the device (n rows, stride ld) into planes.
}  // namespace

// Packing LUT and plane layout.  DNA needs nothing from the data; protein ranks
// the residue bytes present (mask: 256-bit byte-presence mask).
void lut_for(int type, int flags, const uint32_t *mask, uint8_t lut[256], int *kind) {
  const bool naive = (flags & RNJ_FASTDIST) == 0;
  if (type == RNJ_DNA) {
    *kind = naive ? KIND_NAIVE : KIND_DNA;
    dna_lut(naive, lut);
    return;
  }
  int rank = 0;
  for (int c = 0; c < 256; ++c) {
    const bool present = (mask[c >> 5] >> (c & 31)) & 1u;
    if (resolve_char((char)c, RNJ_PROTEIN) == '-') lut[c] = 0xFF;
    else if (present) lut[c] = (uint8_t)(rank++);
    else lut[c] = 0xFF;
  }
  *kind = rank <= 4 ? KIND_MISM2 : (rank <= 32 ? KIND_MISM5 : KIND_MISM7);
}

// (pack_prepared, declared in rnj_objects.h: allocation, pack kernel and TMA
// map of an alignment whose LUT is known; no synchronisation.)

namespace {

int pack_from_device_chars(rnj_ctx *ctx, const uint8_t *d_chars, int n, int L, size_t ld,
                           int type, int flags, rnj_aln **out) {
  if (n < 0 || L < 0 || (n > 0 && ld < (size_t)L))
    return set_error(RNJ_ERR_INVALID, "invalid alignment shape");
  if (type != RNJ_DNA && type != RNJ_PROTEIN)
    return set_error(RNJ_ERR_INVALID, "sequence type must be resolved before packing");
  uint8_t lut[256];
  int kind;
  if (type == RNJ_DNA) {
    lut_for(type, flags, nullptr, lut, &kind);
  } else {
    // Rank the residue alphabet present in the alignment.
    RNJ_CUDA(cudaMemsetAsync(ctx->d_mask, 0, 8 * sizeof(uint32_t), ctx->stream), "mask clear");
    if (n > 0 && L > 0)
      RNJ_CUDA(launch_presence(d_chars, ld, n, L, ctx->d_mask, ctx->stream), "presence kernel");
    RNJ_CUDA(cudaMemcpyAsync(ctx->h_mask, ctx->d_mask, 8 * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, ctx->stream),
             "mask copy");
    RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "mask sync");
    lut_for(type, flags, ctx->h_mask, lut, &kind);
  }
  return pack_prepared(ctx, d_chars, n, L, ld, type, flags, kind, lut, out);
}

}  // namespace

size_t packed_layout(Packed &p, int n, int L, int type, int flags, int kind, const uint8_t *lut,
                     bool tuned_kernel) {
  const bool tc_choice = !tuned_kernel || tune_lookup(n, L, type, flags).dna_kernel == 0;
  p.n = n;
  p.L = L;
  p.type = type;
  p.flags = flags;
  p.kind = kind;
  p.W = (L + 31) / 32;
  p.Wp = std::max(kKW, (p.W + kKW - 1) / kKW * kKW);
  p.Np = std::max(kTile, (n + kTile - 1) / kTile * kTile);
  if (kind == KIND_DNA && !(flags & RNJ_POPCOUNT) && L <= kMaxTcColumns && tc_choice) {
    // FP4 feature rows for the tensor-core kernel instead of bit planes.
    p.kind = KIND_DNA_TC;
    p.NP = 0;
    p.nfb = 4;
    p.Lk = std::max(256, (L + 255) / 256 * 256);
    return (size_t)p.Np * 4 * p.Lk / 2;
  }
  if (type == RNJ_PROTEIN && lut && !(flags & RNJ_POPCOUNT) && L <= kMaxTcColumns && tc_choice) {
    // Protein on the tensor cores: a valid block and one one-hot block per
    // residue rank present, when there are at most kMaxTcRanks ranks.
    int ranks = 0;
    for (int c = 0; c < 256; ++c)
      if (lut[c] != 0xFF) ranks = std::max(ranks, lut[c] + 1);
    if (ranks >= 1 && ranks <= kMaxTcRanks) {
      p.kind = KIND_PROT_TC;
      p.NP = 0;
      p.nfb = 1 + ranks;
      p.Lk = std::max(256, (L + 255) / 256 * 256);
      return (size_t)p.Np * p.nfb * (p.Lk / 2);
    }
  }
  p.NP = planes_of(kind);
  return (size_t)p.NP * p.Wp * p.Np * sizeof(uint32_t);
}

int pack_prepared(rnj_ctx *ctx, const uint8_t *d_chars, int n, int L, size_t ld, int type,
                  int flags, int kind, const uint8_t lut[256], rnj_aln **out, bool tuned_kernel) {
  rnj_aln *a = new rnj_aln();
  a->ctx = ctx;
  Packed &p = a->p;
  const size_t pbytes = packed_layout(p, n, L, type, flags, kind, lut, tuned_kernel);
  if (is_tc_kind(p.kind)) {
    const size_t fbytes = pbytes;
    cudaError_t e = cudaMallocAsync((void **)&p.feat, fbytes, ctx->stream);
    if (e != cudaSuccess) {
      delete a;
      return cuda_error(e, "feature allocation");
    }
    mark(ctx, 0, 0);
    e = p.kind == KIND_DNA_TC
            ? launch_pack_features(d_chars, ld, n, L, p.Np, p.Lk, p.feat, ctx->stream)
            : launch_pack_features_prot(d_chars, ld, n, L, p.Np, p.Lk, p.nfb, lut, p.feat,
                                        ctx->stream);
    mark(ctx, 0, 1);
    int rc = (e == cudaSuccess) ? encode_features_map(p) : cuda_error(e, "feature pack kernel");
    if (rc != RNJ_OK) {
      cudaFreeAsync(p.feat, ctx->stream);
      delete a;
      return rc;
    }
    *out = a;
    return RNJ_OK;
  }
  const size_t bytes = pbytes;
  cudaError_t e = cudaMallocAsync((void **)&p.planes, bytes, ctx->stream);
  if (e != cudaSuccess) {
    delete a;
    return cuda_error(e, "plane allocation");
  }
  mark(ctx, 0, 0);
  e = launch_pack_chars(d_chars, ld, p, lut, ctx->stream);
  mark(ctx, 0, 1);
  if (e != cudaSuccess) {
    cudaFreeAsync(p.planes, ctx->stream);
    delete a;
    return cuda_error(e, "pack kernel");
  }
  int rc = encode_planes_map(p);
  if (rc != RNJ_OK) {
    cudaFreeAsync(p.planes, ctx->stream);
    delete a;
    return rc;
  }
  *out = a;
  return RNJ_OK;
}

namespace {

int count_kind_for(const Packed &p, int model) {
  if (p.kind == KIND_DNA && model == RNJ_JC) return KIND_MISM2;
  return p.kind;
}

EpiParams epi_for(rnj_ctx *ctx, const Packed &p, int model) {
  EpiParams ep = epi_params_for(p, model);
  ep.max_bits = ctx->scratch.words;
  ep.err = ctx->d_err;
  ep.tile_flags = ctx->scratch.words + 2;
  return ep;
}

}  // namespace

// The error word copied to h_max[1] by a finished stream: RNJ_ERR_TIMEOUT (and
// the device word cleared) when a bounded wait ran out.
int take_device_error(rnj_ctx *ctx) {
  if (ctx->h_max[1] == 0) return RNJ_OK;
  ctx->h_max[1] = 0;
  cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
  return set_error(RNJ_ERR_TIMEOUT, "a bounded device wait ran out (pipeline stage lost)");
}

namespace {

// One alignment through the persistent tensor-core kernel: its triangle tiles
// are the work list, one CTA per SM.  Distances go through the packed counts
// and the transform kernel; EPI_COUNTS writes the raw counts directly.
int run_tc_single(rnj_ctx *ctx, const Packed &p, const EpiParams &ep, int epi_mode) {
  const int nt = tiles_of(p.n);
  const long long ntiles = ep.full ? (long long)nt * nt : tri_tiles(nt);
  const TuneParams tp = tune_lookup(p.n, p.L, p.type, p.flags);
  AlnDesc d = desc_for(p, ep);
  d.band = tp.tile_band;
  // Pageable source: the copy is taken before the call returns, so the stack
  // descriptor may go out of scope.
  RNJ_CUDA(cudaMemcpyAsync(ctx->d_desc, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream),
           "descriptor upload");
  if (epi_mode == EPI_COUNTS) {
    const int grid = (int)std::min<long long>(ntiles, ctx->num_sms);
    RNJ_CUDA(launch_tc_batch(ctx->d_desc, nullptr, nullptr, (int)ntiles, 0, (int)ntiles, nullptr,
                             grid, EPI_COUNTS, ctx->stream, tp.tc_stages),
             "tensor-core kernel");
    return RNJ_OK;
  }
  return run_tc_distances(ctx, p, ep, ctx->d_desc, nullptr, ntiles, ctx->stream, tp);
}

// Waits for the context's stream and reports (and clears) the sticky device
// error word: a timeout of any earlier call on this context, including calls
// that returned without waiting.
int check_device_error(rnj_ctx *ctx) {
  RNJ_CUDA(cudaMemcpyAsync(ctx->h_max + 1, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "error word copy");
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "distance sync");
  return take_device_error(ctx);
}

int run_popcount(rnj_ctx *ctx, const Packed &p, int ckind, int nk, int nt, EpiParams &ep);

// The distance pipeline on the context's stream: counts and transform (the
// tensor-core path through packed counts, the bit-plane path fused or split),
// then the saturation fix-up.
int run_distance(rnj_ctx *ctx, const Packed &p, int model, float *d_out, size_t ld,
                 int *d_max_copy) {
  const int nt = tiles_of(p.n);
  const long long ntiles = (p.kind == KIND_NAIVE && (p.flags & RNJ_FULL_ROWS))
                               ? (long long)nt * nt
                               : tri_tiles(nt);
  int rc = ensure_scratch_words(ctx, (size_t)ntiles + 2);
  if (rc != RNJ_OK) return rc;
  RNJ_CUDA(cudaMemsetAsync(ctx->scratch.words, 0, ((size_t)ntiles + 2) * sizeof(int), ctx->stream),
           "scratch clear");
  EpiParams ep = epi_for(ctx, p, model);
  ep.out = d_out;
  ep.ld = ld;
  if (p.n == 1) RNJ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float), ctx->stream), "diagonal");
  const int ckind = count_kind_for(p, model);
  const int nk = p.Wp / kKW;
  if (is_tc_kind(p.kind)) {
    // Marks stage 1 (the counting kernels) and opens stage 2 (the transforms).
    rc = run_tc_single(ctx, p, ep, EPI_PACKED);
    if (rc != RNJ_OK) return rc;
  } else {
    mark(ctx, 1, 0);
    rc = run_popcount(ctx, p, ckind, nk, nt, ep);
    if (rc != RNJ_OK) return rc;
    mark(ctx, 1, 1);
    mark(ctx, 2, 0);
  }
  RNJ_CUDA(launch_fixup(ep, nt, ctx->stream), "fix-up kernel");
  mark(ctx, 2, 1);
  if (d_max_copy)
    RNJ_CUDA(cudaMemcpyAsync(d_max_copy, ctx->scratch.words, sizeof(int), cudaMemcpyDeviceToDevice,
                             ctx->stream),
             "max copy");
  return RNJ_OK;
}

// The bit-plane counting kernels: fused counts + transform, or split counts +
// transform for alignments longer than one 16-bit accumulator pass.
int run_popcount(rnj_ctx *ctx, const Packed &p, int ckind, int nk, int nt, EpiParams &ep) {
  // K split (tuned per bucket): short triangles of long alignments leave most
  // SMs idle with one CTA per tile; splitting the columns over several CTAs
  // per tile (atomic count accumulation, then the transform) fills them.
  const TuneParams tp = tune_lookup(p.n, p.L, p.type, p.flags);
  ep.stages = tp.pop_stages;
  const bool split = tp.ksplit > 1 && nk >= 2 && !ep.full &&
                     (size_t)p.n * p.n * 3 * sizeof(uint32_t) <= (size_t)1 << 30;
  if (nk <= kMaxFusedWords / kKW && !split) {
    RNJ_CUDA(launch_count_tiles(p, ckind, EPI_DIST, ep, ctx->stream), "count kernel");
  } else {
    const size_t cbytes = (size_t)p.n * p.n * 3 * sizeof(uint32_t);
    uint32_t *counts = nullptr;
    RNJ_CUDA(cudaMallocAsync((void **)&counts, cbytes, ctx->stream), "count buffer");
    ep.counts = counts;
    cudaError_t e = cudaMemsetAsync(counts, 0, cbytes, ctx->stream);
    const int kchunk = split ? (nk + tp.ksplit - 1) / tp.ksplit * kKW : 0;
    if (e == cudaSuccess) e = launch_count_tiles(p, ckind, EPI_ATOMIC, ep, ctx->stream, kchunk);
    if (e == cudaSuccess) e = launch_transform_counts(ep, nt, ctx->stream);
    cudaFreeAsync(counts, ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "split count pipeline");
  }
  return RNJ_OK;
}

}  // namespace

void ctx_mark(rnj_ctx *ctx, int stage, int end) { mark(ctx, stage, end); }

int ctx_scratch(rnj_ctx *ctx, size_t words) { return ensure_scratch_words(ctx, words); }

EpiParams ctx_epi(rnj_ctx *ctx, const Packed &p, int model) { return epi_for(ctx, p, model); }

int ctx_check_error(rnj_ctx *ctx) { return check_device_error(ctx); }

bool ctx_block_pinned(const void *p, size_t bytes) {
  if (!p || bytes == 0) return false;
  cudaPointerAttributes a0, a1;
  if (cudaPointerGetAttributes(&a0, p) != cudaSuccess ||
      cudaPointerGetAttributes(&a1, (const char *)p + bytes - 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a0.type == cudaMemoryTypeHost && a1.type == cudaMemoryTypeHost;
}

int ensure_packed(rnj_ctx *ctx, long long tiles) {
  if (ctx->packed_tiles >= tiles) return RNJ_OK;
  if (ctx->d_packed) cudaFreeAsync(ctx->d_packed, ctx->stream);
  ctx->d_packed = nullptr;
  ctx->packed_tiles = 0;
  RNJ_CUDA(cudaMallocAsync((void **)&ctx->d_packed, (size_t)tiles * kPackedTileWords * 8,
                           ctx->stream),
           "packed-count buffer");
  ctx->packed_tiles = tiles;
  return RNJ_OK;
}

int run_tc_distances(rnj_ctx *ctx, const Packed &p, const EpiParams &ep, const AlnDesc *d_desc,
                     const WorkItem *d_items, long long nitems, cudaStream_t s,
                     const TuneParams &tp) {
  if (tp.tc_epilogue == 0 && p.L <= kMaxFusedColumns) {
    // Counts and transform in one launch (rnj_tcf.cu).
    mark(ctx, 1, 0);
    RNJ_CUDA(launch_tc_fused(d_desc, d_items, nullptr, (int)nitems, 0, (int)nitems,
                             (int)std::min<long long>(nitems, ctx->num_sms),
                             fused_variant_for(ep.model, ep.type, ep.compat_wrap, 0), s,
                             tp.tc_stages),
             "fused tensor-core kernel");
    mark(ctx, 1, 1);
    mark(ctx, 2, 0);
    return RNJ_OK;
  }
  int rc = ensure_packed(ctx, std::min<long long>(nitems, kTcChunkTiles));
  if (rc != RNJ_OK) return rc;
  return run_tc_chunks(ctx, d_desc, d_items, nitems, ctx->d_packed, s, tp.transform_ctas,
                       tp.tc_stages);
}

int run_tc_chunks(rnj_ctx *ctx, const AlnDesc *d_desc, const WorkItem *d_items, long long nitems,
                  uint64_t *packed, cudaStream_t s, int transform_ctas, int stages) {
  const int ctas = transform_ctas > 0 ? std::min(transform_ctas, kTransformCtasPerSm)
                                      : kTransformCtasPerSm;
  const int chunk = (int)std::min<long long>(nitems, kTcChunkTiles);
  for (long long i0 = 0; i0 < nitems; i0 += chunk) {
    const int cnt = (int)std::min<long long>(chunk, nitems - i0);
    if (i0 == 0) mark(ctx, 1, 0);
    RNJ_CUDA(launch_tc_batch(d_desc, d_items, nullptr, (int)nitems, (int)i0, cnt, packed,
                             std::min(cnt, ctx->num_sms), EPI_PACKED, s, stages),
             "tensor-core kernel");
    if (i0 + chunk >= nitems) mark(ctx, 1, 1);
    if (i0 + chunk >= nitems) mark(ctx, 2, 0);
    RNJ_CUDA(launch_tc_transform(d_desc, d_items, nullptr, (int)nitems, (int)i0, cnt, packed,
                                 std::min(cnt, ctas * ctx->num_sms), s),
             "transform kernel");
  }
  return RNJ_OK;
}

extern "C" {

const char *rnj_version(void) { return "rapidnj-b200 0.1.0 (sm_100a)"; }

const char *rnj_last_error(void) { return g_error.c_str(); }

int rnj_ctx_create(int device, rnj_ctx **out) {
  if (!out) return set_error(RNJ_ERR_INVALID, "out is NULL");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
  if (device < 0 || device >= count) return set_error(RNJ_ERR_INVALID, "no such CUDA device");
  DeviceGuard g(device);
  rnj_ctx *c = new rnj_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  // A blocking stream: it orders with the legacy default stream, so buffers that
  // callers fill on the default stream (as torch does) are complete before the
  // library reads them, and the caller's later default-stream work sees our results.
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_mask, 8 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_mask, 8 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_max, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e == cudaSuccess) memset(c->h_max, 0, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_desc, sizeof(AlnDesc));
  if (e != cudaSuccess) {
    rnj_ctx_destroy(c);
    return cuda_error(e, "context setup");
  }
  if (!encode_fn()) {
    rnj_ctx_destroy(c);
    return set_error(RNJ_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  }
  // Packed alignments and matrices come from the device's stream-ordered pool;
  // keep freed blocks in the pool instead of returning them at every
  // synchronisation, so repeated calls of one shape do not remap memory.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = c;
  return RNJ_OK;
}

int rnj_ctx_destroy(rnj_ctx *ctx) {
  if (!ctx) return RNJ_OK;
  DeviceGuard g(ctx->device);
  if (ctx->boot) rnj_batch_destroy(ctx->boot);  // uses the context's stream
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch.words) cudaFree(ctx->scratch.words);
  if (ctx->d_mask) cudaFree(ctx->d_mask);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->d_desc) cudaFree(ctx->d_desc);
  if (ctx->d_packed) cudaFree(ctx->d_packed);
  if (ctx->h_mask) cudaFreeHost(ctx->h_mask);
  if (ctx->h_max) cudaFreeHost(ctx->h_max);
  for (int b = 0; b < 2; ++b)
    if (ctx->h_stage[b]) cudaFreeHost(ctx->h_stage[b]);
  for (int k = 0; k < 6; ++k)
    if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
  if (ctx->h_words) cudaFreeHost(ctx->h_words);
  if (ctx->h_file) cudaFreeHost(ctx->h_file);
  if (ctx->s_up) {
    cudaStreamSynchronize(ctx->s_up);
    cudaStreamDestroy(ctx->s_up);
  }
  if (ctx->s_down) {
    cudaStreamSynchronize(ctx->s_down);
    cudaStreamDestroy(ctx->s_down);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return RNJ_OK;
}

int rnj_ctx_stream(rnj_ctx *ctx, void **stream) {
  if (!ctx || !stream) return set_error(RNJ_ERR_INVALID, "null argument");
  *stream = (void *)ctx->stream;
  return RNJ_OK;
}

int rnj_ctx_set_profiling(rnj_ctx *ctx, int on) {
  if (!ctx) return set_error(RNJ_ERR_INVALID, "null context");
  DeviceGuard g(ctx->device);
  if (on && !ctx->ev[0])
    for (int k = 0; k < 6; ++k) RNJ_CUDA(cudaEventCreate(&ctx->ev[k]), "event");
  ctx->profiling = on != 0;
  for (int k = 0; k < 3; ++k) ctx->ev_used[k] = false;
  return RNJ_OK;
}

int rnj_ctx_stage_times(rnj_ctx *ctx, float *ms) {
  if (!ctx || !ms) return set_error(RNJ_ERR_INVALID, "null argument");
  DeviceGuard g(ctx->device);
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "stage sync");
  for (int k = 0; k < 3; ++k) {
    ms[k] = 0.0f;
    if (ctx->profiling && ctx->ev_used[k])
      RNJ_CUDA(cudaEventElapsedTime(&ms[k], ctx->ev[2 * k], ctx->ev[2 * k + 1]), "stage time");
  }
  return RNJ_OK;
}

int rnj_ctx_memory(rnj_ctx *ctx, size_t *free_bytes, size_t *total_bytes) {
  if (!ctx) return set_error(RNJ_ERR_INVALID, "null context");
  DeviceGuard g(ctx->device);
  size_t f = 0, t = 0;
  RNJ_CUDA(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return RNJ_OK;
}

int rnj_set_wait_limit(unsigned int microseconds) {
  g_wait_us.store(microseconds, std::memory_order_relaxed);
  return RNJ_OK;
}

int rnj_test_wait_on_unset_flag(int on) {
  g_wait_stall.store(on ? 1 : 0, std::memory_order_relaxed);
  return RNJ_OK;
}

int rnj_ctx_synchronize(rnj_ctx *ctx) {
  if (!ctx) return set_error(RNJ_ERR_INVALID, "null context");
  DeviceGuard g(ctx->device);
  return check_device_error(ctx);
}

int rnj_detect_type(const char *seq0, int L) {
  for (int i = 0; i < L; ++i) {
    const signed char c = (signed char)seq0[i];
    if (!(c < 65 || c == 'A' || c == 'a' || c == 'C' || c == 'c' || c == 'G' || c == 'g' ||
          c == 'T' || c == 't' || c == 'U' || c == 'u' || c == 'N' || c == 'n'))
      return RNJ_PROTEIN;
  }
  return RNJ_DNA;
}

int rnj_aln_from_device(rnj_ctx *ctx, const void *d_chars, int n, int L, size_t ld, int type,
                        int flags, rnj_aln **out) {
  if (!ctx || !out || (n > 0 && L > 0 && !d_chars))
    return set_error(RNJ_ERR_INVALID, "null argument");
  DeviceGuard g(ctx->device);
  if (type == RNJ_UNKNOWN) {
    std::vector<char> row((size_t)std::max(L, 1));
    if (n > 0 && L > 0) {
      RNJ_CUDA(cudaMemcpyAsync(row.data(), d_chars, (size_t)L, cudaMemcpyDeviceToHost, ctx->stream),
               "first row copy");
      RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "first row sync");
    }
    type = rnj_detect_type(row.data(), n > 0 ? L : 0);
  }
  return pack_from_device_chars(ctx, (const uint8_t *)d_chars, n, L, ld, type, flags, out);
}

int rnj_aln_from_host_buffer(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld, int type,
                             int flags, rnj_aln **out) {
  if (!ctx || !out || (n > 0 && L > 0 && !chars))
    return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 0 || L < 0 || (n > 0 && ld < (size_t)L))
    return set_error(RNJ_ERR_INVALID, "invalid alignment shape");
  DeviceGuard g(ctx->device);
  if (type == RNJ_UNKNOWN) type = (n > 0) ? rnj_detect_type(chars, L) : RNJ_DNA;
  uint8_t *d = nullptr;
  const size_t bytes = std::max<size_t>((size_t)n * L, 1);
  RNJ_CUDA(cudaMallocAsync((void **)&d, bytes, ctx->stream), "upload buffer");
  cudaError_t e = cudaSuccess;
  if (n > 0 && L > 0)
    e = cudaMemcpy2DAsync(d, (size_t)L, chars, ld, (size_t)L, (size_t)n, cudaMemcpyHostToDevice,
                          ctx->stream);
  int rc = RNJ_OK;
  if (e != cudaSuccess) rc = cuda_error(e, "alignment upload");
  else rc = pack_from_device_chars(ctx, d, n, L, (size_t)std::max(L, 1), type, flags, out);
  cudaFreeAsync(d, ctx->stream);
  return rc;
}

int rnj_aln_from_host(rnj_ctx *ctx, const char *const *seqs, int n, int L, int type, int flags,
                      rnj_aln **out) {
  if (!ctx || !out || (n > 0 && !seqs)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 0 || L < 0) return set_error(RNJ_ERR_INVALID, "invalid alignment shape");
  DeviceGuard g(ctx->device);
  const size_t bytes = std::max<size_t>((size_t)n * L, 1);
  int rc = ensure_stage(ctx, bytes);
  if (rc != RNJ_OK) return rc;
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "staging reuse");
  char *stage = (char *)ctx->h_stage[0];
  for (int i = 0; i < n; ++i) memcpy(stage + (size_t)i * L, seqs[i], (size_t)L);
  return rnj_aln_from_host_buffer(ctx, stage, n, L, (size_t)L, type, flags, out);
}

int rnj_aln_from_bitstrings(rnj_ctx *ctx, const unsigned int *const *bit_strings,
                            const unsigned int *const *gap_filters, int n, int L,
                            int bit_strings_count, int type, int flags, rnj_aln **out) {
  if (!ctx || !out || (n > 0 && !bit_strings)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 0 || L < 0 || bit_strings_count < 0) return set_error(RNJ_ERR_INVALID, "invalid shape");
  if (type != RNJ_DNA && type != RNJ_PROTEIN)
    return set_error(RNJ_ERR_INVALID, "type must be RNJ_DNA or RNJ_PROTEIN");
  DeviceGuard g(ctx->device);
  const int bs_words = bit_strings_count * 4;  // 128-bit vectors -> uint32 words
  if (type == RNJ_PROTEIN) {
    // One resolved byte per site, bit_strings_count * 16 bytes per sequence.
    const size_t row = (size_t)bit_strings_count * 16;
    if (row < (size_t)L) return set_error(RNJ_ERR_INVALID, "bit strings shorter than L");
    const size_t bytes = std::max<size_t>((size_t)n * row, 1);
    int rc = ensure_stage(ctx, bytes);
    if (rc != RNJ_OK) return rc;
    RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "staging reuse");
    char *stage = (char *)ctx->h_stage[0];
    for (int i = 0; i < n; ++i) memcpy(stage + (size_t)i * row, bit_strings[i], row);
    return rnj_aln_from_host_buffer(ctx, stage, n, L, row, RNJ_PROTEIN,
                                    flags | RNJ_FASTDIST, out);
  }
  if (!gap_filters && n > 0) return set_error(RNJ_ERR_INVALID, "DNA needs gap filters");
  if ((size_t)bs_words * 16 < (size_t)L) return set_error(RNJ_ERR_INVALID, "bit strings shorter than L");
  const size_t words = (size_t)n * bs_words;
  int rc = ensure_stage(ctx, std::max<size_t>(words * 4, 1));
  if (rc != RNJ_OK) return rc;
  RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "staging reuse");
  uint32_t *sb = (uint32_t *)ctx->h_stage[0];
  uint32_t *sg = (uint32_t *)ctx->h_stage[1];
  for (int i = 0; i < n; ++i) {
    memcpy(sb + (size_t)i * bs_words, bit_strings[i], (size_t)bs_words * 4);
    memcpy(sg + (size_t)i * bs_words, gap_filters[i], (size_t)bs_words * 4);
  }
  rnj_aln *a = new rnj_aln();
  a->ctx = ctx;
  Packed &p = a->p;
  p.n = n;
  p.L = L;
  p.type = RNJ_DNA;
  p.flags = flags | RNJ_FASTDIST;
  p.kind = KIND_DNA;
  p.W = (L + 31) / 32;
  p.Wp = std::max(kKW, (p.W + kKW - 1) / kKW * kKW);
  p.Np = std::max(kTile, (n + kTile - 1) / kTile * kTile);
  p.NP = 3;
  const bool tc = !(flags & RNJ_POPCOUNT) && L <= kMaxTcColumns;
  uint32_t *db = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&db, std::max<size_t>(words * 8, 8), ctx->stream);
  if (tc) {
    p.kind = KIND_DNA_TC;
    p.NP = 0;
    p.Lk = std::max(256, (L + 255) / 256 * 256);
    if (e == cudaSuccess)
      e = cudaMallocAsync((void **)&p.feat, (size_t)p.Np * 4 * p.Lk / 2, ctx->stream);
  } else if (e == cudaSuccess) {
    e = cudaMallocAsync((void **)&p.planes, (size_t)p.NP * p.Wp * p.Np * 4, ctx->stream);
  }
  if (e == cudaSuccess && words)
    e = cudaMemcpyAsync(db, sb, words * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && words)
    e = cudaMemcpyAsync(db + words, sg, words * 4, cudaMemcpyHostToDevice, ctx->stream);
  mark(ctx, 0, 0);
  if (e == cudaSuccess)
    e = tc ? launch_pack_features_bits(db, db + words, bs_words, n, L, p.Np, p.Lk, p.feat,
                                       ctx->stream)
           : launch_pack_bitstrings_dna(db, db + words, bs_words, p, ctx->stream);
  mark(ctx, 0, 1);
  if (db) cudaFreeAsync(db, ctx->stream);
  if (e != cudaSuccess) {
    if (p.planes) cudaFreeAsync(p.planes, ctx->stream);
    if (p.feat) cudaFreeAsync(p.feat, ctx->stream);
    delete a;
    return cuda_error(e, "bit-string upload");
  }
  rc = tc ? encode_features_map(p) : encode_planes_map(p);
  if (rc != RNJ_OK) {
    if (p.planes) cudaFreeAsync(p.planes, ctx->stream);
    if (p.feat) cudaFreeAsync(p.feat, ctx->stream);
    delete a;
    return rc;
  }
  *out = a;
  return RNJ_OK;
}

int rnj_aln_info(const rnj_aln *aln, int *n, int *L, int *type) {
  if (!aln) return set_error(RNJ_ERR_INVALID, "null alignment");
  if (n) *n = aln->p.n;
  if (L) *L = aln->p.L;
  if (type) *type = aln->p.type;
  return RNJ_OK;
}

int rnj_aln_destroy(rnj_aln *aln) {
  if (!aln) return RNJ_OK;
  DeviceGuard g(aln->ctx->device);
  if (aln->owns_mem && aln->p.planes) cudaFreeAsync(aln->p.planes, aln->ctx->stream);
  if (aln->owns_mem && aln->p.feat) cudaFreeAsync(aln->p.feat, aln->ctx->stream);
  delete aln;
  return RNJ_OK;
}

int rnj_distance_into(rnj_ctx *ctx, rnj_aln *aln, int model, float *d_out, size_t ld,
                      float *max_out) {
  if (!ctx || !aln || (!d_out && aln->p.n > 0)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (ld < (size_t)aln->p.n) return set_error(RNJ_ERR_INVALID, "ld < n");
  DeviceGuard g(ctx->device);
  if (aln->p.n == 0) {
    if (max_out) *max_out = 0.0f;
    return RNJ_OK;
  }
  int rc = run_distance(ctx, aln->p, model, d_out, ld, nullptr);
  if (rc != RNJ_OK) return rc;
  if (max_out) {
    RNJ_CUDA(cudaMemcpyAsync(ctx->h_max, ctx->scratch.words, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream),
             "max copy");
    rc = check_device_error(ctx);
    if (rc != RNJ_OK) return rc;
    float m;
    memcpy(&m, ctx->h_max, sizeof(float));
    *max_out = m;
  }
  return RNJ_OK;
}

int rnj_distance(rnj_ctx *ctx, rnj_aln *aln, int model, rnj_mat **out) {
  if (!ctx || !aln || !out) return set_error(RNJ_ERR_INVALID, "null argument");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  DeviceGuard g(ctx->device);
  rnj_mat *m = new rnj_mat();
  m->ctx = ctx;
  m->n = aln->p.n;
  m->ld = (size_t)std::max(4, (aln->p.n + 3) / 4 * 4);
  cudaError_t e = cudaMallocAsync((void **)&m->d, std::max<size_t>(m->ld * m->n * 4, 4), ctx->stream);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&m->d_max, sizeof(int), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->d_max, 0, sizeof(int), ctx->stream);
  if (e != cudaSuccess) {
    rnj_mat_destroy(m);
    return cuda_error(e, "matrix allocation");
  }
  if (m->n > 0) {
    int rc = run_distance(ctx, aln->p, model, m->d, m->ld, m->d_max);
    if (rc != RNJ_OK) {
      rnj_mat_destroy(m);
      return rc;
    }
  }
  *out = m;
  return RNJ_OK;
}

int rnj_counts_into(rnj_ctx *ctx, rnj_aln *aln, unsigned int *d_counts) {
  if (!ctx || !aln || (!d_counts && aln->p.n > 0)) return set_error(RNJ_ERR_INVALID, "null argument");
  DeviceGuard g(ctx->device);
  const Packed &p = aln->p;
  if (p.n == 0) return RNJ_OK;
  const int nt = tiles_of(p.n);
  const long long ntiles = (p.flags & RNJ_FULL_ROWS) ? (long long)nt * nt : tri_tiles(nt);
  int rc = ensure_scratch_words(ctx, (size_t)ntiles + 2);
  if (rc != RNJ_OK) return rc;
  RNJ_CUDA(cudaMemsetAsync(ctx->scratch.words, 0, ((size_t)ntiles + 2) * sizeof(int), ctx->stream),
           "scratch clear");
  RNJ_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)p.n * p.n * 3 * sizeof(uint32_t), ctx->stream),
           "count clear");
  EpiParams ep = epi_for(ctx, p, RNJ_KIMURA);
  ep.full = (p.flags & RNJ_FULL_ROWS) ? 1 : 0;
  ep.counts = d_counts;
  if (is_tc_kind(p.kind)) {
    rc = run_tc_single(ctx, p, ep, EPI_COUNTS);
    if (rc != RNJ_OK) return rc;
    return check_device_error(ctx);
  }
  const int nk = p.Wp / kKW;
  const int mode = (nk <= kMaxFusedWords / kKW) ? EPI_COUNTS : EPI_ATOMIC;
  RNJ_CUDA(launch_count_tiles(p, p.kind, mode, ep, ctx->stream), "count kernel");
  return check_device_error(ctx);
}

int rnj_mat_info(rnj_mat *mat, int *n, float *max_distance) {
  if (!mat) return set_error(RNJ_ERR_INVALID, "null matrix");
  if (n) *n = mat->n;
  if (max_distance && mat->has_host_max) {
    *max_distance = mat->host_max;
  } else if (max_distance) {
    DeviceGuard g(mat->ctx->device);
    rnj_ctx *ctx = mat->ctx;
    if (!mat->d_max) return set_error(RNJ_ERR_INVALID, "matrix carries no maximum");
    RNJ_CUDA(cudaMemcpyAsync(ctx->h_max, mat->d_max, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream),
             "max copy");
    int rc = check_device_error(ctx);
    if (rc != RNJ_OK) return rc;
    memcpy(max_distance, ctx->h_max, sizeof(float));
  }
  return RNJ_OK;
}

int rnj_mat_device_ptr(rnj_mat *mat, float **d_ptr, size_t *ld) {
  if (!mat) return set_error(RNJ_ERR_INVALID, "null matrix");
  if (d_ptr) *d_ptr = mat->d;
  if (ld) *ld = mat->ld;
  return RNJ_OK;
}

int rnj_mat_copy_rows(rnj_ctx *ctx, rnj_mat *mat, int row0, int nrows, float **rows, int threads) {
  if (!ctx || !mat || (nrows > 0 && !rows)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (row0 < 0 || nrows < 0 || row0 + nrows > mat->n)
    return set_error(RNJ_ERR_INVALID, "row range outside the matrix");
  if (nrows == 0) return RNJ_OK;
  DeviceGuard g(ctx->device);
  const int n = mat->n;
  const size_t row_bytes = (size_t)n * sizeof(float);
  if (rows_pinned_block(rows, nrows, n)) {
    // One 2-D DMA straight into the caller's page-locked rows.
    RNJ_CUDA(cudaMemcpy2DAsync(rows[0], row_bytes, mat->d + (size_t)row0 * mat->ld,
                               mat->ld * sizeof(float), row_bytes, (size_t)nrows,
                               cudaMemcpyDeviceToHost, ctx->stream),
             "row copy");
    RNJ_CUDA(cudaStreamSynchronize(ctx->stream), "row copy sync");
    return RNJ_OK;
  }
  const size_t chunk_target = 32u << 20;  // 32 MB per staging buffer
  int rows_per_chunk = (int)std::max<size_t>(1, chunk_target / row_bytes);
  rows_per_chunk = std::min(rows_per_chunk, nrows);
  int rc = ensure_stage(ctx, (size_t)rows_per_chunk * row_bytes);
  if (rc != RNJ_OK) return rc;
  const int T = host_threads(threads);
  cudaEvent_t ev[2];
  RNJ_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "event");
  RNJ_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "event");
  const int nchunks = (nrows + rows_per_chunk - 1) / rows_per_chunk;
  cudaError_t e = cudaSuccess;
  auto enqueue = [&](int c) {
    const int r0 = row0 + c * rows_per_chunk;
    const int rn = std::min(rows_per_chunk, row0 + nrows - r0);
    const int b = c & 1;
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(ctx->h_stage[b], row_bytes, mat->d + (size_t)r0 * mat->ld,
                            mat->ld * sizeof(float), row_bytes, (size_t)rn,
                            cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], ctx->stream);
  };
  enqueue(0);
  for (int c = 0; c < nchunks && e == cudaSuccess; ++c) {
    if (c + 1 < nchunks) enqueue(c + 1);  // DMA of the next chunk overlaps this scatter
    const int b = c & 1;
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[b]);
    if (e != cudaSuccess) break;
    const int r0 = c * rows_per_chunk;
    const int rn = std::min(rows_per_chunk, nrows - r0);
    scatter_rows((const float *)ctx->h_stage[b], rows + r0, rn, n, T);
    // Buffer b is refilled by chunk c + 2, enqueued on the next iteration only
    // after this scatter has finished.
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (e != cudaSuccess) return cuda_error(e, "row copy");
  return RNJ_OK;
}

int rnj_mat_destroy(rnj_mat *mat) {
  if (!mat) return RNJ_OK;
  DeviceGuard g(mat->ctx->device);
  if (mat->owns && mat->d) cudaFreeAsync(mat->d, mat->ctx->stream);
  if (mat->d_max) cudaFreeAsync(mat->d_max, mat->ctx->stream);
  delete mat;
  return RNJ_OK;
}

int rnj_distance_matrix_host(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld, int type,
                             int model, int flags, float *out, float *max_out) {
  return rnj_distance_matrix_host_ex(ctx, chars, n, L, ld, type, model, flags, 0, out, max_out);
}

int rnj_distance_matrix_host_ex(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld,
                                int type, int model, int flags, int band_tiles, float *out,
                                float *max_out) {
  if (!ctx || (n > 0 && !out)) return set_error(RNJ_ERR_INVALID, "null argument");
  if (n > 0 && L > 0 && !chars) return set_error(RNJ_ERR_INVALID, "null argument");
  if (n < 0 || L < 0 || (n > 0 && ld < (size_t)L))
    return set_error(RNJ_ERR_INVALID, "invalid alignment shape");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (type == RNJ_UNKNOWN && n > 0) type = rnj_detect_type(chars, L);
  if ((type == RNJ_DNA || type == RNJ_PROTEIN) && band_tiles >= 0) {
    const int rc = distance_host_streamed(ctx, chars, n, L, ld, type, model, flags, band_tiles, out,
                                          max_out);
    if (rc != RNJ_ERR_UNSUPPORTED) return rc;
  }
  rnj_aln *a = nullptr;
  int rc = rnj_aln_from_host_buffer(ctx, chars, n, L, ld, type, flags, &a);
  if (rc != RNJ_OK) return rc;
  rnj_mat *m = nullptr;
  rc = rnj_distance(ctx, a, model, &m);
  rnj_aln_destroy(a);
  if (rc != RNJ_OK) return rc;
  if (n > 0 && ctx_block_pinned(out, (size_t)n * n * sizeof(float))) {
    // A page-locked output: the matrix as one 2-D download, the maximum and the
    // error word behind it, and one synchronisation for all three.
    cudaError_t e = cudaMemcpy2DAsync(out, (size_t)n * sizeof(float), m->d, m->ld * sizeof(float),
                                      (size_t)n * sizeof(float), (size_t)n,
                                      cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ctx->h_max, m->d_max, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ctx->h_max + 1, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    rc = e == cudaSuccess ? take_device_error(ctx) : cuda_error(e, "matrix download");
    if (rc == RNJ_OK && max_out) memcpy(max_out, ctx->h_max, sizeof(float));
    rnj_mat_destroy(m);
    return rc;
  }
  std::vector<float *> rows((size_t)n);
  for (int i = 0; i < n; ++i) rows[i] = out + (size_t)i * n;
  rc = rnj_mat_copy_rows(ctx, m, 0, n, rows.data(), 0);
  if (rc == RNJ_OK) rc = check_device_error(ctx);
  if (rc == RNJ_OK && max_out) rc = rnj_mat_info(m, nullptr, max_out);
  rnj_mat_destroy(m);
  return rc;
}

}  // extern "C"
