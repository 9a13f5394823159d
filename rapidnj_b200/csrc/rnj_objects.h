// rnj_objects.h -- the opaque C-ABI objects (context, packed alignment, device
// matrix), shared by the translation units that implement the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"

// A parsed alignment: names and n * L bytes (row-major), on the host, or on the
// device when read by rnj_msa_read_device (its host bytes are then copied on
// the first rnj_msa_chars).
struct rnj_msa {
  std::vector<std::string> names;
  mutable std::vector<char> chars;  // n * L (host)
  int n = 0;
  int L = 0;
  int type = RNJ_DNA;
  uint8_t *d_chars = nullptr;  // n * L on device `device` (owned), or null
  int device = -1;
};

// Parses a FASTA (fasta) or Stockholm file's bytes already in memory with the
// host rules (rnj_io.cpp); the format of a path as rnj_msa_read picks it.
int msa_parse_buffer(const char *bytes, size_t size, bool fasta, rnj_msa *m);
int msa_format(const char *path, const char *format, bool *fasta);

struct rnj_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  rnj::Scratch scratch;
  uint32_t *d_mask = nullptr;             // presence mask (8 words)
  uint32_t *h_mask = nullptr;             // pinned
  int *h_max = nullptr;                   // pinned max bits / error word
  // Device error word of the single-alignment calls (bit 0: a bounded wait ran
  // out).  Sticky: a call that does not wait for the GPU leaves it set, and the
  // next call that does (rnj_ctx_synchronize, a max read) reports and clears it.
  int *d_err = nullptr;
  void *h_stage[2] = {nullptr, nullptr};  // pinned staging for copy-out / upload
  size_t stage_cap = 0;
  bool profiling = false;
  cudaEvent_t ev[6] = {};                 // pack, count, fix-up: begin/end pairs
  bool ev_used[3] = {false, false, false};
  cudaStream_t s_up = nullptr;            // host-to-host calls: uploads (created on first use)
  cudaStream_t s_down = nullptr;          // host-to-host calls: downloads
  int *h_words = nullptr;                 // pinned copy of the scratch words (flags, max, error)
  size_t h_words_cap = 0;
  rnj_batch *boot = nullptr;              // rnj_bootstrap's batch, kept for the next call
  int boot_aln = 0;                       // its capacity: alignments and tiles
  long long boot_tiles = 0;
  rnj::AlnDesc *d_desc = nullptr;         // one-alignment work list of the persistent kernel
  uint64_t *d_packed = nullptr;           // packed counts of the tensor-core path
  long long packed_tiles = 0;             // its capacity in tiles
  char *h_file = nullptr;                 // pinned file bytes of rnj_msa_read_device
  size_t h_file_cap = 0;
};

// Grows the context's packed-count buffer to `tiles` tiles (rnj_api.cu).
int ensure_packed(rnj_ctx *ctx, long long tiles);
// Counts + transform of work items [0, nitems) of the tensor-core path in
// passes of at most kTcChunkTiles tiles through `packed` (capacity
// min(nitems, kTcChunkTiles) tiles), on stream s.  Profiling marks: stage 1
// spans the counting kernels, stage 2 the transforms (rnj_api.cu).
// transform_ctas > 0: resident CTAs per SM of the transform grid (else 5);
// stages > 0: the counting kernel's ring depth (else its default).
int run_tc_chunks(rnj_ctx *ctx, const rnj::AlnDesc *d_desc, const rnj::WorkItem *d_items,
                  long long nitems, uint64_t *packed, cudaStream_t s, int transform_ctas = 0,
                  int stages = 0);
// Distances of work items [0, nitems) of one tensor-core alignment (descriptor
// d_desc on the device; d_items == nullptr: its banded triangle): the fused
// kernel (rnj_tcf.cu) when the alignment takes it (at most kMaxFusedColumns
// columns, and the tuned choice), else run_tc_chunks (rnj_api.cu).
int run_tc_distances(rnj_ctx *ctx, const rnj::Packed &p, const rnj::EpiParams &ep,
                     const rnj::AlnDesc *d_desc, const rnj::WorkItem *d_items, long long nitems,
                     cudaStream_t s, const rnj::TuneParams &tp);

struct rnj_aln {
  rnj_ctx *ctx = nullptr;
  rnj::Packed p;
  bool owns_mem = true;  // false: planes / features live in a batch's shared arena
};

struct rnj_mat {
  rnj_ctx *ctx = nullptr;  // stream the matrix is freed and read on
  float *d = nullptr;
  int n = 0;
  size_t ld = 0;
  int *d_max = nullptr;    // device copy of the max bits (single calls)
  bool has_host_max = false;  // batch and served results carry the max on the host
  float host_max = 0.0f;
  bool owns = true;
};

// Packing in two steps (rnj_api.cu): the LUT and plane layout of an alignment
// (protein needs its byte-presence mask), then allocation + pack kernel + map.
void lut_for(int type, int flags, const uint32_t *mask, uint8_t lut[256], int *kind);
int pack_prepared(rnj_ctx *ctx, const uint8_t *d_chars, int n, int L, size_t ld, int type,
                  int flags, int kind, const uint8_t lut[256], rnj_aln **out,
                  bool tuned_kernel = true);
// The packed layout of an alignment (kind: from lut_for; a tensor-core layout
// when DNA or protein takes one) without allocating; returns the bytes of its
// planes or features.
// lut (lut_for's table) decides the protein tensor-core layout (its ranks).
// tuned_kernel: follow the tuner's choice of counting kernel for the bucket
// (bit planes where they were faster for a single call); false for the work
// lists of batches and of the server, whose bit-plane kernel has no K split,
// so that every alignment the tensor cores can take goes to them.
size_t packed_layout(rnj::Packed &p, int n, int L, int type, int flags, int kind,
                     const uint8_t *lut, bool tuned_kernel = true);

// Helpers of rnj_api.cu shared with the streamed host-to-host path
// (rnj_stream.cu): grow the scratch words, transform parameters wired to the
// scratch, the error-word check (synchronises the context stream), and whether
// [p, p + bytes) is page-locked host memory.
int ctx_scratch(rnj_ctx *ctx, size_t words);
rnj::EpiParams ctx_epi(rnj_ctx *ctx, const rnj::Packed &p, int model);
int ctx_check_error(rnj_ctx *ctx);
// After the stream has finished with ctx->d_err copied into ctx->h_max[1]: the
// timeout status of that word (clearing it), else RNJ_OK (rnj_api.cu).
int take_device_error(rnj_ctx *ctx);
bool ctx_block_pinned(const void *p, size_t bytes);
// The context's upload and download streams, created on first use (rnj_stream.cu).
int ensure_side_streams(rnj_ctx *ctx);
// The streamed host-to-host distance call of the tensor-core path, DNA and
// protein (rnj_stream.cu).  Returns RNJ_ERR_UNSUPPORTED, having done nothing, when the
// input does not take that path.
int distance_host_streamed(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld, int type,
                           int model, int flags, int band_tiles, float *out, float *max_out);

// Profiling marks on the context stream (stage 0 pack, 1 count, 2 fix-up;
// end 0 = begin), read back by rnj_ctx_stage_times.
void ctx_mark(rnj_ctx *ctx, int stage, int end);

// A batch whose runs do not make the context stream wait (the server follows
// completion through the batch's event and keeps packing the next batch).
void batch_set_join(rnj_batch *b, bool join);

namespace rnj {
// Sets the calling thread's current device for a scope.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
}  // namespace rnj
