// rnj_internal.h -- host-side internals of librnjgpu.so shared by the C-ABI
// implementation and the kernel launchers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "rnj.h"

namespace rnj {

// Counting kernels, by bit-plane layout of the packed alignment.
//   KIND_DNA    planes {hi, lo, valid}         -> {ts, tv, valid}
//   KIND_NAIVE  planes {hi, lo, valid, upper}  -> {ts, tv, valid} (naive -f rules)
//   KIND_MISM2  planes {c0, c1, valid}         -> {mismatch, valid}
//   KIND_MISM5  planes {c0..c4, valid}         -> {mismatch, valid}
//   KIND_MISM7  planes {c0..c6, valid}         -> {mismatch, valid}
//   KIND_DNA_TC FP4 features {v | r | t | u}    -> {ts, tv, valid} on tensor cores
//   KIND_PROT_TC FP4 features {v | one-hot rank 0 | ... | rank R-1}
//                                              -> {mismatch, valid} on tensor cores
enum Kind {
  KIND_DNA = 0, KIND_NAIVE = 1, KIND_MISM2 = 2, KIND_MISM5 = 3, KIND_MISM7 = 4, KIND_DNA_TC = 5,
  KIND_PROT_TC = 6
};

__host__ __device__ inline bool is_tc_kind(int kind) {
  return kind == KIND_DNA_TC || kind == KIND_PROT_TC;
}
// Protein on the tensor cores: at most this many residue ranks (1 + ranks
// feature blocks); larger alphabets are counted on the bit planes.
constexpr int kMaxTcRanks = 31;

constexpr int kTile = 128;        // pairs per tile edge (rows and columns)
constexpr int kWordBits = 32;     // sites per plane word
constexpr int kKW = 8;            // words per pipeline stage
constexpr int kMaxFusedWords = 2047;  // 16-bit packed accumulators: L <= 65504 per pass
// The tensor-core sums reach 2L in magnitude and stay exact in f32 while below
// 2^24, and the packed counts hold 21 bits; longer DNA alignments are counted on
// the bit-plane kernels.
constexpr int kMaxTcColumns = (1 << 21) - 1;
// The fused tensor-core kernel keeps each pair's counts in 16 bits between the
// accumulators and the transform; longer alignments take the two-kernel form.
constexpr int kMaxFusedColumns = 65535;

__host__ __device__ inline int planes_of(int kind) {
  switch (kind) {
    case KIND_DNA: return 3;
    case KIND_NAIVE: return 4;
    case KIND_MISM2: return 3;
    case KIND_MISM5: return 6;
    default: return 8;
  }
}

// Packed alignment on the device.
struct Packed {
  int n = 0, L = 0;
  int type = RNJ_DNA;
  int flags = 0;
  int kind = KIND_DNA;   // plane layout (for DNA JC the DNA layout is counted as MISM2)
  int W = 0;             // words per sequence holding sites (ceil(L/32))
  int Wp = 0;            // padded to a multiple of kKW
  int Np = 0;            // sequences padded to a multiple of kTile
  int NP = 0;            // planes
  uint32_t *planes = nullptr;  // NP * Wp * Np words, word-major, sequence fastest
  CUtensorMap tmap;      // 3-D map over (Np, Wp, NP), box (kTile, kKW, NP)
  // Tensor-core layout (KIND_DNA_TC): the Np x (4 * Lk) FP4 feature matrix
  // [v | r | t | u], two columns per byte, cut into K blocks of 256 columns
  // (128 bytes), block-major: column k of row i in byte
  // ((k / 256) * Np + i) * 128 + (k % 256) / 2, so the 128-row slab of one K
  // block is a contiguous 16 KB run.
  uint8_t *feat = nullptr;
  int Lk = 0;            // L rounded up to 256
  int nfb = 4;           // feature blocks of Lk columns: 4 (DNA), 1 + ranks (protein)
  CUtensorMap fmap;      // 3-D map over (128, Np, nfb * Lk / 256), box (128, 128, 1), 128-byte swizzle
};

struct EpiParams {
  int n = 0;
  int L = 0;
  int model = RNJ_KIMURA;
  int type = RNJ_DNA;
  int compat_wrap = 0;
  int full = 0;
  double jc_b = 0.75;
  float *out = nullptr;
  size_t ld = 0;
  int *max_bits = nullptr;    // float bits, atomicMax target (init 0 = +0.0f)
  int *tile_flags = nullptr;  // per tile: 1 if it holds a saturated (-1) entry
  uint32_t *counts = nullptr; // n*n*3 counts (count-output and split modes)
  int *err = nullptr;         // device error word (bit 0: a bounded wait ran out)
  uint32_t wait_us = 0;       // bound of the pipeline waits in microseconds (0: 2 s)
  int stall = 0;              // test of the failure path: wait on a barrier nothing completes
  int row0 = 0;               // output row offset: row i is stored at out + (i - row0) * ld
  int tile0 = 0;              // bit-plane kernel: tile of block 0 (a band of full-square tiles)
  int stages = 0;             // bit-plane kernel: ring depth (0: its plane layout's deepest)
};

// One alignment of a work list, as the persistent kernels read it from device
// memory: its TMA map, output, scratch slots and transform parameters.
struct alignas(128) AlnDesc {
  CUtensorMap map;            // features (tensor-core kind) or planes (popcount kinds)
  float *out;                 // n rows of ld floats (distances), or null in count mode
  uint32_t *counts;           // n*n*3 counts (count mode), or null
  unsigned long long ld;
  int *max_bits;              // per-alignment max slot (float bits)
  int *tile_flags;            // per-alignment saturation flags, one per triangle tile
  int *err;                   // shared error word
  int n, L, nt, kdim;         // kdim: Lk columns (tensor-core) or Wp words (popcount)
  int model, type, compat, full;
  int kind, np, band, wait_us; // np: planes, or feature blocks (tensor-core kinds);
                               // band: tile-order band height (single alignment), 0 = 12;
                               // wait_us: bound of the pipeline waits (0: 2 s)
  int stall, row0;             // stall, row0: as EpiParams
  int stages, pad_;            // stages: the tensor-core ring depth of a work-list launch
                               // (read from the first descriptor; 0: the launch's own)
  double jc_b;
};
static_assert(sizeof(AlnDesc) % 128 == 0, "descriptors of a work list share no 128-byte line");

// A work item: alignment index and linear triangle-tile index within it.
struct WorkItem {
  int aln;
  int tile;
};

// Scratch of one distance call: the max slot, the error word and the per-tile
// saturation flags (device), plus the split-K count buffer for long alignments.
struct Scratch {
  int *words = nullptr;       // [0] max bits, [1] error, [2..] tile flags
  size_t words_cap = 0;
  uint32_t *counts = nullptr; // split-K counts
  size_t counts_cap = 0;
};

// Tuned launch parameters of one (alphabet, rules, n, L) bucket (rnj_tune.cu).
// Zero means the built-in default.
struct TuneParams {
  int dna_kernel = 0;      // DNA fast rules and protein: 0 tensor cores, 1 bit-plane popcount
  int ksplit = 1;          // bit-plane kernel: K (columns) split over this many CTAs per tile
  int tile_band = 0;       // tensor-core kernel: tile-order band height in tile rows (0 = 12)
  int transform_ctas = 0;  // tensor-core transform: resident CTAs per SM (0 = 5)
  int stream_band = 0;     // streamed host call: band height in tile rows (0 = automatic)
  int tc_epilogue = 0;     // tensor-core distances: 0 transform fused into the counting
                           // kernel, 1 packed counts + separate transform kernel
  int tc_stages = 0;       // tensor-core ring depth (0 = 6 fused, 7 two-kernel)
  int pop_stages = 0;      // bit-plane kernel ring depth (0 = its plane layout's deepest)
};
// The parameters of the bucket of (n, L, type, flags): the tuned entry if the
// table (filled by rnj_tune / rnj_tune_load / RNJ_TUNE_CACHE) holds one, else
// the defaults (*found, when given, says which).
TuneParams tune_lookup(int n, int L, int type, int flags, bool *found = nullptr);

// One alignment of a batched pack (rnj_batch_add_many): the multi-alignment
// pack kernels take an array of these and find the alignment of each work unit
// by its first unit (unit0, ascending).
struct alignas(16) PackJob {
  const uint8_t *chars;
  unsigned long long ld;
  void *dst;              // bit planes (uint32 words) or FP4 features (bytes)
  long long unit0;        // first work unit of this alignment
  int n, L, Np, W;        // W: Wp words (bit planes) or Lk columns (features)
  int kind, nfb, pad[2];  // nfb: feature blocks (tensor-core kinds)
  uint8_t lut[256];       // bit planes: the per-byte table of lut_for
};

// Launchers (rnj_kernels.cu).
cudaError_t launch_pack_chars(const uint8_t *d_chars, size_t ld, const Packed &p,
                              const uint8_t lut[256], cudaStream_t s);
cudaError_t launch_presence(const uint8_t *d_chars, size_t ld, int n, int L,
                            uint32_t *d_mask /*8 words*/, cudaStream_t s);
// Row segment of a presence-scan work unit (one warp), bytes.
constexpr int kPresenceSeg = 4096;
// Many alignments in one launch each.  Presence: units = sum of
// n * ceil(L / kPresenceSeg) (row segments), 8 mask words per job.  Planes:
// units = sum of (Np/32) * (Wp/8) pack tiles.  Features (rnj_tc.cu): units =
// sum of Np * Lk/32, each job's a multiple of 256 (a block's 256 units share a
// job).
cudaError_t launch_presence_multi(const PackJob *d_jobs, int njobs, long long units,
                                  uint32_t *d_masks, cudaStream_t s);
cudaError_t launch_pack_chars_multi(const PackJob *d_jobs, int njobs, long long units,
                                    cudaStream_t s);
cudaError_t launch_pack_features_multi(const PackJob *d_jobs, int njobs, long long units,
                                       cudaStream_t s);
cudaError_t launch_pack_bitstrings_dna(const uint32_t *d_bits, const uint32_t *d_gaps,
                                       int bs_words, const Packed &p, cudaStream_t s);
// kchunk > 0: words of K per CTA (EPI_ATOMIC splits K over grid.y).  ntiles > 0:
// only tiles [ep.tile0, ep.tile0 + ntiles) (EPI_DIST; a band of full-square tiles).
cudaError_t launch_count_tiles(const Packed &p, int count_kind, int epi_mode,
                               const EpiParams &ep, cudaStream_t s, int kchunk = 0,
                               long long ntiles = 0);
cudaError_t launch_fixup(const EpiParams &ep, int nt, cudaStream_t s);
// Loads every bit-plane kernel a fused distance call can launch (pack, presence
// scan, counts of each plane layout, fix-up).  Under CUDA's lazy module loading a
// kernel's code is loaded, into device memory, at its first launch or attribute
// query; the no-allocation entry point does this at its set-up instead.
cudaError_t preload_bitplane_kernels();
cudaError_t launch_transform_counts(const EpiParams &ep, int nt, cudaStream_t s);
// Tensor-core DNA path (rnj_tc.cu).
// Rows [row0, row0 + rows) of the feature matrix (rows < 0: through Np).
cudaError_t launch_pack_features(const uint8_t *d_chars, size_t ld, int n, int L, int Np, int Lk,
                                 uint8_t *F, cudaStream_t s, int row0 = 0, int rows = -1);
// Protein residues -> FP4 features [v | one-hot rank 0 .. nfb-2]: lut = the rank
// of each byte (0xFF: gap), rows [row0, row0 + rows).
cudaError_t launch_pack_features_prot(const uint8_t *d_chars, size_t ld, int n, int L, int Np,
                                      int Lk, int nfb, const uint8_t lut[256], uint8_t *F,
                                      cudaStream_t s, int row0 = 0, int rows = -1);
cudaError_t launch_pack_features_bits(const uint32_t *d_bits, const uint32_t *d_gaps, int bs_words,
                                      int n, int L, int Np, int Lk, uint8_t *F, cudaStream_t s);
int encode_features_map(Packed &p);
// Batched popcount path (rnj_kernels.cu): persistent, atomic item counter.
cudaError_t launch_count_batch(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                               int *d_counter, int grid, int epi_mode, cudaStream_t s);
cudaError_t launch_fixup_batch(const AlnDesc *d_descs, const WorkItem *items_a, const int *n_a,
                               const WorkItem *items_b, const int *n_b, int grid, cudaStream_t s);
// Host helpers shared by the single and batched paths (rnj_api.cu).
// The process-wide wait settings (rnj_set_wait_limit, rnj_test_wait_on_unset_flag)
// copied into a kernel's parameters.
void apply_wait_settings(EpiParams &ep);
EpiParams epi_params_for(const Packed &p, int model);
AlnDesc desc_for(const Packed &p, const EpiParams &ep);
// Persistent over work items [item0, min(n, item0 + count)); d_items == nullptr
// means the tiles of d_descs[0] in banded order; d_nitems == nullptr means
// nitems is n.  EPI_PACKED writes packed counts (kPackedTileWords per item) for
// launch_tc_transform; EPI_COUNTS writes each alignment's n x n x 3 counts.
// stages: the ring depth (0: the default, 7; the tuner's tc_stages).
cudaError_t launch_tc_batch(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                            int nitems, int item0, int count, uint64_t *packed, int grid,
                            int epi_mode, cudaStream_t s, int stages = 0);
// Tensor-pipe probe (rnj_probe_tc_peak): one CTA per SM, `iters` FP4 MMAs each.
cudaError_t launch_tc_peak_probe(int grid, int iters, int *err, cudaStream_t s);
cudaError_t launch_tc_transform(const AlnDesc *d_descs, const WorkItem *d_items,
                                const int *d_nitems, int nitems, int item0, int count,
                                const uint64_t *packed, int grid, cudaStream_t s);
// The fused form (rnj_tcf.cu): counts and the exact transform in one persistent
// launch over work items [item0, min(n, item0 + count)) (d_items == nullptr: the
// banded tiles of d_descs[0]; d_nitems == nullptr: n = nitems); distances
// straight into each alignment's output, with its max slot and saturation
// flags.  Every alignment has at most kMaxFusedColumns columns.
// variant: the transform of every item (fused_variant_for), or FUSED_ANY to
// choose per item from its descriptor.  stages: the ring depth (0: the
// default, 6; the tuner's tc_stages).
enum FusedVariant {
  FUSED_K2P = 0, FUSED_JC = 1, FUSED_PROTEIN = 2, FUSED_GENERIC = 3, FUSED_FULL = 4, FUSED_ANY = 5
};
int fused_variant_for(int model, int type, int compat, int full);
cudaError_t launch_tc_fused(const AlnDesc *d_descs, const WorkItem *d_items, const int *d_nitems,
                            int nitems, int item0, int count, int grid, int variant,
                            cudaStream_t s, int stages = 0);
// The ring depth launch_tc_fused runs with for a requested `stages`.
int fused_ring_depth(int stages);

// The live work list of the served form (rnj_server.cu): triangle tiles of
// tensor-core alignments appended while tc_live_kernel runs.  The publisher
// (launch_live_publish, on another stream) writes items [first, first + count)
// of alignment slot aln and then raises *tail with a release store; the live
// kernel's CTAs claim indices below *tail (compare-and-swap on *head) and,
// when there is none, poll *tail for idle_us before they exit.  tiles_done[a]
// counts the finished tiles of slot a and sat[a] says whether one held a
// saturated pair.  The CTA that finishes slot a's last tile appends a fix-up
// item per flagged tile to the second list (fix_items: reserved by
// atomicAdd on *fix_tail, written with a release store, claimed by any CTA
// before the main list's items); fix_pending[a] counts the fix-ups not yet
// done (plus one held by the appending CTA), and whoever brings it to zero --
// or the last tile's CTA when nothing saturated -- writes done[a] = {1, max
// bits} (mapped page-locked host memory).  err: the error word of the launch.
struct LiveList {
  WorkItem *items;
  unsigned int *head;
  unsigned int *tail;
  unsigned int *tiles_done;
  int *sat;
  unsigned long long *fix_items;  // (tile << 32) | (slot + 1); 0 = not yet written
  unsigned int *fix_head;
  unsigned int *fix_tail;
  unsigned int *fix_pending;
  // The exit vote: a CTA that has found nothing to claim for idle_us counts
  // itself in *idle_ctas; when every CTA of the launch is counted, *closing is
  // set and every CTA leaves at its next claim (items published after that go
  // to the next launch).  Both are cleared before each launch.
  unsigned int *idle_ctas;
  unsigned int *closing;
  int2 *done;
  int *err;
  int cap_items, cap_aln;
  unsigned int idle_us;
};
// grid CTAs of the live kernel (fewer than the SMs: the others pack arriving
// requests); stages: the ring depth (0: 6).
cudaError_t launch_tc_live(const AlnDesc *d_descs, const LiveList &live, int grid, int stages,
                           cudaStream_t s);
// Clears the scratch of slot aln (its max slot, tile flags and counters),
// appends its count triangle tiles (band order of height band) at items[first
// ..] and publishes them.
cudaError_t launch_live_publish(const LiveList &live, int aln, int nt, int band,
                                unsigned int first, unsigned int count, int *max_bits,
                                int *tile_flags, cudaStream_t s);

enum EpiMode { EPI_DIST = 0, EPI_COUNTS = 1, EPI_ATOMIC = 2, EPI_PACKED = 3 };

// Packed counts of one pair for the tensor-core path: ts, tv and valid in 21
// bits each (the tensor-core path takes L < 2^21).
__host__ __device__ inline uint64_t pack_counts(uint32_t ts, uint32_t tv, uint32_t valid) {
  return (uint64_t)ts | ((uint64_t)tv << 21) | ((uint64_t)valid << 42);
}
__host__ __device__ inline void unpack_counts(uint64_t x, uint32_t &ts, uint32_t &tv,
                                              uint32_t &valid) {
  ts = (uint32_t)(x & 0x1FFFFFu);
  tv = (uint32_t)((x >> 21) & 0x1FFFFFu);
  valid = (uint32_t)(x >> 42);
}
// Tiles per pass of the tensor-core path: the packed-count buffer holds this
// many 128 x 128 tiles (8 bytes per pair, 512 MiB).
constexpr int kTcChunkTiles = 4096;
// Resident CTAs per SM of the transform kernel (256 threads of at most 51
// registers, 34 KB of transpose buffers each): the persistent grid is exactly
// this many per SM, so the tiles spread evenly.
constexpr int kTransformCtasPerSm = 5;
constexpr size_t kPackedTileWords = (size_t)kTile * kTile;

inline int tiles_of(int n) { return (n + kTile - 1) / kTile; }
inline long long tri_tiles(int nt) { return (long long)nt * (nt + 1) / 2; }

// Error plumbing (rnj_api.cu).
int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);

// Packing helpers (rnj_api.cu).
char resolve_char(char c, int type);
void dna_lut(bool naive, uint8_t lut[256]);
int encode_planes_map(Packed &p);

}  // namespace rnj
