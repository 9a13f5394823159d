// rnj_noalloc.cu -- distances for callers that cannot allocate device memory.
//
// Some hosts of this library own every byte of device memory themselves: a
// process that runs under a fixed memory budget with its own pool (an inference
// or database server that reserves the GPU up front), or an embedding where
// cudaMalloc is forbidden because it synchronises the device.
// rnj_distance_noalloc serves them: it runs
// the same pack -> count -> fix-up kernels as rnj_distance_into, on the caller's
// stream, with every intermediate buffer (the packed bit planes, the running
// maximum, the error word and the per-tile saturation flags) placed in one
// fixed array compiled into the library.
//
// Properties a caller must know:
//   * The array holds kNoAllocScratchBytes (16 MiB) on every GPU that loads the
//     library, for the life of the process.
//   * It bounds the alignment: planes of n x L sites must fit (about 0.375 byte
//     per site for DNA on the fast path, 0.5 with -f, 1 byte for protein, with
//     n rounded up to 128 and L to 256); larger inputs are rejected with
//     RNJ_ERR_INVALID before anything runs.  L is also limited to 65280 columns
//     (one counting pass; longer alignments need the split count buffer of
//     rnj_distance_into).
//   * All calls share the array.  Two calls whose work overlaps on the GPU (on
//     different streams, or from different threads) race and corrupt each
//     other; calls issued one after another on one stream are safe.  The parts
//     that must start at zero are cleared at the start of each call.
//   * The first call on each device looks the array's device address up with
//     cudaGetSymbolAddress (host code cannot use the array's name as a device
//     address) and loads the kernels the entry point launches, so that no later
//     call takes device memory for kernel code.  Make that first call before any
//     stream capture begins.
//   * Every call waits for its work on the caller's stream to finish, then reads
//     the array's error word, so that a bounded device wait that ran out is
//     returned as RNJ_ERR_TIMEOUT whether or not the caller asked for the
//     maximum.  On a stream that is being captured the call returns
//     RNJ_ERR_UNSUPPORTED before it touches the stream.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "rnj.h"
#include "rnj_internal.h"

namespace rnj {
namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;
constexpr size_t kHeaderBytes = 256;  // [0] max bits, [1] error word, [2..9] presence mask
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once.
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_error(RNJ_ERR_UNSUPPORTED, "device index too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-allocation scratch)");
    // Load now every kernel a later call may launch: with lazy module loading
    // (CUDA's default) a kernel's first launch would take device memory for its
    // code in the middle of a call that promises to take none.
    e = preload_bitplane_kernels();
    if (e != cudaSuccess) return cuda_error(e, "kernel loading (no-allocation set-up)");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return RNJ_OK;
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace
}  // namespace rnj

using namespace rnj;

extern "C" int rnj_distance_noalloc(const void *d_chars, int n, int L, size_t ld, int type,
                                    int model, int flags, float *d_out, size_t ld_out,
                                    void *stream, float *max_out) {
  if (n < 0 || L < 0 || (n > 0 && (!d_chars || !d_out)))
    return set_error(RNJ_ERR_INVALID, "null argument or negative size");
  if (type != RNJ_DNA && type != RNJ_PROTEIN)
    return set_error(RNJ_ERR_INVALID, "type must be RNJ_DNA or RNJ_PROTEIN");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (n > 0 && (ld < (size_t)L || ld_out < (size_t)n))
    return set_error(RNJ_ERR_INVALID, "row stride smaller than the row");
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    if (max_out) *max_out = 0.0f;
    return RNJ_OK;
  }
  // The call ends by waiting for the stream; a stream being captured cannot be
  // waited for, and trying would invalidate the caller's capture.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t ce = cudaStreamIsCapturing(s, &cap);
  if (ce != cudaSuccess) return cuda_error(ce, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return set_error(RNJ_ERR_UNSUPPORTED,
                     "rnj_distance_noalloc waits for the GPU before it returns; it cannot be "
                     "called on a stream that is being captured");

  // Size check against the worst plane count of the type, before any work.
  const bool naive = (flags & RNJ_FASTDIST) == 0;
  const int worst_planes = (type == RNJ_DNA) ? (naive ? 4 : 3) : 8;
  Packed p;
  p.n = n;
  p.L = L;
  p.type = type;
  p.flags = flags;
  p.W = (L + 31) / 32;
  p.Wp = std::max(kKW, (p.W + kKW - 1) / kKW * kKW);
  p.Np = std::max(kTile, (n + kTile - 1) / kTile * kTile);
  if (p.Wp / kKW > kMaxFusedWords / kKW)
    return set_error(RNJ_ERR_INVALID, "the no-allocation entry point handles at most 65280 columns");
  const int nt = tiles_of(n);
  const bool full = type == RNJ_DNA && naive && (flags & RNJ_FULL_ROWS);
  const long long ntiles = full ? (long long)nt * nt : tri_tiles(nt);
  const size_t flags_off = kHeaderBytes;
  const size_t planes_off = round_up(flags_off + (size_t)ntiles * sizeof(int), 256);
  const size_t need = planes_off + (size_t)worst_planes * p.Wp * p.Np * sizeof(uint32_t);
  if (need > kNoAllocScratchBytes)
    return set_error(RNJ_ERR_INVALID,
                     "alignment of " + std::to_string(n) + " x " + std::to_string(L) + " needs " +
                         std::to_string(need) + " bytes of scratch; the no-allocation entry point "
                         "holds " + std::to_string(kNoAllocScratchBytes) + " (16 MiB)");

  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc != RNJ_OK) return rc;
  uint8_t *scratch = static_cast<uint8_t *>(base);
  int *words = reinterpret_cast<int *>(scratch);
  int *tile_flags = reinterpret_cast<int *>(scratch + flags_off);

  // Clear the header and the tile flags (the planes are fully rewritten by the pack).
  cudaError_t e = cudaMemsetAsync(scratch, 0, planes_off, s);
  if (e != cudaSuccess) return cuda_error(e, "scratch clear");

  uint8_t lut[256];
  if (type == RNJ_DNA) {
    p.kind = naive ? KIND_NAIVE : KIND_DNA;
    dna_lut(naive, lut);
  } else {
    uint32_t *d_mask = reinterpret_cast<uint32_t *>(words + 2);
    uint32_t mask[8];
    e = launch_presence((const uint8_t *)d_chars, ld, n, L, d_mask, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mask, d_mask, sizeof(mask), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "residue presence");
    int rank = 0;
    for (int c = 0; c < 256; ++c) {
      const bool present = (mask[c >> 5] >> (c & 31)) & 1u;
      if (resolve_char((char)c, RNJ_PROTEIN) == '-' || !present) lut[c] = 0xFF;
      else lut[c] = (uint8_t)(rank++);
    }
    p.kind = rank <= 4 ? KIND_MISM2 : (rank <= 32 ? KIND_MISM5 : KIND_MISM7);
  }
  p.NP = planes_of(p.kind);
  p.planes = reinterpret_cast<uint32_t *>(scratch + planes_off);
  e = launch_pack_chars((const uint8_t *)d_chars, ld, p, lut, s);
  if (e != cudaSuccess) return cuda_error(e, "pack kernel");
  rc = encode_planes_map(p);
  if (rc != RNJ_OK) return rc;

  EpiParams ep;
  ep.n = n;
  ep.L = L;
  ep.model = model;
  ep.type = type;
  ep.compat_wrap = (type == RNJ_PROTEIN && !naive && (flags & RNJ_COMPAT_PROTEIN_WRAP)) ? 1 : 0;
  ep.full = full ? 1 : 0;
  ep.jc_b = (type == RNJ_PROTEIN) ? (20.0 - 1) / 20.0 : (4.0 - 1) / 4.0;
  ep.out = d_out;
  ep.ld = ld_out;
  ep.max_bits = words;
  ep.err = words + 1;
  ep.tile_flags = tile_flags;
  apply_wait_settings(ep);
  if (n == 1) {
    e = cudaMemsetAsync(d_out, 0, sizeof(float), s);
    if (e != cudaSuccess) return cuda_error(e, "diagonal");
  }
  const int ckind = (p.kind == KIND_DNA && model == RNJ_JC) ? KIND_MISM2 : p.kind;
  e = launch_count_tiles(p, ckind, EPI_DIST, ep, s);
  if (e == cudaSuccess) e = launch_fixup(ep, nt, s);
  if (e != cudaSuccess) return cuda_error(e, "distance kernels");
  // The maximum and the error word, always: a timeout must not pass as success.
  int hw[2];
  e = cudaMemcpyAsync(hw, words, sizeof(hw), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_error(e, "max copy");
  if (hw[1] != 0) return set_error(RNJ_ERR_TIMEOUT, "a bounded device wait ran out");
  if (max_out) memcpy(max_out, &hw[0], sizeof(float));
  return RNJ_OK;
}
