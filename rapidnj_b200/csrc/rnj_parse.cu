// rnj_parse.cu -- FASTA parsing on the device (rnj_msa_read_device).
//
// The reference reads its input with a character loop (dataloaderFasta::
// parseData, dataloaderFasta.hpp:78-133): at the start of every unit a ';'
// begins a comment (to the newline), a '>' ends the sequence being read and
// begins a name (bytes > 31, parseSequenceName :209-216), anything else begins a
// sequence line whose bytes > 32 are appended (parseSequenceLine :200-207); a
// sequence is stored when the next name or the end of the file comes, and must
// have the first one's length (storeSequence :252-276).  A unit begins at every
// line start, and also right after a name that ended on a control byte before
// its newline.
//
// Here the file's bytes are read by several host threads into page-locked
// memory, each 4 MB chunk copied to the device as soon as it is read, and:
//   1. the newlines are found by a two-pass compaction over 64 KB chunks (count
//      per chunk, scan on the host, positions in order);
//   2. a warp per line reads its first byte: names, comments and sequence lines;
//      a sequence line's bytes > 32 are counted; a name line is checked to hold
//      no control byte but a final '\r' (else the line's rest would be a unit of
//      its own);
//   3. a scan over the lines (names count up, kept bytes sum up per sequence;
//      block totals, their scan on the host, then each block from its prefix)
//      gives each line's sequence and offset, each sequence's length and name
//      line;
//   4. after the host has checked the lengths, a warp per sequence line
//      compacts its kept bytes (ballot + prefix count) into the n x L array.
// Names are cut from the host copy of the name lines.  Inputs the kernels leave
// to the host rules (names ended by a control byte, data before the first
// name, names without data, no name at all, Stockholm, files of 4 GB or more)
// are parsed by rnj_io.cpp's reader from the same bytes and copied to the
// device, so that every input gives the host reader's result.
#include <cuda_runtime.h>
#include <errno.h>
#include <fcntl.h>
#include <stdint.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

constexpr int kChunkThreads = 256;
constexpr int kSegBytes = 256;                        // per thread of the newline passes
constexpr size_t kChunk = (size_t)kChunkThreads * kSegBytes;  // 64 KB per CTA

enum : uint8_t { kLineSeq = 0, kLineName = 1, kLineComment = 2 };
enum : uint32_t { kFlagComplexName = 1u, kFlagLeadingData = 2u };

// Newline bytes ('\n') of a 32-bit word, as a mask of their bit positions /8.
__device__ __forceinline__ uint32_t newline_bytes(uint32_t w) { return __vcmpeq4(w, 0x0A0A0A0Au); }

// Thread t of chunk c owns bytes [c kChunk + t kSegBytes, +kSegBytes) clipped to S.
__device__ __forceinline__ void segment(size_t S, size_t &a, size_t &b) {
  a = min(S, (size_t)blockIdx.x * kChunk + (size_t)threadIdx.x * kSegBytes);
  b = min(S, a + (size_t)kSegBytes);
}

__device__ __forceinline__ uint32_t count_newlines(const uint8_t *B, size_t a, size_t b) {
  uint32_t c = 0;
  if (b - a == (size_t)kSegBytes) {  // a is a multiple of 256: 16-byte loads
    const uint4 *v = reinterpret_cast<const uint4 *>(B + a);
#pragma unroll 4
    for (int k = 0; k < kSegBytes / 16; ++k) {
      const uint4 q = v[k];
      c += (__popc(newline_bytes(q.x)) + __popc(newline_bytes(q.y)) + __popc(newline_bytes(q.z)) +
            __popc(newline_bytes(q.w))) >> 3;
    }
  } else {
    for (size_t i = a; i < b; ++i) c += B[i] == '\n';
  }
  return c;
}

// Exclusive sum over the CTA (blockDim.x = kChunkThreads); *total the sum.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sum[kChunkThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int w = 0; w < kChunkThreads / 32; ++w) {
    if (w < warp) before += warp_sum[w];
    all += warp_sum[w];
  }
  *total = all;
  return before + incl - v;
}

// Pass 1a: newlines per chunk.
__global__ void __launch_bounds__(kChunkThreads)
    nl_count_kernel(const uint8_t *__restrict__ B, size_t S, uint32_t *__restrict__ chunk_cnt) {
  size_t a, b;
  segment(S, a, b);
  const uint32_t c = a < b ? count_newlines(B, a, b) : 0u;
  uint32_t total;
  block_exclusive(c, &total);
  if (threadIdx.x == 0) chunk_cnt[blockIdx.x] = total;
}

// Pass 1b: the newline positions in file order (chunk_off: newlines before
// each chunk).
__global__ void __launch_bounds__(kChunkThreads)
    nl_positions_kernel(const uint8_t *__restrict__ B, size_t S,
                        const uint32_t *__restrict__ chunk_off, uint32_t *__restrict__ pos) {
  size_t a, b;
  segment(S, a, b);
  const uint32_t c = a < b ? count_newlines(B, a, b) : 0u;
  uint32_t total;
  uint32_t k = chunk_off[blockIdx.x] + block_exclusive(c, &total);
  if (c == 0) return;
  if (b - a == (size_t)kSegBytes) {
    const uint4 *v = reinterpret_cast<const uint4 *>(B + a);
    for (int q = 0; q < kSegBytes / 16; ++q) {
      const uint4 x = v[q];
      const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        uint32_t m = newline_bytes(w[j]) & 0x01010101u;  // one bit per newline byte
        while (m) {
          const int bit = __ffs(m) - 1;
          pos[k++] = (uint32_t)(a + 16 * q + 4 * j + (bit >> 3));
          m &= m - 1;
        }
      }
    }
  } else {
    for (size_t i = a; i < b; ++i)
      if (B[i] == '\n') pos[k++] = (uint32_t)i;
  }
}

// Line w spans [start, end): after the previous newline, up to its own (the
// last line ends at the end of the file, which reads as a newline).
__device__ __forceinline__ void line_span(const uint32_t *pos, uint32_t nnl, size_t S, uint32_t w,
                                          size_t &start, size_t &end) {
  start = w == 0 ? 0 : (size_t)pos[w - 1] + 1;
  end = w < nnl ? (size_t)pos[w] : S;
}

// Pass 2: a warp per line: its kind, its kept bytes, the name-line check.
__global__ void __launch_bounds__(256)
    line_classify_kernel(const uint8_t *__restrict__ B, size_t S, const uint32_t *__restrict__ pos,
                         uint32_t nnl, uint8_t *__restrict__ type, uint32_t *__restrict__ cnt,
                         uint32_t *__restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const uint64_t lines = (uint64_t)nnl + 1;
  const uint64_t stride = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < lines; w += stride) {
    size_t start, end;
    line_span(pos, nnl, S, (uint32_t)w, start, end);
    const int b0 = start < end ? B[start] : '\n';
    if (b0 == '>') {
      bool bad = false;
      for (size_t i = start + 1 + lane; i < end; i += 32) {
        const signed char ch = (signed char)B[i];
        if (ch <= 31 && !(ch == '\r' && i + 1 == end)) bad = true;
      }
      bad = __any_sync(0xffffffffu, bad);
      if (lane == 0) {
        type[w] = kLineName;
        cnt[w] = 0;
        atomicAdd(&flags[1], 1u);
        if (bad) atomicOr(&flags[0], kFlagComplexName);
      }
    } else if (b0 == ';') {
      if (lane == 0) {
        type[w] = kLineComment;
        cnt[w] = 0;
      }
    } else {
      uint32_t c = 0;
      for (size_t i = start + lane; i < end; i += 32) c += (signed char)B[i] > 32;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) {
        type[w] = kLineSeq;
        cnt[w] = c;
      }
    }
  }
}

// (names seen, kept bytes since the last name): the scan's element and operator.
struct Seg {
  uint32_t h, s;
};
__device__ __forceinline__ Seg seg_combine(Seg a, Seg b) {
  Seg r;
  r.h = a.h + b.h;
  r.s = b.h ? b.s : a.s + b.s;
  return r;
}
__device__ __forceinline__ Seg seg_shfl_up(Seg v, int o) {
  Seg r;
  r.h = __shfl_up_sync(0xffffffffu, v.h, o);
  r.s = __shfl_up_sync(0xffffffffu, v.s, o);
  return r;
}

// Pass 3, over blocks of kScanLines lines (a CTA each, kScanPer consecutive
// lines a thread): the scan of (names, kept bytes since the last name).  3a
// writes each block's total; the host scans the totals; 3b rescans a block from
// its prefix and walks its lines: line w's sequence rec[w] (-1 before the first
// name) and offset off[w], sequence r's length rec_len[r] and name line span
// rec_start[r] .. rec_end[r].
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr uint32_t kScanLines = kScanThreads * kScanPer;

__device__ __forceinline__ Seg line_seg(const uint8_t *type, const uint32_t *cnt, uint32_t i) {
  Seg e;
  const uint8_t t = type[i];
  e.h = t == kLineName ? 1u : 0u;
  e.s = t == kLineSeq ? cnt[i] : 0u;
  return e;
}

// The CTA's exclusive scan of v (identity (0, 0)); *total the CTA's sum.
__device__ __forceinline__ Seg block_seg_exclusive(Seg v, Seg *total) {
  __shared__ Seg wsum[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Seg incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const Seg y = seg_shfl_up(incl, o);
    if (lane >= o) incl = seg_combine(y, incl);
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  Seg before = {0u, 0u}, all = {0u, 0u};
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) before = seg_combine(before, wsum[w]);
    all = seg_combine(all, wsum[w]);
  }
  *total = all;
  Seg ex = seg_shfl_up(incl, 1);
  if (lane == 0) ex = Seg{0u, 0u};
  return seg_combine(before, ex);
}

__global__ void __launch_bounds__(kScanThreads)
    seq_scan_totals_kernel(const uint8_t *__restrict__ type, const uint32_t *__restrict__ cnt,
                           uint32_t lines, uint2 *__restrict__ block_total) {
  const uint32_t a = min(lines, blockIdx.x * kScanLines + threadIdx.x * kScanPer);
  const uint32_t b = min(lines, a + kScanPer);
  Seg mine = {0u, 0u};
  for (uint32_t i = a; i < b; ++i) mine = seg_combine(mine, line_seg(type, cnt, i));
  Seg total;
  block_seg_exclusive(mine, &total);
  if (threadIdx.x == 0) block_total[blockIdx.x] = make_uint2(total.h, total.s);
}

__global__ void __launch_bounds__(kScanThreads)
    seq_scan_walk_kernel(const uint8_t *__restrict__ type, const uint32_t *__restrict__ cnt,
                         const uint32_t *__restrict__ pos, uint32_t nnl, size_t S,
                         const uint2 *__restrict__ block_prefix, int *__restrict__ rec,
                         uint32_t *__restrict__ off, uint32_t *__restrict__ rec_len,
                         uint32_t *__restrict__ rec_start, uint32_t *__restrict__ rec_end,
                         uint32_t *__restrict__ flags) {
  const uint32_t lines = nnl + 1;
  const uint32_t a = min(lines, blockIdx.x * kScanLines + threadIdx.x * kScanPer);
  const uint32_t b = min(lines, a + kScanPer);
  Seg mine = {0u, 0u};
  for (uint32_t i = a; i < b; ++i) mine = seg_combine(mine, line_seg(type, cnt, i));
  Seg total;
  const Seg ex = block_seg_exclusive(mine, &total);
  Seg run = seg_combine(Seg{block_prefix[blockIdx.x].x, block_prefix[blockIdx.x].y}, ex);
  for (uint32_t i = a; i < b; ++i) {
    const uint8_t t = type[i];
    if (t == kLineName) {
      if (run.h >= 1) rec_len[run.h - 1] = run.s;
      else if (run.s > 0) atomicOr(&flags[0], kFlagLeadingData);
      size_t s0, e0;
      line_span(pos, nnl, S, i, s0, e0);
      rec_start[run.h] = (uint32_t)s0;
      rec_end[run.h] = (uint32_t)e0;
      run.h += 1;
      run.s = 0;
      rec[i] = (int)run.h - 1;
      off[i] = 0;
    } else {
      rec[i] = (int)run.h - 1;
      off[i] = run.s;
      if (t == kLineSeq) run.s += cnt[i];
    }
  }
  if (a < b && b == lines) {  // the last line's thread closes the last sequence
    if (run.h >= 1) rec_len[run.h - 1] = run.s;
    else if (run.s > 0) atomicOr(&flags[0], kFlagLeadingData);
  }
}

// Pass 4: a warp per sequence line: its bytes > 32, in order, to
// out[rec][off ..] (every sequence's length was checked to be L).
__global__ void __launch_bounds__(256)
    compact_kernel(const uint8_t *__restrict__ B, size_t S, const uint32_t *__restrict__ pos,
                   uint32_t nnl, const uint8_t *__restrict__ type, const uint32_t *__restrict__ cnt,
                   const int *__restrict__ rec, const uint32_t *__restrict__ off, int L,
                   uint8_t *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint64_t lines = (uint64_t)nnl + 1;
  const uint64_t stride = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < lines; w += stride) {
    if (type[w] != kLineSeq || cnt[w] == 0) continue;  // uniform per warp
    size_t start, end;
    line_span(pos, nnl, S, (uint32_t)w, start, end);
    uint8_t *dst = out + (size_t)rec[w] * L + off[w];
    uint32_t k = 0;
    for (size_t i0 = start; i0 < end; i0 += 32) {
      const size_t i = i0 + lane;
      const uint8_t ch = i < end ? B[i] : 0;
      const bool keep = (signed char)ch > 32;
      const uint32_t m = __ballot_sync(0xffffffffu, keep);
      if (keep) dst[k + __popc(m & lt)] = ch;
      k += __popc(m);
    }
  }
}

#define PARSE_CUDA(call, what)                           \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_error(e_, what);  \
  } while (0)

// Device buffers of one call, freed on every return path.
struct ParseBuffers {
  cudaStream_t s;
  std::vector<void *> ptrs;
  explicit ParseBuffers(cudaStream_t st) : s(st) {}
  template <class T>
  cudaError_t alloc(T **p, size_t bytes) {
    cudaError_t e = cudaMallocAsync((void **)p, std::max<size_t>(bytes, 16), s);
    if (e == cudaSuccess) ptrs.push_back((void *)*p);
    return e;
  }
  ~ParseBuffers() {
    for (void *p : ptrs) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  }
};

// The file into the context's page-locked buffer: up to eight threads read
// 4 MB chunks in turn and, when d_raw is given (room for the file's bytes on the
// context's device), each copies its chunk there as soon as it is read, so that
// the copies overlap the reading.  *size: the file's bytes.
constexpr size_t kReadChunk = (size_t)4 << 20;

int file_size(const char *path, size_t *size) {
  struct stat st;
  if (stat(path, &st) != 0 || !S_ISREG(st.st_mode))
    return set_error(RNJ_ERR_IO, std::string("ERROR: Could not read file: ") + path);
  *size = (size_t)st.st_size;
  return RNJ_OK;
}

int read_pinned(rnj_ctx *ctx, const char *path, size_t S, uint8_t *d_raw) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return set_error(RNJ_ERR_IO, std::string("ERROR: Could not read file: ") + path);
  if (S + 16 > ctx->h_file_cap) {
    if (ctx->h_file) cudaFreeHost(ctx->h_file);
    ctx->h_file = nullptr;
    ctx->h_file_cap = 0;
    const size_t cap = std::max<size_t>(S + 16, (size_t)1 << 20);
    const cudaError_t e = cudaMallocHost((void **)&ctx->h_file, cap);
    if (e != cudaSuccess) {
      close(fd);
      return cuda_error(e, "page-locked file buffer");
    }
    ctx->h_file_cap = cap;
  }
  const size_t chunks = (S + kReadChunk - 1) / kReadChunk;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int T = (int)std::max<size_t>(1, std::min<size_t>(std::min(8u, hw), chunks));
  std::atomic<size_t> next{0};
  std::vector<int> ok(T, 1);
  std::vector<cudaError_t> err(T, cudaSuccess);
  auto work = [&](int k) {
    if (d_raw && k > 0) cudaSetDevice(ctx->device);  // the current device is per thread
    for (;;) {
      const size_t c = next.fetch_add(1);
      if (c >= chunks) return;
      size_t a = c * kReadChunk;
      const size_t a0 = a, b = std::min(S, a + kReadChunk);
      while (a < b) {
        const ssize_t r = pread(fd, ctx->h_file + a, b - a, (off_t)a);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) {
          ok[k] = 0;
          return;
        }
        a += (size_t)r;
      }
      if (d_raw) {
        const cudaError_t e =
            cudaMemcpyAsync(d_raw + a0, ctx->h_file + a0, b - a0, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) {
          err[k] = e;
          return;
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int k = 1; k < T; ++k) th.emplace_back(work, k);
  work(0);
  for (auto &x : th) x.join();
  close(fd);
  for (int k = 0; k < T; ++k) {
    if (!ok[k]) return set_error(RNJ_ERR_IO, std::string("ERROR: Could not read file: ") + path);
    if (err[k] != cudaSuccess) return cuda_error(err[k], "file upload");
  }
  return RNJ_OK;
}

// The host rules on the bytes read, then the bytes to the device.
int host_parse_to_device(rnj_ctx *ctx, size_t S, bool fasta, rnj_msa **out) {
  rnj_msa *m = new rnj_msa();
  int rc = msa_parse_buffer(ctx->h_file, S, fasta, m);
  if (rc != RNJ_OK) {
    delete m;
    return rc;
  }
  m->device = ctx->device;
  const size_t bytes = (size_t)m->n * m->L;
  if (bytes > 0) {
    cudaError_t e = cudaMalloc((void **)&m->d_chars, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_chars, m->chars.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (m->d_chars) cudaFree(m->d_chars);
      delete m;
      return cuda_error(e, "alignment upload");
    }
  }
  *out = m;
  return RNJ_OK;
}

}  // namespace

extern "C" int rnj_msa_read_device(rnj_ctx *ctx, const char *path, const char *format,
                                   rnj_msa **out) {
  if (!ctx || !path || !out) return set_error(RNJ_ERR_INVALID, "null argument");
  bool fasta = true;
  int rc = msa_format(path, format, &fasta);
  if (rc != RNJ_OK) return rc;
  DeviceGuard guard(ctx->device);
  size_t S = 0;
  rc = file_size(path, &S);
  if (rc != RNJ_OK) return rc;
  if (!fasta || S == 0 || S >= ((size_t)1 << 32) - 1) {
    rc = read_pinned(ctx, path, S, nullptr);
    if (rc != RNJ_OK) return rc;
    return host_parse_to_device(ctx, S, fasta, out);
  }

  cudaStream_t st = ctx->stream;
  int fallback = 0;
  rnj_msa *m = nullptr;
  {
    ParseBuffers buf(st);
    uint8_t *d_raw = nullptr;
    PARSE_CUDA(buf.alloc(&d_raw, S + 16), "parse buffers");
    rc = read_pinned(ctx, path, S, d_raw);
    if (rc != RNJ_OK) return rc;
    const unsigned nchunks = (unsigned)((S + kChunk - 1) / kChunk);
    uint32_t *d_chunk = nullptr;
    PARSE_CUDA(buf.alloc(&d_chunk, (size_t)nchunks * sizeof(uint32_t)), "parse buffers");
    nl_count_kernel<<<nchunks, kChunkThreads, 0, st>>>(d_raw, S, d_chunk);
    PARSE_CUDA(cudaGetLastError(), "newline count");
    std::vector<uint32_t> chunk(nchunks);
    PARSE_CUDA(cudaMemcpyAsync(chunk.data(), d_chunk, (size_t)nchunks * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, st),
               "parse copy");
    PARSE_CUDA(cudaStreamSynchronize(st), "newline count sync");
    uint32_t nnl = 0;
    for (unsigned c = 0; c < nchunks; ++c) {
      const uint32_t v = chunk[c];
      chunk[c] = nnl;
      nnl += v;
    }
    const uint32_t lines = nnl + 1;
    uint32_t *d_pos = nullptr, *d_cnt = nullptr, *d_off = nullptr, *d_flags = nullptr;
    uint8_t *d_type = nullptr;
    int *d_rec = nullptr;
    PARSE_CUDA(buf.alloc(&d_pos, (size_t)std::max<uint32_t>(nnl, 1) * sizeof(uint32_t)), "parse buffers");
    PARSE_CUDA(buf.alloc(&d_type, (size_t)lines), "parse buffers");
    PARSE_CUDA(buf.alloc(&d_cnt, (size_t)lines * sizeof(uint32_t)), "parse buffers");
    PARSE_CUDA(buf.alloc(&d_rec, (size_t)lines * sizeof(int)), "parse buffers");
    PARSE_CUDA(buf.alloc(&d_off, (size_t)lines * sizeof(uint32_t)), "parse buffers");
    PARSE_CUDA(buf.alloc(&d_flags, 2 * sizeof(uint32_t)), "parse buffers");
    PARSE_CUDA(cudaMemsetAsync(d_flags, 0, 2 * sizeof(uint32_t), st), "parse flags");
    // d_chunk now holds the newlines before each chunk
    PARSE_CUDA(cudaMemcpyAsync(d_chunk, chunk.data(), (size_t)nchunks * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, st),
               "parse copy");
    nl_positions_kernel<<<nchunks, kChunkThreads, 0, st>>>(d_raw, S, d_chunk, d_pos);
    PARSE_CUDA(cudaGetLastError(), "newline positions");
    const unsigned grid_lines =
        (unsigned)std::min<uint64_t>(((uint64_t)lines * 32 + 255) / 256, (uint64_t)ctx->num_sms * 16);
    line_classify_kernel<<<grid_lines, 256, 0, st>>>(d_raw, S, d_pos, nnl, d_type, d_cnt, d_flags);
    PARSE_CUDA(cudaGetLastError(), "line classify");
    uint32_t flags[2] = {0u, 0u};
    PARSE_CUDA(cudaMemcpyAsync(flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, st), "parse copy");
    PARSE_CUDA(cudaStreamSynchronize(st), "line classify sync");
    const uint32_t H = flags[1];
    if ((flags[0] & kFlagComplexName) || H == 0) {
      fallback = 1;
    } else {
      uint32_t *d_len = nullptr, *d_rs = nullptr, *d_re = nullptr;
      PARSE_CUDA(buf.alloc(&d_len, (size_t)H * sizeof(uint32_t)), "parse buffers");
      PARSE_CUDA(buf.alloc(&d_rs, (size_t)H * sizeof(uint32_t)), "parse buffers");
      PARSE_CUDA(buf.alloc(&d_re, (size_t)H * sizeof(uint32_t)), "parse buffers");
      const unsigned nblk = (unsigned)((lines + kScanLines - 1) / kScanLines);
      uint2 *d_blk = nullptr;
      PARSE_CUDA(buf.alloc(&d_blk, (size_t)nblk * sizeof(uint2)), "parse buffers");
      seq_scan_totals_kernel<<<nblk, kScanThreads, 0, st>>>(d_type, d_cnt, lines, d_blk);
      PARSE_CUDA(cudaGetLastError(), "sequence scan");
      std::vector<uint2> blk(nblk);
      PARSE_CUDA(cudaMemcpyAsync(blk.data(), d_blk, (size_t)nblk * sizeof(uint2),
                                 cudaMemcpyDeviceToHost, st),
                 "parse copy");
      PARSE_CUDA(cudaStreamSynchronize(st), "sequence scan sync");
      uint2 run = make_uint2(0u, 0u);  // exclusive scan of the block totals
      for (unsigned k = 0; k < nblk; ++k) {
        const uint2 v = blk[k];
        blk[k] = run;
        run.y = v.x ? v.y : run.y + v.y;
        run.x += v.x;
      }
      PARSE_CUDA(cudaMemcpyAsync(d_blk, blk.data(), (size_t)nblk * sizeof(uint2),
                                 cudaMemcpyHostToDevice, st),
                 "parse copy");
      seq_scan_walk_kernel<<<nblk, kScanThreads, 0, st>>>(d_type, d_cnt, d_pos, nnl, S, d_blk, d_rec,
                                                          d_off, d_len, d_rs, d_re, d_flags);
      PARSE_CUDA(cudaGetLastError(), "sequence scan");
      std::vector<uint32_t> len(H), rs(H), re(H);
      PARSE_CUDA(cudaMemcpyAsync(len.data(), d_len, (size_t)H * 4, cudaMemcpyDeviceToHost, st), "parse copy");
      PARSE_CUDA(cudaMemcpyAsync(rs.data(), d_rs, (size_t)H * 4, cudaMemcpyDeviceToHost, st), "parse copy");
      PARSE_CUDA(cudaMemcpyAsync(re.data(), d_re, (size_t)H * 4, cudaMemcpyDeviceToHost, st), "parse copy");
      PARSE_CUDA(cudaMemcpyAsync(flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, st), "parse copy");
      PARSE_CUDA(cudaStreamSynchronize(st), "sequence scan sync");
      for (uint32_t r = 0; r < H && !fallback; ++r)
        if (len[r] == 0) fallback = 1;  // a name without data: the host rules
      if (flags[0] & kFlagLeadingData) fallback = 1;
      if (!fallback) {
        const uint32_t L = len[0];
        for (uint32_t r = 1; r < H; ++r)
          if (len[r] != L)
            return set_error(RNJ_ERR_FORMAT,
                             "ERROR: Sequence " + std::to_string(r) + " has length " +
                                 std::to_string(len[r]) +
                                 " while the preceding sequences in the alignment which have "
                                 "length " + std::to_string(L) + ".");
        if ((uint64_t)L > (uint64_t)INT32_MAX || (uint64_t)H > (uint64_t)INT32_MAX)
          return set_error(RNJ_ERR_UNSUPPORTED, "alignment too large");
        m = new rnj_msa();
        m->n = (int)H;
        m->L = (int)L;
        m->device = ctx->device;
        cudaError_t e = cudaMalloc((void **)&m->d_chars, (size_t)H * L);
        if (e != cudaSuccess) {
          delete m;
          return cuda_error(e, "alignment allocation");
        }
        compact_kernel<<<grid_lines, 256, 0, st>>>(d_raw, S, d_pos, nnl, d_type, d_cnt, d_rec,
                                                    d_off, (int)L, m->d_chars);
        e = cudaGetLastError();
        std::vector<char> row0(L);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(row0.data(), m->d_chars, L, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
          rnj_msa_destroy(m);
          return cuda_error(e, "sequence compaction");
        }
        m->type = rnj_detect_type(row0.data(), (int)L);
        m->names.reserve(H);
        for (uint32_t r = 0; r < H; ++r) {
          const char *a = ctx->h_file + rs[r] + 1, *z = ctx->h_file + re[r], *c = a;
          while (c < z && (signed char)*c > 31) ++c;
          m->names.emplace_back(a, c);
        }
      }
    }
  }
  if (fallback) return host_parse_to_device(ctx, S, fasta, out);
  *out = m;
  return RNJ_OK;
}
