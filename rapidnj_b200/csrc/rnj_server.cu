// rnj_server.cu -- served form: continuous batching of distance requests
// through a live work list.
//
// Clients submit alignments from any thread; a scheduler thread owns the GPU
// work:
//   * admission: a request is admitted when the device memory it needs (its
//     bytes, packed operands and output matrix) fits the server's budget;
//     otherwise it waits (first come, first served);
//   * a submitted alignment is copied into the server's page-locked staging
//     area (pageable memory when it is full), so that its upload is an
//     asynchronous DMA;
//   * an admitted request is uploaded and packed on the server's stream, its
//     descriptor is written, and a one-block publisher kernel appends its
//     triangle tiles to the live work list and raises the list's tail;
//   * one persistent kernel (tc_live_kernel, on its own stream, on all SMs but
//     a few that the packing kernels of arriving requests run on) claims tiles
//     from the list as they appear: a request that arrives while others run
//     is admitted into the running launch, and its tiles are computed as soon
//     as CTAs finish their current ones.  When every CTA has had nothing to
//     claim for a while (a grid-wide vote, so that the launch never thins out
//     to a few CTAs under a light load) the kernel exits; the scheduler
//     launches it again when work arrives;
//   * the CTA that finishes a request's last tile applies its saturation
//     fix-up and writes the request's maximum and a completion flag to
//     page-locked host memory, which the scheduler polls: each request
//     completes on its own, not with a batch;
//   * packed inputs are released at completion, the output matrix stays on the
//     device until the client takes it.
// Requests the tensor-core kernel cannot take (protein alphabets of more than
// 31 residues, the -f rules, RNJ_POPCOUNT, more than 65,535 columns) run as
// plain calls on the server's stream.
// Latency is measured from submit to the moment the scheduler sees the
// request's completion flag (the matrix complete on the device).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <iterator>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { REQ_QUEUED = 0, REQ_RUNNING = 1, REQ_DONE = 2, REQ_FAILED = 3 };

struct Request {
  uint64_t id = 0;
  std::vector<char> chars;  // host copy of the alignment (n * L) when not staged
  size_t pin_off = SIZE_MAX;  // staged: offset of the copy in the server's page-locked area
  int n = 0, L = 0, type = RNJ_DNA, model = RNJ_KIMURA, flags = RNJ_FASTDIST;
  size_t need = 0;          // device bytes reserved while the server holds it
  int state = REQ_QUEUED;
  Clock::time_point t_submit, t_done;
  rnj_mat *mat = nullptr;   // result (device), until taken
  std::string error;
  // in flight
  uint8_t *d_chars = nullptr;
  rnj_aln *aln = nullptr;
  float *d_out = nullptr;   // live: the output matrix (n x n)
  int slot = -1;            // live: the alignment slot of the work list
  size_t held = 0;          // bytes still counted against the budget
};

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Device bytes a request needs: raw bytes, packed operands, output.
size_t bytes_needed(int n, int L, int type, int flags) {
  const size_t np = round_up((size_t)std::max(n, 1), 128);
  const size_t raw = (size_t)n * L;
  size_t packed;
  if (type == RNJ_DNA && (flags & RNJ_FASTDIST) && !(flags & RNJ_POPCOUNT))
    packed = np * 2 * round_up((size_t)std::max(L, 1), 256);  // 4 FP4 features per site
  else
    packed = (size_t)8 * np * round_up((size_t)(L + 31) / 32, 8) * 4;
  const size_t out = (size_t)n * round_up((size_t)std::max(n, 4), 4) * 4;
  return raw + packed + out + 4096;
}

}  // namespace

struct rnj_server {
  rnj_ctx *ctx = nullptr;
  size_t budget = 0, in_use = 0;
  int max_batch = 0;
  long long max_tiles = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Request *> reqs;
  std::atomic<uint64_t> next_id{1};
  std::atomic<bool> stop{false};
  std::thread worker;
  // Page-locked staging of submitted alignments: submit copies a request into
  // memory that is already mapped and locked (a fresh host buffer would page
  // fault on first touch), and the scheduler's upload is then an asynchronous
  // DMA instead of a pageable copy that blocks it.  First fit over free extents.
  char *pin = nullptr;
  size_t pin_cap = 0;
  std::map<size_t, size_t> pin_free;  // offset -> bytes
  std::mutex pin_mu;
  // The live work list (device), its alignment slots and their descriptors.
  // Slots and items are handed out in order and reset together once nothing
  // is in flight and the kernel has exited.
  LiveList live{};
  AlnDesc *d_descs = nullptr;
  AlnDesc *h_descs = nullptr;   // page-locked staging of the descriptor uploads
  unsigned int *d_ctr = nullptr;  // head, tail, fix-up head and tail, exit vote (2)
  uint32_t *d_masks = nullptr, *h_masks = nullptr;  // residue presence, 8 words per admitted request
  int *d_max = nullptr, *d_flags = nullptr;
  int2 *h_done = nullptr;       // mapped page-locked: per slot {done, max bits}
  int next_slot = 0;
  unsigned int published = 0;   // items handed out (and published, in stream order)
  cudaStream_t s_live = nullptr;
  cudaEvent_t ev_live = nullptr, ev_pub = nullptr;
  bool live_running = false;
  // Trace (RNJ_SERVER_TRACE set: printed to stderr when the server is
  // destroyed): live launches, their host-observed running time, generation
  // resets, time in request preparation.
  bool trace = false;
  std::unique_ptr<std::atomic<int64_t>[]> pub_ns;
  uint64_t n_launch = 0, n_reset = 0, n_prepared = 0, n_passes = 0;
  double t_running = 0.0, t_prepare = 0.0, t_upload = 0.0, t_sync = 0.0, t_pack = 0.0,
         t_collect = 0.0, t_to_pub = 0.0, t_pub_to_done = 0.0, t_alloc = 0.0, t_copy = 0.0,
         t_out = 0.0, t_publish = 0.0;
  Clock::time_point t_launch;
  int live_grid = 0;
  std::vector<Request *> inflight;  // live requests not yet complete
  // statistics
  uint64_t completed = 0;
  double work_units = 0;  // pair-columns of completed requests
  Clock::time_point t_first, t_last;
  std::string fatal;
};

namespace {

constexpr size_t kPinAlign = 256;
// Staging area per server: 1 GiB (RNJ_SERVER_STAGING_MB overrides), so that a
// burst of requests is staged in page-locked memory rather than in pageable
// buffers that fault on first touch and make the uploads synchronous.
constexpr size_t kPinBytes = (size_t)1 << 30;

size_t pin_alloc(rnj_server *s, size_t bytes) {
  if (!s->pin || bytes == 0) return SIZE_MAX;
  bytes = round_up(bytes, kPinAlign);
  std::lock_guard<std::mutex> lk(s->pin_mu);
  for (auto it = s->pin_free.begin(); it != s->pin_free.end(); ++it) {
    if (it->second < bytes) continue;
    const size_t off = it->first, left = it->second - bytes;
    s->pin_free.erase(it);
    if (left) s->pin_free[off + bytes] = left;
    return off;
  }
  return SIZE_MAX;
}

void pin_release(rnj_server *s, Request *r) {
  if (r->pin_off == SIZE_MAX) return;
  size_t off = r->pin_off, bytes = round_up((size_t)r->n * r->L, kPinAlign);
  r->pin_off = SIZE_MAX;
  std::lock_guard<std::mutex> lk(s->pin_mu);
  auto next = s->pin_free.lower_bound(off);
  if (next != s->pin_free.end() && off + bytes == next->first) {
    bytes += next->second;
    next = s->pin_free.erase(next);
  }
  if (next != s->pin_free.begin()) {
    auto prev = std::prev(next);
    if (prev->first + prev->second == off) {
      prev->second += bytes;
      return;
    }
  }
  s->pin_free[off] = bytes;
}

// n rows of L bytes (source stride ld) into dst, packed.  Large requests are
// copied by several threads: one thread's copy bandwidth, not the device,
// bounds how fast requests can be submitted.
void copy_rows(char *dst, const char *src, int n, int L, size_t ld) {
  const size_t bytes = (size_t)n * L;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  // Four threads (measured on a 16-core host: 3.6-4.1x plain per-request calls
  // at saturation with p99 1.7-2.1 ms at 1000 req/s; eight threads gave 3.4x with
  // p99 2.7-3.2 ms, one thread 2.5x with p99 1.2-1.3 ms).
  const int T = bytes >= ((size_t)4 << 20) ? (int)std::min<unsigned>(4, std::max(1u, hw / 4)) : 1;
  auto part = [&](int t) {
    const int r0 = (int)((long long)n * t / T), r1 = (int)((long long)n * (t + 1) / T);
    if (ld == (size_t)L)
      memcpy(dst + (size_t)r0 * L, src + (size_t)r0 * L, (size_t)(r1 - r0) * L);
    else
      for (int i = r0; i < r1; ++i) memcpy(dst + (size_t)i * L, src + (size_t)i * ld, L);
  };
  if (T == 1) {
    part(0);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 1; t < T; ++t) pool.emplace_back(part, t);
  part(0);
  for (auto &th : pool) th.join();
}

const char *host_bytes(const rnj_server *s, const Request *r) {
  return r->pin_off != SIZE_MAX ? s->pin + r->pin_off : r->chars.data();
}

constexpr int kLiveSlots = 16384;          // alignments per work-list generation
constexpr int kLiveItems = 1 << 20;        // tiles per generation (8 MB of items)
constexpr int kLiveReserveSms = 16;        // SMs left to the packing kernels
constexpr unsigned int kLiveIdleUs = 500;  // the live kernel's idle time before it exits

size_t out_bytes(const Request *r) {
  return (size_t)r->n * round_up((size_t)std::max(r->n, 4), 4) * 4;
}

// Called with s->mu held: the request's matrix is complete (m) or it failed.
void finish_request(rnj_server *s, Request *r, rnj_mat *m, const std::string &error) {
  const auto now = Clock::now();
  if (m) {
    r->mat = m;
    r->state = REQ_DONE;
    s->completed++;
    s->work_units += (double)r->n * (r->n - 1) / 2.0 * r->L;
    s->t_last = now;
  } else {
    r->state = REQ_FAILED;
    r->error = error;
    if (r->d_out) cudaFreeAsync(r->d_out, s->ctx->stream);
  }
  r->d_out = nullptr;
  r->t_done = now;
  pin_release(s, r);  // its upload ran before its kernels on the same stream
  if (r->d_chars) cudaFreeAsync(r->d_chars, s->ctx->stream);
  r->d_chars = nullptr;
  if (r->aln) rnj_aln_destroy(r->aln);
  r->aln = nullptr;
  if (m) {
    const size_t out = out_bytes(r);
    s->in_use -= (r->held - out);  // the output stays counted until taken
    r->held = out;
  } else {
    s->in_use -= r->held;
    r->held = 0;
  }
  s->cv_done.notify_all();
}

// The requests admitted in one scheduling pass, outside the lock, on the
// server's stream: (1) every upload, and for protein the residue-presence scan
// into the request's own mask slot; (2) one synchronisation for all the masks;
// (3) per request the pack, then the live path (descriptor, scratch, publish)
// or, for what the tensor-core kernel cannot take, a plain call.
void prepare_all(rnj_server *s, const std::vector<Request *> &reqs) {
  rnj_ctx *ctx = s->ctx;
  auto ms_since = [](Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
  };
  auto t0 = Clock::now();
  const size_t nr = reqs.size();
  std::vector<int> rc(nr, RNJ_OK);
  std::vector<std::string> err(nr);
  bool any_protein = false;
  for (size_t k = 0; k < nr; ++k) {
    Request *r = reqs[k];
    auto ta = Clock::now();
    cudaError_t e = cudaMallocAsync((void **)&r->d_chars,
                                    std::max<size_t>((size_t)r->n * r->L, 1), ctx->stream);
    s->t_alloc += ms_since(ta);
    ta = Clock::now();
    if (e == cudaSuccess && r->n * (size_t)r->L > 0)
      e = cudaMemcpyAsync(r->d_chars, host_bytes(s, r), (size_t)r->n * r->L,
                          cudaMemcpyHostToDevice, ctx->stream);
    s->t_copy += ms_since(ta);
    if (e != cudaSuccess) {
      rc[k] = cuda_error(e, "request upload");
      err[k] = rnj_last_error();
    }
  }
  // The presence scans after every upload, so that the copies run back to back.
  for (size_t k = 0; k < nr; ++k) {
    Request *r = reqs[k];
    cudaError_t e = cudaSuccess;
    if (rc[k] == RNJ_OK && r->type == RNJ_PROTEIN) {
      uint32_t *dm = s->d_masks + 8 * k;
      e = cudaMemsetAsync(dm, 0, 8 * sizeof(uint32_t), ctx->stream);
      if (e == cudaSuccess && r->n > 0 && r->L > 0)
        e = launch_presence(r->d_chars, (size_t)r->L, r->n, r->L, dm, ctx->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_masks + 8 * k, dm, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            ctx->stream);
      any_protein = true;
    }
    if (e != cudaSuccess) {
      rc[k] = cuda_error(e, "residue presence scan");
      err[k] = rnj_last_error();
    }
  }
  s->t_upload += ms_since(t0);
  t0 = Clock::now();
  if (any_protein) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
      for (size_t k = 0; k < nr; ++k)
        if (rc[k] == RNJ_OK) {
          rc[k] = cuda_error(e, "presence scan");
          err[k] = rnj_last_error();
        }
  }
  s->t_sync += ms_since(t0);
  bool published = false;
  for (size_t k = 0; k < nr; ++k) {
    Request *r = reqs[k];
    t0 = Clock::now();
    if (rc[k] == RNJ_OK) {
      uint8_t lut[256];
      int kind = 0;
      lut_for(r->type, r->flags, r->type == RNJ_PROTEIN ? s->h_masks + 8 * k : nullptr, lut,
              &kind);
      rc[k] = pack_prepared(ctx, r->d_chars, r->n, r->L, (size_t)std::max(r->L, 1), r->type,
                            r->flags, kind, lut, &r->aln, false);
      if (rc[k] != RNJ_OK) err[k] = rnj_last_error();
    }
    s->t_pack += ms_since(t0);
    if (rc[k] != RNJ_OK) {
      std::lock_guard<std::mutex> lk(s->mu);
      finish_request(s, r, nullptr, err[k]);
      continue;
    }
    if (!is_tc_kind(r->aln->p.kind) || r->L > kMaxFusedColumns) {
      // a plain call on the server's stream
      rnj_mat *m = nullptr;
      int rc2 = rnj_distance(ctx, r->aln, r->model, &m);
      float mx = 0.0f;
      if (rc2 == RNJ_OK) rc2 = rnj_mat_info(m, nullptr, &mx);
      std::lock_guard<std::mutex> lk(s->mu);
      if (rc2 == RNJ_OK) {
        finish_request(s, r, m, "");
      } else {
        if (m) rnj_mat_destroy(m);
        finish_request(s, r, nullptr, rnj_last_error());
      }
      continue;
    }
    const Packed &p = r->aln->p;
    const int slot = s->next_slot++;
    const unsigned int first = s->published;
    const int nt = tiles_of(r->n);
    const unsigned int ntiles = (unsigned int)tri_tiles(nt);
    s->published += ntiles;
    r->slot = slot;
    auto tb = Clock::now();
    cudaError_t e =
        cudaMallocAsync((void **)&r->d_out, (size_t)r->n * r->n * sizeof(float), ctx->stream);
    s->t_out += ms_since(tb);
    tb = Clock::now();
    if (e == cudaSuccess) {
      EpiParams ep = epi_params_for(p, r->model);
      ep.out = r->d_out;
      ep.ld = (size_t)r->n;
      ep.max_bits = s->d_max + slot;
      ep.tile_flags = s->d_flags + first;
      ep.err = s->live.err;
      s->h_descs[slot] = desc_for(p, ep);
      s->h_done[slot] = make_int2(0, 0);
      e = cudaMemcpyAsync(s->d_descs + slot, s->h_descs + slot, sizeof(AlnDesc),
                          cudaMemcpyHostToDevice, ctx->stream);
    }
    const TuneParams tp = tune_lookup(p.n, p.L, p.type, p.flags);
    if (e == cudaSuccess)
      e = launch_live_publish(s->live, slot, nt, tp.tile_band, first, ntiles, s->d_max + slot,
                              s->d_flags + first, ctx->stream);
    s->t_publish += ms_since(tb);
    if (e == cudaSuccess && s->trace) {
      // trace: when the server's stream passed the publish (a server-owned
      // word per slot, so that a late callback never touches a freed request)
      s->pub_ns[slot].store(0);
      e = cudaLaunchHostFunc(
          ctx->stream,
          [](void *p) {
            static_cast<std::atomic<int64_t> *>(p)->store(
                std::chrono::duration_cast<std::chrono::nanoseconds>(
                    Clock::now().time_since_epoch())
                    .count());
          },
          &s->pub_ns[slot]);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (e == cudaSuccess) {
      s->inflight.push_back(r);
      published = true;
    } else {
      // Its slot and items stay unused until the next generation.
      const int rc3 = cuda_error(e, "request publish");
      (void)rc3;
      cudaStreamSynchronize(ctx->stream);
      finish_request(s, r, nullptr, rnj_last_error());
    }
  }
  // A launch of the live kernel waits for this (the pass's last publish).
  if (published) cudaEventRecord(s->ev_pub, ctx->stream);
}

// Called with s->mu held: the completion flags of the live requests.
bool collect(rnj_server *s) {
  bool any = false;
  for (size_t k = 0; k < s->inflight.size();) {
    Request *r = s->inflight[k];
    volatile int2 *f = s->h_done + r->slot;
    if (f->x != 1) {
      ++k;
      continue;
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    const int bits = f->y;
    if (s->trace) {
      const auto now = Clock::now();
      const int64_t pub = s->pub_ns[r->slot].load();
      const Clock::time_point tp{std::chrono::nanoseconds(pub)};
      if (pub) {
        s->t_to_pub += std::chrono::duration<double, std::milli>(tp - r->t_submit).count();
        s->t_pub_to_done += std::chrono::duration<double, std::milli>(now - tp).count();
      }
    }
    rnj_mat *m = new rnj_mat();
    m->ctx = s->ctx;
    m->d = r->d_out;
    m->n = r->n;
    m->ld = (size_t)r->n;
    m->owns = true;
    m->has_host_max = true;
    memcpy(&m->host_max, &bits, sizeof(float));
    finish_request(s, r, m, "");
    s->inflight[k] = s->inflight.back();
    s->inflight.pop_back();
    any = true;
  }
  return any;
}

void scheduler(rnj_server *s) {
  DeviceGuard g(s->ctx->device);
  while (!s->stop.load()) {
    bool progress = false;
    {
      const auto t0 = Clock::now();
      std::lock_guard<std::mutex> lock(s->mu);
      progress |= collect(s);
      s->t_collect += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    }
    // The live kernel exited: an error fails the requests in flight; requests
    // published after its CTAs stopped looking get a new launch below.
    if (s->live_running && cudaEventQuery(s->ev_live) != cudaErrorNotReady) {
      s->live_running = false;
      s->t_running += std::chrono::duration<double, std::milli>(Clock::now() - s->t_launch).count();
      int err = 0;
      cudaError_t e = cudaMemcpyAsync(&err, s->live.err, sizeof(int), cudaMemcpyDeviceToHost,
                                      s->s_live);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s->s_live);
      std::lock_guard<std::mutex> lock(s->mu);
      collect(s);
      if (e != cudaSuccess || err) {
        const std::string msg = e != cudaSuccess ? std::string(cudaGetErrorString(e))
                                                 : "a bounded device wait ran out in the server";
        cudaMemsetAsync(s->live.err, 0, sizeof(int), s->s_live);
        cudaStreamSynchronize(s->ctx->stream);
        for (Request *r : s->inflight) finish_request(s, r, nullptr, msg);
        s->inflight.clear();
      }
      progress = true;
    }
    // A new generation of slots and items once nothing is in flight.
    if (!s->live_running && s->inflight.empty() && s->published > 0) {
      cudaMemsetAsync(s->d_ctr, 0, 4 * sizeof(unsigned int), s->ctx->stream);
      cudaMemsetAsync(s->live.fix_items, 0, sizeof(unsigned long long) * kLiveItems,
                      s->ctx->stream);
      cudaEventRecord(s->ev_pub, s->ctx->stream);
      s->published = 0;
      ++s->n_reset;
      s->next_slot = 0;
    }
    // Admission, first come first served, within the budget and the list.
    std::vector<Request *> admitted;
    {
      std::lock_guard<std::mutex> lock(s->mu);
      unsigned int items = s->published;
      int slots = s->next_slot;
      while (!s->queue.empty() && (int)admitted.size() < s->max_batch) {
        Request *r = s->reqs[s->queue.front()];
        const unsigned int rt = (unsigned int)tri_tiles(tiles_of(r->n));
        if (s->in_use + r->need > s->budget) break;  // wait for memory (FIFO)
        if (slots + 1 > kLiveSlots || (long long)items + rt > kLiveItems) break;
        s->queue.pop_front();
        s->in_use += r->need;
        r->held = r->need;
        r->state = REQ_RUNNING;
        items += rt;
        ++slots;
        admitted.push_back(r);
      }
    }
    if (!admitted.empty()) {
      const auto t0 = Clock::now();
      prepare_all(s, admitted);
      s->t_prepare += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
      s->n_prepared += admitted.size();
      ++s->n_passes;
    }
    progress |= !admitted.empty();
    // A launch while live requests wait for tiles and none is running.
    bool waiting = false;
    {
      std::lock_guard<std::mutex> lock(s->mu);
      waiting = !s->inflight.empty();
    }
    if (waiting && !s->live_running) {
      cudaError_t e = cudaStreamWaitEvent(s->s_live, s->ev_pub, 0);
      if (e == cudaSuccess)  // a fresh exit vote
        e = cudaMemsetAsync(s->live.idle_ctas, 0, 2 * sizeof(unsigned int), s->s_live);
      if (e == cudaSuccess) e = launch_tc_live(s->d_descs, s->live, s->live_grid, 0, s->s_live);
      if (e == cudaSuccess) e = cudaEventRecord(s->ev_live, s->s_live);
      if (e == cudaSuccess) {
        s->live_running = true;
        s->t_launch = Clock::now();
        ++s->n_launch;
      } else {
        std::lock_guard<std::mutex> lock(s->mu);
        const std::string msg = std::string("live kernel launch: ") + cudaGetErrorString(e);
        for (Request *r : s->inflight) finish_request(s, r, nullptr, msg);
        s->inflight.clear();
      }
      progress = true;
    }
    if (!progress) {
      std::unique_lock<std::mutex> lock(s->mu);
      if (s->inflight.empty() && !s->live_running && s->queue.empty())
        s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
      else {
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(10));
      }
    }
  }
}

// Releases everything of a server whose scheduler has stopped.  The live
// kernel exits by itself once it has had nothing to claim for its idle time.
void free_server(rnj_server *s) {
  if (s->ctx) {
    DeviceGuard g(s->ctx->device);
    if (s->s_live) cudaStreamSynchronize(s->s_live);
    cudaStreamSynchronize(s->ctx->stream);
    for (auto &kv : s->reqs) {
      Request *r = kv.second;
      if (r->mat) rnj_mat_destroy(r->mat);
      if (r->d_out) cudaFreeAsync(r->d_out, s->ctx->stream);
      if (r->d_chars) cudaFreeAsync(r->d_chars, s->ctx->stream);
      if (r->aln) rnj_aln_destroy(r->aln);
      delete r;
    }
    s->reqs.clear();
    cudaStreamSynchronize(s->ctx->stream);
    cudaFree(s->d_descs);
    cudaFree(s->live.items);
    cudaFree(s->d_ctr);
    cudaFree(s->live.tiles_done);
    cudaFree(s->live.fix_pending);
    cudaFree(s->live.sat);
    cudaFree(s->live.fix_items);
    cudaFree(s->d_max);
    cudaFree(s->d_flags);
    cudaFree(s->live.err);
    if (s->h_descs) cudaFreeHost(s->h_descs);
    cudaFree(s->d_masks);
    if (s->h_masks) cudaFreeHost(s->h_masks);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->ev_live) cudaEventDestroy(s->ev_live);
    if (s->ev_pub) cudaEventDestroy(s->ev_pub);
    if (s->s_live) cudaStreamDestroy(s->s_live);
    rnj_ctx_destroy(s->ctx);  // synchronises its stream: no upload still reads the staging area
  }
  if (s->pin) cudaFreeHost(s->pin);
  delete s;
}

}  // namespace

extern "C" {

int rnj_server_create(int device, size_t memory_budget, int max_batch, rnj_server **out) {
  if (!out) return set_error(RNJ_ERR_INVALID, "out is NULL");
  rnj_server *s = new rnj_server();
  int rc = rnj_ctx_create(device, &s->ctx);
  if (rc != RNJ_OK) {
    delete s;
    return rc;
  }
  DeviceGuard g(device);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  s->budget = memory_budget ? memory_budget : (size_t)(0.6 * (double)free_b);
  s->max_batch = max_batch > 0 ? max_batch : 256;
  s->max_tiles = 255 * 256 / 2;  // n <= 32640 (one request's tiles in the work list)
  // Freed device memory stays in the device's default pool (stream-ordered
  // allocations of every request: bytes, packed operands, outputs) instead of
  // going back to the system at each synchronisation, so that the next
  // request's buffers come from the pool rather than from new mappings.  This
  // is the pool of the whole process on this device.
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  // The live work list and its slots.
  cudaError_t e = cudaStreamCreateWithFlags(&s->s_live, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_live, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_pub, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_descs, sizeof(AlnDesc) * kLiveSlots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->live.items, sizeof(WorkItem) * kLiveItems);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_ctr, 8 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->live.tiles_done, sizeof(unsigned int) * kLiveSlots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->live.fix_pending, sizeof(unsigned int) * kLiveSlots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->live.sat, sizeof(int) * kLiveSlots);
  if (e == cudaSuccess)
    e = cudaMalloc((void **)&s->live.fix_items, sizeof(unsigned long long) * kLiveItems);
  if (e == cudaSuccess)
    e = cudaMemset(s->live.fix_items, 0, sizeof(unsigned long long) * kLiveItems);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_max, sizeof(int) * kLiveSlots);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->d_flags, sizeof(int) * kLiveItems);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->live.err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s->d_ctr, 0, 8 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(s->live.err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_descs, sizeof(AlnDesc) * kLiveSlots, 0);
  if (e == cudaSuccess)
    e = cudaMalloc((void **)&s->d_masks, 8 * sizeof(uint32_t) * (size_t)s->max_batch);
  if (e == cudaSuccess)
    e = cudaHostAlloc((void **)&s->h_masks, 8 * sizeof(uint32_t) * (size_t)s->max_batch, 0);
  if (e == cudaSuccess)
    e = cudaHostAlloc((void **)&s->h_done, sizeof(int2) * kLiveSlots, cudaHostAllocMapped);
  int2 *d_done = nullptr;
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&d_done, s->h_done, 0);
  if (e != cudaSuccess) {
    rc = cuda_error(e, "server allocation");
    free_server(s);
    return rc;
  }
  memset(s->h_done, 0, sizeof(int2) * kLiveSlots);
  s->live.head = s->d_ctr;
  s->live.tail = s->d_ctr + 1;
  s->live.fix_head = s->d_ctr + 2;
  s->live.fix_tail = s->d_ctr + 3;
  s->live.idle_ctas = s->d_ctr + 4;
  s->live.closing = s->d_ctr + 5;
  s->live.done = d_done;
  s->live.cap_items = kLiveItems;
  s->live.cap_aln = kLiveSlots;
  s->live.idle_us = kLiveIdleUs;
  int reserve = kLiveReserveSms;
  if (const char *v = getenv("RNJ_SERVER_RESERVE_SMS")) reserve = std::max(1, atoi(v));
  if (const char *v = getenv("RNJ_SERVER_IDLE_US")) s->live.idle_us = (unsigned)std::max(1, atoi(v));
  s->live_grid = std::max(1, s->ctx->num_sms - reserve);
  {
    const char *t = getenv("RNJ_SERVER_TRACE");
    s->trace = t && *t && strcmp(t, "0") != 0;
    if (s->trace) s->pub_ns.reset(new std::atomic<int64_t>[kLiveSlots]());
  }
  // Staging area (best effort: without it requests are copied to pageable memory).
  size_t pin_bytes = kPinBytes;
  if (const char *v = getenv("RNJ_SERVER_STAGING_MB")) pin_bytes = (size_t)std::max(1, atoi(v)) << 20;
  if (cudaHostAlloc((void **)&s->pin, pin_bytes, cudaHostAllocDefault) == cudaSuccess) {
    s->pin_cap = pin_bytes;
    s->pin_free[0] = pin_bytes;
  } else {
    cudaGetLastError();
    s->pin = nullptr;
  }
  s->worker = std::thread(scheduler, s);
  *out = s;
  return RNJ_OK;
}

int rnj_server_submit(rnj_server *s, const char *chars, int n, int L, size_t ld, int type,
                      int model, int flags, uint64_t *id) {
  if (!s || (!chars && n > 0 && L > 0) || n < 1 || L < 0 || ld < (size_t)L)
    return set_error(RNJ_ERR_INVALID, "invalid request");
  if (model != RNJ_JC && model != RNJ_KIMURA) return set_error(RNJ_ERR_INVALID, "unknown model");
  if (type == RNJ_UNKNOWN) type = rnj_detect_type(chars, L);
  if (tri_tiles(tiles_of(n)) > s->max_tiles)
    return set_error(RNJ_ERR_INVALID, "alignment has more tiles than the server takes for one "
                                      "request (n > " + std::to_string(kTile * 255) +
                                          "); use rnj_distance");
  Request *r = new Request();
  r->id = s->next_id.fetch_add(1);
  r->n = n;
  r->L = L;
  r->type = type;
  r->model = model;
  r->flags = flags;
  const size_t bytes = (size_t)n * L;
  r->pin_off = pin_alloc(s, bytes);
  char *dst = r->pin_off != SIZE_MAX ? s->pin + r->pin_off : nullptr;
  if (!dst) {
    r->chars.resize(bytes);
    dst = r->chars.data();
  }
  copy_rows(dst, chars, n, L, ld);
  r->need = bytes_needed(n, L, type, flags);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (r->need > s->budget) {
      pin_release(s, r);
      delete r;
      return set_error(RNJ_ERR_BUSY, "request larger than the server's memory budget");
    }
    if (s->completed == 0 && s->reqs.empty()) s->t_first = r->t_submit;
    s->reqs[r->id] = r;
    s->queue.push_back(r->id);
  }
  s->cv_work.notify_one();
  if (id) *id = r->id;
  return RNJ_OK;
}

int rnj_server_poll(rnj_server *s, uint64_t id, int *state) {
  if (!s || !state) return set_error(RNJ_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(RNJ_ERR_INVALID, "unknown request");
  *state = it->second->state;
  return RNJ_OK;
}

int rnj_server_wait(rnj_server *s, uint64_t id, int timeout_ms) {
  if (!s) return set_error(RNJ_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(RNJ_ERR_INVALID, "unknown request");
  Request *r = it->second;
  const bool ok = s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] {
    return r->state == REQ_DONE || r->state == REQ_FAILED;
  });
  if (!ok) return set_error(RNJ_ERR_TIMEOUT, "request not finished within the timeout");
  if (r->state == REQ_FAILED) return set_error(RNJ_ERR_CUDA, "request failed: " + r->error);
  return RNJ_OK;
}

int rnj_server_result(rnj_server *s, uint64_t id, rnj_ctx *owner, rnj_mat **out,
                      double *latency_ms) {
  if (!s || !out) return set_error(RNJ_ERR_INVALID, "null argument");
  if (owner && owner->device != s->ctx->device)
    return set_error(RNJ_ERR_INVALID, "owner context on another device");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(RNJ_ERR_INVALID, "unknown request");
  Request *r = it->second;
  if (r->state == REQ_FAILED) return set_error(RNJ_ERR_CUDA, "request failed: " + r->error);
  if (r->state != REQ_DONE) return set_error(RNJ_ERR_NOTREADY, "request still running");
  // The matrix leaves the server: it is freed and read on the owner's stream
  // from now on, so it outlives the server.
  if (owner) r->mat->ctx = owner;
  *out = r->mat;
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  s->in_use -= r->held;
  s->reqs.erase(it);
  delete r;
  return RNJ_OK;
}

int rnj_server_stats(rnj_server *s, uint64_t *completed, double *pair_columns, double *seconds,
                     size_t *bytes_in_use) {
  if (!s) return set_error(RNJ_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lock(s->mu);
  if (completed) *completed = s->completed;
  if (pair_columns) *pair_columns = s->work_units;
  if (seconds)
    *seconds = s->completed ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
  if (bytes_in_use) *bytes_in_use = s->in_use;
  return RNJ_OK;
}

int rnj_server_destroy(rnj_server *s) {
  if (!s) return RNJ_OK;
  s->stop.store(true);
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->trace)
    fprintf(stderr,
            "rnj server: %llu requests prepared in %llu passes, %.3f ms (uploads %.3f, mask "
            "sync %.3f, packs %.3f); collect %.3f ms; %llu live launches running %.3f ms; %llu "
            "list generations; summed over live requests: submit -> published %.3f ms, "
            "published -> complete seen %.3f ms; input allocations %.3f, input copies %.3f, "
            "output allocations %.3f, publishes %.3f ms\n",
            (unsigned long long)s->n_prepared, (unsigned long long)s->n_passes, s->t_prepare,
            s->t_upload, s->t_sync, s->t_pack, s->t_collect, (unsigned long long)s->n_launch,
            s->t_running, (unsigned long long)s->n_reset, s->t_to_pub, s->t_pub_to_done, s->t_alloc,
            s->t_copy, s->t_out, s->t_publish);
  free_server(s);
  return RNJ_OK;
}

}  // extern "C"
