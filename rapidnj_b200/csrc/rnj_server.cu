// rnj_server.cu -- served form: continuous batching of distance requests.
//
// Clients submit alignments from any thread; a scheduler thread owns the GPU
// work:
//   * admission: a request is admitted when the device memory it needs (its
//     bytes, packed operands and output matrix) fits the server's budget;
//     otherwise it waits (first come, first served);
//   * a submitted alignment is copied into the server's page-locked staging
//     area (pageable memory when it is full), so that its upload is an
//     asynchronous DMA;
//   * every admitted request is uploaded and packed on the server's stream and
//     added to the batch being formed;
//   * up to two batches are in flight: a new batch is launched as soon as it has
//     requests, while the previous one may still run, so the new batch's
//     persistent CTAs take SMs as the old batch's finish and the two overlap on
//     the device;
//   * completion is observed on the batch's event; packed inputs are released
//     at once, the output matrix stays on the device until the client takes it.
// Latency is measured from submit to the moment the matrix is complete on the
// device (as the scheduler observes the batch's completion event).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <iterator>
#include <map>
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
  int batch = -1, slot = -1;
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
  rnj_batch *batch[2] = {nullptr, nullptr};
  bool busy[2] = {false, false};
  std::vector<uint64_t> members[2];
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Request *> reqs;
  std::atomic<uint64_t> next_id{1};
  std::atomic<bool> stop{false};
  std::thread worker;
  // statistics
  // Page-locked staging of submitted alignments: submit copies a request into
  // memory that is already mapped and locked (a fresh host buffer would page
  // fault on first touch), and the scheduler's upload is then an asynchronous
  // DMA instead of a pageable copy that blocks it.  First fit over free extents.
  char *pin = nullptr;
  size_t pin_cap = 0;
  std::map<size_t, size_t> pin_free;  // offset -> bytes
  std::mutex pin_mu;
  uint64_t completed = 0;
  double work_units = 0;  // pair-columns of completed requests
  Clock::time_point t_first, t_last;
  std::string fatal;
};

namespace {

constexpr size_t kPinAlign = 256;
constexpr size_t kPinBytes = (size_t)256 << 20;  // staging area per server

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

void finish_batch(rnj_server *s, int b) {
  // Called with s->mu held, after the batch's completion.
  const auto now = Clock::now();
  for (uint64_t id : s->members[b]) {
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) continue;
    Request *r = it->second;
    rnj_mat *m = nullptr;
    int rc = rnj_batch_take(s->batch[b], r->slot, &m);
    if (rc == RNJ_OK) {
      r->mat = m;
      r->state = REQ_DONE;
    } else {
      r->state = REQ_FAILED;
      r->error = rnj_last_error();
    }
    r->t_done = now;
    pin_release(s, r);  // its upload ran before the batch on the same stream
    if (r->d_chars) cudaFreeAsync(r->d_chars, s->ctx->stream);
    r->d_chars = nullptr;
    r->aln = nullptr;  // owned by the batch, freed by rnj_batch_clear
    const size_t out = (size_t)r->n * round_up((size_t)std::max(r->n, 4), 4) * 4;
    s->in_use -= (r->held - out);  // keep the output counted until taken
    r->held = out;
    if (r->state == REQ_DONE) {
      s->completed++;
      s->work_units += (double)r->n * (r->n - 1) / 2.0 * r->L;
      s->t_last = now;
    }
  }
  rnj_batch_clear(s->batch[b]);
  s->members[b].clear();
  s->busy[b] = false;
  s->cv_done.notify_all();
}

void scheduler(rnj_server *s) {
  DeviceGuard g(s->ctx->device);
  while (!s->stop.load()) {
    std::unique_lock<std::mutex> lock(s->mu);
    // Completed batches.
    for (int b = 0; b < 2; ++b) {
      if (!s->busy[b]) continue;
      int done = 0;
      if (rnj_batch_poll(s->batch[b], &done) != RNJ_OK) done = 1;
      if (done) finish_batch(s, b);
    }
    // Form a batch from admitted requests if a batch slot is free.
    int free_b = !s->busy[0] ? 0 : (!s->busy[1] ? 1 : -1);
    if (free_b < 0 || s->queue.empty()) {
      if (s->busy[0] || s->busy[1]) {
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      } else {
        s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
      }
      continue;
    }
    std::vector<Request *> admitted;
    long long tiles = 0;
    while (!s->queue.empty() && (int)admitted.size() < s->max_batch) {
      Request *r = s->reqs[s->queue.front()];
      const int nt = tiles_of(r->n);
      const long long rt = tri_tiles(nt);
      if (s->in_use + r->need > s->budget) break;  // wait for memory (FIFO)
      if (tiles + rt > s->max_tiles) break;
      s->queue.pop_front();
      s->in_use += r->need;
      r->held = r->need;
      r->state = REQ_RUNNING;
      tiles += rt;
      admitted.push_back(r);
    }
    if (admitted.empty()) {
      lock.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(50));
      continue;
    }
    lock.unlock();
    // Upload and pack outside the lock (clients may keep submitting).
    std::vector<const void *> ptrs;
    std::vector<int> ns, Ls, types, models;
    std::vector<size_t> lds;
    int flags = admitted[0]->flags;
    std::vector<Request *> ok;
    for (Request *r : admitted) {
      cudaError_t e = cudaMallocAsync((void **)&r->d_chars, std::max<size_t>((size_t)r->n * r->L, 1),
                                      s->ctx->stream);
      if (e == cudaSuccess && r->n * (size_t)r->L > 0)
        e = cudaMemcpyAsync(r->d_chars, host_bytes(s, r), (size_t)r->n * r->L,
                            cudaMemcpyHostToDevice, s->ctx->stream);
      if (e != cudaSuccess) {
        cudaStreamSynchronize(s->ctx->stream);
        pin_release(s, r);
        std::lock_guard<std::mutex> l2(s->mu);
        r->state = REQ_FAILED;
        r->error = cudaGetErrorString(e);
        r->t_done = Clock::now();
        s->in_use -= r->held;
        r->held = 0;
        continue;
      }
      ok.push_back(r);
    }
    // Requests of one batch share the flag set of the first; others go alone.
    std::vector<Request *> same, later;
    for (Request *r : ok) (r->flags == flags ? same : later).push_back(r);
    for (Request *r : same) {
      ptrs.push_back(r->d_chars);
      ns.push_back(r->n);
      Ls.push_back(r->L);
      lds.push_back((size_t)std::max(r->L, 1));
      types.push_back(r->type);
      models.push_back(r->model);
    }
    std::vector<int> slots(same.size());
    int rc = rnj_batch_add_many(s->batch[free_b], (int)same.size(), ptrs.data(), ns.data(),
                                Ls.data(), lds.data(), types.data(), models.data(), flags, nullptr,
                                nullptr, slots.data());
    if (rc == RNJ_OK) rc = rnj_batch_run(s->batch[free_b]);
    lock.lock();
    for (Request *r : later) {  // back to the front of the queue for the next batch
      s->in_use -= r->held;
      r->held = 0;
      r->state = REQ_QUEUED;
      if (r->d_chars) cudaFreeAsync(r->d_chars, s->ctx->stream);
      r->d_chars = nullptr;
      s->queue.push_front(r->id);
    }
    if (rc != RNJ_OK) {
      cudaStreamSynchronize(s->ctx->stream);
      for (Request *r : same) {
        pin_release(s, r);
        r->state = REQ_FAILED;
        r->error = rnj_last_error();
        r->t_done = Clock::now();
        s->in_use -= r->held;
        r->held = 0;
      }
      rnj_batch_clear(s->batch[free_b]);
      s->cv_done.notify_all();
      continue;
    }
    for (size_t k = 0; k < same.size(); ++k) {
      same[k]->batch = free_b;
      same[k]->slot = slots[k];
      s->members[free_b].push_back(same[k]->id);
    }
    s->busy[free_b] = true;
  }
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
  s->max_tiles = 255 * 256 / 2;  // n <= 32640; eight tensor-core passes per batch graph
  for (int b = 0; b < 2; ++b) {
    rc = rnj_batch_create(s->ctx, s->max_batch, s->max_tiles, &s->batch[b]);
    if (rc != RNJ_OK) {
      for (int k = 0; k < b; ++k) rnj_batch_destroy(s->batch[k]);
      rnj_ctx_destroy(s->ctx);
      delete s;
      return rc;
    }
    batch_set_join(s->batch[b], false);
  }
  // Staging area (best effort: without it requests are copied to pageable memory).
  if (cudaHostAlloc((void **)&s->pin, kPinBytes, cudaHostAllocDefault) == cudaSuccess) {
    s->pin_cap = kPinBytes;
    s->pin_free[0] = kPinBytes;
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
    return set_error(RNJ_ERR_INVALID, "alignment has more tiles than a server batch holds (n > " +
                                          std::to_string(kTile * 255) + "); use rnj_distance");
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
  {
    DeviceGuard g(s->ctx->device);
    for (int b = 0; b < 2; ++b) {
      if (s->busy[b]) rnj_batch_synchronize(s->batch[b]);
      rnj_batch_destroy(s->batch[b]);
    }
    for (auto &kv : s->reqs) {
      if (kv.second->mat) rnj_mat_destroy(kv.second->mat);
      if (kv.second->d_chars) cudaFreeAsync(kv.second->d_chars, s->ctx->stream);
      delete kv.second;
    }
  }
  rnj_ctx_destroy(s->ctx);  // synchronises its stream: no upload still reads the staging area
  if (s->pin) cudaFreeHost(s->pin);
  delete s;
  return RNJ_OK;
}

}  // extern "C"
