// rnj_tune.cu -- the launch-parameter autotuner and its per-bucket table.
//
// A bucket is (alphabet, counting rules, floor(log2 n), floor(log2 L)).  For
// each bucket the table holds the choices that only change the time of a
// distance call, never its result:
//   * tensor-core or bit-plane popcount counting (DNA fast rules, protein);
//   * bit-plane kernel: how many CTAs share the columns of one tile (K split,
//     counts accumulated atomically, then the transform) -- one CTA per tile
//     leaves most SMs idle when a long alignment has few sequences -- and the
//     depth of its ring of staged K blocks;
//   * tensor-core kernels: the band height of the tile order (L2 reuse of the
//     operand slabs), the depth of the ring of staged K blocks, and the
//     epilogue form: the transform in the counting kernel's own warps, or
//     packed counts and a transform kernel with its resident CTAs per SM;
//   * the streamed host call: its band height.
// rnj_tune measures the candidates on a seeded synthetic alignment of the
// caller's shape through the library's own calls and keeps the fastest.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "rnj_internal.h"
#include "rnj_objects.h"

using namespace rnj;

namespace {

using Key = std::tuple<int, int, int, int>;  // type, naive rules, log2 n, log2 L

std::mutex g_mu;
std::map<Key, rnj_tune_params> g_table;
std::once_flag g_env_once;

int floor_log2(long long x) {
  int r = 0;
  while (x > 1) {
    x >>= 1;
    ++r;
  }
  return r;
}

Key key_of(int n, int L, int type, int flags) {
  return Key(type, (flags & RNJ_FASTDIST) ? 0 : 1, floor_log2(std::max(1, n)),
             floor_log2(std::max(1, L)));
}

bool valid_params(const rnj_tune_params &p) {
  return (p.dna_kernel == 0 || p.dna_kernel == 1) && p.ksplit >= 0 && p.ksplit <= 64 &&
         p.tile_band >= 0 && p.tile_band <= 4096 && p.transform_ctas >= 0 &&
         p.transform_ctas <= kTransformCtasPerSm && p.stream_band >= 0 && p.stream_band <= 4096 &&
         (p.tc_epilogue == 0 || p.tc_epilogue == 1) && p.tc_stages >= 0 && p.tc_stages <= 7 &&
         p.pop_stages >= 0 && p.pop_stages <= 4;
}

const char *cache_path() {
  const char *p = getenv("RNJ_TUNE_CACHE");
  return (p && *p) ? p : nullptr;
}

// Text form: a header comment, then one bucket per line:
//   <dna|protein> <naive 0/1> <log2 n> <log2 L> <dna_kernel> <ksplit> <tile_band>
//   <transform_ctas> <stream_band> <tc_epilogue> <tc_stages> <pop_stages> <ms>
// Lines of the earlier forms are read too: without the two ring depths (11
// fields) or also without tc_epilogue (10 fields); the missing fields are 0.
int load_locked(const char *path) {
  FILE *f = fopen(path, "r");
  if (!f) return set_error(RNJ_ERR_IO, std::string("cannot open ") + path);
  char line[512];
  int lineno = 0;
  while (fgets(line, sizeof line, f)) {
    ++lineno;
    if (line[0] == '#' || line[0] == '\n') continue;
    // tokens after the type: naive log2n log2L, then the integer fields, ms last
    char type[16];
    int consumed = 0;
    bool ok = sscanf(line, "%15s%n", type, &consumed) == 1;
    std::vector<double> v;
    for (const char *c = line + consumed; ok;) {
      char *end = nullptr;
      const double x = strtod(c, &end);
      if (end == c) break;
      v.push_back(x);
      c = end;
    }
    rnj_tune_params p;
    memset(&p, 0, sizeof p);
    const size_t nv = v.size();  // 9, 10 or 12 numbers after the type
    ok = ok && (nv == 9 || nv == 10 || nv == 12);
    int *const ints[] = {&p.dna_kernel, &p.ksplit,      &p.tile_band, &p.transform_ctas,
                         &p.stream_band, &p.tc_epilogue, &p.tc_stages, &p.pop_stages};
    for (size_t k = 0; ok && k + 1 < nv; ++k)
      ok = std::fabs(v[k]) < 1e9 && v[k] == std::floor(v[k]);  // integer fields
    int naive = 0, ln = 0, ll = 0;
    if (ok) {
      naive = (int)v[0];
      ln = (int)v[1];
      ll = (int)v[2];
      for (size_t k = 3; k + 1 < nv; ++k) *ints[k - 3] = (int)v[k];
      p.ms = (float)v[nv - 1];
    }
    const int t = strcmp(type, "dna") == 0 ? RNJ_DNA : (strcmp(type, "protein") == 0 ? RNJ_PROTEIN : -1);
    if (!ok || t < 0 || (naive != 0 && naive != 1) || ln < 0 || ln > 40 || ll < 0 || ll > 40 ||
        !valid_params(p)) {
      fclose(f);
      return set_error(RNJ_ERR_FORMAT, std::string(path) + ": bad tune entry on line " +
                                           std::to_string(lineno));
    }
    g_table[Key(t, naive, ln, ll)] = p;
  }
  fclose(f);
  return RNJ_OK;
}

int save_locked(const char *path) {
  FILE *f = fopen(path, "w");
  if (!f) return set_error(RNJ_ERR_IO, std::string("cannot write ") + path);
  fprintf(f, "# rapidnj-b200 tune table v3: type naive log2n log2L dna_kernel ksplit tile_band "
             "transform_ctas stream_band tc_epilogue tc_stages pop_stages ms\n");
  for (const auto &kv : g_table) {
    const rnj_tune_params &p = kv.second;
    fprintf(f, "%s %d %d %d %d %d %d %d %d %d %d %d %.4f\n",
            std::get<0>(kv.first) == RNJ_DNA ? "dna" : "protein", std::get<1>(kv.first),
            std::get<2>(kv.first), std::get<3>(kv.first), p.dna_kernel, p.ksplit, p.tile_band,
            p.transform_ctas, p.stream_band, p.tc_epilogue, p.tc_stages, p.pop_stages, p.ms);
  }
  const bool ok = fclose(f) == 0;
  return ok ? RNJ_OK : set_error(RNJ_ERR_IO, std::string("cannot write ") + path);
}

// The table shipped beside the library (tune_b200.txt in the directory of
// librnjgpu.so, made by make_tune_table.py on a B200), or "" if not found.
std::string shipped_table() {
  Dl_info info;
  if (dladdr(reinterpret_cast<void *>(&rnj_tune_get), &info) == 0 || !info.dli_fname) return "";
  std::string path(info.dli_fname);
  const size_t slash = path.rfind('/');
  path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/tune_b200.txt";
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return "";
  fclose(f);
  return path;
}

// First use: the file RNJ_TUNE_CACHE names (if it exists yet), else the
// shipped table unless RNJ_NO_TUNE_TABLE is set.  A shipped table that does
// not parse is ignored (the defaults stay); rnj_tune_load reports errors.
void load_env_once() {
  std::call_once(g_env_once, [] {
    const char *p = cache_path();
    std::string path;
    if (p) {
      path = p;
    } else {
      const char *off = getenv("RNJ_NO_TUNE_TABLE");
      if (off && *off && strcmp(off, "0") != 0) return;
      path = shipped_table();
    }
    if (path.empty()) return;
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return;  // no cache yet: the first rnj_tune writes it
    fclose(f);
    std::lock_guard<std::mutex> lk(g_mu);
    if (load_locked(path.c_str()) != RNJ_OK) g_table.clear();
  });
}

}  // namespace

namespace rnj {

TuneParams tune_lookup(int n, int L, int type, int flags, bool *found) {
  load_env_once();
  TuneParams t;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find(key_of(n, L, type, flags));
  if (found) *found = it != g_table.end();
  if (it == g_table.end()) return t;
  t.dna_kernel = it->second.dna_kernel;
  t.ksplit = std::max(1, it->second.ksplit);
  t.tile_band = it->second.tile_band;
  t.transform_ctas = it->second.transform_ctas;
  t.stream_band = it->second.stream_band;
  t.tc_epilogue = it->second.tc_epilogue;
  t.tc_stages = it->second.tc_stages;
  t.pop_stages = it->second.pop_stages;
  return t;
}

}  // namespace rnj

namespace {

// Seeded synthetic alignment of related sequences: a random root, every row
// the root with 8 % of its sites replaced by a random letter and 3 % gaps.
std::vector<char> synthetic(int n, int L, int type, uint64_t seed) {
  static const char dna[] = "ACGT";
  static const char aa[] = "ACDEFGHIKLMNPQRSTVWY";
  const char *alpha = type == RNJ_DNA ? dna : aa;
  const int na = type == RNJ_DNA ? 4 : 20;
  uint64_t s = seed;
  auto next = [&s]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<char> root((size_t)L), out((size_t)n * L);
  for (int j = 0; j < L; ++j) root[j] = alpha[next() % na];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < L; ++j) {
      const uint64_t r = next() % 1000;
      out[(size_t)i * L + j] = r < 30 ? '-' : (r < 110 ? alpha[next() % na] : root[j]);
    }
  return out;
}

// Device buffers and pinned host buffers of one tuning call.
struct TuneBuffers {
  rnj_ctx *ctx;
  void *d_chars = nullptr;
  float *d_out = nullptr;
  char *h_chars = nullptr;
  float *h_out = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  explicit TuneBuffers(rnj_ctx *c) : ctx(c) {}
  ~TuneBuffers() {
    cudaStreamSynchronize(ctx->stream);
    if (d_chars) cudaFree(d_chars);
    if (d_out) cudaFree(d_out);
    if (h_chars) cudaFreeHost(h_chars);
    if (h_out) cudaFreeHost(h_out);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Repetitions of one candidate's timing: at least `reps`, and more (up to
// kMaxReps) until the timed calls add up to kMinTimedMs, so that the median of
// a small shape's calls (tens of microseconds each) is not one noisy sample.
constexpr int kMaxReps = 41;
constexpr float kMinTimedMs = 25.0f;
// A candidate replaces the best so far only when it is faster by this
// fraction: the first candidate of each search is the default, which stays
// unless another is clearly faster.
constexpr float kTuneMargin = 0.02f;

bool more_reps(const std::vector<float> &t, int reps) {
  if ((int)t.size() < reps) return true;
  float sum = 0.0f;
  for (float x : t) sum += x;
  return sum < kMinTimedMs && (int)t.size() < kMaxReps;
}

// Median device time (ms) of pack + distances with the bucket's table entry
// set to `p`, after one untimed call.
int time_plain(rnj_ctx *ctx, TuneBuffers &b, int n, int L, int type, int flags, int model,
               const rnj_tune_params &p, int reps, float *ms) {
  rnj_tune_set(n, L, type, flags, &p);
  std::vector<float> t;
  for (int r = -1; r < 0 || more_reps(t, reps); ++r) {
    if (cudaEventRecord(b.ev[0], ctx->stream) != cudaSuccess) return cuda_error(cudaGetLastError(), "event");
    rnj_aln *a = nullptr;
    int rc = rnj_aln_from_device(ctx, b.d_chars, n, L, (size_t)L, type, flags, &a);
    if (rc == RNJ_OK) rc = rnj_distance_into(ctx, a, model, b.d_out, (size_t)n, nullptr);
    if (a) rnj_aln_destroy(a);
    if (rc != RNJ_OK) return rc;
    cudaEventRecord(b.ev[1], ctx->stream);
    const cudaError_t e = cudaEventSynchronize(b.ev[1]);
    if (e != cudaSuccess) return cuda_error(e, "tuning run");
    float x = 0.0f;
    cudaEventElapsedTime(&x, b.ev[0], b.ev[1]);
    if (r >= 0) t.push_back(x);
  }
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return RNJ_OK;
}

// Median host time (ms) of the host-to-host call with band height `band`.
int time_host(rnj_ctx *ctx, TuneBuffers &b, int n, int L, int type, int flags, int model,
              const rnj_tune_params &p, int reps, float *ms) {
  rnj_tune_set(n, L, type, flags, &p);
  std::vector<float> t;
  for (int r = -1; r < 0 || more_reps(t, reps); ++r) {
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = rnj_distance_matrix_host_ex(ctx, b.h_chars, n, L, (size_t)L, type, model,
                                               flags, 0, b.h_out, nullptr);
    if (rc != RNJ_OK) return rc;
    const auto t1 = std::chrono::steady_clock::now();
    if (r >= 0) t.push_back(std::chrono::duration<float, std::milli>(t1 - t0).count());
  }
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return RNJ_OK;
}

}  // namespace

extern "C" {

int rnj_tune_get(int n, int L, int type, int flags, rnj_tune_params *out) {
  if (!out) return set_error(RNJ_ERR_INVALID, "out is NULL");
  if (type != RNJ_DNA && type != RNJ_PROTEIN) return set_error(RNJ_ERR_INVALID, "type must be DNA or protein");
  load_env_once();
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find(key_of(n, L, type, flags));
  if (it == g_table.end()) return set_error(RNJ_ERR_NOTREADY, "no tuned entry for this bucket");
  *out = it->second;
  return RNJ_OK;
}

int rnj_tune_set(int n, int L, int type, int flags, const rnj_tune_params *params) {
  if (!params) return set_error(RNJ_ERR_INVALID, "params is NULL");
  if (type != RNJ_DNA && type != RNJ_PROTEIN) return set_error(RNJ_ERR_INVALID, "type must be DNA or protein");
  if (!valid_params(*params)) return set_error(RNJ_ERR_INVALID, "tune parameter out of range");
  load_env_once();
  std::lock_guard<std::mutex> lk(g_mu);
  g_table[key_of(n, L, type, flags)] = *params;
  return RNJ_OK;
}

int rnj_tune_clear(void) {
  load_env_once();
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
  return RNJ_OK;
}

int rnj_tune_save(const char *path) {
  if (!path) return set_error(RNJ_ERR_INVALID, "path is NULL");
  load_env_once();
  std::lock_guard<std::mutex> lk(g_mu);
  return save_locked(path);
}

int rnj_tune_load(const char *path) {
  if (!path) return set_error(RNJ_ERR_INVALID, "path is NULL");
  load_env_once();
  std::lock_guard<std::mutex> lk(g_mu);
  return load_locked(path);
}

}  // extern "C"

extern "C" int rnj_tune(rnj_ctx *ctx, int n, int L, int type, int flags, rnj_tune_params *out) {
  if (!ctx) return set_error(RNJ_ERR_INVALID, "ctx is NULL");
  if (type != RNJ_DNA && type != RNJ_PROTEIN) return set_error(RNJ_ERR_INVALID, "type must be DNA or protein");
  if (n < 2 || L < 1) return set_error(RNJ_ERR_INVALID, "tuning needs n >= 2 and L >= 1");
  if ((long long)n * L > (2LL << 30) || n > 65536)
    return set_error(RNJ_ERR_INVALID, "tuning shape too large (n * L <= 2^31, n <= 65536)");
  DeviceGuard guard(ctx->device);
  const int model = RNJ_KIMURA;
  const int reps = 5;
  TuneBuffers b(ctx);
  {
    const std::vector<char> h = synthetic(n, L, type, 0x5EEDull + (uint64_t)n * 131 + (uint64_t)L);
    cudaError_t e = cudaMalloc(&b.d_chars, (size_t)n * L);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b.d_out, (size_t)n * n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(b.d_chars, h.data(), h.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaEventCreate(&b.ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&b.ev[1]);
    if (e != cudaSuccess) return cuda_error(e, "tuning buffers");
  }
  // The bucket's previous entry is restored if tuning fails part-way.
  rnj_tune_params prev;
  const bool had_prev = rnj_tune_get(n, L, type, flags, &prev) == RNJ_OK;
  auto restore = [&]() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (had_prev) g_table[key_of(n, L, type, flags)] = prev;
    else g_table.erase(key_of(n, L, type, flags));
  };

  const int nt = tiles_of(n);
  const int nk = std::max(1, ((L + 31) / 32 + kKW - 1) / kKW);  // 8-word K blocks of the bit planes
  // Tensor cores: DNA with the fast rules; protein with either (its synthetic
  // alphabet has 20 residues, within the tensor-core limit).
  const bool tc_ok = (type == RNJ_PROTEIN || (flags & RNJ_FASTDIST)) && !(flags & RNJ_POPCOUNT) &&
                     L <= kMaxTcColumns;
  const bool split_ok = (size_t)n * n * 3 * sizeof(uint32_t) <= ((size_t)1 << 30);
  rnj_tune_params best;
  memset(&best, 0, sizeof best);
  best.ms = 1e30f;
  auto consider = [&](rnj_tune_params c, bool host, float *ms_out = nullptr) -> int {
    float ms = 0.0f;
    const int rc = host ? time_host(ctx, b, n, L, type, flags, model, c, reps, &ms)
                        : time_plain(ctx, b, n, L, type, flags, model, c, reps, &ms);
    if (rc != RNJ_OK) return rc;
    if (ms_out) *ms_out = ms;
    if (best.ms >= 1e29f || ms < best.ms * (1.0f - kTuneMargin)) {
      best = c;
      best.ms = ms;
    }
    return RNJ_OK;
  };
  int rc = RNJ_OK;
  // 1. Tensor cores: tile-order band, then the ring depth, then the
  //    two-kernel form (its ring depth and the transform's occupancy).
  if (tc_ok) {
    const bool fused_ok = L <= kMaxFusedColumns;
    rnj_tune_params base;
    memset(&base, 0, sizeof base);
    base.tc_epilogue = fused_ok ? 0 : 1;
    for (int band : {12, 4, 8, 24}) {
      if (band != 12 && band >= nt) continue;
      rnj_tune_params c = base;
      c.tile_band = band;
      if ((rc = consider(c, false)) != RNJ_OK) break;
    }
    const int band = best.tile_band;
    for (int st : {5, 4, 3}) {
      if (rc != RNJ_OK || !fused_ok) break;
      rnj_tune_params c = base;
      c.tile_band = band;
      c.tc_stages = st;
      rc = consider(c, false);
    }
    if (fused_ok && rc == RNJ_OK) {
      rnj_tune_params c = base;
      c.tile_band = band;
      c.tc_epilogue = 1;
      rc = consider(c, false);
    }
    if (best.tc_epilogue == 1) {
      for (int ctas : {3, 4}) {
        if (rc != RNJ_OK) break;
        rnj_tune_params c = best;
        c.transform_ctas = ctas;
        rc = consider(c, false);
      }
      const rnj_tune_params two = best;
      for (int st : {6, 5}) {
        if (rc != RNJ_OK) break;
        rnj_tune_params c = two;
        c.tc_stages = st;
        rc = consider(c, false);
      }
    }
  }
  // 2. Bit planes (every protein and -f bucket; DNA as the alternative):
  //    columns split over 1, 2, 4, ... CTAs per tile, then the ring depth.
  if (rc == RNJ_OK) {
    rnj_tune_params pbest;
    memset(&pbest, 0, sizeof pbest);
    pbest.ms = 1e30f;
    for (int ks : {1, 2, 4, 8, 16}) {
      if (ks > 1 && (!split_ok || ks > nk)) break;
      rnj_tune_params c;
      memset(&c, 0, sizeof c);
      c.dna_kernel = tc_ok ? 1 : 0;
      c.ksplit = ks;
      float ms = 0.0f;
      if ((rc = consider(c, false, &ms)) != RNJ_OK) break;
      if (ms < pbest.ms) {
        pbest = c;
        pbest.ms = ms;
      }
    }
    // One shallower ring than the default (the deepest): 3 stages of DNA
    // planes, 2 of the synthetic protein's 5-bit codes (the least each
    // layout's distance staging takes).
    if (rc == RNJ_OK && pbest.ms < 1e29f) {
      rnj_tune_params c = pbest;
      c.pop_stages = type == RNJ_DNA ? 3 : 2;
      rc = consider(c, false);
    }
  }
  // 3. The streamed host call's band height (tensor-core DNA and protein; the
  //    host buffers are page-locked like a caller's would be for this path).
  if (rc == RNJ_OK && tc_ok && best.dna_kernel == 0 && nt >= 8 && n <= 16384) {
    cudaError_t e = cudaMallocHost((void **)&b.h_chars, (size_t)n * L);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&b.h_out, (size_t)n * n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(b.h_chars, b.d_chars, (size_t)n * L, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      rc = cuda_error(e, "tuning host buffers");
    } else {
      const rnj_tune_params plain_best = best;
      rnj_tune_params host_best = plain_best;
      float host_ms = 1e30f;
      for (int band : {0, 4, 8, 16, 32}) {  // 0: the automatic height, the default
        if (band >= nt) continue;
        rnj_tune_params c = plain_best;
        c.stream_band = band;
        float ms = 0.0f;
        if ((rc = time_host(ctx, b, n, L, type, flags, model, c, reps, &ms)) != RNJ_OK) break;
        if (host_ms >= 1e29f || ms < host_ms * (1.0f - kTuneMargin)) {
          host_ms = ms;
          host_best = c;
        }
      }
      if (rc == RNJ_OK) {
        best = host_best;
        best.ms = plain_best.ms;  // the device time of pack + distances
      }
    }
  }
  if (rc != RNJ_OK) {
    restore();
    return rc;
  }
  rnj_tune_set(n, L, type, flags, &best);
  if (const char *p = cache_path()) {
    std::lock_guard<std::mutex> lk(g_mu);
    rc = save_locked(p);
    if (rc != RNJ_OK) return rc;
  }
  if (out) *out = best;
  return RNJ_OK;
}
