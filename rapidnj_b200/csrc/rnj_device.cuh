// rnj_device.cuh -- device helpers shared by the sm_100a kernels: mbarrier and
// TMA wrappers (inline PTX), bounded waits, and the exact distance transforms.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rnj_logtab.h"

namespace rnj {

// ------------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// The same test, letting the thread sleep until the phase completes for at
// most hint_ns (the try_wait suspend-time hint) instead of the system's own
// limit: a waiting warp issues far fewer instructions, leaving the issue slots
// of its scheduler to the warps that work.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t *bar, uint32_t parity,
                                                   uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A wait on an mbarrier phase that gives up after limit_ns of wall time (or an
// iteration cap), so that a lost transfer turns into an error status instead of
// a hung GPU.  Pipeline waits take the limit the host chose (rnj_set_wait_limit,
// wait_limit_ns below); the drains that let a CTA's own copies land before it
// exits always allow the full default.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s
constexpr uint32_t kWaitIterCap = 1u << 26;

__device__ __forceinline__ uint64_t wait_limit_ns(uint32_t us) {
  return us ? (uint64_t)us * 1000ull : kWaitLimitNs;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < kWaitIterCap; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && global_timer_ns() - t0 > limit_ns) break;
  }
  return false;
}

// 3-D tiled TMA load (no multicast): box lands in shared memory with dim0
// fastest.  c0 is always 16-byte aligned as TMA requires: for bit planes it is
// a sequence index (4-byte elements) that is a multiple of the 128-row tile, for
// the K-blocked tensor-core features it is 0.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------------ exact transforms
//
// Each transform restates the reference's float/double arithmetic operation by
// operation with explicitly rounded intrinsics, so that no multiply-add is
// contracted (the reference is compiled for SSE2 without FMA).  The logarithm
// is CUDA's double log(), except on the K2P fast path (ln_table, below), whose
// result is only used where a rounding check with a proven error bound decides.

// ln(x) for x in [2^-1022, 1] by Tang's table-driven method (ACM TOMS 16(4),
// 1990): x = 2^k m, m in [1, 2); F = 1 + j/128 with j the top 7 bits of m's
// fraction, so f = m - F is exact and in [0, 2^-7); r = f * (1/F) (table);
// ln x = k ln 2 + ln F + ln(1 + r), the last by its series to r^6.  Error:
//   series remainder        |r|^7 / 7 < 2^-51.8
//   r against f / F         <= 2^-52 |f / F| < 2^-59   (so is ln(1 + r) against ln(1 + f/F))
//   series arithmetic       < 2^-58 (terms below 2^-7, each fma rounded once)
//   ln F from the table     <= 2^-54 (nearest double, ln F < 1)
//   k ln 2                  k * kLn2Hi exact (42-bit kLn2Hi, |k| < 2^11), k * kLn2Lo
//                           and the table sum rounded: < 2^-52
//   final fma               <= 2^-53 |ln x|
// so |ln_table(x) - ln x| < 2^-50.5 + 2^-53 |ln x|.
__device__ __forceinline__ double ln_table(double x) {
  const long long bits = __double_as_longlong(x);
  const int k = (int)((bits >> 52) & 0x7FF) - 1023;
  const int j = (int)((bits >> 45) & 127);
  const double m = __longlong_as_double((bits & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
  const double F = __longlong_as_double(0x3FF0000000000000LL | ((long long)j << 45));
  const double lnF = __ldg(&c_log_tab[j][0]);
  const double inv = __ldg(&c_log_tab[j][1]);
  const double r = __dmul_rn(__dsub_rn(m, F), inv);
  double p = -1.0 / 6.0;
  p = __fma_rn(p, r, 0.2);
  p = __fma_rn(p, r, -0.25);
  p = __fma_rn(p, r, 1.0 / 3.0);
  p = __fma_rn(p, r, -0.5);
  p = __fma_rn(p, r, 1.0);
  p = __dmul_rn(p, r);
  const double dk = (double)k;
  return __fma_rn(dk, kLn2Hi, __dadd_rn(__fma_rn(dk, kLn2Lo, lnF), p));
}

// -ln(x) / 4, the K2P fast path's logarithm, with the table read from `tab`
// (a copy of c_log_tab in shared memory, each entry scaled by -1/4: a warp's
// 32 random entries are one shared-memory request instead of up to 16 L1
// lines) and k turned into a double by the 2^52 bias (an integer add and a
// double subtraction, both exact, instead of a conversion).  The arithmetic
// is ln_table's with every operand scaled by a power of two: r' = -r / 4 (the
// table's -1/(4F)), Horner coefficients c_k (-4)^k, so the k-th Horner value
// is (-4)^k times ln_table's and the product with r' is -1/4 of its; ln F and
// ln 2 scaled by -1/4.  Rounding to nearest commutes with a power-of-two
// scale (no operand comes near overflow or underflow), so the result is
// exactly -ln_table(x) / 4, with ln_table's error bound divided by 4.
constexpr double kNegQuarterLn2Hi = -0.25 * kLn2Hi, kNegQuarterLn2Lo = -0.25 * kLn2Lo;
__device__ __forceinline__ double neg_quarter_ln_table_k(double x, const double2 *tabq) {
  const long long bits = __double_as_longlong(x);
  const int ebits = (int)((bits >> 52) & 0x7FF);  // k + 1023
  const int j = (int)((bits >> 45) & 127);
  const double m = __longlong_as_double((bits & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
  const double F = __longlong_as_double(0x3FF0000000000000LL | ((long long)j << 45));
  const double2 e = tabq[j];  // {-ln F / 4, -1 / (4 F)}
  const double r = __dmul_rn(__dsub_rn(m, F), e.y);
  double p = (-1.0 / 6.0) * -1024.0;
  p = __fma_rn(p, r, 0.2 * 256.0);
  p = __fma_rn(p, r, -0.25 * -64.0);
  p = __fma_rn(p, r, (1.0 / 3.0) * 16.0);
  p = __fma_rn(p, r, -0.5 * -4.0);
  p = __fma_rn(p, r, 1.0);
  p = __dmul_rn(p, r);
  // 2^52 + ebits, exactly, minus 2^52 + 1023: the double k (|k| < 2^11).
  const double dk =
      __dsub_rn(__hiloint2double(0x43300000, ebits), 4503599627370496.0 + 1023.0);
  return __fma_rn(dk, kNegQuarterLn2Hi, __dadd_rn(__fma_rn(dk, kNegQuarterLn2Lo, e.x), p));
}

// The double of an integer 0 <= v < 2^32: 2^52 + v has v in its low mantissa
// bits, so the subtraction of 2^52 is exact.
__device__ __forceinline__ double u32_to_double(uint32_t v) {
  return __dsub_rn(__hiloint2double(0x43300000, (int)v), 4503599627370496.0);
}

// y rounded to 24 significant bits, to nearest, in double arithmetic: Veltkamp
// splitting with C = 2^29 + 1 (Dekker 1971): g = fl(C y), h = fl(g - fl(g - y))
// keeps the 53 - 29 = 24 leading bits of y rounded to nearest (Boldo 2006; a
// tie may round either way).  For 2^-126 <= |y| < 2^127 that is (double)(float)y
// unless y lies exactly halfway between two floats.
__device__ __forceinline__ double round_to_float_bits(double y) {
  const double g = __dmul_rn(y, 536870913.0);
  return __dsub_rn(g, __dsub_rn(g, y));
}

// Valid-site count as the fast protein estimator reports it for L % 128 == 0
// (bitDistanceProtein.cpp:15-16,59): padded length minus the gaps counted over
// one extra 128-byte block, stored in an unsigned long long.
__device__ __forceinline__ unsigned long long protein_fast_valid(unsigned long long valid, int L) {
  const long long padded = ((long long)L + 127) & ~127LL;
  const long long span = 128LL * (((long long)L / 16 + 8) / 8);
  const long long gaps_total = ((long long)L - (long long)valid) + (span - (long long)L);
  return (unsigned long long)(padded - gaps_total);
}

// The float nearest to -c ln(arg), arg in (0, 1], c in {0.75, 0.95, 1}, when
// the table logarithm decides it; else NaN.  The reference evaluates
// (float)(-c log(arg)) in double (log within 1 ulp, one rounded product):
// |d_ref - D| <= 1.5 * 2^-52 D for D = -c ln(arg) >= 0.  Here dd = fl(-c
// ln_table(arg)) with |dd - D| < 2^-50.5 + 2^-52 D (ln_table's bound, c <= 1),
// so |dd - d_ref| < eps = 2^-49 (1 + 4 dd) and, as on the K2P fast path, if
// dd - eps and dd + eps round to the same float so does d_ref.
__device__ __forceinline__ float neg_log_checked(double c, double arg) {
  const double dd = __dmul_rn(-c, ln_table(arg));
  const double eps = __dmul_rn(0x1p-49, __dadd_rn(1.0, __dmul_rn(4.0, dd)));
  const float lo = __double2float_rn(__dsub_rn(dd, eps));
  const float hi = __double2float_rn(__dadd_rn(dd, eps));
  return __float_as_int(lo) == __float_as_int(hi) ? lo : __int_as_float(0x7fc00000);
}

// neg_log_checked with the table read from `tabq`, the shared-memory copy scaled
// by -1/4 (neg_quarter_ln_table_k): ln_table(arg) is exactly -4 times that value
// (a power-of-two scale), so dd, the check and the result are neg_log_checked's
// bit for bit.
__device__ __forceinline__ float neg_log_checked_tab(double c, double arg, const double2 *tabq) {
  const double dd = __dmul_rn(c, __dmul_rn(4.0, neg_quarter_ln_table_k(arg, tabq)));
  const double eps = __dmul_rn(0x1p-49, __dadd_rn(1.0, __dmul_rn(4.0, dd)));
  const float lo = __double2float_rn(__dsub_rn(dd, eps));
  const float hi = __double2float_rn(__dadd_rn(dd, eps));
  return __float_as_int(lo) == __float_as_int(hi) ? lo : __int_as_float(0x7fc00000);
}

// The float quotient fl32(num / den) of integers 0 <= num <= den < 2^24, the
// value of both (float)num / (float)den and (float)((double)num / (double)den)
// in the reference.  Given rn within 2^-51 (relative) of 1 / den (recip_nr),
// d = fl64(num * rn) is within 2^-50 of num / den.  A float rounding boundary
// m (the midpoint of two floats) has 25 significant bits, m = (2k + 1) 2^-s
// with 2k + 1 >= 2^24; num / den = m would need 2k + 1 to divide num < 2^24, so
// num / den != m and |num / den - m| >= 1 / (den 2^s), at least 2^-49 relative
// to m.  d therefore lies on the same side of every boundary as num / den and
// rounds to the same float.  rn == 0 divides instead.
__device__ __forceinline__ float ratio_f32(unsigned long long num, unsigned long long den,
                                           double rn) {
  if (rn != 0.0) return __double2float_rn(__dmul_rn((double)num, rn));
  return __fdiv_rn(__ull2float_rn(num), __ull2float_rn(den));
}

// The PTX fast reciprocal of a float (rcp.approx: within a couple of ulps of
// 1 / x; one instruction, where a correctly rounded reciprocal takes several).
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// 1 / n for an integer 1 <= n < 2^24, within 2^-52.9 (relative), by Newton-
// Raphson iteration for the reciprocal, r <- r + r (1 - n r), from the fast
// float reciprocal of n.  With r = (1 / n)(1 - e), one step gives
// (1 / n)(1 - e^2) before rounding:
//   r0 = rcp_approx(n)       |e0| <= 2^-21 (a float within 4 ulps of 1 / n)
//   t0 = fma(-n, r0, 1) = e0 exactly (n r0 has at most 48 significant bits and
//        lies within 2^-21 of 1, so the product and the difference are exact)
//   r1 = fma(r0, t0, r0)     |e1| <= 2^-42 + 2^-53
//   t1 = fma(-n, r1, 1)      = e1 (1 + 2^-53 at most)
//   r2 = fma(r1, t1, r1)     |e2| <= e1^2 + 2^-53 + ... < 2^-52.9
// which is well inside the 2^-51 that ratio_f32 needs.  n = 0 gives a NaN
// (callers treat valid == 0 before any quotient).
__device__ __forceinline__ double recip_nr(uint32_t n) {
  const double dn = (double)n;
  const double r0 = (double)rcp_approx((float)n);
  const double r1 = __fma_rn(r0, __fma_rn(-dn, r0, 1.0), r0);
  return __fma_rn(r1, __fma_rn(-dn, r1, 1.0), r1);
}

// The undecided cases of the table logarithm (about one pair in 10^6): the
// reference's own formulas with CUDA's log, kept out of line so that the
// registers they need do not weigh on the common path.
static __device__ __noinline__ float neg_log_slow(double c, double arg) {
  return __double2float_rn(__dmul_rn(-c, log(arg)));
}
static __device__ __noinline__ float k2p_two_logs(double a, double b) {
  return __double2float_rn(__dsub_rn(__dmul_rn(-0.5, log(a)), __dmul_rn(0.25, log(b))));
}

// JCdistance.cpp:171-183.  b = (alpha - 1) / alpha in double, alpha 4 or 20.
// rn: an approximate reciprocal of valid (recip_nr; see ratio_f32), or 0.
__device__ __forceinline__ float jc_of_p(float distance, double b);

__device__ __forceinline__ float jc_distance(unsigned long long total,
                                             unsigned long long valid, double b,
                                             double rn = 0.0) {
  float distance;
  if (valid == 0) distance = 0.0f;
  else if (rn != 0.0) distance = ratio_f32(total, valid, rn);
  else distance = __fdiv_rn(__ll2float_rn((long long)total), __ull2float_rn(valid));
  return jc_of_p(distance, b);
}

// JCdistance.cpp:177-183 from the float p (0 when valid is 0).
__device__ __forceinline__ float jc_of_q(double q, double b, const double2 *tabq = nullptr);

__device__ __forceinline__ float jc_of_p(float distance, double b) {
  return jc_of_q(__ddiv_rn((double)distance, b), b);
}

// (double)p / b for a float p in [0, 1] from y = 1 / b correctly rounded
// (b = 3/4 or 19/20, JCdistance.cpp:171-177): q0 = fl(p y) is within one ulp
// of p / b, the residual p - b q0 is then exact as one fused multiply-add, and
// fl(q0 + r y), one more, is the correctly rounded quotient (Markstein's
// theorem for a correctly rounded reciprocal) -- checked on the device for
// every float p in [0, 1] and both b (rnj_check_quotient16).
__device__ __forceinline__ double div_by_b(double p, double b, double inv_b) {
  const double q0 = __dmul_rn(p, inv_b);
  return __fma_rn(__fma_rn(-q0, b, p), inv_b, q0);
}

// JCdistance.cpp:177-183 from q = (double)p / b.  tabq: the logarithm table in
// shared memory (neg_log_checked_tab), or null for the global one.
__device__ __forceinline__ float jc_of_q(double q, double b, const double2 *tabq) {
  if (q >= 1.0) return -1.0f;
  const double arg = __dsub_rn(1.0, q);
  if (arg == 1.0) return __double2float_rn(__dmul_rn(-b, 0.0));  // -0.0, as the reference
  const float fast = tabq ? neg_log_checked_tab(b, arg, tabq) : neg_log_checked(b, arg);
  if (fast == fast) return fast;
  return neg_log_slow(b, arg);
}

// KimuraDistance.cpp:339-349.  rn: an approximate reciprocal of valid
// (recip_nr; see ratio_f32), or 0.
__device__ __forceinline__ float k2p_distance(unsigned long long ts_count,
                                              unsigned long long tv_count,
                                              unsigned long long valid, double rn = 0.0) {
  if (valid == 0) return -1.0f;
  // ts = (float)((double)P / (double)n): for integers P <= n < 2^24 this equals
  // the float quotient rounded once.  A float midpoint m has at most 25
  // significant bits, so a quotient P / n that is not m lies at least
  // 1 / (n * 2^25) > 2^-49 (relative) away from it, while the double rounding
  // moves it by at most 2^-53: both roundings land on the same float.
  float ts, tv;
  if (rn != 0.0) {
    ts = ratio_f32(ts_count, valid, rn);
    tv = ratio_f32(tv_count, valid, rn);
  } else if (valid < (1u << 24)) {
    const float fn = (float)valid;
    ts = __fdiv_rn((float)ts_count, fn);
    tv = __fdiv_rn((float)tv_count, fn);
  } else {
    const double dn = (double)valid;
    ts = __double2float_rn(__ddiv_rn((double)ts_count, dn));
    tv = __double2float_rn(__ddiv_rn((double)tv_count, dn));
  }
  const double a = __dsub_rn(__dsub_rn(1.0, __dmul_rn(2.0, (double)ts)), (double)tv);
  const double b = __dsub_rn(1.0, __dmul_rn(2.0, (double)tv));
  const float temp1 = __double2float_rn(a);
  const float temp2 = __double2float_rn(b);
  if (temp1 <= 0.0f || temp2 <= 0.0f) return -1.0f;
  // Identical pairs: -0.5 log(1) - 0.25 log(1) = -0.0 - 0.0 = -0.0.
  if ((ts_count | tv_count) == 0) return -0.0f;
  // Fast path, one logarithm: D = -0.5 log a - 0.25 log b = -0.25 log(a^2 b),
  // a, b in (0, 1], so D >= 0 and 0.5|log a| + 0.25|log b| = D.
  //   reference  d_ref = (-0.5 log a) - (0.25 log b), each log within 1 ulp,
  //              one rounded subtraction:   |d_ref - D| <= 1.5 * 2^-52 * D
  //   this path  dd = -0.25 ln_table(fl(fl(a a) b)): the product is within
  //              2^-52 (relative) of a^2 b, so its log within 2^-52 of log(a^2 b);
  //              ln_table adds < 2^-50.5 + 2^-53 |log x| (its comment), and the
  //              scaling by -0.25 is exact:
  //                                  |dd - D| < 2^-52.5 + 2^-54 + 2^-53 (D + ...)
  // so |dd - d_ref| < 2^-51.9 + 2^-50.4 D < eps = 2^-49 (1 + 4 dd).  (a^2 b
  // stays far from the double underflow range: a, b >= 2^-46 when positive.)
  // If dd - eps and dd + eps round to the same float, so does every value
  // between them (rounding is monotone), d_ref included: the float result is
  // the reference's.  Otherwise -- about one pair in 10^7 -- the reference's
  // own two-logarithm formula decides (with CUDA's log).
  const double x = __dmul_rn(__dmul_rn(a, a), b);
  const double dd = __dmul_rn(-0.25, ln_table(x));
  const double eps = __dmul_rn(0x1p-49, __dadd_rn(1.0, __dmul_rn(4.0, dd)));
  const float lo = __double2float_rn(__dsub_rn(dd, eps));
  const float hi = __double2float_rn(__dadd_rn(dd, eps));
  if (__float_as_int(lo) == __float_as_int(hi)) return lo;
  return k2p_two_logs(a, b);
}

// The K2P distance of k2p_distance for 1 <= n < 2^24 (the fused kernel's
// counts), without branches, so that the pairs of a group interleave: the
// saturated (-1) and identical (-0.0) cases and the one-logarithm value are
// computed for every pair and selected.  *slow is set when the rounding check
// cannot decide (about one pair in 10^6-10^7); the caller then evaluates
// k2p_distance for that pair.  n == 0 gives -1 like k2p_distance.
__device__ __forceinline__ float k2p_decide(uint32_t P, uint32_t Q, uint32_t n, bool &slow) {
  const double rn = recip_nr(n == 0 ? 1u : n);
  const float ts = __double2float_rn(__dmul_rn((double)P, rn));
  const float tv = __double2float_rn(__dmul_rn((double)Q, rn));
  const double a = __dsub_rn(__dsub_rn(1.0, __dmul_rn(2.0, (double)ts)), (double)tv);
  const double b = __dsub_rn(1.0, __dmul_rn(2.0, (double)tv));
  const bool sat = (n == 0) | (__double2float_rn(a) <= 0.0f) | (__double2float_rn(b) <= 0.0f);
  const bool same = (P | Q) == 0;
  // a, b in (0, 1] unless saturated: ln_table's argument stays positive.
  const double x = sat ? 1.0 : __dmul_rn(__dmul_rn(a, a), b);
  const double dd = __dmul_rn(-0.25, ln_table(x));
  const double eps = __dmul_rn(0x1p-49, __dadd_rn(1.0, __dmul_rn(4.0, dd)));
  const float lo = __double2float_rn(__dsub_rn(dd, eps));
  const float hi = __double2float_rn(__dadd_rn(dd, eps));
  slow = !sat && !same && (__float_as_int(lo) != __float_as_int(hi));
  return sat ? -1.0f : (same ? -0.0f : lo);
}

// 1 / d for an integer 1 <= d < 2^16 given as a float: one Newton-Raphson step
// r0 + r0 (1 - d r0) from the fast reciprocal (|d r0 - 1| <= 2^-21).  1 - d r0
// is exact as a fused multiply-add (d r0 has at most 40 significant bits and
// lies within 2^-21 of 1; the difference is a multiple of 2^-39), so the
// result has |d y - 1| <= 2^-42 + 2^-24 < 2^-23.9.
__device__ __forceinline__ float recip16(float d) {
  const float r0 = rcp_approx(d);
  return __fmaf_rn(r0, __fmaf_rn(-d, r0, 1.0f), r0);
}

// fl32(num / d) for integers 0 <= num <= d < 2^16 (d as a float, y = recip16(d))
// in float arithmetic.  q0 = fl(num y) is within 2^-22.9 (relative) of num / d;
// the residual num - d q0 is a multiple of ulp(q0) with fewer than 2^17 of them,
// so one fused multiply-add gives it exactly; q = fl(q0 + r y), one more fused
// multiply-add, rounds num / d + (num / d - q0)(d y - 1), which is within
// 2^-22 ulp of num / d.  num / d lies at least 2^-18 ulp from every float
// midpoint (a midpoint is M 2^-e with M odd of 25 bits, and num / d = M 2^-e
// would need M | num < 2^16), so q is the correctly rounded quotient: the
// reference's (float)((double)num / (double)d) and (float)num / (float)d (the
// double quotient is no midpoint either, so its float rounding agrees).
__device__ __forceinline__ float quotient16(uint32_t num, float d, float y) {
  const float fnum = __fsub_rn(__uint_as_float(0x4B000000u | num), 8388608.0f);
  const float q0 = __fmul_rn(fnum, y);
  return __fmaf_rn(__fmaf_rn(-q0, d, fnum), y, q0);
}

// k2p_decide for 16-bit counts (the fused kernel): P, Q, n < 2^16 given as
// integers packed by the epilogue.  The same decision and result, computed
// with fewer conversions:
//   * the floats of P, Q and n by the 2^23 bias; ts, tv = quotient16, the
//     reference's float quotients, converted to double exactly;
//   * temp1 = (float)a <= 0 exactly when a <= 0: a and b are sums of doubles
//     of floats in [0, 1] with at most 24 significant bits and exponents above
//     -17, so a nonzero a or b exceeds 2^-70 in magnitude and its float is not 0;
//   * neg_quarter_ln_table_k for -ln(x) / 4 (tab: the table in shared memory,
//     scaled by -1/4).
__device__ __forceinline__ float k2p_decide16(uint32_t P, uint32_t Q, uint32_t n, bool &slow,
                                              const double2 *tab) {
  const uint32_t nn = n == 0 ? 1u : n;
  const float fn = __fsub_rn(__uint_as_float(0x4B000000u | nn), 8388608.0f);
  const float y = recip16(fn);
  const double ts = (double)quotient16(P, fn, y);
  const double tv = (double)quotient16(Q, fn, y);
  // fl(1 - 2 ts) as one fused multiply-add: 2 ts is exact, so both forms are
  // the exact 1 - 2 ts rounded once (the reference's double arithmetic).
  const double a = __dsub_rn(__fma_rn(-2.0, ts, 1.0), tv);
  const double b = __fma_rn(-2.0, tv, 1.0);
  const bool sat = (n == 0) | (a <= 0.0) | (b <= 0.0);
  const bool same = (P | Q) == 0;
  const double x = sat ? 1.0 : __dmul_rn(__dmul_rn(a, a), b);
  const double dd = neg_quarter_ln_table_k(x, tab);  // -ln(x) / 4, exactly as scaled
  // eps = 2^-49 (1 + 4 dd), one fused multiply-add (rounded once, as close to
  // the bound as the three-operation form)
  const double eps = __fma_rn(0x1p-47, dd, 0x1p-49);
  const float lo = __double2float_rn(__dsub_rn(dd, eps));
  const float hi = __double2float_rn(__dadd_rn(dd, eps));
  slow = !sat && !same && (__float_as_int(lo) != __float_as_int(hi));
  return sat ? -1.0f : (same ? -0.0f : lo);
}

// KimuraDistance.cpp:322-338 with the Dayhoff table of KimuraDistance.cpp:30-49.
// rn: an approximate reciprocal of valid (recip_nr; see ratio_f32), or 0.
__device__ __forceinline__ float kimura_protein_of_p(float distance, const float *pam_dist,
                                                     const double2 *tabq = nullptr);

__device__ __forceinline__ float kimura_protein_distance(unsigned long long mism,
                                                         unsigned long long valid,
                                                         const float *pam_dist, double rn = 0.0) {
  float distance = -1.0f;
  if (valid != 0)
    distance = rn != 0.0 ? ratio_f32(mism, valid, rn)
                         : __fdiv_rn(__ll2float_rn((long long)mism), __ull2float_rn(valid));
  return kimura_protein_of_p(distance, pam_dist);
}

// KimuraDistance.cpp:325-338 from the float p (-1 when valid is 0).  pam_dist:
// the Dayhoff table's distances, (float)(PAM / 100.0) per entry; tabq: as jc_of_q.
__device__ __forceinline__ float kimura_protein_of_p(float distance, const float *pam_dist,
                                                     const double2 *tabq) {
  const double dd = (double)distance;
  if (dd < 0.75) {
    if (dd > 0.0) {
      const double sq = (double)__fmul_rn(distance, distance);
      const double arg = __dsub_rn(__dsub_rn(1.0, dd), __dmul_rn(sq, 0.20));
      const float fast = tabq ? neg_log_checked_tab(1.0, arg, tabq) : neg_log_checked(1.0, arg);
      distance = fast == fast ? fast : neg_log_slow(1.0, arg);
    }
  } else {
    if (dd > 0.930) {
      distance = 10.0f;
    } else {
      const int idx = (int)__dsub_rn(__dmul_rn(dd, 1000.0), 750.0);
      distance = __ldg(pam_dist + idx);
    }
  }
  return distance;
}

}  // namespace rnj
