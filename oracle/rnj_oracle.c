/*
 * rnj_oracle.c -- CPU restatement of rapidNJ's distance-estimation path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py load this library, and only as the
 * checker.  The product path (librnjgpu.so) never links or calls it.
 *
 * Parity status: pinned.  tests/test_oracle_golden.py checks every function
 * here against golden vectors produced by the reference itself (its own
 * estimator objects and its own JCdistance / KimuraDistance drivers, built
 * from source by oracle/Makefile) on the reference's test_data fixtures and
 * on crafted edge alignments.
 *
 * Restated reference behaviour (paths relative to the rapidNJ source tree):
 *   - DNA fast-path packing: src/distanceCalculation/dataloaderFasta.hpp:147-182
 *     (A=0, G=1, T=2, C=3 from src/stdinclude.h:25; only A/C/G/T in either case
 *     are valid, every other byte is a gap).
 *   - resolveChar: dataloaderFasta.hpp:184-199.
 *   - DNA fast counts: src/distanceCalculation/bitDistanceGap.cpp:134-203
 *     (tv = high bit of the code XOR, ts = low bit and not tv, both masked by
 *     the AND of the gap filters; valid = popcount of that AND).
 *   - Protein fast counts: src/distanceCalculation/bitDistanceProtein.cpp:31-84
 *     (byte compare of resolved bytes, gap = '-' in either, valid =
 *     paddedSeqLength - gaps with paddedSeqLength = (L+127)&~127).
 *   - Naive counts (-f): src/distanceCalculation/simpleDistanceCalculator.cpp:40-98.
 *   - JC transform: src/distanceCalculation/JCdistance.cpp:171-187.
 *   - Kimura transforms: src/distanceCalculation/KimuraDistance.cpp:319-353.
 *   - Post-process: KimuraDistance.cpp:366-395, JCdistance.cpp:201-230.
 *
 * Compiled with -ffp-contract=off so that no multiply-add is fused (the
 * reference is built for SSE2 without FMA), against glibc's log().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rnj_oracle.h"

/* Dayhoff PAM distances (x100) for p = 0.750 .. 0.930 in steps of 0.001, as used
 * by the protein Kimura estimate (KimuraDistance.cpp:30-49).  The values are the
 * published table; parity requires them value for value. */
static const int kDayhoffPam[181] = {
    195, 196, 197, 198, 199, 200, 200, 201, 202, 203, 204, 205, 206, 207, 208,
    209, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222,
    223, 224, 226, 227, 228, 229, 230, 231, 232, 233, 234, 236, 237, 238, 239,
    240, 241, 243, 244, 245, 246, 248, 249, 250, 252, 253, 254, 255, 257, 258,
    260, 261, 262, 264, 265, 267, 268, 270, 271, 273, 274, 276, 277, 279, 281,
    282, 284, 285, 287, 289, 291, 292, 294, 296, 298, 299, 301, 303, 305, 307,
    309, 311, 313, 315, 317, 319, 321, 323, 325, 328, 330, 332, 335, 337, 339,
    342, 344, 347, 349, 352, 354, 357, 360, 362, 365, 368, 371, 374, 377, 380,
    383, 386, 389, 393, 396, 399, 403, 407, 410, 414, 418, 422, 426, 430, 434,
    438, 442, 447, 451, 456, 461, 466, 471, 476, 482, 487, 493, 498, 504, 511,
    517, 524, 531, 538, 545, 553, 560, 569, 577, 586, 595, 605, 615, 626, 637,
    649, 661, 675, 688, 703, 719, 736, 754, 775, 796, 819, 845, 874, 907, 945,
    988};

int orc_pam_value(int idx) { return (idx >= 0 && idx < 181) ? kDayhoffPam[idx] : -1; }

/* dataloaderFasta.hpp:54-76: first sequence decides; any byte >= 65 outside
 * ACGTUN/acgtun makes the alignment protein. */
int orc_detect_type(const char *seq0, int L) {
  for (int i = 0; i < L; i++) {
    signed char c = (signed char)seq0[i];
    if (!(c < 65 || c == 'A' || c == 'a' || c == 'C' || c == 'c' || c == 'G' ||
          c == 'g' || c == 'T' || c == 't' || c == 'U' || c == 'u' || c == 'N' ||
          c == 'n'))
      return ORC_PROTEIN;
  }
  return ORC_DNA;
}

/* dataloaderFasta.hpp:184-199 */
char orc_resolve_char(char c, int type) {
  if (type == ORC_DNA) {
    if (!(c == 'a' || c == 'A' || c == 'c' || c == 'C' || c == 'g' || c == 'G' ||
          c == 't' || c == 'T' || c == 'u' || c == 'U'))
      return '-';
    return c;
  }
  if (c == '-' || c == '.' || c == 'X' || c == 'x' || c == 'z' || c == 'Z' ||
      c == 'b' || c == 'B' || c == 'J' || c == 'j' || c == '?')
    return '-';
  return c;
}

/* dataloaderFasta.hpp:155-180: 2-bit code of the fast path, -1 for a gap. */
static int dna_fast_code(char c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'G': case 'g': return 1;
    case 'T': case 't': return 2;
    case 'C': case 'c': return 3;
    default: return -1;
  }
}

/* bitDistanceGap.cpp:134-203, one site at a time. */
static void count_dna_fast(const char *a, const char *b, int L, uint64_t out[3]) {
  uint64_t ts = 0, tv = 0, valid = 0;
  for (int k = 0; k < L; k++) {
    int ca = dna_fast_code(a[k]), cb = dna_fast_code(b[k]);
    if (ca < 0 || cb < 0) continue;
    valid++;
    int x = ca ^ cb;
    if (x & 2) tv++;
    else if (x & 1) ts++;
  }
  out[0] = ts; out[1] = tv; out[2] = valid;
}

/* simpleDistanceCalculator.cpp:58-98 on resolved characters.  Note the
 * asymmetry: only an upper-case A/C/G/T in the first sequence classifies a
 * difference; any other differing valid pair adds to the length only. */
static void count_dna_naive(const char *a, const char *b, int L, uint64_t out[3]) {
  uint64_t ts = 0, tv = 0, len = 0;
  for (int k = 0; k < L; k++) {
    char x = orc_resolve_char(a[k], ORC_DNA), y = orc_resolve_char(b[k], ORC_DNA);
    if (x == '-' || y == '-') continue;
    if (x != y) {
      if (x == 'A') { if (y == 'G') ts++; else tv++; }
      else if (x == 'C') { if (y == 'T') ts++; else tv++; }
      else if (x == 'G') { if (y == 'A') ts++; else tv++; }
      else if (x == 'T') { if (y == 'C') ts++; else tv++; }
    }
    len++;
  }
  out[0] = ts; out[1] = tv; out[2] = len;
}

/* bitDistanceProtein.cpp:73-84 (fast) and simpleDistanceCalculator.cpp:40-55
 * (naive) agree on the mismatch count; both skip sites where either resolved
 * byte is a gap.  The valid count returned here is the correct one,
 * L - (sites with a gap); orc_protein_fast_valid() restates the fast path's
 * arithmetic on it. */
static void count_protein(const char *a, const char *b, int L, uint64_t out[3]) {
  uint64_t mism = 0, valid = 0;
  for (int k = 0; k < L; k++) {
    char x = orc_resolve_char(a[k], ORC_PROTEIN), y = orc_resolve_char(b[k], ORC_PROTEIN);
    if (x == '-' || y == '-' || x == '.' || y == '.') continue;
    valid++;
    if (x != y) mism++;
  }
  out[0] = mism; out[1] = 0; out[2] = valid;
}

/* bitDistanceProtein.cpp:15-16,59.  The fast path counts gaps over
 * 128*floor((L/16+8)/8) byte positions (the alignment plus '-' padding) and
 * subtracts them from (L+127)&~127.  For L % 128 != 0 both spans are equal and
 * the result is the true valid count; for L % 128 == 0 the span exceeds the
 * padded length by 128 and the long difference is stored in an unsigned long
 * long (it wraps when negative). */
uint64_t orc_protein_fast_valid(uint64_t valid, int L) {
  long padded = ((long)L + 127) & ~127L;
  long span = 128L * (((long)L / 16 + 8) / 8);
  long gaps_total = ((long)L - (long)valid) + (span - (long)L);
  return (unsigned long long)(padded - gaps_total);
}

void orc_pair_counts(const char *a, const char *b, int L, int type, int naive,
                     uint64_t out[3]) {
  if (type == ORC_PROTEIN) count_protein(a, b, L, out);
  else if (naive) count_dna_naive(a, b, L, out);
  else count_dna_fast(a, b, L, out);
}

void orc_counts(const char *seqs, int n, int L, int type, int naive, int full,
                uint32_t *out) {
  orc_counts_rows(seqs, n, L, type, naive, full, 0, n, out);
}

/* Rows [row0, row1) of orc_counts (several host threads can each take a range). */
void orc_counts_rows(const char *seqs, int n, int L, int type, int naive, int full, int row0,
                     int row1, uint32_t *out) {
  for (int i = row0; i < row1; i++) {
    for (int j = full ? 0 : i + 1; j < n; j++) {
      uint64_t c[3];
      orc_pair_counts(seqs + (size_t)i * L, seqs + (size_t)j * L, L, type, naive, c);
      uint32_t *o = out + ((size_t)i * n + j) * 3;
      o[0] = (uint32_t)c[0]; o[1] = (uint32_t)c[1]; o[2] = (uint32_t)c[2];
    }
  }
}

/* JCdistance.cpp:171-183 */
float orc_jc(uint64_t c0, uint64_t c1, uint64_t valid, int type) {
  double alpha = (type == ORC_PROTEIN) ? 20.0 : 4.0;
  long total = (long)(c0 + c1);
  float distance;
  if (valid == 0) distance = 0;
  else distance = (float)total / (float)valid;
  if (distance / ((alpha - 1) / alpha) >= 1.0) return -1.0f;
  return (float)(-((alpha - 1) / alpha) * log(1.0 - distance / ((alpha - 1) / alpha)));
}

/* KimuraDistance.cpp:339-349 */
float orc_k2p(uint64_t ts_count, uint64_t tv_count, uint64_t valid) {
  float distance = -1.0f;
  if (valid != 0) {
    float ts = (float)((double)ts_count / (double)valid);
    float tv = (float)((double)tv_count / (double)valid);
    float temp1 = (float)(1.0 - 2.0 * ts - tv);
    float temp2 = (float)(1.0 - 2.0 * tv);
    if (!(temp1 <= 0 || temp2 <= 0))
      distance = (float)(-0.5 * log(1.0 - 2.0 * ts - tv) - 0.25 * log(1.0 - 2.0 * tv));
  }
  return distance;
}

/* KimuraDistance.cpp:322-338 */
float orc_kimura_protein(uint64_t mism, uint64_t valid) {
  long total = (long)mism;
  float distance = -1.0f;
  if (valid != 0) distance = ((float)total / (float)valid);
  if (distance < 0.75) {
    if (distance > 0.0) distance = (float)(-log(1.0 - distance - (double)(distance * distance) * 0.20));
  } else {
    if (distance > 0.930) {
      distance = 10.0f;
    } else {
      int table_index = (int)((distance * 1000.0) - 750.0);
      distance = (float)(kDayhoffPam[table_index] / 100.0);
    }
  }
  return distance;
}

float orc_distance(const uint32_t c[3], int L, int type, int model, int naive,
                   int compat_wrap) {
  uint64_t valid = c[2];
  if (type == ORC_PROTEIN && !naive && compat_wrap) valid = orc_protein_fast_valid(valid, L);
  if (model == ORC_JC) return orc_jc(c[0], c[1], valid, type);
  if (type == ORC_PROTEIN) return orc_kimura_protein(c[0], valid);
  return orc_k2p(c[0], c[1], valid);
}

/* The same three transforms returning the double each reference expression
 * has before its (float) cast (the value of a saturated pair stays -1). */
double orc_jc_d(uint64_t c0, uint64_t c1, uint64_t valid, int type) {
  double alpha = (type == ORC_PROTEIN) ? 20.0 : 4.0;
  long total = (long)(c0 + c1);
  float distance;
  if (valid == 0) distance = 0;
  else distance = (float)total / (float)valid;
  if (distance / ((alpha - 1) / alpha) >= 1.0) return -1.0;
  return -((alpha - 1) / alpha) * log(1.0 - distance / ((alpha - 1) / alpha));
}

double orc_k2p_d(uint64_t ts_count, uint64_t tv_count, uint64_t valid) {
  if (valid == 0) return -1.0;
  float ts = (float)((double)ts_count / (double)valid);
  float tv = (float)((double)tv_count / (double)valid);
  float temp1 = (float)(1.0 - 2.0 * ts - tv);
  float temp2 = (float)(1.0 - 2.0 * tv);
  if (temp1 <= 0 || temp2 <= 0) return -1.0;
  return -0.5 * log(1.0 - 2.0 * ts - tv) - 0.25 * log(1.0 - 2.0 * tv);
}

double orc_kimura_protein_d(uint64_t mism, uint64_t valid) {
  long total = (long)mism;
  float distance = -1.0f;
  if (valid != 0) distance = ((float)total / (float)valid);
  if (distance < 0.75) {
    if (distance > 0.0) return -log(1.0 - distance - (double)(distance * distance) * 0.20);
    return distance;
  }
  if (distance > 0.930) return 10.0;
  int table_index = (int)((distance * 1000.0) - 750.0);
  return kDayhoffPam[table_index] / 100.0;
}

/* The double matrix: raw doubles for i < j (every i != j with full), maximum
 * over them, -1 -> 2 * max, mirror (unless full), diagonal 0. */
double orc_matrix_d(const uint32_t *counts, int n, int L, int type, int model, int naive,
                    int compat_wrap, int full, double *out) {
  double maxd = 0.0;
  for (int i = 0; i < n; i++) {
    for (int j = full ? 0 : i + 1; j < n; j++) {
      if (i == j) continue;
      const uint32_t *c = counts + ((size_t)i * n + j) * 3;
      uint64_t valid = c[2];
      if (type == ORC_PROTEIN && !naive && compat_wrap) valid = orc_protein_fast_valid(valid, L);
      double d = model == ORC_JC ? orc_jc_d(c[0], c[1], valid, type)
                                 : (type == ORC_PROTEIN ? orc_kimura_protein_d(c[0], valid)
                                                        : orc_k2p_d(c[0], c[1], valid));
      if (d > maxd) maxd = d;
      out[(size_t)i * n + j] = d;
    }
  }
  for (int i = 0; i < n; i++) {
    double *row = out + (size_t)i * n;
    for (int j = 0; j < n; j++) {
      if (!full && j < i) row[j] = out[(size_t)j * n + i];
      if (i == j) row[j] = 0.0;
      if (row[j] == -1.0) row[j] = maxd * 2;
    }
  }
  return maxd;
}

/* Raw (pre post-process) distances for i<j plus the running maximum, then the
 * post-process of KimuraDistance.cpp:366-395 / JCdistance.cpp:201-230:
 * mirror, zero diagonal, -1 -> 2*max. */
float orc_matrix(const uint32_t *counts, int n, int L, int type, int model,
                 int naive, int compat_wrap, float *out) {
  float maxd = 0.0f;
  for (int i = 0; i < n; i++) {
    for (int j = i + 1; j < n; j++) {
      float d = orc_distance(counts + ((size_t)i * n + j) * 3, L, type, model, naive,
                             compat_wrap);
      if (d > maxd) maxd = d;
      out[(size_t)i * n + j] = d;
    }
  }
  for (int i = 0; i < n; i++) {
    float *row = out + (size_t)i * n;
    for (int j = 0; j < n; j++) {
      if (j < i) row[j] = out[(size_t)j * n + i];
      if (i == j) row[j] = 0.0f;
      if (row[j] == -1) row[j] = maxd * 2;
    }
  }
  return maxd;
}

/* Full-row variant (the disk-matrix mode, KimuraDistance.cpp:308-354 with
 * dm != NULL): every (i, j) is computed in (row, column) order, no mirror. */
float orc_matrix_full(const uint32_t *counts, int n, int L, int type, int model,
                      int naive, int compat_wrap, float *out) {
  float maxd = 0.0f;
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) {
      float d = orc_distance(counts + ((size_t)i * n + j) * 3, L, type, model, naive,
                             compat_wrap);
      if (d > maxd) maxd = d;
      out[(size_t)i * n + j] = d;
    }
  }
  for (size_t k = 0; k < (size_t)n * n; k++) {
    size_t i = k / n, j = k % n;
    if (i == j) out[k] = 0.0f;
    if (out[k] == -1) out[k] = maxd * 2;
  }
  return maxd;
}

/* Distances before the post-process (saturated pairs stay -1, no mirror, no
 * diagonal rule): every j > i, or every (i, j) when full.  Other entries are
 * left as they are.  Checker for split computations that post-process later
 * (the multi-GPU shards). */
void orc_raw_distances(const uint32_t *counts, int n, int L, int type, int model, int naive,
                       int compat_wrap, int full, float *out) {
  for (int i = 0; i < n; i++)
    for (int j = full ? 0 : i + 1; j < n; j++)
      out[(size_t)i * n + j] = orc_distance(counts + ((size_t)i * n + j) * 3, L, type, model,
                                            naive, compat_wrap);
}
