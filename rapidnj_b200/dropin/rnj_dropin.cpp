// rnj_dropin.cpp -- the GPU distance matrix for rapidNJ's distance classes,
// through the C ABI of librnjgpu.so (include/rnj.h).
#include "rnj_dropin.hpp"

#include <stdlib.h>

#include <algorithm>
#include <iostream>
#include <vector>

#include "rnj.h"

namespace rnj_dropin {
namespace {

void check(int rc, const char *what) {
  if (rc == RNJ_OK) return;
  std::cerr << "ERROR: " << what << ": " << rnj_last_error() << std::endl;
  exit(1);
}

// One context for the process (the driver may build several matrices: one per
// bootstrap replicate, main.cpp:519-532).  RNJ_DEVICE selects the GPU.
rnj_ctx *context() {
  static rnj_ctx *ctx = nullptr;
  if (!ctx) {
    const char *dev = getenv("RNJ_DEVICE");
    check(rnj_ctx_create(dev ? atoi(dev) : 0, &ctx), "GPU distance context");
  }
  return ctx;
}

// Where the rows of a banded computation go: the caller's row arrays or the
// disk matrix; which rows hold saturated pairs (-1) for the post-process.
struct RowSink {
  distType **rows;
  diskMatrix *dm;
  int n;
  std::vector<char> saturated;
};

int take_rows(void *user, int row0, int nrows, const float *band, size_t ld) {
  RowSink *s = static_cast<RowSink *>(user);
  for (int k = 0; k < nrows; ++k) {
    const float *src = band + (size_t)k * ld;
    const int i = row0 + k;
    s->saturated[i] = std::find(src, src + s->n, -1.0f) != src + s->n;
    if (s->rows) {
      std::copy(src, src + s->n, s->rows[i]);
    } else {
      // diskMatrix::writeArray takes a non-const row; the band buffer is ours
      // only for the call, so the row goes through a copy.
      std::vector<distType> row(src, src + s->n);
      s->dm->writeArray(row.data(), i, s->n);
    }
  }
  return 0;
}

// Device bytes the n x n matrix may take: RNJ_DEVICE_MATRIX_BUDGET when set,
// else 80 % of the free device memory.
double matrix_budget(rnj_ctx *ctx) {
  if (const char *b = getenv("RNJ_DEVICE_MATRIX_BUDGET")) return atof(b);
  size_t free_bytes = 0;
  check(rnj_ctx_memory(ctx, &free_bytes, nullptr), "device memory");
  return 0.8 * (double)free_bytes;
}

}  // namespace

distType compute(dataloader *loader, bool fastdist, int model, distType **rows, diskMatrix *dm,
                 int numThreads, bool verbose) {
  rnj_ctx *ctx = context();
  const int n = (int)loader->getSequenceCount();
  const int L = (int)loader->getSequenceLength();
  const int type = (loader->type == PROTEIN) ? RNJ_PROTEIN : RNJ_DNA;
  if (verbose)
    std::cerr << "Computing " << (model == RNJ_JC ? "JC" : "Kimura") << " distances of " << n
              << " sequences (" << L << " columns) on the GPU" << std::endl;
  const double budget = matrix_budget(ctx);
  const double need = (double)n * n * sizeof(float);
  // Rows in bands when the reference keeps the matrix on disk, or when the whole
  // matrix would not fit the device budget.
  const bool banded = dm != nullptr || need > budget;
  rnj_aln *aln = nullptr;
  if (fastdist) {
    check(rnj_aln_from_bitstrings(ctx, loader->getBitStrings(),
                                  type == RNJ_DNA ? loader->getGapFilters() : nullptr, n, L,
                                  (int)loader->getBitStringsCount(), type, RNJ_FASTDIST, &aln),
          "alignment upload");
  } else {
    // The naive estimator is asymmetric (only an upper-case row classifies a
    // difference), so the row-band mode, which keeps both triangles as
    // computed (as the reference's disk-matrix drivers do), needs every ordered pair.
    std::vector<char *> &seqs = *loader->getSequences();
    check(rnj_aln_from_host(ctx, seqs.data(), n, L, type, banded ? RNJ_FULL_ROWS : 0, &aln),
          "alignment upload");
  }
  float mx = 0.0f;
  if (banded) {
    // Two bands of at most half the budget (at least one 128-row tile each).
    const int band = std::max(128, (int)std::min<double>(n, budget / (2.0 * n * sizeof(float))));
    RowSink sink{rows, dm, n, std::vector<char>((size_t)n, 0)};
    int saturated = 0;
    check(rnj_distance_rows(ctx, aln, model, band, take_rows, &sink, &mx, &saturated),
          "distance computation");
    rnj_aln_destroy(aln);
    if (saturated) {
      // The reference's post-process of the saturated pairs
      // (KimuraDistance.cpp:366-395, JCdistance.cpp:201-230), on the rows that hold one.
      const distType cap = mx * 2;
      std::vector<distType> buf(dm ? (size_t)n : 0);
      for (int i = 0; i < n; ++i) {
        if (!sink.saturated[i]) continue;
        distType *row = rows ? rows[i] : buf.data();
        if (dm) dm->readArray(row, i, n);
        for (int j = 0; j < n; ++j)
          if (row[j] == -1) row[j] = cap;
        if (dm) dm->writeArray(row, i, n);
      }
    }
    return mx;
  }
  rnj_mat *m = nullptr;
  check(rnj_distance(ctx, aln, model, &m), "distance computation");
  rnj_aln_destroy(aln);
  check(rnj_mat_copy_rows(ctx, m, 0, n, rows, numThreads), "distance copy");
  check(rnj_mat_info(m, nullptr, &mx), "distance maximum");
  rnj_mat_destroy(m);
  return mx;
}

}  // namespace rnj_dropin
