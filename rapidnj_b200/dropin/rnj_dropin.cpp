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
  rnj_aln *aln = nullptr;
  if (fastdist) {
    check(rnj_aln_from_bitstrings(ctx, loader->getBitStrings(),
                                  type == RNJ_DNA ? loader->getGapFilters() : nullptr, n, L,
                                  (int)loader->getBitStringsCount(), type, RNJ_FASTDIST, &aln),
          "alignment upload");
  } else {
    // The naive estimator is asymmetric (only an upper-case row classifies a
    // difference), so the disk-backed mode, which keeps both triangles as
    // computed, needs every ordered pair.
    std::vector<char *> &seqs = *loader->getSequences();
    check(rnj_aln_from_host(ctx, seqs.data(), n, L, type, dm ? RNJ_FULL_ROWS : 0, &aln),
          "alignment upload");
  }
  rnj_mat *m = nullptr;
  check(rnj_distance(ctx, aln, model, &m), "distance computation");
  rnj_aln_destroy(aln);
  if (rows) {
    check(rnj_mat_copy_rows(ctx, m, 0, n, rows, numThreads), "distance copy");
  } else if (dm) {
    // Bands of rows through one host buffer, then the disk matrix row by row.
    const int band = std::max(1, std::min(n, 256));
    std::vector<distType> buf((size_t)band * n);
    std::vector<distType *> ptrs(band);
    for (int r0 = 0; r0 < n; r0 += band) {
      const int k = std::min(band, n - r0);
      for (int i = 0; i < k; ++i) ptrs[i] = buf.data() + (size_t)i * n;
      check(rnj_mat_copy_rows(ctx, m, r0, k, ptrs.data(), numThreads), "distance copy");
      for (int i = 0; i < k; ++i) dm->writeArray(ptrs[i], r0 + i, n);
    }
  }
  float mx = 0.0f;
  check(rnj_mat_info(m, nullptr, &mx), "distance maximum");
  rnj_mat_destroy(m);
  return mx;
}

}  // namespace rnj_dropin
