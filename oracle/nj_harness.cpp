// nj_harness.cpp -- drives the reference's own neighbour-joining initialisation
// (rapidNJ::initialize, rapidNJ.cpp:94-141, and rapidNJMem::initialize,
// rapidNJMem.cpp:92-135), compiled from its sources by oracle/Makefile into
// oracle/_ref/.  TEST INFRASTRUCTURE ONLY: golden-vector generator and timed CPU
// baseline of the NJ set-up, never the product.
//
// initialize() and the arrays it fills are private members; this file alone
// opens them by defining `private` as `public` around the reference headers
// (after every standard header they include, so that only the reference's own
// classes are affected).  The reference sources are compiled unchanged.
//
// Usage:
//   nj_harness <in.bin> <out.bin|-> [reps]
//     in.bin:  int32 n, int32 cap, then n*n float32 (row-major distance matrix).
//              cap <= 0: rapidNJ (every row fully sorted); cap > 0: rapidNJMem
//              with sortedMatrixSize = cap.
//     out.bin: int32 n; float32 separationsums[n], separations[n],
//              maxRowSeparations[n], max_separation; int32 indexToId[n],
//              redundantToMasterMap[n], redundantCount[n], row_lengths[n]
//              (0 for redundant rows, which the reference leaves unset); then per
//              row: int32 length and the redundantMap list in list order; then per
//              non-redundant row its row_lengths[i] cluster_pairs {uint32 id,
//              float32 distance}.
//     Prints one JSON line with the seconds of each initialize() call.
#include <sys/time.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <list>
#include <map>
#include <stack>
#include <string>
#include <utility>
#include <vector>

#define private public
#include "rapidNJ.h"
#include "rapidNJMem.hpp"
#undef private

static double now_s() {
  timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}

template <class T>
static void put(FILE *f, const T *p, size_t count) {
  if (fwrite(p, sizeof(T), count, f) != count) {
    fprintf(stderr, "write failed\n");
    exit(1);
  }
}

template <class NJ>
static void dump(FILE *f, NJ *nj, int n, cluster_pair **rows) {
  put(f, &n, 1);
  put(f, nj->separationsums, n);
  put(f, nj->separations, n);
  put(f, nj->maxRowSeparations, n);
  put(f, &nj->max_separation, 1);
  put(f, nj->indexToId, n);
  put(f, nj->redundantToMasterMap, n);
  put(f, nj->redundantCount, n);
  std::vector<int> lengths(n, 0);
  for (int i = 0; i < n; i++)
    if (nj->indexToId[i] != -1) lengths[i] = nj->row_lengths[i];
  put(f, lengths.data(), n);
  for (int i = 0; i < n; i++) {
    int len = (int)nj->redundantMap[i].size();
    put(f, &len, 1);
    for (std::list<int>::iterator it = nj->redundantMap[i].begin();
         it != nj->redundantMap[i].end(); ++it) {
      int v = *it;
      put(f, &v, 1);
    }
  }
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < lengths[i]; k++) {
      unsigned int id = rows[i][k].id;
      float d = rows[i][k].distance;
      put(f, &id, 1);
      put(f, &d, 1);
    }
  }
}

int main(int argc, char **argv) {
  if (argc != 3 && argc != 4) {
    fprintf(stderr, "usage: see header\n");
    return 2;
  }
  FILE *in = fopen(argv[1], "rb");
  if (!in) {
    fprintf(stderr, "cannot open %s\n", argv[1]);
    return 1;
  }
  int hdr[2];
  if (fread(hdr, sizeof(int), 2, in) != 2) return 1;
  const int n = hdr[0], cap = hdr[1];
  const int reps = argc == 4 ? atoi(argv[3]) : 1;
  std::vector<float> flat((size_t)n * n);
  if (fread(flat.data(), sizeof(float), flat.size(), in) != flat.size()) return 1;
  fclose(in);
  std::vector<std::string> *names = new std::vector<std::string>();
  for (int i = 0; i < n; i++) names->push_back("s" + std::to_string(i));

  printf("{\"n\": %d, \"cap\": %d, \"init_s\": [", n, cap);
  for (int r = 0; r < reps; r++) {
    // A fresh copy of the rows per call: the NJ classes own and mutate them.
    distType **m = new distType *[n];
    for (int i = 0; i < n; i++) {
      m[i] = new distType[n];
      memcpy(m[i], &flat[(size_t)i * n], sizeof(float) * n);
    }
    distMatrixReader *reader = new distMatrixReader(false, n, false, names, m);
    ProgressBar *pb = new ProgressBar();
    double t0, t1;
    FILE *f = NULL;
    if (r == reps - 1 && strcmp(argv[2], "-") != 0) f = fopen(argv[2], "wb");
    if (cap <= 0) {
      rapidNJ *nj = new rapidNJ(reader, n, false, pb);
      t0 = now_s();
      nj->initialize();
      t1 = now_s();
      if (f) dump(f, nj, n, nj->cluster_data);
      delete nj;  // frees the rows, the sorted rows and the reader
    } else {
      rapidNJMem *nj = new rapidNJMem(reader, n, cap, false, false, pb);
      t0 = now_s();
      nj->initialize();
      t1 = now_s();
      if (f) dump(f, nj, n, nj->cluster_data);
      delete nj;
    }
    delete pb;
    if (f) fclose(f);
    printf("%s%.6f", r ? ", " : "", t1 - t0);
  }
  printf("]}\n");
  return 0;
}
