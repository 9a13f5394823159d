// ref_harness.cpp -- drives the reference's own distance code, compiled from its
// sources by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY: it is
// the golden-vector generator and the timed CPU baseline, never the product.
//
// Usage:
//   ref_harness counts <aln> <fa|sth> <d|p|auto> <fastdist 0|1> <full 0|1> <out.bin>
//       Per-pair {c0, c1, valid} from the reference estimator
//       (DistanceEstimate::computeDistance, DistanceEstimate.hpp:14), for j>i or
//       every (i, j) when full=1.  Output: int32 n, L, type, then n*n*3 uint32.
//   ref_harness matrix <aln> <fa|sth> <d|p|auto> <fastdist 0|1> <jc|kim> <threads> <out.bin|-> [disk]
//       The post-processed float matrix from JCdistance::computeDistanceMatrix /
//       KimuraDistance::computeDistances (main.cpp:259-270), with the disk-matrix
//       row path (diskMatrix.cpp) when "disk" is given.  Output: int32 n, then n*n
//       float.  Prints one JSON line with the timing of the compute call.
#include <sys/time.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "JCdistance.hpp"
#include "KimuraDistance.hpp"
#include "bitDistanceGap.hpp"
#include "bitDistanceProtein.hpp"
#include "dataloader.hpp"
#include "dataloaderFasta.hpp"
#include "dataloaderStockholm.hpp"
#include "diskMatrix.h"
#include "simpleDistanceCalculator.hpp"

static double now_s() {
  timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}

static dataloader *load(const char *path, const std::string &fmt, const std::string &t,
                        bool fastdist) {
  InputType type = UNKNOWN;
  if (t == "d") type = DNA;
  if (t == "p") type = PROTEIN;
  dataloader *dl;
  if (fmt == "sth") dl = new dataloaderStockholm();
  else dl = new dataloaderFasta();
  dl->readData(path, fastdist, false, type, false);
  return dl;
}

static DistanceEstimate *estimator(dataloader *dl) {
  if (!dl->fastdist) return new simpleDistanceCalculator(dl);
  if (dl->type == DNA) return new bitDistanceGap(dl);
  return new bitDistanceProtein(dl);
}

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: see header\n");
    return 2;
  }
  std::string mode = argv[1];
  if (mode == "counts" && argc == 8) {
    bool fastdist = atoi(argv[5]) != 0;
    bool full = atoi(argv[6]) != 0;
    dataloader *dl = load(argv[2], argv[3], argv[4], fastdist);
    int n = dl->getSequenceCount();
    int L = dl->getSequenceLength();
    int type = dl->type;
    DistanceEstimate *de = estimator(dl);
    unsigned int *out = (unsigned int *)calloc((size_t)n * n * 3, sizeof(unsigned int));
    unsigned long long d[3];
    for (int i = 0; i < n; i++)
      for (int j = full ? 0 : i + 1; j < n; j++) {
        de->computeDistance(i, j, d);
        unsigned int *o = out + ((size_t)i * n + j) * 3;
        o[0] = (unsigned int)d[0];
        o[1] = (unsigned int)d[1];
        o[2] = (unsigned int)d[2];
      }
    FILE *f = fopen(argv[7], "wb");
    if (!f) return 1;
    int hdr[3] = {n, L, type};
    fwrite(hdr, sizeof(int), 3, f);
    fwrite(out, sizeof(unsigned int), (size_t)n * n * 3, f);
    fclose(f);
    delete de;
    return 0;
  }
  if (mode == "matrix" && (argc == 9 || argc == 10)) {
    bool fastdist = atoi(argv[5]) != 0;
    std::string model = argv[6];
    int threads = atoi(argv[7]);
    bool disk = (argc == 10 && std::string(argv[9]) == "disk");
    double t0 = now_s();
    dataloader *dl = load(argv[2], argv[3], argv[4], fastdist);
    double t1 = now_s();
    int n = dl->getSequenceCount();
    int L = dl->getSequenceLength();
    diskMatrix *dm = NULL;
    if (disk) dm = new diskMatrix("", n);
    distType **m = NULL;
    double t2 = now_s();
    if (model == "jc") {
      JCdistance *alg = new JCdistance(false, fastdist, dl, dm);
      alg->computeDistanceMatrix(threads);
      m = alg->getDistanceMatrix();
      delete alg;
    } else {
      KimuraDistance *alg = new KimuraDistance(false, fastdist, dl, dm);
      alg->computeDistances(threads);
      m = alg->getDistanceMatrix();
      delete alg;
    }
    double t3 = now_s();
    printf("{\"n\": %d, \"L\": %d, \"type\": %d, \"threads\": %d, \"load_s\": %.6f, \"compute_s\": %.6f}\n",
           n, L, (int)dl->type, threads, t1 - t0, t3 - t2);
    if (std::string(argv[8]) != "-") {
      FILE *f = fopen(argv[8], "wb");
      if (!f) return 1;
      fwrite(&n, sizeof(int), 1, f);
      distType *row = new distType[n];
      for (int i = 0; i < n; i++) {
        if (dm) dm->readArray(row, i, n);
        else memcpy(row, m[i], sizeof(distType) * n);
        fwrite(row, sizeof(distType), n, f);
      }
      delete[] row;
      fclose(f);
    }
    return 0;
  }
  if (mode == "bench" && argc == 10) {
    // bench <aln> <fmt> <type> <fastdist> <jc|kim> <threads> <warmup> <steps>:
    // repeated driver calls on one loaded alignment; each call allocates and
    // frees its own matrix, as main.cpp's computeDistanceMatrix does.
    bool fastdist = atoi(argv[5]) != 0;
    std::string model = argv[6];
    int threads = atoi(argv[7]);
    int warmup = atoi(argv[8]);
    int steps = atoi(argv[9]);
    dataloader *dl = load(argv[2], argv[3], argv[4], fastdist);
    int n = dl->getSequenceCount();
    printf("{\"n\": %d, \"L\": %d, \"threads\": %d, \"step_s\": [", n, (int)dl->getSequenceLength(),
           threads);
    for (int s = 0; s < warmup + steps; s++) {
      double t0 = now_s();
      distType **m;
      if (model == "jc") {
        JCdistance *alg = new JCdistance(false, fastdist, dl, NULL);
        alg->computeDistanceMatrix(threads);
        m = alg->getDistanceMatrix();
        delete alg;
      } else {
        KimuraDistance *alg = new KimuraDistance(false, fastdist, dl, NULL);
        alg->computeDistances(threads);
        m = alg->getDistanceMatrix();
        delete alg;
      }
      double t1 = now_s();
      for (int i = 0; i < n; i++) delete[] m[i];
      delete[] m;
      if (s >= warmup) printf("%s%.6f", s > warmup ? ", " : "", t1 - t0);
    }
    printf("]}\n");
    return 0;
  }
  fprintf(stderr, "bad arguments\n");
  return 2;
}
