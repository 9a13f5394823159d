// KimuraDistance.cpp -- rapidNJ's KimuraDistance class (declared in its
// src/distanceCalculation/KimuraDistance.hpp:9-41) computed on the GPU.
//
// Same constructors and calls as the reference (KimuraDistance.cpp:50-99):
// computeDistances(numThreads) fills a new n x n matrix of new[] rows, or the
// caller's preallocated rows (the bootstrap replicates, main.cpp:519-532), or,
// with a disk matrix, the disk.  The preallocated form with a disk matrix is
// refused with the reference's message.  computeDistancesGPU() is the same
// computation (every call here runs on the GPU).
#include "KimuraDistance.hpp"

#include <iostream>

#include "rnj.h"
#include "rnj_dropin.hpp"

KimuraDistance::KimuraDistance(bool verbose, bool fastdist, dataloader *loader, diskMatrix *dm) {
  KimuraDistance::verbose = verbose;
  KimuraDistance::fastdist = fastdist;
  KimuraDistance::popcnt = false;
  KimuraDistance::loader = loader;
  KimuraDistance::seqCount = loader->getSequenceCount();
  KimuraDistance::sequenceNames = *loader->getSequenceNames();
  KimuraDistance::gpuInitialised = false;
  KimuraDistance::dm = dm;
  distMatrix = NULL;
  distanceMatrixTS = NULL;
  distanceMatrixTV = NULL;
  maxDistance = 0.0;
}

KimuraDistance::KimuraDistance(bool verbose, bool fastdist, dataloader *loader,
                               distType **_distMatrix, diskMatrix *dm) {
  KimuraDistance::verbose = verbose;
  KimuraDistance::fastdist = fastdist;
  KimuraDistance::popcnt = false;
  KimuraDistance::loader = loader;
  KimuraDistance::seqCount = loader->getSequenceCount();
  KimuraDistance::sequenceNames = *loader->getSequenceNames();
  KimuraDistance::gpuInitialised = false;
  KimuraDistance::dm = dm;
  distMatrix = _distMatrix;
  distanceMatrixTS = NULL;
  distanceMatrixTV = NULL;
  maxDistance = 0.0;
}

// The matrix belongs to the caller (getDistanceMatrix), as in the reference.
KimuraDistance::~KimuraDistance(void) {}

void KimuraDistance::computeDistances(int numThreads) {
  maxDistance = 0.0;
  if (distMatrix != NULL && dm != NULL) {
    std::cerr << "ERROR: computation of bootstrap values is not supported for trees which use "
                 "I/O efficient computation."
              << std::endl;
    exit(1);
  }
  if (dm == NULL && distMatrix == NULL) {
    distMatrix = new distType *[seqCount];
    for (int i = 0; i < seqCount; i++) distMatrix[i] = new distType[seqCount];
  }
  maxDistance = rnj_dropin::compute(loader, fastdist, RNJ_KIMURA, dm == NULL ? distMatrix : NULL,
                                    dm, numThreads, verbose);
  gpuInitialised = true;
}

void KimuraDistance::computeDistancesGPU() { computeDistances(0); }

distType **KimuraDistance::getDistanceMatrix() { return distMatrix; }
