// JCdistance.cpp -- rapidNJ's JCdistance class (declared in its
// src/distanceCalculation/JCdistance.hpp:11-35) computed on the GPU.
//
// Same constructor and calls as the reference (JCdistance.cpp:14-44): the
// driver constructs it, calls computeDistanceMatrix(numThreads) and takes the
// n rows of getDistanceMatrix(), each a new[]-allocated distType array that the
// join loops later mutate and delete[].  With a disk matrix the rows go to
// disk instead and getDistanceMatrix() returns NULL.
#include "JCdistance.hpp"

#include "rnj.h"
#include "rnj_dropin.hpp"

JCdistance::JCdistance(bool verbose, bool fastdist, dataloader *loader, diskMatrix *dm) {
  JCdistance::verbose = verbose;
  JCdistance::fastdist = fastdist;
  JCdistance::loader = loader;
  JCdistance::seqCount = loader->getSequenceCount();
  JCdistance::seqLength = loader->getSequenceLength();
  JCdistance::sequenceNames = *loader->getSequenceNames();
  JCdistance::dm = dm;
  jcDistMatrix = NULL;
  distanceMatrixTS = NULL;
  distanceMatrixTV = NULL;
  maxDistance = 0.0;
}

void JCdistance::computeDistanceMatrix(int numThreads) {
  maxDistance = 0.0;
  jcDistMatrix = NULL;
  if (dm == NULL) {
    jcDistMatrix = new distType *[seqCount];
    for (int i = 0; i < seqCount; i++) jcDistMatrix[i] = new distType[seqCount];
  }
  maxDistance = rnj_dropin::compute(loader, fastdist, RNJ_JC, jcDistMatrix, dm, numThreads, verbose);
}

distType **JCdistance::getDistanceMatrix() { return jcDistMatrix; }
