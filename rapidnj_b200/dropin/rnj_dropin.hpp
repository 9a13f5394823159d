// rnj_dropin.hpp -- shared part of the JCdistance / KimuraDistance drop-in.
//
// The two classes rapidNJ's driver constructs (main.cpp:255-270) are declared by
// rapidNJ's own headers (src/distanceCalculation/JCdistance.hpp:11-35,
// KimuraDistance.hpp:9-41).  JCdistance.cpp and KimuraDistance.cpp in this
// directory implement those declarations on top of librnjgpu.so, so a rapidNJ
// build links them in place of its CPU implementations and nothing else in
// rapidNJ changes.  This header needs rapidNJ's include paths (stdinclude.h,
// dataloader.hpp, diskMatrix.h) and include/rnj.h.
#ifndef RNJ_DROPIN_HPP
#define RNJ_DROPIN_HPP

#include "dataloader.hpp"
#include "diskMatrix.h"
#include "stdinclude.h"

namespace rnj_dropin {

// The post-processed distance matrix of the loader's alignment under `model`
// (RNJ_JC or RNJ_KIMURA), computed on the GPU:
//   rows != NULL: rows[i][0..n) of the caller's n row arrays receive row i;
//   dm != NULL:   every full row goes through dm->writeArray(row, i, n), the
//                 disk-backed mode of the reference (KimuraDistance.cpp:267-281),
//                 and rows holding saturated pairs are post-processed through
//                 readArray / writeArray (KimuraDistance.cpp:366-395).
// With a disk matrix, or when the n x n floats exceed the device budget
// (RNJ_DEVICE_MATRIX_BUDGET bytes, else 80 % of the free device memory), the
// rows are computed in bands (rnj_distance_rows) with device buffers for two
// bands only; otherwise the whole matrix is computed on the device and copied.
// fastdist reads the loader's bit strings (getBitStrings / getGapFilters /
// getBitStringsCount), otherwise its sequences with the naive -f rules.
// numThreads is used for the host copy of the rows.  Returns the maximum
// distance.  On failure it prints the library's message on stderr and exits
// with status 1, as the reference's drivers do.
distType compute(dataloader *loader, bool fastdist, int model, distType **rows, diskMatrix *dm,
                 int numThreads, bool verbose);

}  // namespace rnj_dropin

#endif
