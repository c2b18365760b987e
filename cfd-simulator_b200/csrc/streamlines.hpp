// streamlines.hpp - the device streamline tracer (post::traceStreamlines,
// src/post/Streamlines.cpp:80-197) for the solver front end.
#pragma once

#include <cuda_runtime.h>

#include "common.hpp"

namespace cfdb {

/// StreamlineOptions (include/cfd/post/Streamlines.hpp:16-33), with the stall
/// speed already formed (max(stallFraction, 0) * max(referenceSpeed, 0)).
struct StreamlineSettings {
  int maxSteps;
  double stepFraction;
  double stallSpeed;
  int traceBackwards;
};

/// Trace `seeds` seeds (device xy pairs) through the cell velocities (u, v)
/// of an NI x NJ block with node coordinates `nodes` (device, (x, y) per node,
/// NI + 1 per row). points gets 2 * seeds curves of up to maxSteps + 1
/// points (seed s upstream at 2s, downstream at 2s + 1) and lengths their
/// point counts; seedCell gets each seed's cell (a value >= NI*NJ when no
/// cell contains it).
Status launchStreamlines(int NI, int NJ, const double* nodes, const double* area, const int* acrossJ0,
                         const double* u, const double* v, int seeds, const double* seedXY,
                         const StreamlineSettings& o, int* seedCell, double* points, int* lengths,
                         cudaStream_t stream);

}  // namespace cfdb
