// streamlines.cu - post::traceStreamlines (src/post/Streamlines.cpp:80-197)
// on the device: classical RK4 through the piecewise-constant cell velocity
// of a structured block, with the reference's point location (a walk out of
// the worst edge from a hint cell, across the wake cut, and a first-cell scan
// where no hint is usable; Streamlines.cpp:47-100).
//
// One thread per seed and direction. The seeds are placed first by a scan in
// which every (seed, cell) pair is tested and the lowest containing cell wins,
// which is the cell the reference's sequential scan finds. Arithmetic follows
// the reference's expressions and their order (no contraction), so curves
// agree with the reference's to rounding: the speed is CUDA's hypot (within
// its documented error of the host's std::hypot), the one operation that may
// round differently.

#include <cuda_runtime.h>

#include <cmath>

#include "streamlines.hpp"

namespace cfdb {
namespace {

#define SDEV __device__ __forceinline__

struct Block {
  int NI, NJ;           // cells
  const double* nodes;  // (x, y) per node, node (i, j) at j*(NI+1) + i
  const double* area;   // per cell
  const int* acrossJ0;  // cell across the j = 0 face of column i, or -1
  const double *u, *v;  // per cell
};

/// -turn(a, b, p): how far p lies outside the edge a -> b of an anticlockwise
/// cell (Streamlines.cpp:13-29), negative inside.
SDEV double edgeDistance(const Block& B, int c, int k, double px, double py) {
  const int i = c % B.NI, j = c / B.NI;
  const int stride = B.NI + 1;
  // corners (i, j), (i+1, j), (i+1, j+1), (i, j+1) (Mesh.cpp:130-136)
  const int corner[5] = {j * stride + i, j * stride + i + 1, (j + 1) * stride + i + 1,
                         (j + 1) * stride + i, j * stride + i};
  const double ax = B.nodes[2 * corner[k]], ay = B.nodes[2 * corner[k] + 1];
  const double bx = B.nodes[2 * corner[k + 1]], by = B.nodes[2 * corner[k + 1] + 1];
  const double ex = bx - ax, ey = by - ay;
  const double qx = px - ax, qy = py - ay;
  return -(ex * qy - ey * qx);
}

/// The cell across edge k (0 below, 1 right, 2 above, 3 left: Mesh::cellFaces
/// order, Mesh.cpp:204-213) as the walk leaves through it: the face's owner
/// when that is another cell, else oppositeCell (neighbour, or the partner
/// across the wake cut), or -1 through a real boundary.
SDEV int acrossEdge(const Block& B, int c, int k) {
  const int i = c % B.NI, j = c / B.NI;
  switch (k) {
    case 0: return (j > 0) ? c - B.NI : B.acrossJ0[i];
    case 1: return (i < B.NI - 1) ? c + 1 : -1;
    case 2: return (j < B.NJ - 1) ? c + B.NI : -1;
    default: return (i > 0) ? c - 1 : -1;
  }
}

/// locateCell (Streamlines.cpp:47-100): from a usable hint, walk towards the
/// point, leaving each cell through the edge it lies furthest beyond (-1 when
/// that is a real boundary); after 4096 steps without arriving, or without a
/// hint, the first cell that contains the point (a scan: rare on a walk, and
/// costly, but it is the reference's answer).
SDEV int locate(const Block& B, double px, double py, int hint) {
  const int cells = B.NI * B.NJ;
  if (hint >= 0 && hint < cells) {
    int current = hint;
    for (int step = 0; step < 4096; ++step) {
      int worstEdge = -1;
      double worst = 0.0;
      for (int k = 0; k < 4; ++k) {
        const double outside = edgeDistance(B, current, k, px, py);
        if (outside > worst) {
          worst = outside;
          worstEdge = k;
        }
      }
      if (worstEdge < 0) return current;
      const int next = acrossEdge(B, current, worstEdge);
      if (next < 0) return -1;
      current = next;
    }
  }
  for (int c = 0; c < cells; ++c) {
    bool inside = true;
    for (int k = 0; k < 4 && inside; ++k) inside = !(edgeDistance(B, c, k, px, py) > 0.0);
    if (inside) return c;
  }
  return -1;
}

/// Lowest-index cell containing each seed (the reference's scan), by atomicMin.
__global__ void seedKernel(Block B, int seeds, const double* __restrict__ xy, int* __restrict__ cell) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long cells = static_cast<long long>(B.NI) * B.NJ;
  if (t >= cells * seeds) return;
  const int s = static_cast<int>(t / cells);
  const int c = static_cast<int>(t % cells);
  const double px = xy[2 * s], py = xy[2 * s + 1];
  for (int k = 0; k < 4; ++k) {
    if (edgeDistance(B, c, k, px, py) > 0.0) return;
  }
  atomicMin(cell + s, c);
}

/// One seed in one direction (odd threads downstream, even upstream): the
/// points from the seed onwards, at most maxSteps + 1 (Streamlines.cpp:132-183).
__global__ void traceKernel(Block B, int seeds, const double* __restrict__ xy, const int* __restrict__ seedCell,
                            StreamlineSettings o, double* __restrict__ points, int* __restrict__ lengths) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * seeds) return;
  const int s = t >> 1;
  const bool downstream = (t & 1) != 0;
  double* out = points + static_cast<long long>(t) * 2 * (o.maxSteps + 1);
  const int start = seedCell[s];
  if (start < 0 || start >= B.NI * B.NJ || (!downstream && !o.traceBackwards)) {
    lengths[t] = 0;
    return;
  }
  const double sense = downstream ? 1.0 : -1.0;
  double px = xy[2 * s], py = xy[2 * s + 1];
  int cell = start;
  int n = 0;
  out[2 * n] = px;
  out[2 * n + 1] = py;
  ++n;
  // velocityAt: the cell holding the point (walking from the carried cell),
  // its velocity times the sense; zero outside the domain
  auto velocityAt = [&](double x, double y, int& carried, double& vx, double& vy) {
    const int found = locate(B, x, y, carried);
    if (found < 0) {
      vx = 0.0;
      vy = 0.0;
      return;
    }
    carried = found;
    vx = B.u[found] * sense;
    vy = B.v[found] * sense;
  };
  for (int step = 0; step < o.maxSteps; ++step) {
    int probe = cell;
    double k1x, k1y;
    velocityAt(px, py, probe, k1x, k1y);
    const double speed = hypot(k1x, k1y);
    if (!(speed > o.stallSpeed)) break;
    const double step0 = o.stepFraction * sqrt(fmax(B.area[cell], 0.0));
    const double dt = (speed > 0.0) ? step0 / speed : 0.0;
    if (!(dt > 0.0)) break;
    int probe2 = probe;
    double k2x, k2y;
    velocityAt(px + k1x * (0.5 * dt), py + k1y * (0.5 * dt), probe2, k2x, k2y);
    int probe3 = probe2;
    double k3x, k3y;
    velocityAt(px + k2x * (0.5 * dt), py + k2y * (0.5 * dt), probe3, k3x, k3y);
    int probe4 = probe3;
    double k4x, k4y;
    velocityAt(px + k3x * dt, py + k3y * dt, probe4, k4x, k4y);
    const double h = dt / 6.0;
    const double ax = (((k1x + k2x * 2.0) + k3x * 2.0) + k4x) * h;
    const double ay = (((k1y + k2y * 2.0) + k3y * 2.0) + k4y) * h;
    const double nx = px + ax, ny = py + ay;
    const int nextCell = locate(B, nx, ny, cell);
    if (nextCell < 0) break;  // left the domain
    px = nx;
    py = ny;
    cell = nextCell;
    out[2 * n] = px;
    out[2 * n + 1] = py;
    ++n;
  }
  lengths[t] = n;
}

}  // namespace

Status launchStreamlines(int NI, int NJ, const double* nodes, const double* area, const int* acrossJ0,
                         const double* u, const double* v, int seeds, const double* seedXY,
                         const StreamlineSettings& o, int* seedCell, double* points, int* lengths,
                         cudaStream_t stream) {
  const Block B{NI, NJ, nodes, area, acrossJ0, u, v};
  const long long pairs = static_cast<long long>(NI) * NJ * seeds;
  const int block = 256;
  cudaError_t e = cudaMemsetAsync(seedCell, 0x7f, sizeof(int) * seeds, stream);  // above any cell index
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  seedKernel<<<static_cast<unsigned>((pairs + block - 1) / block), block, 0, stream>>>(B, seeds, seedXY, seedCell);
  traceKernel<<<(2 * seeds + 127) / 128, 128, 0, stream>>>(B, seeds, seedXY, seedCell, o, points, lengths);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  return CFD_OK;
}

}  // namespace cfdb
