// forces.cu - wall surface data and force integration on the device, FP64:
// post::extractSurface and post::integrateForces (src/post/SurfaceData.cpp:101-348,
// src/post/Forces.cpp:23-130) on the solver's current field.
//
// Everything that depends only on the mesh (the wall stations in contour
// order, their normals, tangents and lengths, the two wall distances of the
// shear fit, the leading edge) is tabulated on the host once, in the
// reference's arithmetic. The device reads the wall-adjacent cells, finds the
// stagnation station, evaluates each station in parallel and then sums the
// forces and moments in the reference's order (upper surface from the
// leading edge, then the lower surface outwards from it) so the coefficients
// round as the reference's do.

#include <cuda_runtime.h>

#include <cmath>

#include "forces.hpp"

namespace cfdb {
namespace {

#define FDEV __device__ __forceinline__

struct ForceParams {
  double dynamicPressure, referencePressure, chord, cosA, sinA;
};

/// Per station: Cp, wall shear, Cf and the force/moment increments, in wall
/// order. Thread 0 first finds the stagnation station (highest owner
/// pressure, first of equals), then every thread evaluates its stations.
__global__ void forcesKernel(WallTable w, const double* __restrict__ p, const double* __restrict__ u,
                             const double* __restrict__ v, const double* __restrict__ mu,
                             ForceParams fp, double* __restrict__ station, double* __restrict__ out) {
  __shared__ int stagnation;
  const int S = w.count;
  if (threadIdx.x == 0) {
    int best = 0;
    double highest = -1.7976931348623157e308;
    for (int k = 0; k < S; ++k) {
      const double pk = p[w.owner[k]];
      if (pk > highest) {
        highest = pk;
        best = k;
      }
    }
    stagnation = best;
  }
  __syncthreads();
  const int stag = stagnation;
  for (int k = threadIdx.x; k < S; k += blockDim.x) {
    const int o = w.owner[k];
    const double nx = w.nx[k], ny = w.ny[k];
    // flowTangent (SurfaceData.cpp:278-288)
    double tx = w.tx[k], ty = w.ty[k];
    const bool forward = (k == stag) ? (k >= w.leadingEdge) : (k > stag);
    if (!forward) {
      tx = tx * -1.0;
      ty = ty * -1.0;
    }
    const double pressure = p[o];
    const double cp = (fp.dynamicPressure > 0.0) ? (pressure - fp.referencePressure) / fp.dynamicPressure : 0.0;
    const double uc = u[o], vc = v[o];
    const double dn = uc * nx + vc * ny;
    const double px = uc - nx * dn, py = vc - ny * dn;
    double shear = 0.0;
    const double d1 = w.wallDistance[k];
    if (d1 > 0.0) {
      double gradient = (px * tx + py * ty) / d1;
      const int second = w.second[k];
      if (second >= 0) {
        const double d2 = w.outerDistance[k];
        if (d2 > d1 * 1.05) {
          const double ou = u[second], ov = v[second];
          const double odn = ou * nx + ov * ny;
          const double opx = ou - nx * odn, opy = ov - ny * odn;
          const double u1 = px * tx + py * ty;
          const double u2 = opx * tx + opy * ty;
          gradient = (u1 * d2 * d2 - u2 * d1 * d1) / (d1 * d2 * (d2 - d1));
        }
      }
      shear = mu[o] * gradient;
    }
    const double cf = (fp.dynamicPressure > 0.0) ? shear / fp.dynamicPressure : 0.0;
    double* s = station + static_cast<size_t>(k) * kStationValues;
    s[0] = pressure;
    s[1] = cp;
    s[2] = shear;
    s[3] = cf;
    s[4] = tx;
    s[5] = ty;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  // Accumulator::add over upper then lower (Forces.cpp:23-45, :76-80)
  double pfx = 0.0, pfy = 0.0, ffx = 0.0, ffy = 0.0, pm = 0.0, fm = 0.0;
  int stations = 0;
  const double refX = 0.25 * fp.chord, refY = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    const int count = (pass == 0) ? S - w.leadingEdge : w.leadingEdge;
    for (int m = 0; m < count; ++m) {
      const int k = (pass == 0) ? w.leadingEdge + m : w.leadingEdge - 1 - m;
      const double* s = station + static_cast<size_t>(k) * kStationValues;
      const double ds = w.length[k];
      if (!(ds > 0.0)) continue;
      const double scale = -(s[0] - fp.referencePressure) * ds;
      const double dpx = w.nx[k] * scale, dpy = w.ny[k] * scale;
      const double fs = s[2] * ds;
      const double dfx = s[4] * fs, dfy = s[5] * fs;
      pfx = pfx + dpx;
      pfy = pfy + dpy;
      ffx = ffx + dfx;
      ffy = ffy + dfy;
      const double ax = w.cx[k] - refX, ay = w.cy[k] - refY;
      pm += ax * dpy - ay * dpx;
      fm += ax * dfy - ay * dfx;
      ++stations;
    }
  }
  const double pd = pfx * fp.cosA + pfy * fp.sinA;
  const double fd = ffx * fp.cosA + ffy * fp.sinA;
  const double pl = pfy * fp.cosA - pfx * fp.sinA;
  const double fl = ffy * fp.cosA - ffx * fp.sinA;
  const double drag = pd + fd;
  const double lift = pl + fl;
  const double moment = -pm - fm;
  const double forceScale = fp.dynamicPressure * fp.chord;
  const double momentScale = forceScale * fp.chord;
  out[0] = lift / forceScale;
  out[1] = drag / forceScale;
  out[2] = moment / momentScale;
  out[3] = pd / forceScale;
  out[4] = fd / forceScale;
  out[5] = lift;
  out[6] = drag;
  out[7] = moment;
  out[8] = (fp.chord > 0.0) ? w.cx[stag] / fp.chord : w.cx[stag];
  out[9] = static_cast<double>(stations);
  // findSeparation (SurfaceData.cpp:179-203) on each surface, walked from the
  // leading edge: the first pair of stations, neither of them the stagnation
  // station, whose wall shear goes from positive to negative; the chordwise
  // station is interpolated linearly between them. -1 where none is found.
  for (int side = 0; side < 2; ++side) {
    const int count = (side == 0) ? S - w.leadingEdge : w.leadingEdge;
    double found = -1.0;
    for (int m = 1; m < count; ++m) {
      const int k = (side == 0) ? w.leadingEdge + m : w.leadingEdge - 1 - m;
      const int kp = (side == 0) ? k - 1 : k + 1;  // the station before it
      if (k == stag || kp == stag) continue;
      const double before = station[static_cast<size_t>(kp) * kStationValues + 2];
      const double after = station[static_cast<size_t>(k) * kStationValues + 2];
      if (!(before > 0.0) || !(after < 0.0)) continue;
      const double span = before - after;
      const double fraction = (span > 0.0) ? before / span : 0.0;
      const double xp = (fp.chord > 0.0) ? w.cx[kp] / fp.chord : w.cx[kp];
      const double xk = (fp.chord > 0.0) ? w.cx[k] / fp.chord : w.cx[k];
      found = xp + fraction * (xk - xp);
      break;
    }
    out[10 + side] = found;
  }
}

}  // namespace

Status buildWallTable(const HostMesh& m, const double* nodes, HostWallTable* out) {
  HostWallTable& t = *out;
  t = HostWallTable{};
  if (nodes == nullptr) return ok();
  const int ni = m.nodesI, NI = ni - 1, NJ = m.nodesJ - 1;
  const int jFaces = NI * m.nodesJ;
  // collectWallFaces (SurfaceData.cpp:27-59): the j = 0 faces marked Wall.
  for (int i = 0; i < NI; ++i) {
    const int f = i;
    if (m.boundary[f] != 1) continue;  // mesh::BoundaryType::Wall
    const double ax = nodes[2 * i], ay = nodes[2 * i + 1];
    const double bx = nodes[2 * (i + 1)], by = nodes[2 * (i + 1) + 1];
    const double alx = bx - ax, aly = by - ay;
    const double len = std::hypot(alx, aly);
    if (!(len > 0.0)) continue;
    const int owner = m.owner[f];
    const double cx = m.faceCentre[2 * f], cy = m.faceCentre[2 * f + 1];
    const double nx = m.faceNormal[2 * f] * -1.0, ny = m.faceNormal[2 * f + 1] * -1.0;
    t.face.push_back(f);
    t.owner.push_back(owner);
    t.cx.push_back(cx);
    t.cy.push_back(cy);
    t.tx.push_back(alx * (1.0 / len));
    t.ty.push_back(aly * (1.0 / len));
    t.nx.push_back(nx);
    t.ny.push_back(ny);
    t.length.push_back(len);
    t.node0x.push_back(ax);
    // wall distance of the owner centroid (SurfaceData.cpp:118-119)
    const double ox = m.centroid[2 * owner] - cx, oy = m.centroid[2 * owner + 1] - cy;
    t.wallDistance.push_back(std::abs(ox * nx + oy * ny));
    // secondCellFromWall (SurfaceData.cpp:67-98): the cell across the owner's
    // face that points most nearly along the wall normal (alignment > 0.5),
    // faces visited below, right, above, left.
    const int oi = owner % NI, oj = owner / NI;
    const int cellFaces[4] = {oj * NI + oi, jFaces + (oi + 1) * NJ + oj, (oj + 1) * NI + oi,
                              jFaces + oi * NJ + oj};
    int best = -1;
    double bestAlignment = 0.5;
    for (int q = 0; q < 4; ++q) {
      const int g = cellFaces[q];
      if (g == f) continue;
      int across = m.neighbour[g];
      if (across < 0 && m.boundary[g] == 4 && m.partner[g] >= 0) across = m.owner[m.partner[g]];
      if (across < 0 || across == owner) continue;
      double ux = m.faceNormal[2 * g], uy = m.faceNormal[2 * g + 1];
      if (m.owner[g] != owner) {
        ux = ux * -1.0;
        uy = uy * -1.0;
      }
      const double alignment = ux * nx + uy * ny;
      if (alignment > bestAlignment) {
        bestAlignment = alignment;
        best = across;
      }
    }
    t.second.push_back(best);
    double d2 = 0.0;
    if (best >= 0) {
      const double qx = m.centroid[2 * best] - cx, qy = m.centroid[2 * best + 1] - cy;
      d2 = std::abs(qx * nx + qy * ny);
    }
    t.outerDistance.push_back(d2);
  }
  // leading edge: the first station whose first node is furthest forward
  // (SurfaceData.cpp:238-250)
  double forward = 1.7976931348623157e308;
  t.leadingEdge = 0;
  for (std::size_t k = 0; k < t.node0x.size(); ++k) {
    if (t.node0x[k] < forward) {
      forward = t.node0x[k];
      t.leadingEdge = static_cast<int>(k);
    }
  }
  return ok();
}

Status launchForces(const WallTable& w, const double* p, const double* u, const double* v,
                    const double* mu, double dynamicPressure, double referencePressure,
                    double chord, double cosA, double sinA, double* station, double* out,
                    cudaStream_t stream) {
  ForceParams fp{dynamicPressure, referencePressure, chord, cosA, sinA};
  forcesKernel<<<1, 256, 0, stream>>>(w, p, u, v, mu, fp, station, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  return ok();
}

}  // namespace cfdb
