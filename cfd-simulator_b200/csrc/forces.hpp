// forces.hpp - the wall station table and the device force integration.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.hpp"

namespace cfdb {

/// Values stored per station by the force kernel: pressure, Cp, wall shear,
/// Cf, flow-direction tangent (x, y).
constexpr int kStationValues = 6;

/// Mesh-only data of the wall stations, in contour (i) order, on the host.
struct HostWallTable {
  std::vector<int> face, owner, second;
  std::vector<double> cx, cy, tx, ty, nx, ny, length, node0x, wallDistance, outerDistance;
  int leadingEdge{0};
  int count() const { return static_cast<int>(owner.size()); }
};

/// The same, as device pointers (passed by value to the kernel).
struct WallTable {
  int count{0};
  int leadingEdge{0};
  const int* owner{nullptr};
  const int* second{nullptr};
  const double *cx{nullptr}, *cy{nullptr}, *tx{nullptr}, *ty{nullptr}, *nx{nullptr}, *ny{nullptr};
  const double *length{nullptr}, *wallDistance{nullptr}, *outerDistance{nullptr};
};

/// Tabulate the wall stations from a structured C-grid (needs node
/// coordinates; with none, the table stays empty).
Status buildWallTable(const HostMesh& mesh, const double* nodes, HostWallTable* out);

/// Launch the force integration; out gets 12 doubles (cfd_forces order:
/// Cl, Cd, Cm, Cd_p, Cd_f, lift, drag, moment, stagnation x/c, stations,
/// separation x/c on the upper and the lower surface or -1).
Status launchForces(const WallTable& w, const double* p, const double* u, const double* v,
                    const double* mu, double dynamicPressure, double referencePressure,
                    double chord, double cosA, double sinA, double* station, double* out,
                    cudaStream_t stream);

}  // namespace cfdb
