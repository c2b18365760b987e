// common.hpp - host-side types shared by the mesh builder, the solver front
// end and the C ABI: status codes with a thread-local message, and the
// face-based host mesh (the arrays of cfd::mesh::Mesh, Mesh.hpp:121-190).
#pragma once

#include <string>
#include <vector>

#include "cfd_gpu.h"

namespace cfdb {

using Status = cfd_status;

/// Record a failure message for cfd_last_error() and return the code.
Status fail(Status code, const std::string& message);
inline Status ok() { return CFD_OK; }

struct HostMesh {
  int nodesI{0}, nodesJ{0};
  int cells{0}, faces{0};
  std::vector<double> nodes;       // 2 * nodes
  std::vector<double> centroid;    // 2 * cells
  std::vector<double> cellArea;    // cells
  std::vector<double> faceCentre;  // 2 * faces
  std::vector<double> faceNormal;  // 2 * faces
  std::vector<double> faceArea;    // faces
  std::vector<int> owner, neighbour, boundary, partner;  // faces
  double totalArea{0.0};
};

inline void describe(const HostMesh& g, cfd_mesh_desc* d) {
  d->nodes_i = g.nodesI;
  d->nodes_j = g.nodesJ;
  d->cell_count = g.cells;
  d->face_count = g.faces;
  d->cell_centroids = g.centroid.data();
  d->cell_areas = g.cellArea.data();
  d->face_centres = g.faceCentre.data();
  d->face_normals = g.faceNormal.data();
  d->face_areas = g.faceArea.data();
  d->face_owner = g.owner.data();
  d->face_neighbour = g.neighbour.data();
  d->face_boundary = g.boundary.data();
  d->face_partner = g.partner.data();
  d->nodes = g.nodes.data();
}

}  // namespace cfdb
