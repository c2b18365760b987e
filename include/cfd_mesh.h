/* cfd_mesh.h - host-side generation of the structured meshes the solver runs
 * on: NACA 4-digit C-grids and Cartesian boxes.
 *
 * The reference builds these in C++ (include/cfd/mesh/CGrid.hpp:95-96,
 * include/cfd/mesh/BoxGrid.hpp:282, include/cfd/mesh/Mesh.hpp:209); a caller
 * that already holds a cfd::mesh::Mesh passes its arrays to cfd_gpu_create
 * directly and never needs this file. It exists so the library can also mesh
 * a request on its own (batch and serving front ends, benchmarks). Results
 * match the reference's meshes to the last bit on the same host libm.
 */
#ifndef CFD_MESH_H
#define CFD_MESH_H

#include "cfd_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfd_mesh_t* cfd_mesh;

/* mesh::CGridOptions (CGrid.hpp:53-81) for a closed-trailing-edge NACA
 * section of chord 1 (geom::makeNaca4Digit, Airfoil.hpp:485-486). */
typedef struct cfd_cgrid_options {
  double upstream_chords;        /* 12 */
  double downstream_chords;      /* 25 */
  double vertical_chords;        /* 12 */
  int surface_points;            /* 160 */
  int wake_points;               /* 56 */
  int normal_points;             /* 72 */
  double first_layer_height;     /* 3e-4 */
  double normal_blend_length;    /* 0.06 */
  int normal_smoothing_passes;   /* 6 */
} cfd_cgrid_options;

void cfd_default_cgrid_options(cfd_cgrid_options* out);

/* generateCGrid (CGrid.cpp:98-399). designation is four digits ("0012"). */
cfd_status cfd_mesh_cgrid(const char* designation, const cfd_cgrid_options* options,
                          cfd_mesh* out);

/* generateBox (BoxGrid.cpp:7-65). grading: 0 uniform, 1 toward lower, 2 both.
 * Sides take CFD_FACE_* boundary types. */
cfd_status cfd_mesh_box(double origin_x, double origin_y, double length, double height,
                        int cells_x, int cells_y, int grading, double first_cell_height,
                        int left, int right, int lower, int upper, cfd_mesh* out);

/* Borrowed view of the mesh's arrays, valid until cfd_mesh_free. */
cfd_status cfd_mesh_describe(cfd_mesh m, cfd_mesh_desc* out);
/* Node coordinates, 2 * nodes_i * nodes_j doubles, row-major (j, i). */
const double* cfd_mesh_nodes(cfd_mesh m);

/* buildFaceConditions with the default BoundaryConditions
 * (BoundaryConditions.cpp:73-97): wall -> no-slip, far field -> FarField,
 * outlet -> Outlet, interior and wake cut -> Internal; pressure = 0,
 * velocity = freestream (zero on walls). kind: faces ints; velocity 2*faces. */
cfd_status cfd_mesh_face_conditions(cfd_mesh m, double speed, double alpha_deg, int* kind,
                                    double* velocity, double* pressure);

void cfd_mesh_free(cfd_mesh m);

#ifdef __cplusplus
}
#endif
#endif /* CFD_MESH_H */
