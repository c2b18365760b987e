/* cfd_oracle.h - CPU restatement of the reference's steady SIMPLE solve
 * (laminar and k-omega SST) on a face-based structured mesh.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the device solver is compared with.
 * It is never linked into, called by, or substituted for the product library.
 *
 * It follows, loop for loop, src/solver/SimpleSolver.cpp, LinearSystem.cpp,
 * Gradient.cpp, KOmegaSST.cpp and TurbulenceModel.cpp of the reference, in
 * the reference's own face-loop (scatter) form. Two Gauss-Seidel orders are
 * offered: lexicographic (the reference's) and red-black (the device
 * solver's). Field and stage identifiers are the CFD_FIELD_* / CFD_STAGE_*
 * values of include/cfd_gpu.h.
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_mesh {
  int nodes_i, nodes_j, cells, faces;
  const double* centroid;     /* 2*cells */
  const double* cell_area;    /* cells */
  const double* face_centre;  /* 2*faces */
  const double* face_normal;  /* 2*faces */
  const double* face_area;    /* faces */
  const int* owner;
  const int* neighbour;
  const int* boundary;        /* mesh::BoundaryType */
  const int* partner;
} or_mesh;

typedef struct or_solver or_solver;

/* settings: the 12 SimpleSettings values {alphaU, alphaP, sweeps, cgMax,
 * cgTol, scheme, alphaT, intensity, viscosityRatio, lengthScale, nCorr,
 * blend}. model: 0 none, 1 laminar closure, 2 SST. gs_order is a bit mask:
 * bit 0 sweeps the momentum equations red-black, bit 1 the k and omega
 * equations; 0 is the reference (all lexicographic), 1 the device solver.
 * The mesh arrays must outlive the solver. NULL on invalid input. */
or_solver* or_create(const or_mesh* mesh, const int* kind, const double* velocity,
                     const double* pressure, const double* settings, int model, int gs_order);
int or_initialise(or_solver* s, const double* u, const double* v, const double* p,
                  const double* rho, const double* mu);
/* n iterations; the first one stops after stop_stage (CFD_STAGE_END = 10 for
 * whole ones). monitor: 16 doubles per iteration (cfd_monitor's layout
 * without the padding int: continuity, momX, momY, massImbalance, maxDiv,
 * cgIterations, turb1, turb2, minK, maxK, minW, maxW, minMut, maxMut,
 * maxRatio, maxYPlus). Returns iterations run. */
int or_iterate(or_solver* s, int n, int stop_stage, double* monitor);
int or_read(or_solver* s, int which, double* out);
void or_load_state(or_solver* s, const double* u, const double* v, const double* p,
                   const double* mass_flux, const double* k, const double* omega,
                   const double* mut, const double* mu_eff);
/* {kInflow, omegaInflow, referenceMassFlow} */
void or_scalars(or_solver* s, double* out3);
void or_free(or_solver* s);
const char* or_last_error(void);

/* LDU primitives (LinearSystem.cpp), on the same mesh layout; gs_order 0
 * lexicographic, 1 red-black. */
void or_ldu_multiply(const or_mesh* m, const double* diag, const double* upper,
                     const double* lower, const double* x, double* y);
void or_ldu_gauss_seidel(const or_mesh* m, const double* diag, const double* source,
                         const double* upper, const double* lower, double* x, int sweeps,
                         int gs_order);
/* report = {iterations, initialResidual, finalResidual, converged} */
void or_ldu_cg(const or_mesh* m, const double* diag, const double* source, const double* upper,
               const double* lower, double* x, double tolerance, int max_iterations,
               double* report);
void or_green_gauss(const or_mesh* m, const double* face_values, double* out);

#ifdef __cplusplus
}
#endif
#endif /* CFD_ORACLE_H */
