// ref_harness.cpp - a thin C accessor over the reference's own solver
// libraries, compiled from the reference sources by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product links this file; it exists
// so that golden fixtures (tests/golden/make_golden.py) and the CPU baseline
// leg of bench.py can drive the unmodified reference code path:
//
//   generateCGrid / generateBox -> buildFaceConditions -> SimpleSolver::create
//   -> setTurbulenceModel -> initialise(FlowField::uniform) -> iterate()
//   (src/solver/SimpleSolver.cpp:30-80, :133-210, :662-794)
//
// Stage outputs that the reference keeps private (face values, gradients, the
// momentum and pressure-correction LDU systems, SST blending fields) are read
// by compiling this one translation unit with `private`/`protected` mapped to
// `public` *after* every standard header has been included. The reference's
// own translation units are compiled unchanged; GCC lays out a class the same
// way regardless of access specifiers, so the accessors read the real objects.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <deque>
#include <format>
#include <memory>
#include <optional>
#include <source_location>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

#define private public
#define protected public
#include "cfd/flow/BoundaryConditions.hpp"
#include "cfd/flow/FlowField.hpp"
#include "cfd/flow/Freestream.hpp"
#include "cfd/geom/Airfoil.hpp"
#include "cfd/geom/Naca4.hpp"
#include "cfd/mesh/BoxGrid.hpp"
#include "cfd/mesh/CGrid.hpp"
#include "cfd/mesh/Mesh.hpp"
#include "cfd/post/Forces.hpp"
#include "cfd/post/Polar.hpp"
#include "cfd/post/Streamlines.hpp"
#include "cfd/post/SurfaceData.hpp"
#include "cfd/solver/Gradient.hpp"
#include "cfd/solver/KOmegaSST.hpp"
#include "cfd/solver/LinearSystem.hpp"
#include "cfd/solver/SimpleSolver.hpp"
#include "cfd/solver/TurbulenceModel.hpp"
#undef private
#undef protected

using cfd::Vec2;
namespace mesh = cfd::mesh;
namespace flow = cfd::flow;
namespace solver = cfd::solver;

namespace {

thread_local std::string g_error;

struct RefMesh {
  mesh::Mesh mesh;
};

struct RefSolver {
  const RefMesh* mesh{nullptr};
  std::optional<solver::SimpleSolver> solver;
  solver::KOmegaSST* sst{nullptr};  // owned by the solver once attached
  solver::SolverMonitor last{};
};

void copyVec2(const std::vector<Vec2>& in, double* out) {
  for (std::size_t k = 0; k < in.size(); ++k) {
    out[2 * k] = in[k].x;
    out[2 * k + 1] = in[k].y;
  }
}

void copyDouble(const std::vector<double>& in, double* out) {
  std::memcpy(out, in.data(), in.size() * sizeof(double));
}

solver::SimpleSettings unpackSettings(const double* s) {
  solver::SimpleSettings settings;
  settings.velocityRelaxation = s[0];
  settings.pressureRelaxation = s[1];
  settings.momentumSweeps = static_cast<int>(s[2]);
  settings.pressureIterations = static_cast<int>(s[3]);
  settings.pressureTolerance = s[4];
  settings.scheme = (s[5] != 0.0) ? solver::ConvectionScheme::SecondOrderUpwind
                                  : solver::ConvectionScheme::Upwind;
  settings.turbulenceRelaxation = s[6];
  settings.inflow.intensity = s[7];
  settings.inflow.viscosityRatio = s[8];
  settings.inflow.lengthScale = s[9];
  settings.nonOrthogonalCorrectors = static_cast<int>(s[10]);
  settings.nonOrthogonalBlend = s[11];
  return settings;
}

void packMonitor(const solver::SolverMonitor& m, double* out) {
  out[0] = m.residuals.continuity;
  out[1] = m.residuals.momentumX;
  out[2] = m.residuals.momentumY;
  out[3] = m.massImbalance;
  out[4] = m.maxDivergence;
  out[5] = static_cast<double>(m.pressureIterations);
  out[6] = m.turbulence.first;
  out[7] = m.turbulence.second;
  out[8] = m.turbulenceRanges.minEnergy;
  out[9] = m.turbulenceRanges.maxEnergy;
  out[10] = m.turbulenceRanges.minDissipation;
  out[11] = m.turbulenceRanges.maxDissipation;
  out[12] = m.turbulenceRanges.minEddyViscosity;
  out[13] = m.turbulenceRanges.maxEddyViscosity;
  out[14] = m.maxEddyViscosityRatio;
}

solver::TurbulenceContext contextOf(RefSolver* r) {
  solver::SimpleSolver& s = *r->solver;
  solver::TurbulenceContext context;
  context.mesh = s.mesh_;
  context.field = &s.field_;
  context.conditions = &s.conditions_;
  context.massFlux = &s.massFlux_;
  context.gradU = &s.gradU_;
  context.gradV = &s.gradV_;
  context.molecularViscosity = &s.molecularViscosity_;
  context.relaxation = s.settings_.turbulenceRelaxation;
  return context;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// ---------------------------------------------------------------- meshes ---

void* ref_mesh_cgrid(const char* designation, int surfacePoints, int wakePoints,
                     int normalPoints, double firstLayer, double upstream, double downstream,
                     double vertical, double blendLength, int smoothingPasses) {
  auto section = cfd::geom::makeNaca4Digit(
      designation, {.chord = 1.0, .trailingEdge = cfd::geom::TrailingEdge::Closed});
  if (!section) {
    g_error = section.error().format();
    return nullptr;
  }
  mesh::CGridOptions options;
  options.surfacePoints = surfacePoints;
  options.wakePoints = wakePoints;
  options.normalPoints = normalPoints;
  options.firstLayerHeight = firstLayer;
  options.upstreamChords = upstream;
  options.downstreamChords = downstream;
  options.verticalChords = vertical;
  options.normalBlendLength = blendLength;
  options.normalSmoothingPasses = smoothingPasses;
  auto grid = mesh::generateCGrid(section.value(), options);
  if (!grid) {
    g_error = grid.error().format();
    return nullptr;
  }
  return new RefMesh{std::move(grid).value()};
}

void* ref_mesh_box(double originX, double originY, double length, double height, int cellsX,
                   int cellsY, int grading, double firstCellHeight, int left, int right,
                   int lower, int upper) {
  mesh::BoxOptions options;
  options.originX = originX;
  options.originY = originY;
  options.length = length;
  options.height = height;
  options.cellsX = cellsX;
  options.cellsY = cellsY;
  options.grading = static_cast<mesh::Grading>(grading);
  options.firstCellHeight = firstCellHeight;
  options.left = static_cast<mesh::BoundaryType>(left);
  options.right = static_cast<mesh::BoundaryType>(right);
  options.lower = static_cast<mesh::BoundaryType>(lower);
  options.upper = static_cast<mesh::BoundaryType>(upper);
  auto grid = mesh::generateBox(options);
  if (!grid) {
    g_error = grid.error().format();
    return nullptr;
  }
  return new RefMesh{std::move(grid).value()};
}

void ref_mesh_free(void* m) { delete static_cast<RefMesh*>(m); }

/// out = {nodesI, nodesJ, cells, faces}
void ref_mesh_counts(void* m, int* out) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  out[0] = g.nodesI();
  out[1] = g.nodesJ();
  out[2] = static_cast<int>(g.cellCount());
  out[3] = static_cast<int>(g.faceCount());
}

/// Every array the Mesh exposes, in its own order. Vec2 arrays are (x, y)
/// pairs. boundary uses mesh::BoundaryType's enumerator values.
void ref_mesh_arrays(void* m, double* nodes, double* centroids, double* cellAreas,
                     double* faceCentres, double* faceNormals, double* faceAreas, int* owner,
                     int* neighbour, int* boundary, int* partner) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  copyVec2(g.nodes(), nodes);
  copyVec2(g.cellCentroids(), centroids);
  copyDouble(g.cellAreas(), cellAreas);
  copyVec2(g.faceCentres(), faceCentres);
  copyVec2(g.faceNormals(), faceNormals);
  copyDouble(g.faceAreas(), faceAreas);
  for (std::size_t f = 0; f < g.faceCount(); ++f) {
    owner[f] = g.faces()[f].owner;
    neighbour[f] = g.faces()[f].neighbour;
    boundary[f] = static_cast<int>(g.faces()[f].boundary);
    partner[f] = g.faces()[f].partner;
  }
}

/// buildFaceConditions with default BoundaryConditions (wall = NoSlipWall,
/// far field = FarField, outlet = Outlet). kinds use flow::BoundaryKind values.
int ref_face_conditions(void* m, double speed, double alphaDeg, double density,
                        double reynolds, int* kinds, double* velocity, double* pressure) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  flow::FreestreamConditions stream;
  stream.speed = speed;
  stream.angleOfAttackDeg = alphaDeg;
  stream.density = density;
  stream.reynoldsNumber = reynolds;
  auto conditions = flow::buildFaceConditions(g, flow::BoundaryConditions{}, stream);
  if (!conditions) {
    g_error = conditions.error().format();
    return 1;
  }
  for (std::size_t f = 0; f < g.faceCount(); ++f) {
    kinds[f] = static_cast<int>(conditions.value()[f].kind);
    velocity[2 * f] = conditions.value()[f].velocity.x;
    velocity[2 * f + 1] = conditions.value()[f].velocity.y;
    pressure[f] = conditions.value()[f].pressure;
  }
  return 0;
}

/// FlowField::uniform for a freestream; out arrays are per cell.
int ref_uniform_field(void* m, double speed, double alphaDeg, double density, double reynolds,
                      double chord, double* u, double* v, double* p, double* rho, double* mu) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  flow::FreestreamConditions stream;
  stream.speed = speed;
  stream.angleOfAttackDeg = alphaDeg;
  stream.density = density;
  stream.reynoldsNumber = reynolds;
  auto field = flow::FlowField::uniform(g.cellCount(), stream, chord);
  if (!field) {
    g_error = field.error().format();
    return 1;
  }
  for (std::size_t c = 0; c < g.cellCount(); ++c) {
    u[c] = field.value().velocity[c].x;
    v[c] = field.value().velocity[c].y;
    p[c] = field.value().pressure[c];
    rho[c] = field.value().density[c];
    mu[c] = field.value().viscosity[c];
  }
  return 0;
}

// ---------------------------------------------------------------- solver ---

/// turbulence: 0 = none (laminar), 1 = LaminarModel, 2 = KOmegaSST.
void* ref_solver_create(void* m, const int* kinds, const double* velocity,
                        const double* pressure, const double* settings, int turbulence) {
  RefMesh* rm = static_cast<RefMesh*>(m);
  const mesh::Mesh& g = rm->mesh;
  flow::FaceConditions conditions(g.faceCount());
  for (std::size_t f = 0; f < g.faceCount(); ++f) {
    conditions[f].kind = static_cast<flow::BoundaryKind>(kinds[f]);
    conditions[f].velocity = Vec2{velocity[2 * f], velocity[2 * f + 1]};
    conditions[f].pressure = pressure[f];
  }
  auto created = solver::SimpleSolver::create(g, std::move(conditions), unpackSettings(settings));
  if (!created) {
    g_error = created.error().format();
    return nullptr;
  }
  auto* r = new RefSolver;
  r->mesh = rm;
  r->solver.emplace(std::move(created).value());
  if (turbulence == 1) {
    (void)r->solver->setTurbulenceModel(std::make_unique<solver::LaminarModel>());
  } else if (turbulence == 2) {
    auto model = std::make_unique<solver::KOmegaSST>();
    r->sst = model.get();
    (void)r->solver->setTurbulenceModel(std::move(model));
  }
  return r;
}

void ref_solver_free(void* s) { delete static_cast<RefSolver*>(s); }

int ref_solver_initialise(void* s, const double* u, const double* v, const double* p,
                          const double* rho, const double* mu) {
  RefSolver* r = static_cast<RefSolver*>(s);
  const std::size_t n = r->mesh->mesh.cellCount();
  flow::FlowField field;
  field.resize(n);
  for (std::size_t c = 0; c < n; ++c) {
    field.velocity[c] = Vec2{u[c], v[c]};
    field.pressure[c] = p[c];
    field.density[c] = rho[c];
    field.viscosity[c] = mu[c];
  }
  const cfd::Status st = r->solver->initialise(field);
  if (!st) {
    g_error = st.error().format();
    return 1;
  }
  return 0;
}

/// Run n outer iterations; monitor (15 doubles, see packMonitor) of the last.
/// history, if not null, receives 15 doubles per iteration.
void ref_solver_iterate(void* s, int n, double* monitor, double* history) {
  RefSolver* r = static_cast<RefSolver*>(s);
  for (int k = 0; k < n; ++k) {
    r->last = r->solver->iterate();
    if (history != nullptr) {
      packMonitor(r->last, history + 15 * k);
    }
  }
  if (monitor != nullptr) {
    packMonitor(r->last, monitor);
  }
}

/// Iterate until worst() < tol (the worker's stop rule) or the cap; returns
/// the iterations taken.
int ref_solver_converge(void* s, int cap, double tol, double* monitor) {
  RefSolver* r = static_cast<RefSolver*>(s);
  int taken = 0;
  while (taken < cap) {
    r->last = r->solver->iterate();
    ++taken;
    if (!std::isfinite(r->last.residuals.worst())) break;
    if (r->last.residuals.worst() < tol) break;
  }
  if (monitor != nullptr) packMonitor(r->last, monitor);
  return taken;
}

// Field identifiers for ref_solver_read. Cell arrays unless marked (F) for
// per-face, (2N) for Vec2 per cell.
enum RefField {
  kU = 0, kV, kP, kRho, kMuEff, kMassFlux /*F*/, kDivergence, kMuMolecular,
  kFaceU /*F*/, kFaceV /*F*/, kFaceP /*F*/, kGradU /*2N*/, kGradV /*2N*/, kGradP /*2N*/,
  kMomDiag, kMomSource, kMomUpper /*F*/, kMomLower /*F*/, kMomentumDiagonal,
  kPDiag, kPSource, kPUpper /*F*/, kPLower /*F*/, kNetFlux, kDeadBand /*F*/,
  kGeomArea /*2F*/, kGeomDelta /*2F*/, kGeomTangential /*2F*/, kGeomDiffusion /*F*/,
  kGeomWeight /*F*/,
  kK, kOmega, kMut, kWallDistance, kStrain, kF1, kF2, kCrossDiffusion, kProduction,
  kGradK /*2N*/, kGradOmega /*2N*/,
};

int ref_solver_read(void* s, int which, double* out) {
  RefSolver* r = static_cast<RefSolver*>(s);
  solver::SimpleSolver& sv = *r->solver;
  const auto& field = sv.field_;
  switch (which) {
    case kU: for (std::size_t c = 0; c < field.size(); ++c) out[c] = field.velocity[c].x; return 0;
    case kV: for (std::size_t c = 0; c < field.size(); ++c) out[c] = field.velocity[c].y; return 0;
    case kP: copyDouble(field.pressure, out); return 0;
    case kRho: copyDouble(field.density, out); return 0;
    case kMuEff: copyDouble(field.viscosity, out); return 0;
    case kMassFlux: copyDouble(sv.massFlux_, out); return 0;
    case kDivergence: copyDouble(sv.divergence(), out); return 0;
    case kMuMolecular: copyDouble(sv.molecularViscosity_, out); return 0;
    case kFaceU: copyDouble(sv.faceU_, out); return 0;
    case kFaceV: copyDouble(sv.faceV_, out); return 0;
    case kFaceP: copyDouble(sv.faceP_, out); return 0;
    case kGradU: copyVec2(sv.gradU_, out); return 0;
    case kGradV: copyVec2(sv.gradV_, out); return 0;
    case kGradP: copyVec2(sv.gradP_, out); return 0;
    case kMomDiag: copyDouble(sv.momentum_.diagonal, out); return 0;
    case kMomSource: copyDouble(sv.momentum_.source, out); return 0;
    case kMomUpper: copyDouble(sv.momentum_.upper, out); return 0;
    case kMomLower: copyDouble(sv.momentum_.lower, out); return 0;
    case kMomentumDiagonal: copyDouble(sv.momentumDiagonal_, out); return 0;
    case kPDiag: copyDouble(sv.pressure_.diagonal, out); return 0;
    case kPSource: copyDouble(sv.pressure_.source, out); return 0;
    case kPUpper: copyDouble(sv.pressure_.upper, out); return 0;
    case kPLower: copyDouble(sv.pressure_.lower, out); return 0;
    case kNetFlux: copyDouble(sv.netFlux_, out); return 0;
    case kDeadBand: copyDouble(sv.farFieldDeadBand_, out); return 0;
    case kGeomArea:
      for (std::size_t f = 0; f < sv.geometry_.size(); ++f) {
        out[2 * f] = sv.geometry_[f].area.x;
        out[2 * f + 1] = sv.geometry_[f].area.y;
      }
      return 0;
    case kGeomDelta:
      for (std::size_t f = 0; f < sv.geometry_.size(); ++f) {
        out[2 * f] = sv.geometry_[f].delta.x;
        out[2 * f + 1] = sv.geometry_[f].delta.y;
      }
      return 0;
    case kGeomTangential:
      for (std::size_t f = 0; f < sv.geometry_.size(); ++f) {
        out[2 * f] = sv.geometry_[f].tangential.x;
        out[2 * f + 1] = sv.geometry_[f].tangential.y;
      }
      return 0;
    case kGeomDiffusion:
      for (std::size_t f = 0; f < sv.geometry_.size(); ++f) out[f] = sv.geometry_[f].diffusion;
      return 0;
    case kGeomWeight:
      for (std::size_t f = 0; f < sv.geometry_.size(); ++f) out[f] = sv.geometry_[f].ownerWeight;
      return 0;
    default: break;
  }
  if (r->sst == nullptr) {
    g_error = "no SST model attached";
    return 1;
  }
  solver::KOmegaSST& t = *r->sst;
  switch (which) {
    case kK: copyDouble(t.k_, out); return 0;
    case kOmega: copyDouble(t.omega_, out); return 0;
    case kMut: copyDouble(t.eddyViscosity_, out); return 0;
    case kWallDistance: copyDouble(t.wallDistance_, out); return 0;
    case kStrain: copyDouble(t.strain_, out); return 0;
    case kF1: copyDouble(t.f1_, out); return 0;
    case kF2: copyDouble(t.f2_, out); return 0;
    case kCrossDiffusion: copyDouble(t.crossDiffusion_, out); return 0;
    case kProduction: copyDouble(t.production_, out); return 0;
    case kGradK: copyVec2(t.gradK_, out); return 0;
    case kGradOmega: copyVec2(t.gradOmega_, out); return 0;
    default: break;
  }
  g_error = "unknown field";
  return 1;
}

/// SST scalars: {kInflow, omegaInflow, maxYPlus, residual k, residual omega}.
int ref_sst_scalars(void* s, double* out) {
  RefSolver* r = static_cast<RefSolver*>(s);
  if (r->sst == nullptr) return 1;
  out[0] = r->sst->kInflow_;
  out[1] = r->sst->omegaInflow_;
  out[2] = r->sst->maxYPlus_;
  out[3] = r->sst->residuals_.first;
  out[4] = r->sst->residuals_.second;
  return 0;
}

/// Solver scalars: {referenceMassFlow, hasPressureReference}.
void ref_solver_scalars(void* s, double* out) {
  RefSolver* r = static_cast<RefSolver*>(s);
  out[0] = r->solver->referenceMassFlow_;
  out[1] = r->solver->hasPressureReference_ ? 1.0 : 0.0;
}

// Stages of one outer iteration, each the reference's own member function.
enum RefStage {
  kInterpolate = 0, kGradients, kAssembleU, kAssembleV, kRelaxU, kRelaxV, kRhieChow,
  kAssemblePressure, kApplyEddyViscosity,
  kSstStrain, kSstBlending, kSstTransport, kSstWall, kSstEddy, kSstRanges,
};

int ref_solver_stage(void* s, int stage) {
  RefSolver* r = static_cast<RefSolver*>(s);
  solver::SimpleSolver& sv = *r->solver;
  switch (stage) {
    case kInterpolate: sv.interpolateFaceValues(); return 0;
    case kGradients: sv.computeGradients(); return 0;
    case kAssembleU: sv.assembleMomentum(0); return 0;
    case kAssembleV: sv.assembleMomentum(1); return 0;
    case kRelaxU: sv.applyRelaxation(0); return 0;
    case kRelaxV: sv.applyRelaxation(1); return 0;
    case kRhieChow: sv.computeRhieChowFluxes(); return 0;
    case kAssemblePressure: sv.assemblePressureCorrection(); return 0;
    case kApplyEddyViscosity: sv.applyEddyViscosity(); return 0;
    default: break;
  }
  if (r->sst == nullptr) return 1;
  const solver::TurbulenceContext context = contextOf(r);
  switch (stage) {
    case kSstStrain: r->sst->computeStrain(context); return 0;
    case kSstBlending: r->sst->computeBlending(context); return 0;
    case kSstTransport: r->sst->solveTransport(context); return 0;
    case kSstWall: r->sst->applyWallConditions(context); return 0;
    case kSstEddy: r->sst->updateEddyViscosity(context); return 0;
    case kSstRanges: r->sst->updateRanges(); return 0;
    default: break;
  }
  return 1;
}

/// correct(p') with a caller-supplied correction (SimpleSolver.cpp:582-660).
void ref_solver_correct(void* s, const double* correction) {
  RefSolver* r = static_cast<RefSolver*>(s);
  std::vector<double> pc(correction, correction + r->mesh->mesh.cellCount());
  r->solver->correct(pc);
}

/// Copy the momentum system's current momentum_.diagonal into
/// momentumDiagonal_, as iterate() does after the x-component solve.
void ref_solver_keep_momentum_diagonal(void* s) {
  RefSolver* r = static_cast<RefSolver*>(s);
  r->solver->momentumDiagonal_ = r->solver->momentum_.diagonal;
}

// ---------------------------------------------------- linear algebra ---

namespace {
solver::LinearSystem systemOf(const mesh::Mesh& g, const double* diag, const double* source,
                              const double* upper, const double* lower) {
  solver::LinearSystem sys(g.cellCount(), g.faceCount());
  std::copy(diag, diag + g.cellCount(), sys.diagonal.begin());
  std::copy(source, source + g.cellCount(), sys.source.begin());
  std::copy(upper, upper + g.faceCount(), sys.upper.begin());
  std::copy(lower, lower + g.faceCount(), sys.lower.begin());
  return sys;
}
}  // namespace

/// y = A x (LinearSystem::multiply, LinearSystem.cpp:18-43).
void ref_ldu_multiply(void* m, const double* diag, const double* upper, const double* lower,
                      const double* x, double* y) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  std::vector<double> zero(g.cellCount(), 0.0);
  const solver::LinearSystem sys = systemOf(g, diag, zero.data(), upper, lower);
  std::vector<double> xv(x, x + g.cellCount());
  std::vector<double> yv;
  sys.multiply(g, xv, yv);
  copyDouble(yv, y);
}

/// gaussSeidel in place (LinearSystem.cpp:77-116).
void ref_ldu_gauss_seidel(void* m, const double* diag, const double* source,
                          const double* upper, const double* lower, double* x, int sweeps) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  const solver::LinearSystem sys = systemOf(g, diag, source, upper, lower);
  std::vector<double> xv(x, x + g.cellCount());
  solver::gaussSeidel(g, sys, xv, sweeps);
  copyDouble(xv, x);
}

/// conjugateGradient (LinearSystem.cpp:118-210); report = {iterations,
/// initialResidual, finalResidual, converged}.
void ref_ldu_cg(void* m, const double* diag, const double* source, const double* upper,
                const double* lower, double* x, double tolerance, int maxIterations,
                double* report) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  const solver::LinearSystem sys = systemOf(g, diag, source, upper, lower);
  std::vector<double> xv(x, x + g.cellCount());
  const solver::SolveReport rep = solver::conjugateGradient(g, sys, xv, tolerance, maxIterations);
  copyDouble(xv, x);
  report[0] = rep.iterations;
  report[1] = rep.initialResidual;
  report[2] = rep.finalResidual;
  report[3] = rep.converged ? 1.0 : 0.0;
}

/// greenGaussGradient (Gradient.cpp:20-50); out is (x, y) per cell.
void ref_green_gauss(void* m, const double* faceValues, double* out) {
  const mesh::Mesh& g = static_cast<RefMesh*>(m)->mesh;
  std::vector<double> fv(faceValues, faceValues + g.faceCount());
  auto grad = solver::greenGaussGradient(g, fv);
  copyVec2(grad.value(), out);
}

// ------------------------------------------------------------------ post ---

/// extractSurface + integrateForces on the solver's current field
/// (SurfaceData.cpp:208-348, Forces.cpp:60-130). out = {Cl, Cd, Cm, Cd_p,
/// Cd_f, stations, upper and lower separation x/c or -1}; cp, if not null,
/// receives Cp for upper then lower stations.
int ref_forces(void* s, double speed, double alphaDeg, double density, double reynolds,
               double chord, double* out, double* cp) {
  RefSolver* r = static_cast<RefSolver*>(s);
  flow::FreestreamConditions stream;
  stream.speed = speed;
  stream.angleOfAttackDeg = alphaDeg;
  stream.density = density;
  stream.reynoldsNumber = reynolds;
  auto surface = cfd::post::extractSurface(r->mesh->mesh, r->solver->field(), stream, chord);
  if (!surface) {
    g_error = surface.error().format();
    return 1;
  }
  auto forces = cfd::post::integrateForces(surface.value(), stream);
  if (!forces) {
    g_error = forces.error().format();
    return 1;
  }
  const auto& fv = forces.value();
  out[0] = fv.liftCoefficient;
  out[1] = fv.dragCoefficient;
  out[2] = fv.momentCoefficient;
  out[3] = fv.pressureDragCoefficient;
  out[4] = fv.frictionDragCoefficient;
  out[5] = static_cast<double>(fv.stations);
  const auto& sd = surface.value();
  out[6] = sd.upperSeparation.found ? sd.upperSeparation.chordFraction : -1.0;
  out[7] = sd.lowerSeparation.found ? sd.lowerSeparation.chordFraction : -1.0;
  if (cp != nullptr) {
    std::size_t k = 0;
    for (const auto& point : surface.value().upper) cp[k++] = point.pressureCoefficient;
    for (const auto& point : surface.value().lower) cp[k++] = point.pressureCoefficient;
  }
  return 0;
}

// ----------------------------------------------------------------- polar ---

/// post::sweepAngles (Polar.cpp:36-77): the angle count, written to `out`
/// when it has room; -1 on the reference's refusal (message in
/// ref_last_error).
int ref_sweep_angles(double start, double end, double step, double* out, int capacity) {
  auto angles = cfd::post::sweepAngles(start, end, step);
  if (!angles) {
    g_error = angles.error().message();
    return -1;
  }
  const auto& a = angles.value();
  for (std::size_t k = 0; k < a.size() && static_cast<int>(k) < capacity; ++k) out[k] = a[k];
  return static_cast<int>(a.size());
}

/// post::toCsv (Polar.cpp:126-164) of a polar given point by point: 13
/// doubles per point {alpha, cl, cd, cd_pressure, cd_friction, cm, l_over_d,
/// upper separation, lower separation, converged, diverged, iterations,
/// continuity residual}. Returns the text's length; writes it (not
/// terminated) when it fits `capacity`.
int ref_polar_csv(const char* section, const char* mesh, double reynolds, double speed, double chord,
                  double momentReference, int continued, int n, const double* points, char* out,
                  int capacity) {
  cfd::post::Polar polar;
  polar.section = section;
  polar.meshResolution = mesh;
  polar.reynoldsNumber = reynolds;
  polar.machEquivalentSpeed = speed;
  polar.chord = chord;
  polar.momentReferenceFraction = momentReference;
  polar.continuedBetweenPoints = continued != 0;
  for (int k = 0; k < n; ++k) {
    const double* v = points + 13 * k;
    cfd::post::PolarPoint p;
    p.angleOfAttackDeg = v[0];
    p.liftCoefficient = v[1];
    p.dragCoefficient = v[2];
    p.pressureDragCoefficient = v[3];
    p.frictionDragCoefficient = v[4];
    p.momentCoefficient = v[5];
    p.liftToDrag = v[6];
    p.upperSeparation = v[7];
    p.lowerSeparation = v[8];
    p.converged = v[9] != 0.0;
    p.diverged = v[10] != 0.0;
    p.iterations = static_cast<long long>(v[11]);
    p.continuityResidual = v[12];
    polar.points.push_back(p);
  }
  const std::string text = cfd::post::toCsv(polar);
  if (static_cast<int>(text.size()) <= capacity) std::memcpy(out, text.data(), text.size());
  return static_cast<int>(text.size());
}

// ----------------------------------------------------------- streamlines ---

/// post::traceStreamlines (Streamlines.cpp:80-197) on the solver's current
/// field. lengths[s] gets each seed's point count (0 where the seed was
/// dropped); points the curves one after another while they fit `capacity`
/// points. Returns the total point count, or -1 on the reference's refusal.
long long ref_streamlines(void* s, const double* seeds, int count, int maxSteps, double stepFraction,
                          double stallFraction, double referenceSpeed, int traceBackwards, int* lengths,
                          double* points, long long capacity) {
  RefSolver* r = static_cast<RefSolver*>(s);
  cfd::post::StreamlineOptions o;
  for (int k = 0; k < count; ++k) o.seeds.push_back(Vec2{seeds[2 * k], seeds[2 * k + 1]});
  o.maxSteps = maxSteps;
  o.stepFraction = stepFraction;
  o.stallFraction = stallFraction;
  o.referenceSpeed = referenceSpeed;
  o.traceBackwards = traceBackwards != 0;
  // which seeds survive: the reference returns only the kept curves, in seed
  // order, so a seed's curve is matched by tracing it alone
  long long total = 0;
  for (int k = 0; k < count; ++k) {
    cfd::post::StreamlineOptions one = o;
    one.seeds = {o.seeds[static_cast<std::size_t>(k)]};
    auto lines = cfd::post::traceStreamlines(r->mesh->mesh, r->solver->field(), one);
    if (!lines) {
      g_error = lines.error().format();
      return -1;
    }
    const std::size_t n = lines.value().empty() ? 0 : lines.value().front().size();
    lengths[k] = static_cast<int>(n);
    for (std::size_t q = 0; q < n; ++q, ++total) {
      if (total < capacity) {
        points[2 * total] = lines.value().front()[q].x;
        points[2 * total + 1] = lines.value().front()[q].y;
      }
    }
  }
  return total;
}

}  // extern "C"
