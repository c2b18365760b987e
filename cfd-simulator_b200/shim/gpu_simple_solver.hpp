// gpu_simple_solver.hpp - the reference's SimpleSolver interface over the B200
// library's C ABI (include/cfd_gpu.h), for the reference's own callers.
//
// Header-only C++20, meant to be compiled inside the reference tree against
// its headers (include/cfd/...) and linked with libcfd_b200.so. It mirrors
// cfd::solver::SimpleSolver (include/cfd/solver/SimpleSolver.hpp:159-274)
// member for member, so that SolverWorker (src/app/SolverWorker.cpp:134-277),
// updateSolver (src/app/Panels.cpp:1274-1315) and the tests' converge() loops
// need only the solver's type name changed (SolverWorker.hpp:107 and :151,
// and the create call in Panels.cpp): every member they use exists here with
// the reference's signature and meaning.
//
//   create(mesh, conditions, settings) -> Result<GpuSimpleSolver>
//   initialise(FlowField), setTurbulenceModel(unique_ptr<TurbulenceModel>),
//   turbulenceModel(), iterate(), field() (const and mutable), massFlux(),
//   settings(), setSettings(), divergence()
//
// Ownership: the solver owns its device handle and is move-only, like the
// reference's (which holds a unique_ptr); a moved-from solver holds no handle.
// The mesh must outlive the solver, as in the reference (SimpleSolver.hpp:156-158).
//
// The turbulence closure runs on the device inside iterate(). The model object
// a caller hands to setTurbulenceModel (LaminarModel or KOmegaSST) selects the
// closure; turbulenceModel() then returns a DeviceTurbulenceModel that answers
// the reference's queries (name, eddyViscosity, turbulentEnergyField,
// dissipationField, residuals, ranges, maxWallYPlus) from the device state.
//
// Field access: field() returns a host mirror of the device state, refreshed
// from the device the first time it is asked for after an iterate(). The
// mutable overload may be edited, as the reference's may; the mirror is then
// uploaded before the next iterate(), so edits take effect as they would in
// the reference.
#pragma once

#include <cmath>
#include <limits>
#include <memory>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#include "cfd/core/Error.hpp"
#include "cfd/core/Vec2.hpp"
#include "cfd/flow/BoundaryConditions.hpp"
#include "cfd/flow/FlowField.hpp"
#include "cfd/mesh/Mesh.hpp"
#include "cfd/solver/SimpleSolver.hpp"
#include "cfd/solver/TurbulenceModel.hpp"
#include "cfd_gpu.h"

namespace cfd::solver::gpu {

static_assert(sizeof(Vec2) == 2 * sizeof(double), "Vec2 arrays are passed as (x, y) pairs");

/// cfd_status -> cfd::ErrorCode (include/cfd/core/Error.hpp:37-46): the C
/// ABI's codes are the enumerators' positions plus one.
inline ErrorCode toErrorCode(cfd_status s) noexcept {
  switch (s) {
    case CFD_INVALID_ARGUMENT: return ErrorCode::InvalidArgument;
    case CFD_OUT_OF_RANGE: return ErrorCode::OutOfRange;
    case CFD_NOT_FOUND: return ErrorCode::NotFound;
    case CFD_IO_FAILURE: return ErrorCode::IoFailure;
    case CFD_NOT_IMPLEMENTED: return ErrorCode::NotImplemented;
    case CFD_INITIALIZATION_FAILURE: return ErrorCode::InitializationFailure;
    case CFD_NUMERICAL_FAILURE: return ErrorCode::NumericalFailure;
    default: return ErrorCode::Internal;
  }
}

/// The failure the library recorded for status `s` on this thread.
inline Error libraryError(cfd_status s) {
  const char* message = cfd_last_error();
  return Error{toErrorCode(s), (message != nullptr) ? message : "B200 solver failure"};
}

inline Status toStatus(cfd_status s) {
  if (s == CFD_OK) return Status::ok();
  return libraryError(s);
}

/// The closure attached to a GpuSimpleSolver, as its callers see it. The
/// equations themselves advance on the device inside the solver's iterate();
/// this object reports their state. Fields are copied from the device the
/// first time they are asked for after an iteration.
class DeviceTurbulenceModel final : public TurbulenceModel {
 public:
  DeviceTurbulenceModel(std::string name, int model, cfd_handle handle, std::size_t cells)
      : name_(std::move(name)), model_(model), handle_(handle), cells_(cells) {}

  [[nodiscard]] std::string_view name() const noexcept override { return name_; }

  /// Nothing to do: the device solver sets the closure up in its own
  /// initialise() (KOmegaSST::initialise, wall distances included).
  [[nodiscard]] Status initialise(const mesh::Mesh&, const flow::FaceConditions&,
                                  const flow::FlowField&, const TurbulenceInflow&) override {
    return Status::ok();
  }

  /// Nothing to do: the device solver advances the closure inside iterate().
  void update(const TurbulenceContext&) override {}

  [[nodiscard]] const std::vector<double>& eddyViscosity() const noexcept override {
    return mirror(CFD_FIELD_MUT, eddyViscosity_, eddyViscosityStale_);
  }
  [[nodiscard]] TurbulenceResiduals residuals() const noexcept override { return residuals_; }
  [[nodiscard]] TurbulenceRanges ranges() const noexcept override { return ranges_; }
  [[nodiscard]] const std::vector<double>* turbulentEnergyField() const noexcept override {
    if (!transported()) return nullptr;
    return &mirror(CFD_FIELD_K, energy_, energyStale_);
  }
  [[nodiscard]] const std::vector<double>* dissipationField() const noexcept override {
    if (!transported()) return nullptr;
    return &mirror(CFD_FIELD_OMEGA, dissipation_, dissipationStale_);
  }
  [[nodiscard]] double maxWallYPlus() const noexcept override { return maxWallYPlus_; }

  /// 1 LaminarModel, 2 KOmegaSST (the C ABI's model codes).
  [[nodiscard]] int code() const noexcept { return model_; }

  /// Record what the latest iteration reported; the fields are now stale.
  void observe(const cfd_monitor& m) noexcept {
    if (transported()) {
      residuals_ = TurbulenceResiduals{m.turbulence_first, m.turbulence_second};
      ranges_ = TurbulenceRanges{m.min_energy, m.max_energy, m.min_dissipation,
                                 m.max_dissipation, m.min_eddy_viscosity, m.max_eddy_viscosity};
      maxWallYPlus_ = m.max_wall_yplus;
    }
    eddyViscosityStale_ = energyStale_ = dissipationStale_ = true;
  }

 private:
  [[nodiscard]] bool transported() const noexcept { return model_ == 2; }

  const std::vector<double>& mirror(int which, std::vector<double>& out, bool& stale) const noexcept {
    if (stale) {
      out.resize(cells_);
      if (cfd_gpu_read_field(handle_, which, out.data()) == CFD_OK) stale = false;
    }
    return out;
  }

  std::string name_;
  int model_;
  cfd_handle handle_;
  std::size_t cells_;
  TurbulenceResiduals residuals_{};
  TurbulenceRanges ranges_{};
  double maxWallYPlus_{0.0};
  mutable std::vector<double> eddyViscosity_, energy_, dissipation_;
  mutable bool eddyViscosityStale_{true}, energyStale_{true}, dissipationStale_{true};
};

/// SimpleSolver on one B200: the steady SIMPLE solve of the reference,
/// resident on the device, behind the reference's own interface.
class GpuSimpleSolver {
 public:
  /// SimpleSolver::create (SimpleSolver.cpp:30-80): validation, geometry and
  /// conditions copied to the device. The settings' form is the plain FP64 one,
  /// the reference-parity drop-in.
  [[nodiscard]] static Result<GpuSimpleSolver> create(const mesh::Mesh& mesh,
                                                      flow::FaceConditions conditions,
                                                      const SimpleSettings& settings) {
    const std::size_t faces = mesh.faceCount();
    if (conditions.size() != faces) {
      return Error{ErrorCode::InvalidArgument, "one face condition per mesh face is required"};
    }
    std::vector<int> owner(faces), neighbour(faces), boundary(faces), partner(faces), kind(faces);
    std::vector<double> velocity(2 * faces), pressure(faces);
    for (std::size_t f = 0; f < faces; ++f) {
      const mesh::Face& face = mesh.faces()[f];
      owner[f] = face.owner;
      neighbour[f] = face.neighbour;
      boundary[f] = static_cast<int>(face.boundary);
      partner[f] = face.partner;
      kind[f] = static_cast<int>(conditions[f].kind);
      velocity[2 * f] = conditions[f].velocity.x;
      velocity[2 * f + 1] = conditions[f].velocity.y;
      pressure[f] = conditions[f].pressure;
    }
    const auto pairs = [](const std::vector<Vec2>& v) {
      return v.empty() ? nullptr : &v.front().x;
    };
    cfd_mesh_desc d{};
    d.nodes_i = mesh.nodesI();
    d.nodes_j = mesh.nodesJ();
    d.cell_count = static_cast<int>(mesh.cellCount());
    d.face_count = static_cast<int>(faces);
    d.cell_centroids = pairs(mesh.cellCentroids());
    d.cell_areas = mesh.cellAreas().data();
    d.face_centres = pairs(mesh.faceCentres());
    d.face_normals = pairs(mesh.faceNormals());
    d.face_areas = mesh.faceAreas().data();
    d.face_owner = owner.data();
    d.face_neighbour = neighbour.data();
    d.face_boundary = boundary.data();
    d.face_partner = partner.data();
    d.nodes = pairs(mesh.nodes());
    cfd_face_bc bc{kind.data(), velocity.data(), pressure.data()};
    const cfd_settings s = toC(settings);
    cfd_handle h = nullptr;
    if (const cfd_status st = cfd_gpu_create(&d, &bc, &s, &h); st != CFD_OK) return libraryError(st);
    return GpuSimpleSolver(mesh, h, settings);
  }

  GpuSimpleSolver(const GpuSimpleSolver&) = delete;
  GpuSimpleSolver& operator=(const GpuSimpleSolver&) = delete;
  GpuSimpleSolver(GpuSimpleSolver&& other) noexcept { *this = std::move(other); }
  GpuSimpleSolver& operator=(GpuSimpleSolver&& other) noexcept {
    if (this != &other) {
      release();
      mesh_ = other.mesh_;
      handle_ = std::exchange(other.handle_, nullptr);
      settings_ = other.settings_;
      field_ = std::move(other.field_);
      massFlux_ = std::move(other.massFlux_);
      model_ = std::move(other.model_);
      fieldStale_ = other.fieldStale_;
      fieldEdited_ = other.fieldEdited_;
      massFluxStale_ = other.massFluxStale_;
    }
    return *this;
  }
  ~GpuSimpleSolver() { release(); }

  /// SimpleSolver::initialise (SimpleSolver.cpp:133-210).
  [[nodiscard]] Status initialise(const flow::FlowField& initial) {
    if (initial.size() != mesh_->cellCount() || !initial.isConsistent()) {
      return Error{ErrorCode::InvalidArgument, "initial field does not match the mesh"};
    }
    std::vector<double> u(initial.size()), v(initial.size());
    for (std::size_t c = 0; c < initial.size(); ++c) {
      u[c] = initial.velocity[c].x;
      v[c] = initial.velocity[c].y;
    }
    if (const cfd_status st = cfd_gpu_initialise(handle_, u.data(), v.data(), initial.pressure.data(),
                                                 initial.density.data(), initial.viscosity.data());
        st != CFD_OK) {
      return libraryError(st);
    }
    field_ = initial;
    fieldStale_ = true;  // the effective viscosity now includes the closure's mu_t
    fieldEdited_ = false;
    massFluxStale_ = true;
    if (model_ != nullptr) model_->observe(cfd_monitor{});
    return Status::ok();
  }

  /// SimpleSolver::setTurbulenceModel (SimpleSolver.cpp:212-230): nullptr for
  /// laminar flow, or a LaminarModel / KOmegaSST, which select the device
  /// closure. Any other model cannot run on the device.
  [[nodiscard]] Status setTurbulenceModel(std::unique_ptr<TurbulenceModel> model) {
    int code = 0;
    std::string name;
    if (model != nullptr) {
      name = std::string(model->name());
      if (name == "laminar") {
        code = 1;
      } else if (name == "k-omega SST") {
        code = 2;
      } else {
        return Error{ErrorCode::NotImplemented,
                     "the B200 solver runs the laminar and k-omega SST closures only, not " + name};
      }
    }
    if (const cfd_status st = cfd_gpu_set_turbulence(handle_, code); st != CFD_OK) return libraryError(st);
    model_ = (code == 0) ? nullptr
                         : std::make_unique<DeviceTurbulenceModel>(name, code, handle_, mesh_->cellCount());
    fieldStale_ = true;
    return Status::ok();
  }

  [[nodiscard]] const TurbulenceModel* turbulenceModel() const noexcept { return model_.get(); }

  /// One outer iteration (SimpleSolver.cpp:662-794) on the device. As in the
  /// reference, a failing solve is not an error: a device failure reports
  /// non-finite residuals, which SolverWorker classifies as diverged.
  SolverMonitor iterate() {
    pushEdits();
    cfd_monitor m{};
    SolverMonitor out;
    if (cfd_gpu_iterate(handle_, 1, &m, nullptr) != CFD_OK) {
      const double nan = std::numeric_limits<double>::quiet_NaN();
      out.residuals = flow::ResidualSet{nan, nan, nan};
      return out;
    }
    out.residuals = flow::ResidualSet{m.continuity, m.momentum_x, m.momentum_y};
    out.massImbalance = m.mass_imbalance;
    out.maxDivergence = m.max_divergence;
    out.pressureIterations = m.pressure_iterations;
    if (model_ != nullptr && model_->code() == 2) {
      out.turbulence = TurbulenceResiduals{m.turbulence_first, m.turbulence_second};
      out.turbulenceRanges = TurbulenceRanges{m.min_energy, m.max_energy, m.min_dissipation,
                                              m.max_dissipation, m.min_eddy_viscosity,
                                              m.max_eddy_viscosity};
      out.maxEddyViscosityRatio = m.max_eddy_viscosity_ratio;
    }
    if (model_ != nullptr) model_->observe(m);
    fieldStale_ = true;
    massFluxStale_ = true;
    return out;
  }

  [[nodiscard]] const flow::FlowField& field() const noexcept {
    refreshField();
    return field_;
  }
  /// The mirror handed out for editing; uploaded before the next iterate().
  [[nodiscard]] flow::FlowField& field() noexcept {
    refreshField();
    fieldEdited_ = true;
    return field_;
  }

  /// Mass flux through each face, positive out of the owner (reference face order).
  [[nodiscard]] const std::vector<double>& massFlux() const noexcept {
    if (massFluxStale_) {
      massFlux_.resize(mesh_->faceCount());
      if (cfd_gpu_read_field(handle_, CFD_FIELD_MASS_FLUX, massFlux_.data()) == CFD_OK) {
        massFluxStale_ = false;
      }
    }
    return massFlux_;
  }

  [[nodiscard]] const SimpleSettings& settings() const noexcept { return settings_; }
  void setSettings(const SimpleSettings& settings) {
    const cfd_settings s = toC(settings);
    if (cfd_gpu_set_settings(handle_, &s) == CFD_OK) settings_ = settings;
  }

  /// SimpleSolver::divergence (SimpleSolver.cpp:796-817).
  [[nodiscard]] std::vector<double> divergence() const {
    std::vector<double> out(mesh_->cellCount());
    if (cfd_gpu_read_field(handle_, CFD_FIELD_DIVERGENCE, out.data()) != CFD_OK) out.clear();
    return out;
  }

  /// The library handle, for the calls the reference has no counterpart for
  /// (cfd_gpu_forces, cfd_gpu_converge, batches).
  [[nodiscard]] cfd_handle handle() const noexcept { return handle_; }

 private:
  GpuSimpleSolver(const mesh::Mesh& mesh, cfd_handle handle, const SimpleSettings& settings)
      : mesh_(&mesh), handle_(handle), settings_(settings) {}

  static cfd_settings toC(const SimpleSettings& in) {
    cfd_settings s;
    cfd_default_settings(&s);
    s.velocity_relaxation = in.velocityRelaxation;
    s.pressure_relaxation = in.pressureRelaxation;
    s.momentum_sweeps = in.momentumSweeps;
    s.pressure_iterations = in.pressureIterations;
    s.pressure_tolerance = in.pressureTolerance;
    s.scheme = (in.scheme == ConvectionScheme::SecondOrderUpwind) ? 1 : 0;
    s.turbulence_relaxation = in.turbulenceRelaxation;
    s.inflow_intensity = in.inflow.intensity;
    s.inflow_viscosity_ratio = in.inflow.viscosityRatio;
    s.inflow_length_scale = in.inflow.lengthScale;
    s.non_orthogonal_correctors = in.nonOrthogonalCorrectors;
    s.non_orthogonal_blend = in.nonOrthogonalBlend;
    return s;
  }

  void release() noexcept {
    model_.reset();
    if (handle_ != nullptr) cfd_gpu_destroy(handle_);
    handle_ = nullptr;
  }

  void refreshField() const noexcept {
    if (!fieldStale_ || handle_ == nullptr) return;
    const std::size_t n = mesh_->cellCount();
    std::vector<double> u(n), v(n);
    field_.velocity.resize(n);
    field_.pressure.resize(n);
    field_.viscosity.resize(n);
    if (cfd_gpu_read_field(handle_, CFD_FIELD_U, u.data()) != CFD_OK ||
        cfd_gpu_read_field(handle_, CFD_FIELD_V, v.data()) != CFD_OK ||
        cfd_gpu_read_field(handle_, CFD_FIELD_P, field_.pressure.data()) != CFD_OK ||
        cfd_gpu_read_field(handle_, CFD_FIELD_MU_EFF, field_.viscosity.data()) != CFD_OK) {
      return;
    }
    if (field_.density.size() != n) {
      field_.density.resize(n);
      cfd_gpu_read_field(handle_, CFD_FIELD_RHO, field_.density.data());
    }
    for (std::size_t c = 0; c < n; ++c) field_.velocity[c] = Vec2{u[c], v[c]};
    fieldStale_ = false;
  }

  /// Upload a mirror the caller may have edited through field().
  void pushEdits() {
    if (!fieldEdited_) return;
    fieldEdited_ = false;
    const std::size_t n = field_.size();
    if (n != mesh_->cellCount()) return;
    std::vector<double> u(n), v(n);
    for (std::size_t c = 0; c < n; ++c) {
      u[c] = field_.velocity[c].x;
      v[c] = field_.velocity[c].y;
    }
    cfd_gpu_load_state(handle_, u.data(), v.data(), field_.pressure.data(), nullptr, nullptr, nullptr,
                       nullptr, field_.viscosity.data());
  }

  const mesh::Mesh* mesh_{nullptr};
  cfd_handle handle_{nullptr};
  SimpleSettings settings_{};
  mutable flow::FlowField field_;
  mutable std::vector<double> massFlux_;
  std::unique_ptr<DeviceTurbulenceModel> model_;
  mutable bool fieldStale_{true};
  bool fieldEdited_{false};
  mutable bool massFluxStale_{true};
};

}  // namespace cfd::solver::gpu
