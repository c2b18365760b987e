// shim_check.cpp - TEST INFRASTRUCTURE. Drives the reference-side binding
// (cfd-simulator_b200/shim/gpu_simple_solver.hpp) the way the reference's own
// callers do, next to the reference's SimpleSolver on the same inputs, and
// checks the device answer with the reference's post-processing.
//
// Built by `make -C oracle shim` against the reference's headers and its
// compiled numerics (oracle/_ref/libcfdref.so) plus libcfd_b200.so; run by
// tests/test_gpu_shim.py on a GPU. The sequence is updateSolver's
// (src/app/Panels.cpp:1274-1315: create, setTurbulenceModel, initialise) and
// SolverWorker::runLoop's (src/app/SolverWorker.cpp:134-277: setSettings,
// iterate until worst() < tolerance, field(), divergence(), and the
// turbulence model's fields and maxWallYPlus), then extractSurface +
// integrateForces (src/post/SurfaceData.cpp, src/post/Forces.cpp) on both
// fields. Prints `key value` lines.
#include <cmath>
#include <cstdio>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "cfd/flow/BoundaryConditions.hpp"
#include "cfd/flow/FlowField.hpp"
#include "cfd/flow/Freestream.hpp"
#include "cfd/geom/Airfoil.hpp"
#include "cfd/geom/Naca4.hpp"
#include "cfd/mesh/CGrid.hpp"
#include "cfd/post/Forces.hpp"
#include "cfd/post/SurfaceData.hpp"
#include "cfd/solver/KOmegaSST.hpp"
#include "cfd/solver/SimpleSolver.hpp"
#include "gpu_simple_solver.hpp"

using namespace cfd;
using solver::gpu::GpuSimpleSolver;

namespace {

int g_failures = 0;

void check(bool ok, const char* what) {
  std::printf("check %s %s\n", what, ok ? "ok" : "FAILED");
  if (!ok) ++g_failures;
}

double relL2(const std::vector<double>& a, const std::vector<double>& b) {
  double num = 0.0, den = 0.0;
  for (std::size_t k = 0; k < a.size(); ++k) {
    num += (a[k] - b[k]) * (a[k] - b[k]);
    den += b[k] * b[k];
  }
  return std::sqrt(num) / std::max(std::sqrt(den), 1e-300);
}

std::vector<double> component(const flow::FlowField& f, int which) {
  std::vector<double> out(f.size());
  for (std::size_t c = 0; c < f.size(); ++c) {
    out[c] = (which == 0) ? f.velocity[c].x : (which == 1) ? f.velocity[c].y : f.pressure[c];
  }
  return out;
}

/// A closure the device cannot run, to see the binding refuse it.
class OtherModel final : public solver::TurbulenceModel {
 public:
  std::string_view name() const noexcept override { return "spalart-allmaras"; }
  Status initialise(const mesh::Mesh&, const flow::FaceConditions&, const flow::FlowField&,
                    const solver::TurbulenceInflow&) override {
    return Status::ok();
  }
  void update(const solver::TurbulenceContext&) override {}
  const std::vector<double>& eddyViscosity() const noexcept override { return none_; }
  solver::TurbulenceResiduals residuals() const noexcept override { return {}; }

 private:
  std::vector<double> none_;
};

struct Case {
  const char* name;
  const char* designation;
  int surface, wake, normal;
  double firstLayer, reynolds, alpha, viscosityRatio, tolerance;
  bool sst;
};

template <typename Solver>
long long converge(Solver& s, double tolerance, int cap, int settle) {
  long long it = 0;
  for (; it < cap; ++it) {
    const solver::SolverMonitor m = s.iterate();
    if (!std::isfinite(m.residuals.worst())) return -1;
    if (m.residuals.worst() < tolerance) break;  // SolverWorker.cpp:182-185
  }
  for (int k = 0; k < settle; ++k) s.iterate();
  return it;
}

void runCase(const Case& c) {
  std::printf("case %s\n", c.name);
  auto section = geom::makeNaca4Digit(c.designation, {.chord = 1.0, .trailingEdge = geom::TrailingEdge::Closed});
  mesh::CGridOptions options;
  options.surfacePoints = c.surface;
  options.wakePoints = c.wake;
  options.normalPoints = c.normal;
  options.firstLayerHeight = c.firstLayer;
  options.upstreamChords = 10.0;
  options.downstreamChords = 15.0;
  options.verticalChords = 10.0;
  const mesh::Mesh grid = mesh::generateCGrid(section.value(), options).value();
  flow::FreestreamConditions stream;
  stream.speed = 1.0;
  stream.angleOfAttackDeg = c.alpha;
  stream.density = 1.0;
  stream.reynoldsNumber = c.reynolds;
  const flow::FaceConditions conditions =
      flow::buildFaceConditions(grid, flow::BoundaryConditions{}, stream).value();
  const flow::FlowField start = flow::FlowField::uniform(grid.cellCount(), stream, 1.0).value();
  solver::SimpleSettings settings;
  settings.inflow.viscosityRatio = c.viscosityRatio;

  // the reference
  auto ref = solver::SimpleSolver::create(grid, conditions, settings);
  solver::SimpleSolver r = std::move(ref).value();
  if (c.sst) {
    check(r.setTurbulenceModel(std::make_unique<solver::KOmegaSST>()).hasValue(), "ref_model");
  }
  check(r.initialise(start).hasValue(), "ref_initialise");

  // the binding, held as SolverWorker holds its solver (an optional, moved in)
  auto created = GpuSimpleSolver::create(grid, conditions, settings);
  check(created.hasValue(), "create");
  GpuSimpleSolver moved = std::move(created).value();
  std::optional<GpuSimpleSolver> held;
  held.emplace(std::move(moved));
  check(moved.handle() == nullptr && held->handle() != nullptr, "move_leaves_no_handle");
  GpuSimpleSolver& g = *held;
  if (c.sst) {
    check(g.setTurbulenceModel(std::make_unique<solver::KOmegaSST>()).hasValue(), "gpu_model");
    check(g.turbulenceModel() != nullptr && g.turbulenceModel()->name() == "k-omega SST", "model_name");
  } else {
    check(g.setTurbulenceModel(std::make_unique<solver::LaminarModel>()).hasValue(), "gpu_model");
    check(g.turbulenceModel() != nullptr && g.turbulenceModel()->name() == "laminar", "model_name");
  }
  check(g.initialise(start).hasValue(), "gpu_initialise");
  g.setSettings(settings);

  const long long refIt = converge(r, c.tolerance, 40000, 2000);
  const long long gpuIt = converge(g, c.tolerance, 40000, 2000);
  std::printf("iterations_ref %lld\niterations_gpu %lld\n", refIt, gpuIt);
  check(refIt > 0 && gpuIt > 0, "both_converged");

  const flow::FlowField& fr = r.field();
  const flow::FlowField& fg = std::as_const(g).field();
  const double du = relL2(component(fg, 0), component(fr, 0));
  const double dv = relL2(component(fg, 1), component(fr, 1));
  const double dp = relL2(component(fg, 2), component(fr, 2));
  std::printf("rel_l2_u %.3e\nrel_l2_v %.3e\nrel_l2_p %.3e\n", du, dv, dp);
  check(du < 1e-9 && dv < 1e-9 && dp < 1e-9, "fields_1e-9");
  const double dm = relL2(g.massFlux(), r.massFlux());
  const double dd = relL2(g.divergence(), r.divergence());
  std::printf("rel_l2_mass_flux %.3e\nrel_l2_divergence %.3e\n", dm, dd);
  check(dm < 1e-9, "mass_flux_1e-9");

  if (c.sst) {
    const solver::TurbulenceModel& mg = *g.turbulenceModel();
    const solver::TurbulenceModel& mr = *r.turbulenceModel();
    const double dk = relL2(*mg.turbulentEnergyField(), *mr.turbulentEnergyField());
    const double dw = relL2(*mg.dissipationField(), *mr.dissipationField());
    const double dt = relL2(mg.eddyViscosity(), mr.eddyViscosity());
    std::printf("rel_l2_k %.3e\nrel_l2_omega %.3e\nrel_l2_mut %.3e\n", dk, dw, dt);
    check(dk < 1e-9 && dw < 1e-9 && dt < 1e-9, "turbulence_fields_1e-9");
    std::printf("yplus_ref %.12e\nyplus_gpu %.12e\n", mr.maxWallYPlus(), mg.maxWallYPlus());
    check(std::abs(mg.maxWallYPlus() - mr.maxWallYPlus()) <= 1e-7 * mr.maxWallYPlus(), "yplus");
  }

  // the reference's own post-processing on both fields
  const auto sr = post::extractSurface(grid, fr, stream, 1.0).value();
  const auto sg = post::extractSurface(grid, fg, stream, 1.0).value();
  const auto forcesR = post::integrateForces(sr, stream).value();
  const auto forcesG = post::integrateForces(sg, stream).value();
  std::printf("cl_ref %.15e\ncl_gpu %.15e\ncd_ref %.15e\ncd_gpu %.15e\ncm_ref %.15e\ncm_gpu %.15e\n",
              forcesR.liftCoefficient, forcesG.liftCoefficient, forcesR.dragCoefficient,
              forcesG.dragCoefficient, forcesR.momentCoefficient, forcesG.momentCoefficient);
  const auto close = [](double a, double b) { return std::abs(a - b) <= 1e-7 * std::abs(b); };
  check(close(forcesG.liftCoefficient, forcesR.liftCoefficient) &&
            close(forcesG.dragCoefficient, forcesR.dragCoefficient) &&
            close(forcesG.momentCoefficient, forcesR.momentCoefficient),
        "forces_1e-7");

  // The mutable field() is uploaded before the next iterate(); handing out
  // the unchanged mirror must not change a bit of what follows.
  auto a = GpuSimpleSolver::create(grid, conditions, settings).value();
  auto b = GpuSimpleSolver::create(grid, conditions, settings).value();
  for (GpuSimpleSolver* s : {&a, &b}) {
    if (c.sst) (void)s->setTurbulenceModel(std::make_unique<solver::KOmegaSST>());
    (void)s->initialise(start);
  }
  for (int k = 0; k < 5; ++k) {
    a.iterate();
    (void)b.field();  // the mutable overload
    b.iterate();
  }
  check(component(std::as_const(a).field(), 0) == component(std::as_const(b).field(), 0) &&
            component(std::as_const(a).field(), 2) == component(std::as_const(b).field(), 2),
        "mutable_field_roundtrip_exact");
}

}  // namespace

int main() {
  std::setvbuf(stdout, nullptr, _IOLBF, 0);
  // errors map one to one onto ErrorCode
  {
    auto section = geom::makeNaca4Digit("0012", {.chord = 1.0, .trailingEdge = geom::TrailingEdge::Closed});
    mesh::CGridOptions options;
    options.surfacePoints = 24;
    options.wakePoints = 12;
    options.normalPoints = 13;
    const mesh::Mesh grid = mesh::generateCGrid(section.value(), options).value();
    flow::FreestreamConditions stream;
    const flow::FaceConditions conditions =
        flow::buildFaceConditions(grid, flow::BoundaryConditions{}, stream).value();
    flow::FaceConditions shortList(conditions.begin(), conditions.end() - 1);
    auto bad = GpuSimpleSolver::create(grid, shortList, solver::SimpleSettings{});
    check(bad.hasError() && bad.error().code() == ErrorCode::InvalidArgument, "short_conditions");
    solver::SimpleSettings wrong;
    wrong.velocityRelaxation = 1.5;  // outside (0, 1]: the library refuses it (SimpleSolver.cpp:33-44)
    auto refused = GpuSimpleSolver::create(grid, conditions, wrong);
    check(refused.hasError() && refused.error().code() == ErrorCode::InvalidArgument, "relaxation_refused");
    auto ok = GpuSimpleSolver::create(grid, conditions, solver::SimpleSettings{});
    if (ok.hasValue()) {
      GpuSimpleSolver s = std::move(ok).value();
      const Status st = s.setTurbulenceModel(std::make_unique<OtherModel>());
      check(st.hasError() && st.error().code() == ErrorCode::NotImplemented, "unsupported_model");
    } else {
      check(false, "create_for_model_check");
    }
  }
  runCase({"laminar", "0012", 24, 12, 13, 2e-3, 500.0, 4.0, 1.0, 1e-12, false});
  runCase({"sst", "0012", 24, 12, 13, 1e-4, 1e6, 4.0, 10.0, 1e-11, true});
  std::printf("failures %d\n", g_failures);
  return (g_failures == 0) ? 0 : 1;
}
