// solver.cu - host side of a device-resident SIMPLE solve and the C ABI
// (include/cfd_gpu.h).

#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>

#include "cfd_gpu.h"

namespace cfdb {

Status launchWallDistance(int n, const double* centroid, int walls, const double* wallCentre,
                          double far, double* out, cudaStream_t stream);

namespace {
thread_local std::string g_message;

constexpr double kTinySolver = 1e-300;
constexpr double kTinySst = 1.0e-30;
constexpr double kMinOmega = 1.0e-10;

inline double hyp(double x, double y) { return std::hypot(x, y); }

#define CUDA_OR_FAIL(expr)                                                              \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e_)); \
  } while (0)
}  // namespace

Status fail(Status code, const std::string& message) {
  g_message = message;
  return code;
}

Status launchFault(int word) {
  std::string what = "the solver kernel stopped waiting";
  if (word & kFaultChainWait) what += " (a k/omega sweep stage for its neighbour)";
  if (word & kFaultHaloWait) what += " (the pressure CG for a neighbour's halo row)";
  return fail(CFD_INTERNAL, what + "; the launch's results are not valid");
}

// ---- settings -----------------------------------------------------------------

Settings fromC(const cfd_settings& s) {
  Settings o;
  o.velocityRelaxation = s.velocity_relaxation;
  o.pressureRelaxation = s.pressure_relaxation;
  o.momentumSweeps = s.momentum_sweeps;
  o.pressureIterations = s.pressure_iterations;
  o.pressureTolerance = s.pressure_tolerance;
  o.scheme = s.scheme;
  o.turbulenceRelaxation = s.turbulence_relaxation;
  o.inflowIntensity = s.inflow_intensity;
  o.inflowViscosityRatio = s.inflow_viscosity_ratio;
  o.inflowLengthScale = s.inflow_length_scale;
  o.nonOrthogonalCorrectors = s.non_orthogonal_correctors;
  o.nonOrthogonalBlend = s.non_orthogonal_blend;
  o.precision = s.precision;
  o.innerIterations = s.inner_iterations;
  return o;
}

void toC(const Settings& s, cfd_settings* o) {
  o->velocity_relaxation = s.velocityRelaxation;
  o->pressure_relaxation = s.pressureRelaxation;
  o->momentum_sweeps = s.momentumSweeps;
  o->pressure_iterations = s.pressureIterations;
  o->pressure_tolerance = s.pressureTolerance;
  o->scheme = s.scheme;
  o->turbulence_relaxation = s.turbulenceRelaxation;
  o->inflow_intensity = s.inflowIntensity;
  o->inflow_viscosity_ratio = s.inflowViscosityRatio;
  o->inflow_length_scale = s.inflowLengthScale;
  o->non_orthogonal_correctors = s.nonOrthogonalCorrectors;
  o->non_orthogonal_blend = s.nonOrthogonalBlend;
  o->precision = s.precision;
  o->inner_iterations = s.innerIterations;
}

// ---- device arena ---------------------------------------------------------------

DeviceArena::~DeviceArena() {
  if (base_ != nullptr) cudaFree(base_);
}

Status DeviceArena::allocate() {
  const std::size_t bytes = used_;
  CUDA_OR_FAIL(cudaMalloc(reinterpret_cast<void**>(&base_), bytes));
  CUDA_OR_FAIL(cudaMemset(base_, 0, bytes));
  used_ = 0;
  return CFD_OK;
}

// ---- create (SimpleSolver.cpp:30-131) -----------------------------------------------

int Solver::idxOf(int f) const {
  if (f < jFaces_) return f;
  const int g = f - jFaces_;
  const int i = g / NJ_, j = g % NJ_;
  return j * (NI_ + 1) + i;
}

Status Solver::create(const cfd_mesh_desc& mesh, const cfd_face_bc& bc, const Settings& s,
                      Solver** out) {
  if (mesh.cell_count <= 0) return fail(CFD_INVALID_ARGUMENT, "cannot solve on an empty mesh");
  if (bc.kind == nullptr || bc.velocity == nullptr || bc.pressure == nullptr) {
    return fail(CFD_INVALID_ARGUMENT, "face conditions are missing");
  }
  if (!(s.velocityRelaxation > 0.0) || s.velocityRelaxation > 1.0 || !(s.pressureRelaxation > 0.0) ||
      s.pressureRelaxation > 1.0) {
    return fail(CFD_INVALID_ARGUMENT, "relaxation factors must lie in (0, 1]");
  }
  if (s.precision != 0 && s.precision != 1) {
    return fail(CFD_INVALID_ARGUMENT, "precision must be 0 (plain FP64) or 1 (mixed FP32/FP64)");
  }
  if (s.innerIterations < 0) return fail(CFD_INVALID_ARGUMENT, "inner_iterations must be >= 0");
  auto* solver = new Solver;
  solver->settings_ = s;
  if (Status st = solver->build(mesh, bc); st != CFD_OK) {
    delete solver;
    return st;
  }
  *out = solver;
  return CFD_OK;
}

Status Solver::build(const cfd_mesh_desc& m, const cfd_face_bc& bc) {
  const int ni = m.nodes_i, nj = m.nodes_j;
  if (ni < 2 || nj < 2) return fail(CFD_NOT_IMPLEMENTED, "the device solver needs a structured mesh (nodesI, nodesJ)");
  NI_ = ni - 1;
  NJ_ = nj - 1;
  N_ = NI_ * NJ_;
  jFaces_ = NI_ * nj;
  F_ = jFaces_ + ni * NJ_;
  if (m.cell_count != N_ || m.face_count != F_) {
    return fail(CFD_INVALID_ARGUMENT, "cell or face count does not match the structured block");
  }
  const std::size_t N = N_, F = F_;
  auto copyIn = [](const auto* src, std::size_t n, auto& dst) { dst.assign(src, src + n); };
  copyIn(m.cell_centroids, 2 * N, centroid_);
  copyIn(m.cell_areas, N, cellArea_);
  copyIn(m.face_centres, 2 * F, faceCentre_);
  copyIn(m.face_normals, 2 * F, faceNormal_);
  copyIn(m.face_areas, F, faceArea_);
  copyIn(m.face_owner, F, owner_);
  copyIn(m.face_neighbour, F, neighbour_);
  copyIn(m.face_boundary, F, boundary_);
  copyIn(m.face_partner, F, partner_);
  copyIn(bc.kind, F, kind_);
  copyIn(bc.velocity, 2 * F, bcVel_);
  copyIn(bc.pressure, F, bcP_);

  // The structured layout of buildStructured (Mesh.cpp:138-170) is what the
  // device indexing assumes; anything else is refused rather than misread.
  for (int f = 0; f < F_; ++f) {
    int o, n;
    if (f < jFaces_) {
      const int i = f % NI_, j = f / NI_;
      o = (j == 0) ? i : (j == NJ_) ? (NJ_ - 1) * NI_ + i : (j - 1) * NI_ + i;
      n = (j == 0 || j == NJ_) ? -1 : j * NI_ + i;
    } else {
      const int g = f - jFaces_, i = g / NJ_, j = g % NJ_;
      o = (i == 0) ? j * NI_ : (i == NI_) ? j * NI_ + NI_ - 1 : j * NI_ + i - 1;
      n = (i == 0 || i == NI_) ? -1 : j * NI_ + i;
    }
    if (owner_[f] != o || neighbour_[f] != n) {
      return fail(CFD_NOT_IMPLEMENTED, "face " + std::to_string(f) + " is not in the structured block layout");
    }
    if (f >= NI_ && partner_[f] >= 0) {
      return fail(CFD_NOT_IMPLEMENTED, "wake-cut partners are supported on the j = 0 boundary only");
    }
    if (kind_[f] < CFD_BC_INTERNAL || kind_[f] > CFD_BC_NOSLIP_WALL) {
      return fail(CFD_INVALID_ARGUMENT, "unknown boundary kind on face " + std::to_string(f));
    }
  }

  // oppositeCell (Mesh.cpp:78-87) and precomputeGeometry (SimpleSolver.cpp:82-131).
  across_.assign(F, -1);
  Sx_.assign(F, 0.0); Sy_.assign(F, 0.0); dx_.assign(F, 0.0); dy_.assign(F, 0.0);
  D_.assign(F, 0.0); w_.assign(F, 1.0);
  std::vector<double> Tx(F, 0.0), Ty(F, 0.0), Dt(F, 0.0);
  for (std::size_t f = 0; f < F; ++f) {
    if (neighbour_[f] >= 0) across_[f] = neighbour_[f];
    else if (boundary_[f] == CFD_FACE_WAKECUT && partner_[f] >= 0) across_[f] = owner_[partner_[f]];
    const double ax = faceNormal_[2 * f] * faceArea_[f];
    const double ay = faceNormal_[2 * f + 1] * faceArea_[f];
    Sx_[f] = ax;
    Sy_[f] = ay;
    const int o = owner_[f];
    const double ocx = centroid_[2 * o], ocy = centroid_[2 * o + 1];
    const double fcx = faceCentre_[2 * f], fcy = faceCentre_[2 * f + 1];
    double ddx, ddy, w;
    if (neighbour_[f] >= 0) {
      const int n = neighbour_[f];
      ddx = centroid_[2 * n] - ocx;
      ddy = centroid_[2 * n + 1] - ocy;
      // ownerWeight (Gradient.cpp:7-18)
      const double toOwner = hyp(ocx - fcx, ocy - fcy);
      const double toNb = hyp(centroid_[2 * n] - fcx, centroid_[2 * n + 1] - fcy);
      const double total = toOwner + toNb;
      w = (total > 0.0) ? toNb / total : 0.5;
    } else if (across_[f] >= 0) {
      const int a = across_[f];
      ddx = centroid_[2 * a] - ocx;
      ddy = centroid_[2 * a + 1] - ocy;
      const double toOwner = hyp(ocx - fcx, ocy - fcy);
      const double toAcross = hyp(centroid_[2 * a] - fcx, centroid_[2 * a + 1] - fcy);
      const double span = toOwner + toAcross;
      w = (span > 0.0) ? toAcross / span : 0.5;
    } else {
      ddx = fcx - ocx;
      ddy = fcy - ocy;
      w = 1.0;
    }
    dx_[f] = ddx;
    dy_[f] = ddy;
    w_[f] = w;
    const double aDd = ax * ddx + ay * ddy;
    const double aSq = ax * ax + ay * ay;
    if (std::abs(aDd) > kTinySolver) {
      D_[f] = aSq / aDd;
      Tx[f] = ax - ddx * D_[f];
      Ty[f] = ay - ddy * D_[f];
    }
    // KOmegaSST.cpp:399-403 / :423-427
    Dt[f] = (std::abs(aDd) > kTinySst) ? std::abs(aSq / aDd) : 0.0;
  }

  // Red-black ordering needs the two cells across each wake pair to differ
  // in colour (always true on a C-grid, where cellsI is even).
  std::vector<int> acrossJ0(NI_, -1);
  for (int i = 0; i < NI_; ++i) {
    const int a = (neighbour_[i] < 0) ? across_[i] : -1;
    acrossJ0[i] = a;
    if (a >= NI_) return fail(CFD_NOT_IMPLEMENTED, "a wake-cut partner must lie in the j = 0 row");
    // The C-grid pairing (CGrid.cpp:368-378): column i meets column NI-1-i.
    if (a >= 0 && a != NI_ - 1 - i) {
      return fail(CFD_NOT_IMPLEMENTED, "wake-cut partners must pair column i with column cellsI-1-i");
    }
    if (a >= 0) {
      const int ai = a % NI_, aj = a / NI_;
      if (((ai + aj) & 1) == (i & 1)) {
        return fail(CFD_NOT_IMPLEMENTED, "wake-cut partners of equal colour (odd cellsI)");
      }
    }
  }

  if (settings_.precision == 1) planMultigrid(acrossJ0);

  bool anchor = false;
  for (int f = 0; f < F_; ++f) {
    if (kind_[f] == CFD_BC_OUTLET || kind_[f] == CFD_BC_FARFIELD) {
      anchor = true;
      break;
    }
  }
  hasPRef_ = anchor;

  // Wall faces: no-slip faces, marked on their owner (KOmegaSST.cpp:312-316).
  std::vector<uint8_t> wallMask(N, 0);
  std::vector<double> wallCentres;
  for (int f = 0; f < F_; ++f) {
    if (kind_[f] != CFD_BC_NOSLIP_WALL) continue;
    wallCentres.push_back(faceCentre_[2 * f]);
    wallCentres.push_back(faceCentre_[2 * f + 1]);
    const int o = owner_[f];
    const int oi = o % NI_, oj = o / NI_;
    int bit;
    if (f < jFaces_) bit = (f / NI_ == oj) ? 0 : 1;  // south (j = 0 row) or north
    else bit = (((f - jFaces_) / NJ_) == oi) ? 2 : 3;  // west (i = 0) or east
    wallMask[o] |= static_cast<uint8_t>(1u << bit);
  }

  // Wall stations for the device force integration (needs node coordinates).
  {
    HostMesh view;
    view.nodesI = ni;
    view.nodesJ = nj;
    view.cells = N_;
    view.faces = F_;
    view.centroid = centroid_;
    view.faceCentre = faceCentre_;
    view.faceNormal = faceNormal_;
    view.owner = owner_;
    view.neighbour = neighbour_;
    view.boundary = boundary_;
    view.partner = partner_;
    if (Status st = buildWallTable(view, m.nodes, &wall_); st != CFD_OK) return st;
  }
  // node coordinates, for the streamline tracer (copied to the device on first use)
  if (m.nodes != nullptr) nodes_.assign(m.nodes, m.nodes + 2 * static_cast<std::size_t>(ni) * nj);
  const std::size_t S = static_cast<std::size_t>(std::max(wall_.count(), 1));

  // ---- device layout ----
  const std::size_t FN = static_cast<std::size_t>(NI_) * (NJ_ + 1);
  const std::size_t FE = static_cast<std::size_t>(NI_ + 1) * NJ_;
  historyCapacity_ = 256;
  auto carve = [&](DeviceArena& a) {
    Instance& I = view_;
    I.vol = a.take<double>(N);
    auto famGeo = [&](FaceGeo& g, std::size_t n) {
      g.Sx = a.take<double>(n); g.Sy = a.take<double>(n); g.D = a.take<double>(n);
      g.Tx = a.take<double>(n); g.Ty = a.take<double>(n); g.w = a.take<double>(n);
      g.Dt = a.take<double>(n); g.nx = a.take<double>(n); g.ny = a.take<double>(n);
    };
    famGeo(I.gN, FN);
    famGeo(I.gE, FE);
    I.acrossJ0 = a.take<int>(NI_);
    I.kindN = a.take<int8_t>(FN); I.kindE = a.take<int8_t>(FE);
    I.bcuN = a.take<double>(FN); I.bcvN = a.take<double>(FN); I.bcpN = a.take<double>(FN);
    I.bcuE = a.take<double>(FE); I.bcvE = a.take<double>(FE); I.bcpE = a.take<double>(FE);
    I.deadN = a.take<double>(FN); I.deadE = a.take<double>(FE);
    I.wallDist = a.take<double>(N);
    I.wallMask = a.take<uint8_t>(N);
    double** cellArrays[] = {&I.u, &I.v, &I.p, &I.rho, &I.mu, &I.muMol, &I.gux, &I.guy, &I.gvx,
                             &I.gvy, &I.gpx, &I.gpy, &I.aD, &I.aS, &I.aN, &I.aW, &I.aE, &I.bU,
                             &I.bV, &I.pD, &I.pB, &I.net, &I.x, &I.r, &I.z, &I.q, &I.d0, &I.d1, &I.s1, &I.cgp,
                             &I.div, &I.k, &I.om, &I.mut, &I.strain, &I.f1, &I.f2, &I.cd, &I.prod,
                             &I.gkx, &I.gky, &I.gwx, &I.gwy, &I.kD, &I.kS, &I.kN, &I.kW, &I.kE,
                             &I.kB, &I.wD, &I.wS, &I.wN, &I.wW, &I.wE, &I.wB};
    for (double** ptr : cellArrays) *ptr = a.take<double>(N);
    I.mfN = a.take<double>(FN); I.mfE = a.take<double>(FE);
    I.pN = a.take<double>(FN); I.pE = a.take<double>(FE);
    I.history = a.take<double>(static_cast<std::size_t>(historyCapacity_) * kMonSlots);
    I.iterations = a.take<int>(2);  // iterations, then the launch's fault word
    dCentroids_ = a.take<double>(2 * N);
    dWallCentres_ = a.take<double>(std::max<std::size_t>(wallCentres.size(), 2));
    dView_ = a.take<Instance>(1);
    dWall_.owner = a.take<int>(S);
    dWall_.second = a.take<int>(S);
    dWall_.cx = a.take<double>(S); dWall_.cy = a.take<double>(S);
    dWall_.tx = a.take<double>(S); dWall_.ty = a.take<double>(S);
    dWall_.nx = a.take<double>(S); dWall_.ny = a.take<double>(S);
    dWall_.length = a.take<double>(S);
    dWall_.wallDistance = a.take<double>(S);
    dWall_.outerDistance = a.take<double>(S);
    dStations_ = a.take<double>(S * kStationValues);
    dFaceStage_ = a.take<double>(static_cast<std::size_t>(F_));
    dForces_ = a.take<double>(16);
    if (!mgShape_.empty()) {
      Multigrid& G = I.mg;
      G.levels = static_cast<int>(mgShape_.size());
      G.distributed = mgDistributed_;
      G.warpFrom = G.levels;
      for (int l = mgDistributed_; l < G.levels; ++l) {
        if (mgShape_[l].NI * mgShape_[l].NJ <= 64) {
          G.warpFrom = l;
          break;
        }
      }
      G.smemBytes = mgSmemBytes_;
      // Red-black sweeps before and after the coarse correction, and on the
      // coarsest level; CFD_MG="pre,post,coarse" overrides for tuning runs.
      G.pre = 1;
      G.post = 1;
      G.coarse = 2;
      if (const char* env = std::getenv("CFD_MG")) {
        int a = 0, b = 0, c = 0;
        if (std::sscanf(env, "%d,%d,%d", &a, &b, &c) == 3 && a >= 1 && b >= 1 && c >= 1 && a <= 8 &&
            b <= 8 && c <= 64) {
          G.pre = a;
          G.post = b;
          G.coarse = c;
        }
      }
      for (int l = 0; l < G.levels; ++l) {
        const MgShape& sh = mgShape_[l];
        const std::size_t n = static_cast<std::size_t>(sh.NI) * sh.NJ;
        MgLevel& L = G.lv[l];
        L.NI = sh.NI;
        L.NJ = sh.NJ;
        L.smem = sh.smem;
        L.smemWake = sh.smemWake;
        L.D = a.take<float>(n); L.S = a.take<float>(n); L.N = a.take<float>(n);
        L.W = a.take<float>(n); L.E = a.take<float>(n); L.inv = a.take<float>(n);
        L.x = a.take<float>(n); L.b = a.take<float>(n);
        L.wake = (l == 0) ? I.acrossJ0 : a.take<int>(sh.NI);
      }
      float** vectors[] = {&G.r, &G.q, &G.e, &G.z0, &G.z1, &G.d0, &G.d1};
      for (float** ptr : vectors) *ptr = a.take<float>(N);
      for (Rows32* rows : {&I.mom, &I.tk, &I.tw}) {
        float** arrays[] = {&rows->D, &rows->S, &rows->N, &rows->W, &rows->E, &rows->r, &rows->x};
        for (float** ptr : arrays) *ptr = a.take<float>(N);
      }
      I.momRv = a.take<float>(N);
      I.momXv = a.take<float>(N);
    }
  };
  carve(arena_);
  arenaBytes_ = arena_.bytes();
  if (Status st = arena_.allocate(); st != CFD_OK) return st;
  carve(arena_);
  dHistory_ = view_.history;
  dIterations_ = view_.iterations;
  CUDA_OR_FAIL(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));

  // Scatter per-face data into the two device families.
  std::vector<double> hN(FN), hE(FE);
  auto put = [&](const std::vector<double>& src, const double* dN, const double* dE) -> Status {
    std::fill(hN.begin(), hN.end(), 0.0);
    std::fill(hE.begin(), hE.end(), 0.0);
    for (int f = 0; f < F_; ++f) (famOf(f) ? hE : hN)[idxOf(f)] = src[f];
    CUDA_OR_FAIL(cudaMemcpy(const_cast<double*>(dN), hN.data(), FN * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OR_FAIL(cudaMemcpy(const_cast<double*>(dE), hE.data(), FE * sizeof(double), cudaMemcpyHostToDevice));
    return CFD_OK;
  };
  std::vector<double> nx(F), ny(F), bu(F), bv(F);
  for (std::size_t f = 0; f < F; ++f) {
    nx[f] = faceNormal_[2 * f];
    ny[f] = faceNormal_[2 * f + 1];
    bu[f] = bcVel_[2 * f];
    bv[f] = bcVel_[2 * f + 1];
  }
  Instance& I = view_;
  Status st = CFD_OK;
  if ((st = put(Sx_, I.gN.Sx, I.gE.Sx)) || (st = put(Sy_, I.gN.Sy, I.gE.Sy)) ||
      (st = put(D_, I.gN.D, I.gE.D)) || (st = put(Tx, I.gN.Tx, I.gE.Tx)) ||
      (st = put(Ty, I.gN.Ty, I.gE.Ty)) || (st = put(w_, I.gN.w, I.gE.w)) ||
      (st = put(Dt, I.gN.Dt, I.gE.Dt)) || (st = put(nx, I.gN.nx, I.gE.nx)) ||
      (st = put(ny, I.gN.ny, I.gE.ny)) || (st = put(bu, I.bcuN, I.bcuE)) ||
      (st = put(bv, I.bcvN, I.bcvE)) || (st = put(bcP_, I.bcpN, I.bcpE))) {
    return st;
  }
  std::vector<int8_t> kN(FN, 0), kE(FE, 0);
  for (int f = 0; f < F_; ++f) (famOf(f) ? kE : kN)[idxOf(f)] = static_cast<int8_t>(kind_[f]);
  CUDA_OR_FAIL(cudaMemcpy(const_cast<int8_t*>(I.kindN), kN.data(), FN, cudaMemcpyHostToDevice));
  CUDA_OR_FAIL(cudaMemcpy(const_cast<int8_t*>(I.kindE), kE.data(), FE, cudaMemcpyHostToDevice));
  CUDA_OR_FAIL(cudaMemcpy(const_cast<int*>(I.acrossJ0), acrossJ0.data(), NI_ * sizeof(int), cudaMemcpyHostToDevice));
  for (std::size_t l = 1; l < mgShape_.size(); ++l) {
    CUDA_OR_FAIL(cudaMemcpy(const_cast<int*>(I.mg.lv[l].wake), mgShape_[l].wake.data(),
                            mgShape_[l].NI * sizeof(int), cudaMemcpyHostToDevice));
  }
  CUDA_OR_FAIL(cudaMemcpy(const_cast<double*>(I.vol), cellArea_.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_OR_FAIL(cudaMemcpy(const_cast<uint8_t*>(I.wallMask), wallMask.data(), N, cudaMemcpyHostToDevice));
  CUDA_OR_FAIL(cudaMemcpy(dCentroids_, centroid_.data(), 2 * N * sizeof(double), cudaMemcpyHostToDevice));
  if (!wallCentres.empty()) {
    CUDA_OR_FAIL(cudaMemcpy(dWallCentres_, wallCentres.data(), wallCentres.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  dWall_.count = wall_.count();
  dWall_.leadingEdge = wall_.leadingEdge;
  if (wall_.count() > 0) {
    const std::size_t n = wall_.owner.size();
    CUDA_OR_FAIL(cudaMemcpy(const_cast<int*>(dWall_.owner), wall_.owner.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OR_FAIL(cudaMemcpy(const_cast<int*>(dWall_.second), wall_.second.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    const std::pair<const double*, const std::vector<double>*> cols[] = {
        {dWall_.cx, &wall_.cx}, {dWall_.cy, &wall_.cy}, {dWall_.tx, &wall_.tx}, {dWall_.ty, &wall_.ty},
        {dWall_.nx, &wall_.nx}, {dWall_.ny, &wall_.ny}, {dWall_.length, &wall_.length},
        {dWall_.wallDistance, &wall_.wallDistance}, {dWall_.outerDistance, &wall_.outerDistance}};
    for (const auto& col : cols) {
      CUDA_OR_FAIL(cudaMemcpy(const_cast<double*>(col.first), col.second->data(), n * sizeof(double),
                              cudaMemcpyHostToDevice));
    }
  }
  // momentumDiagonal_ starts at 1 (SimpleSolver.cpp:64).
  {
    std::vector<double> ones(N, 1.0);
    CUDA_OR_FAIL(cudaMemcpy(I.aD, ones.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  }

  // Wall distance, once, on the device (TurbulenceModel.cpp:28-65).
  double totalArea = 0.0;
  for (double a : cellArea_) totalArea += a;
  const double far = 1.0e6 * std::sqrt(std::abs(totalArea) + 1.0);
  if ((st = launchWallDistance(N_, dCentroids_, static_cast<int>(wallCentres.size() / 2), dWallCentres_,
                               far, const_cast<double*>(I.wallDist), stream_)) != CFD_OK) {
    return st;
  }
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  wallDist_.resize(N);
  CUDA_OR_FAIL(cudaMemcpy(wallDist_.data(), I.wallDist, N * sizeof(double), cudaMemcpyDeviceToHost));

  clusterSize_ = chooseClusterSize(N_);
  // Launch-shape overrides for tuning sweeps: CTAs per solve (1..16) and
  // threads per CTA (a multiple of 32, at most 512).
  if (const char* env = std::getenv("CFD_CLUSTER_SIZE")) {
    const int r = std::atoi(env);
    if (r >= 1 && r <= 16) clusterSize_ = r;
  }
  if (const char* env = std::getenv("CFD_THREADS")) {
    const int t = std::atoi(env);
    if (t >= 32 && t <= 512 && t % 32 == 0) threads_ = t;
  }
  return uploadSettings();
}

std::size_t Solver::estimateBytes(int NI, int NJ) {
  // cell arrays (~60), face arrays of both families (~26), per-face geometry
  // and conditions; rounded up generously.
  const std::size_t N = static_cast<std::size_t>(NI) * NJ;
  const std::size_t F = static_cast<std::size_t>(NI) * (NJ + 1) + static_cast<std::size_t>(NI + 1) * NJ;
  return (64 * N + 16 * F) * 8 + (1u << 20);
}

void Solver::planMultigrid(const std::vector<int>& wake0) {
  mgShape_.clear();
  mgShape_.push_back(MgShape{NI_, NJ_, -1, -1, wake0});
  // Halve both directions while the columns pair up and the wake map stays
  // a map between aggregates (partner aggregates of the two cells agree).
  while (static_cast<int>(mgShape_.size()) < kMaxMgLevels) {
    const MgShape f = mgShape_.back();
    if (f.NI % 2 != 0 || f.NJ < 2 || f.NI * f.NJ <= 16) break;
    MgShape c{f.NI / 2, (f.NJ + 1) / 2, -1, -1, std::vector<int>(f.NI / 2, -1)};
    bool ok = true;
    for (int I = 0; I < c.NI; ++I) {
      const int a = f.wake[2 * I], b = f.wake[2 * I + 1];
      const int pa = (a >= 0) ? a / 2 : -1, pb = (b >= 0) ? b / 2 : -1;
      if (pa >= 0 && pb >= 0 && pa != pb) ok = false;
      c.wake[I] = (pa >= 0) ? pa : pb;
      if (c.wake[I] == I) ok = false;
      // The level's red-black sweeps update a colour's cells concurrently, so
      // partners across the cut must have opposite colours (both in row 0:
      // I + wake[I] odd); with an odd number of columns they would not, and
      // the two cells would read each other while both are written.
      if (c.wake[I] >= 0 && ((I + c.wake[I]) & 1) == 0) ok = false;
    }
    if (!ok) break;
    mgShape_.push_back(std::move(c));
  }
  const int levels = static_cast<int>(mgShape_.size());
  mgDistributed_ = levels;
  for (int l = 1; l < levels; ++l) {
    if (mgShape_[l].NI * mgShape_[l].NJ <= kMgSharedCells) {
      mgDistributed_ = l;
      break;
    }
  }
  int bytes = 0;
  for (int l = mgDistributed_; l < levels; ++l) {
    mgShape_[l].smem = bytes;
    bytes += 8 * ((mgShape_[l].NI * mgShape_[l].NJ + 3) & ~3) * static_cast<int>(sizeof(float));
    mgShape_[l].smemWake = bytes;
    bytes += ((mgShape_[l].NI + 3) & ~3) * static_cast<int>(sizeof(int));
  }
  mgSmemBytes_ = bytes;
}

Status Solver::setLaunchShape(int clusterSize, int threads) {
  if (clusterSize < 1 || clusterSize > 16 || threads < 32 || threads > 512 || threads % 32 != 0) {
    return fail(CFD_INVALID_ARGUMENT, "cluster size must be 1..16 and threads a multiple of 32 up to 512");
  }
  clusterSize_ = clusterSize;
  threads_ = threads;
  return CFD_OK;
}

int Solver::launchSmemBytes(int clusterSize) const {
  if (settings_.precision == 1) {
    const int scan = chainSweepBytes(NI_, 4);  // the chained k/omega row sweeps, FP32
    return std::max(mgSmemBytes_, (scan <= kMaxCgSharedBytes) ? scan : 0);
  }
  return cgSharedBytes(NI_, NJ_, clusterSize);
}

Solver::~Solver() {
  if (stream_ != nullptr) cudaStreamDestroy(stream_);
  if (dNodes_ != nullptr) cudaFree(dNodes_);
}

Status Solver::uploadSettings() {
  Instance& I = view_;
  I.NI = NI_;
  I.NJ = NJ_;
  I.N = N_;
  I.model = model_;
  I.precision = settings_.precision;
  I.mgCap = (settings_.innerIterations > 0) ? std::min(settings_.innerIterations, settings_.pressureIterations)
                                            : settings_.pressureIterations;
  I.alphaU = settings_.velocityRelaxation;
  I.alphaP = settings_.pressureRelaxation;
  I.blend = settings_.nonOrthogonalBlend;
  I.alphaT = settings_.turbulenceRelaxation;
  I.sweeps = settings_.momentumSweeps;
  I.cgMax = settings_.pressureIterations;
  I.cgTol = settings_.pressureTolerance;
  I.sou = (settings_.scheme != 0) ? 1 : 0;
  I.nCorr = settings_.nonOrthogonalCorrectors;
  I.hasPRef = hasPRef_ ? 1 : 0;
  I.refMassFlow = refMassFlow_;
  I.kIn = kIn_;
  I.wIn = wIn_;
  // SSTConstants::gamma1/gamma2 (KOmegaSST.cpp:96-102) and beta*^(1/4).
  const double beta1 = 0.075, beta2 = 0.0828, betaStar = 0.09, kappa = 0.41;
  I.gamma1 = beta1 / betaStar - 0.5 * kappa * kappa / std::sqrt(betaStar);
  I.gamma2 = beta2 / betaStar - 0.856 * kappa * kappa / std::sqrt(betaStar);
  I.betaStarQuarter = std::pow(betaStar, 0.25);
  I.stopTol = -1.0;
  I.iterLimit = 0x7fffffff;
  CUDA_OR_FAIL(cudaMemcpy(dView_, &view_, sizeof(Instance), cudaMemcpyHostToDevice));
  return CFD_OK;
}

Status Solver::setSettings(const Settings& s) {
  if (!(s.velocityRelaxation > 0.0) || s.velocityRelaxation > 1.0 || !(s.pressureRelaxation > 0.0) ||
      s.pressureRelaxation > 1.0) {
    return fail(CFD_INVALID_ARGUMENT, "relaxation factors must lie in (0, 1]");
  }
  if (s.precision != settings_.precision) {
    return fail(CFD_INVALID_ARGUMENT, "the precision form is fixed when the solver is created");
  }
  settings_ = s;
  return uploadSettings();
}

Status Solver::download(const double* dev, std::size_t n, double* host) {
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  CUDA_OR_FAIL(cudaMemcpy(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost));
  return CFD_OK;
}

Status Solver::upload(double* dev, const double* host, std::size_t n) {
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  CUDA_OR_FAIL(cudaMemcpy(dev, host, n * sizeof(double), cudaMemcpyHostToDevice));
  return CFD_OK;
}

// ---- initialise (SimpleSolver.cpp:133-210) ------------------------------------------

Status Solver::initialise(const double* u, const double* v, const double* p, const double* rho,
                          const double* mu) {
  if (u == nullptr || v == nullptr || p == nullptr || rho == nullptr || mu == nullptr) {
    return fail(CFD_INVALID_ARGUMENT, "initial field has missing arrays");
  }
  const std::size_t N = N_, F = F_;
  muMol_.assign(mu, mu + N);
  // Current fluxes decide imposesVelocity during the seed, as in the reference.
  std::vector<double> flux(F, 0.0);
  if (Status st = readField(CFD_FIELD_MASS_FLUX, flux.data()); st != CFD_OK) return st;

  double speed = 0.0;
  for (std::size_t c = 0; c < N; ++c) speed = std::max(speed, hyp(u[c], v[c]));
  std::vector<double> dead(F, 0.0);
  for (std::size_t f = 0; f < F; ++f) {
    if (kind_[f] != CFD_BC_FARFIELD) continue;
    dead[f] = 1.0e-3 * rho[owner_[f]] * speed * hyp(Sx_[f], Sy_[f]);
  }
  auto imposes = [&](std::size_t f) {
    switch (kind_[f]) {
      case CFD_BC_NOSLIP_WALL:
      case CFD_BC_INLET: return true;
      case CFD_BC_FARFIELD: return flux[f] < dead[f];
      default: return false;
    }
  };
  std::vector<double> seeded(F, 0.0);
  for (std::size_t f = 0; f < F; ++f) {
    const int o = owner_[f];
    const int other = across_[f];
    double fu, fv;
    if (other >= 0) {
      const double w = w_[f];
      fu = w * u[o] + (1.0 - w) * u[other];
      fv = w * v[o] + (1.0 - w) * v[other];
    } else if (imposes(f)) {
      fu = bcVel_[2 * f];
      fv = bcVel_[2 * f + 1];
    } else {
      fu = u[o];
      fv = v[o];
    }
    double density = rho[o];
    if (neighbour_[f] >= 0) {
      const double w = w_[f];
      density = w * rho[o] + (1.0 - w) * rho[neighbour_[f]];
    }
    seeded[f] = density * (fu * Sx_[f] + fv * Sy_[f]);
  }
  double ref = 0.0;
  for (std::size_t f = 0; f < F; ++f) {
    if (boundary_[f] == CFD_FACE_INTERIOR || kind_[f] == CFD_BC_INTERNAL) continue;
    ref += std::max(-seeded[f], 0.0);
  }
  if (!(ref > 0.0)) ref = 1.0;
  refMassFlow_ = ref;

  Instance& I = view_;
  Status st = CFD_OK;
  if ((st = upload(I.u, u, N)) || (st = upload(I.v, v, N)) || (st = upload(I.p, p, N)) ||
      (st = upload(I.rho, rho, N)) || (st = upload(I.mu, mu, N)) || (st = upload(I.muMol, mu, N))) {
    return st;
  }
  {
    const std::size_t FN = static_cast<std::size_t>(NI_) * (NJ_ + 1);
    const std::size_t FE = static_cast<std::size_t>(NI_ + 1) * NJ_;
    std::vector<double> hN(FN, 0.0), hE(FE, 0.0), dN(FN, 0.0), dE(FE, 0.0);
    for (int f = 0; f < F_; ++f) {
      (famOf(f) ? hE : hN)[idxOf(f)] = seeded[f];
      (famOf(f) ? dE : dN)[idxOf(f)] = dead[f];
    }
    if ((st = upload(I.mfN, hN.data(), FN)) || (st = upload(I.mfE, hE.data(), FE)) ||
        (st = upload(const_cast<double*>(I.deadN), dN.data(), FN)) ||
        (st = upload(const_cast<double*>(I.deadE), dE.data(), FE))) {
      return st;
    }
  }
  initialised_ = true;
  if (model_ == 2) {
    if ((st = sstInitialise()) != CFD_OK) return st;
  } else if (model_ == 1) {
    // LaminarModel: mu_t = 0, so mu_eff = mu + 0 (TurbulenceModel.cpp:67-71).
    std::vector<double> eff(N);
    for (std::size_t c = 0; c < N; ++c) eff[c] = muMol_[c] + 0.0;
    if ((st = upload(I.mu, eff.data(), N)) != CFD_OK) return st;
  }
  return uploadSettings();
}

// ---- KOmegaSST::initialise (KOmegaSST.cpp:104-200) ------------------------------------

Status Solver::sstInitialise() {
  const std::size_t N = N_;
  const Settings& s = settings_;
  if (!std::isfinite(s.inflowIntensity) || s.inflowIntensity < 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "turbulence intensity must be finite and not negative");
  }
  if (!std::isfinite(s.inflowViscosityRatio) || s.inflowViscosityRatio <= 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "the eddy viscosity ratio must be positive");
  }
  if (!std::isfinite(s.inflowLengthScale) || s.inflowLengthScale < 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "the turbulence length scale must not be negative");
  }
  // The model initialises from the field as the solver holds it now: the
  // effective viscosity is what the reference passes (field_.viscosity).
  std::vector<double> u(N), v(N), rho(N), mu(N);
  Instance& I = view_;
  Status st = CFD_OK;
  if ((st = download(I.u, N, u.data())) || (st = download(I.v, N, v.data())) ||
      (st = download(I.rho, N, rho.data())) || (st = download(I.mu, N, mu.data()))) {
    return st;
  }
  double refSpeed = 0.0, refRho = 0.0, refMu = 0.0;
  for (std::size_t c = 0; c < N; ++c) {
    const double sp = hyp(u[c], v[c]);
    if (sp > refSpeed) refSpeed = sp;
    refRho = std::max(refRho, rho[c]);
    refMu = std::max(refMu, mu[c]);
  }
  if (!(refSpeed > 0.0) || !(refRho > 0.0) || !(refMu > 0.0)) {
    return fail(CFD_INVALID_ARGUMENT, "the starting field has no scale to set freestream turbulence from");
  }
  const double betaStar = 0.09, beta1 = 0.075, kappa = 0.41;
  const double intensity = std::max(s.inflowIntensity, 1.0e-8);
  kIn_ = 1.5 * (intensity * refSpeed) * (intensity * refSpeed);
  double eddy = 0.0;
  if (s.inflowLengthScale > 0.0) {
    wIn_ = std::max(std::sqrt(kIn_) / (std::pow(betaStar, 0.25) * s.inflowLengthScale), kMinOmega);
    eddy = refRho * kIn_ / wIn_;
  } else {
    eddy = s.inflowViscosityRatio * refMu;
    wIn_ = std::max(refRho * kIn_ / eddy, kMinOmega);
  }
  (void)eddy;
  std::vector<double> k(N, kIn_), om(N, wIn_), mut(N), eff(N);
  for (std::size_t c = 0; c < N; ++c) {
    const double d = std::max(wallDist_[c], kTinySst);
    const double nu = mu[c] / std::max(rho[c], kTinySst);
    // wallOmega (KOmegaSST.cpp:86-92)
    const double dd = std::max(d, kTinySst);
    const double viscous = 6.0 * nu / (beta1 * dd * dd);
    const double logarithmic = std::sqrt(std::max(k[c], 0.0)) / (std::pow(betaStar, 0.25) * kappa * dd);
    const double wall = std::sqrt(viscous * viscous + logarithmic * logarithmic);
    om[c] = std::max(wIn_, wall);
    mut[c] = rho[c] * k[c] / om[c];
    eff[c] = muMol_[c] + mut[c];
  }
  if ((st = upload(I.k, k.data(), N)) || (st = upload(I.om, om.data(), N)) ||
      (st = upload(I.mut, mut.data(), N)) || (st = upload(I.mu, eff.data(), N))) {
    return st;
  }
  return uploadSettings();
}

// ---- setTurbulenceModel (SimpleSolver.cpp:212-230) -------------------------------------

Status Solver::setTurbulence(int model) {
  if (model < 0 || model > 2) return fail(CFD_INVALID_ARGUMENT, "unknown turbulence model");
  const int previous = model_;
  model_ = model;
  if (model == 0) {
    if (initialised_) {
      if (Status st = upload(view_.mu, muMol_.data(), N_); st != CFD_OK) return st;
    }
    return uploadSettings();
  }
  if (!initialised_) return uploadSettings();
  (void)previous;
  if (model == 1) {
    std::vector<double> eff(N_);
    for (int c = 0; c < N_; ++c) eff[c] = muMol_[c] + 0.0;
    if (Status st = upload(view_.mu, eff.data(), N_); st != CFD_OK) return st;
    return uploadSettings();
  }
  return sstInitialise();
}

// ---- iterate ---------------------------------------------------------------------------

Status Solver::iterate(int n, int stopStage, double tolerance, std::vector<double>* history, int* taken) {
  if (!initialised_) return fail(CFD_INVALID_ARGUMENT, "initialise() has not been called");
  if (n < 0) return fail(CFD_INVALID_ARGUMENT, "negative iteration count");
  if (history != nullptr) history->clear();
  int total = 0;
  while (total < n) {
    const int chunk = std::min(n - total, historyCapacity_);
    if (Status st = launchSimple(dView_, 1, clusterSize_, threads_, chunk, stopStage, tolerance, stream_,
                                 launchSmemBytes(clusterSize_));
        st != CFD_OK) {
      return st;
    }
    CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
    int words[2] = {0, 0};
    CUDA_OR_FAIL(cudaMemcpy(words, dIterations_, sizeof(words), cudaMemcpyDeviceToHost));
    if (words[1] != 0) return launchFault(words[1]);
    const int ran = words[0];
    if (history != nullptr && ran > 0) {
      const std::size_t old = history->size();
      history->resize(old + static_cast<std::size_t>(ran) * kMonSlots);
      CUDA_OR_FAIL(cudaMemcpy(history->data() + old, dHistory_, static_cast<std::size_t>(ran) * kMonSlots * sizeof(double),
                              cudaMemcpyDeviceToHost));
    }
    total += ran;
    if (ran < chunk || stopStage != kStageEnd) break;
  }
  if (taken != nullptr) *taken = total;
  return CFD_OK;
}

// ---- field access -------------------------------------------------------------------

Status Solver::readField(int which, double* out) {
  if (out == nullptr) return fail(CFD_INVALID_ARGUMENT, "null output");
  const Instance& I = view_;
  const std::size_t N = N_, F = F_;
  const std::size_t FN = static_cast<std::size_t>(NI_) * (NJ_ + 1);
  const std::size_t FE = static_cast<std::size_t>(NI_ + 1) * NJ_;
  auto cell = [&](const double* dev) { return download(dev, N, out); };
  auto faces = [&](const double* dN, const double* dE) -> Status {
    std::vector<double> hN(FN), hE(FE);
    if (Status st = download(dN, FN, hN.data()); st != CFD_OK) return st;
    if (Status st = download(dE, FE, hE.data()); st != CFD_OK) return st;
    for (int f = 0; f < F_; ++f) out[f] = (famOf(f) ? hE : hN)[idxOf(f)];
    return CFD_OK;
  };
  auto vec2 = [&](const double* dx, const double* dy) -> Status {
    std::vector<double> hx(N), hy(N);
    if (Status st = download(dx, N, hx.data()); st != CFD_OK) return st;
    if (Status st = download(dy, N, hy.data()); st != CFD_OK) return st;
    for (std::size_t c = 0; c < N; ++c) {
      out[2 * c] = hx[c];
      out[2 * c + 1] = hy[c];
    }
    return CFD_OK;
  };
  auto rowsToFaces = [&](bool upper) -> Status {
    // Row storage (S, N, W, E coefficients of each cell) back to the LDU
    // upper/lower per face of LinearSystem.hpp:29-71.
    std::vector<double> aS(N), aN(N), aW(N), aE(N);
    Status st = CFD_OK;
    if ((st = download(I.aS, N, aS.data())) || (st = download(I.aN, N, aN.data())) ||
        (st = download(I.aW, N, aW.data())) || (st = download(I.aE, N, aE.data()))) {
      return st;
    }
    for (std::size_t f = 0; f < F; ++f) {
      out[f] = 0.0;
      const int o = owner_[f], n = neighbour_[f];
      if (n >= 0) {
        if (static_cast<int>(f) < jFaces_) out[f] = upper ? aN[o] : aS[n];
        else out[f] = upper ? aE[o] : aW[n];
      } else if (across_[f] >= 0 && upper) {
        out[f] = aS[o];
      }
    }
    return CFD_OK;
  };
  switch (which) {
    case CFD_FIELD_U: return cell(I.u);
    case CFD_FIELD_V: return cell(I.v);
    case CFD_FIELD_P: return cell(I.p);
    case CFD_FIELD_RHO: return cell(I.rho);
    case CFD_FIELD_MU_EFF: return cell(I.mu);
    case CFD_FIELD_MASS_FLUX: return faces(I.mfN, I.mfE);
    case CFD_FIELD_DIVERGENCE: {
      // SimpleSolver::divergence (SimpleSolver.cpp:796-817), on the host.
      std::vector<double> flux(F), rho(N);
      Status st = CFD_OK;
      if ((st = readField(CFD_FIELD_MASS_FLUX, flux.data())) != CFD_OK) return st;
      if ((st = download(I.rho, N, rho.data())) != CFD_OK) return st;
      std::fill(out, out + N, 0.0);
      for (std::size_t f = 0; f < F; ++f) {
        const int o = owner_[f];
        const double vf = flux[f] / std::max(rho[o], kTinySolver);
        out[o] += vf;
        if (neighbour_[f] >= 0) out[neighbour_[f]] -= vf;
      }
      for (std::size_t c = 0; c < N; ++c) out[c] = (cellArea_[c] > 0.0) ? out[c] / cellArea_[c] : 0.0;
      return CFD_OK;
    }
    case CFD_FIELD_MU_MOLECULAR: return cell(I.muMol);
    case CFD_FIELD_GRAD_U: return vec2(I.gux, I.guy);
    case CFD_FIELD_GRAD_V: return vec2(I.gvx, I.gvy);
    case CFD_FIELD_GRAD_P: return vec2(I.gpx, I.gpy);
    case CFD_FIELD_MOM_DIAG: return cell(I.aD);
    case CFD_FIELD_MOM_SOURCE_U: return cell(I.bU);
    case CFD_FIELD_MOM_SOURCE_V: return cell(I.bV);
    case CFD_FIELD_MOM_UPPER: return rowsToFaces(true);
    case CFD_FIELD_MOM_LOWER: return rowsToFaces(false);
    case CFD_FIELD_MOMENTUM_DIAGONAL: return cell(I.aD);
    case CFD_FIELD_P_DIAG: return cell(I.pD);
    case CFD_FIELD_P_SOURCE: return cell(I.pB);
    case CFD_FIELD_P_UPPER: return faces(I.pN, I.pE);
    case CFD_FIELD_NET_FLUX: return cell(I.net);
    case CFD_FIELD_P_CORRECTION: return cell(I.x);
    case CFD_FIELD_K: return cell(I.k);
    case CFD_FIELD_OMEGA: return cell(I.om);
    case CFD_FIELD_MUT: return cell(I.mut);
    case CFD_FIELD_WALL_DISTANCE: return cell(I.wallDist);
    case CFD_FIELD_STRAIN: return cell(I.strain);
    case CFD_FIELD_F1: return cell(I.f1);
    case CFD_FIELD_F2: return cell(I.f2);
    case CFD_FIELD_CROSS_DIFFUSION: return cell(I.cd);
    case CFD_FIELD_PRODUCTION: return cell(I.prod);
    case CFD_FIELD_GRAD_K: return vec2(I.gkx, I.gky);
    case CFD_FIELD_GRAD_OMEGA: return vec2(I.gwx, I.gwy);
    case CFD_FIELD_T_DIAG_K: return cell(I.kD);
    case CFD_FIELD_T_SOURCE_K: return cell(I.kB);
    case CFD_FIELD_T_DIAG_W: return cell(I.wD);
    case CFD_FIELD_T_SOURCE_W: return cell(I.wB);
    default: break;
  }
  return fail(CFD_OUT_OF_RANGE, "unknown field " + std::to_string(which));
}

Status Solver::streamlines(const double* seeds, int count, const StreamlineSettings& o, int* lengths,
                           double* points, long long capacity, long long* total) {
  if (!initialised_) return fail(CFD_INVALID_ARGUMENT, "initialise() has not been called");
  if (nodes_.empty()) return fail(CFD_NOT_FOUND, "the mesh was created without node coordinates");
  if (count < 0 || (count > 0 && seeds == nullptr) || lengths == nullptr) {
    return fail(CFD_INVALID_ARGUMENT, "seeds and lengths are required");
  }
  if (o.maxSteps < 1 || !(o.stepFraction > 0.0)) {
    return fail(CFD_INVALID_ARGUMENT, "streamline step settings are unusable");  // Streamlines.cpp:101-103
  }
  if (count == 0) {
    if (total != nullptr) *total = 0;
    return CFD_OK;
  }
  if (dNodes_ == nullptr) {
    CUDA_OR_FAIL(cudaMalloc(reinterpret_cast<void**>(&dNodes_), nodes_.size() * sizeof(double)));
    CUDA_OR_FAIL(cudaMemcpy(dNodes_, nodes_.data(), nodes_.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  // per call: the seeds, their cells, and both halves of every curve
  const std::size_t perCurve = 2 * static_cast<std::size_t>(o.maxSteps + 1);
  const std::size_t bytes = 2 * count * sizeof(double) + count * sizeof(int) + 2 * count * sizeof(int) +
                            2 * count * perCurve * sizeof(double) + 512;
  char* scratch = nullptr;
  CUDA_OR_FAIL(cudaMalloc(reinterpret_cast<void**>(&scratch), bytes));
  auto release = [&]() { cudaFree(scratch); };
  double* dSeeds = reinterpret_cast<double*>(scratch);
  double* dPoints = dSeeds + 2 * count;
  int* dCells = reinterpret_cast<int*>(dPoints + 2 * count * perCurve);
  int* dLengths = dCells + count;
  cudaError_t e = cudaMemcpyAsync(dSeeds, seeds, 2 * count * sizeof(double), cudaMemcpyHostToDevice, stream_);
  if (e != cudaSuccess) {
    release();
    return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  }
  const Instance& I = view_;
  if (Status st = launchStreamlines(NI_, NJ_, dNodes_, I.vol, I.acrossJ0, I.u, I.v, count, dSeeds, o, dCells,
                                    dPoints, dLengths, stream_);
      st != CFD_OK) {
    release();
    return st;
  }
  std::vector<int> half(2 * static_cast<std::size_t>(count));
  std::vector<double> raw(2 * count * perCurve);
  e = cudaMemcpyAsync(half.data(), dLengths, half.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(raw.data(), dPoints, raw.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  release();
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  // Each curve reads in the direction of the flow: the upstream half
  // reversed, then the downstream half without its repeated seed; a seed
  // outside the domain or a curve of fewer than 4 points is dropped
  // (Streamlines.cpp:185-194).
  long long written = 0;
  Status status = CFD_OK;
  for (int s = 0; s < count; ++s) {
    const int back = half[2 * s], fwd = half[2 * s + 1];
    const int n = (back + fwd < 4) ? 0 : back + (fwd > 0 ? fwd - 1 : 0);
    lengths[s] = n;
    if (n == 0) continue;
    if (points == nullptr || written + n > capacity) {
      status = CFD_OUT_OF_RANGE;
      written += n;
      continue;
    }
    double* out = points + 2 * written;
    const double* b = raw.data() + (2 * s) * perCurve;
    const double* f = raw.data() + (2 * s + 1) * perCurve;
    int k = 0;
    for (int q = back - 1; q >= 0; --q, ++k) {
      out[2 * k] = b[2 * q];
      out[2 * k + 1] = b[2 * q + 1];
    }
    for (int q = (fwd > 0 ? 1 : 0); q < fwd; ++q, ++k) {
      out[2 * k] = f[2 * q];
      out[2 * k + 1] = f[2 * q + 1];
    }
    written += n;
  }
  if (total != nullptr) *total = written;
  if (status != CFD_OK && points != nullptr) return fail(CFD_OUT_OF_RANGE, "points buffer too small for the curves");
  return CFD_OK;
}

Status Solver::forces(double speed, double alphaDeg, double density, double referencePressure,
                      double chord, double* out, double* cp, double* cf, int* stations,
                      int* leadingEdge) {
  if (!initialised_) return fail(CFD_INVALID_ARGUMENT, "initialise() has not been called");
  if (wall_.count() < 4) {
    return fail(CFD_NOT_FOUND, "no aerofoil surface: the mesh has no wall stations (or no node coordinates)");
  }
  if (!std::isfinite(speed) || speed <= 0.0 || !std::isfinite(density) || density <= 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "freestream speed and density must be positive");
  }
  // FreestreamConditions::dynamicPressure and angleOfAttackRad (Freestream.cpp:7-18);
  // the wind-axis rotation uses the host's cos and sin, as the reference does.
  const double dynamicPressure = 0.5 * density * speed * speed;
  const double alpha = alphaDeg * 3.14159265358979323846 / 180.0;
  const double c = (chord > 0.0) ? chord : 1.0;
  const Instance& I = view_;
  if (Status st = launchForces(dWall_, I.p, I.u, I.v, I.mu, dynamicPressure, referencePressure, c,
                               std::cos(alpha), std::sin(alpha), dStations_, dForces_, stream_);
      st != CFD_OK) {
    return st;
  }
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  double h[12];
  CUDA_OR_FAIL(cudaMemcpy(h, dForces_, sizeof(h), cudaMemcpyDeviceToHost));
  std::copy(h, h + 12, out);
  const int S = wall_.count();
  if (stations != nullptr) *stations = S;
  if (leadingEdge != nullptr) *leadingEdge = wall_.leadingEdge;
  if (cp != nullptr || cf != nullptr) {
    std::vector<double> st(static_cast<std::size_t>(S) * kStationValues);
    CUDA_OR_FAIL(cudaMemcpy(st.data(), dStations_, st.size() * sizeof(double), cudaMemcpyDeviceToHost));
    // upper: leading edge onwards; lower: from the leading edge back to 0
    int q = 0;
    for (int k = wall_.leadingEdge; k < S; ++k, ++q) {
      if (cp) cp[q] = st[static_cast<std::size_t>(k) * kStationValues + 1];
      if (cf) cf[q] = st[static_cast<std::size_t>(k) * kStationValues + 3];
    }
    for (int k = wall_.leadingEdge - 1; k >= 0; --k, ++q) {
      if (cp) cp[q] = st[static_cast<std::size_t>(k) * kStationValues + 1];
      if (cf) cf[q] = st[static_cast<std::size_t>(k) * kStationValues + 3];
    }
  }
  return CFD_OK;
}

namespace {

/// Reference face order -> the two device families: j-faces keep their
/// index, i-face offset + i*NJ + j goes to j*(NI+1) + i.
__global__ void scatterFacesKernel(const double* __restrict__ src, double* __restrict__ n,
                                   double* __restrict__ e, int NI, int NJ) {
  const int jFaces = NI * (NJ + 1);
  const int F = jFaces + (NI + 1) * NJ;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
    if (f < jFaces) {
      n[f] = src[f];
    } else {
      const int g = f - jFaces, i = g / NJ, j = g - i * NJ;
      e[j * (NI + 1) + i] = src[f];
    }
  }
}

}  // namespace

Status Solver::loadState(const double* u, const double* v, const double* p, const double* massFlux,
                         const double* k, const double* omega, const double* mut, const double* muEff) {
  if (!initialised_) return fail(CFD_INVALID_ARGUMENT, "initialise() has not been called");
  const Instance& I = view_;
  const std::size_t bytes = static_cast<std::size_t>(N_) * sizeof(double);
  // One wait for the solver's own work, then every copy queued on its
  // stream (the face permutation runs on the device), then one wait so the
  // caller may reuse its buffers on return.
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  auto put = [&](double* dev, const double* host) -> cudaError_t {
    return (host == nullptr) ? cudaSuccess : cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, stream_);
  };
  CUDA_OR_FAIL(put(I.u, u));
  CUDA_OR_FAIL(put(I.v, v));
  CUDA_OR_FAIL(put(I.p, p));
  CUDA_OR_FAIL(put(I.k, k));
  CUDA_OR_FAIL(put(I.om, omega));
  CUDA_OR_FAIL(put(I.mut, mut));
  CUDA_OR_FAIL(put(I.mu, muEff));
  if (massFlux != nullptr) {
    CUDA_OR_FAIL(cudaMemcpyAsync(dFaceStage_, massFlux, static_cast<std::size_t>(F_) * sizeof(double),
                                 cudaMemcpyHostToDevice, stream_));
    scatterFacesKernel<<<std::min((F_ + 255) / 256, 1024), 256, 0, stream_>>>(dFaceStage_, I.mfN, I.mfE, NI_, NJ_);
    CUDA_OR_FAIL(cudaGetLastError());
  }
  CUDA_OR_FAIL(cudaStreamSynchronize(stream_));
  return CFD_OK;
}

}  // namespace cfdb

// ---- C ABI ----------------------------------------------------------------------------

struct cfd_solver_t {
  cfdb::Solver* solver{nullptr};
};

namespace {
void packMonitor(const double* h, cfd_monitor* m) {
  using namespace cfdb;
  m->continuity = h[kMonContinuity];
  m->momentum_x = h[kMonMomX];
  m->momentum_y = h[kMonMomY];
  m->mass_imbalance = h[kMonMassImbalance];
  m->max_divergence = h[kMonMaxDivergence];
  m->pressure_iterations = static_cast<int>(h[kMonPressureIterations]);
  m->pad_ = 0;
  m->turbulence_first = h[kMonTurbFirst];
  m->turbulence_second = h[kMonTurbSecond];
  m->min_energy = h[kMonMinK];
  m->max_energy = h[kMonMaxK];
  m->min_dissipation = h[kMonMinW];
  m->max_dissipation = h[kMonMaxW];
  m->min_eddy_viscosity = h[kMonMinMut];
  m->max_eddy_viscosity = h[kMonMaxMut];
  m->max_eddy_viscosity_ratio = h[kMonMaxRatio];
  m->max_wall_yplus = h[kMonMaxYPlus];
}

cfd_status checkHandle(cfd_handle h) {
  if (h == nullptr || h->solver == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null solver handle");
  return CFD_OK;
}
}  // namespace

extern "C" {

const char* cfd_last_error(void) { return cfdb::g_message.c_str(); }

cfd_status cfd_set_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cfdb::fail(CFD_INVALID_ARGUMENT, cudaGetErrorString(e));
  return CFD_OK;
}

void cfd_default_settings(cfd_settings* out) {
  if (out != nullptr) cfdb::toC(cfdb::Settings{}, out);
}

cfd_status cfd_gpu_create(const cfd_mesh_desc* mesh, const cfd_face_bc* conditions,
                          const cfd_settings* settings, cfd_handle* out) {
  if (mesh == nullptr || conditions == nullptr || out == nullptr) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  }
  const cfdb::Settings s = (settings != nullptr) ? cfdb::fromC(*settings) : cfdb::Settings{};
  cfdb::Solver* solver = nullptr;
  if (cfd_status st = cfdb::Solver::create(*mesh, *conditions, s, &solver); st != CFD_OK) return st;
  *out = new cfd_solver_t{solver};
  return CFD_OK;
}

cfd_status cfd_gpu_set_turbulence(cfd_handle h, int model) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  return h->solver->setTurbulence(model);
}

cfd_status cfd_gpu_initialise(cfd_handle h, const double* u, const double* v, const double* p,
                              const double* rho, const double* mu) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  return h->solver->initialise(u, v, p, rho, mu);
}

cfd_status cfd_gpu_iterate(cfd_handle h, int n, cfd_monitor* last, cfd_monitor* history) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  std::vector<double> hist;
  int taken = 0;
  if (cfd_status st = h->solver->iterate(n, cfdb::kStageEnd, -1.0, &hist, &taken); st != CFD_OK) return st;
  if (history != nullptr) {
    for (int k = 0; k < taken; ++k) packMonitor(hist.data() + k * cfdb::kMonSlots, history + k);
  }
  if (last != nullptr && taken > 0) packMonitor(hist.data() + (taken - 1) * cfdb::kMonSlots, last);
  return CFD_OK;
}

cfd_status cfd_gpu_converge(cfd_handle h, int cap, double tol, int* taken, cfd_monitor* last) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  if (!(tol >= 0.0)) return cfdb::fail(CFD_INVALID_ARGUMENT, "tolerance must be >= 0");
  std::vector<double> hist;
  int ran = 0;
  if (cfd_status st = h->solver->iterate(cap, cfdb::kStageEnd, tol, &hist, &ran); st != CFD_OK) return st;
  if (taken != nullptr) *taken = ran;
  if (last != nullptr && ran > 0) packMonitor(hist.data() + (ran - 1) * cfdb::kMonSlots, last);
  return CFD_OK;
}

cfd_status cfd_gpu_iterate_partial(cfd_handle h, int stage, cfd_monitor* last) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  if (stage < 0 || stage > CFD_STAGE_END) return cfdb::fail(CFD_OUT_OF_RANGE, "unknown stage");
  std::vector<double> hist;
  int taken = 0;
  if (cfd_status st = h->solver->iterate(1, stage, -1.0, &hist, &taken); st != CFD_OK) return st;
  if (last != nullptr && taken > 0 && hist.size() >= static_cast<std::size_t>(cfdb::kMonSlots)) {
    packMonitor(hist.data(), last);
  }
  return CFD_OK;
}

cfd_status cfd_gpu_read_field(cfd_handle h, int which, double* out) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  return h->solver->readField(which, out);
}

cfd_status cfd_gpu_load_state(cfd_handle h, const double* u, const double* v, const double* p,
                              const double* mass_flux, const double* k, const double* omega,
                              const double* mut, const double* mu_eff) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  return h->solver->loadState(u, v, p, mass_flux, k, omega, mut, mu_eff);
}

void cfd_default_streamline_options(cfd_streamline_options* o) {
  if (o == nullptr) return;
  // StreamlineOptions' defaults (include/cfd/post/Streamlines.hpp:16-33)
  o->max_steps = 4000;
  o->step_fraction = 0.35;
  o->stall_fraction = 1e-4;
  o->reference_speed = 1.0;
  o->trace_backwards = 1;
}

cfd_status cfd_gpu_streamlines(cfd_handle h, const double* seeds, int count,
                               const cfd_streamline_options* options, int* lengths, double* points,
                               long long capacity, long long* total) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  cfd_streamline_options o;
  cfd_default_streamline_options(&o);
  if (options != nullptr) o = *options;
  cfdb::StreamlineSettings s{o.max_steps, o.step_fraction,
                             std::max(o.stall_fraction, 0.0) * std::max(o.reference_speed, 0.0),
                             o.trace_backwards};
  return h->solver->streamlines(seeds, count, s, lengths, points, capacity, total);
}

cfd_status cfd_gpu_forces(cfd_handle h, double speed, double alpha_deg, double density,
                          double reference_pressure, double chord, cfd_forces* out, double* cp,
                          double* cf) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  if (out == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null output");
  double v[12];
  int stations = 0, leadingEdge = 0;
  if (cfd_status st = h->solver->forces(speed, alpha_deg, density, reference_pressure, chord, v, cp, cf,
                                        &stations, &leadingEdge);
      st != CFD_OK) {
    return st;
  }
  out->lift_coefficient = v[0];
  out->drag_coefficient = v[1];
  out->moment_coefficient = v[2];
  out->pressure_drag_coefficient = v[3];
  out->friction_drag_coefficient = v[4];
  out->lift = v[5];
  out->drag = v[6];
  out->pitching_moment = v[7];
  out->stagnation_chord_fraction = v[8];
  out->stations = static_cast<int>(v[9]);
  out->leading_edge = leadingEdge;
  out->separation_upper_chord_fraction = v[10];
  out->separation_lower_chord_fraction = v[11];
  (void)stations;
  return CFD_OK;
}

cfd_status cfd_gpu_set_settings(cfd_handle h, const cfd_settings* settings) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  if (settings == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null settings");
  return h->solver->setSettings(cfdb::fromC(*settings));
}

cfd_status cfd_gpu_dims(cfd_handle h, int* out4) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  out4[0] = h->solver->cellsI();
  out4[1] = h->solver->cellsJ();
  out4[2] = h->solver->cells();
  out4[3] = h->solver->faces();
  return CFD_OK;
}

cfd_status cfd_gpu_scalars(cfd_handle h, double* out3) {
  if (cfd_status st = checkHandle(h); st != CFD_OK) return st;
  out3[0] = h->solver->kInflow();
  out3[1] = h->solver->omegaInflow();
  out3[2] = h->solver->referenceMassFlow();
  return CFD_OK;
}

cfd_status cfd_gpu_destroy(cfd_handle h) {
  if (h == nullptr) return CFD_OK;
  delete h->solver;
  delete h;
  return CFD_OK;
}

}  // extern "C"

// ---- batches ------------------------------------------------------------------------------

/// The solves of a batch that share a launch shape: one launch over a
/// contiguous part of the descriptor table, on a stream of its own.
struct BatchGroup {
  int offset{0}, count{0};
  int clusterSize{1}, threads{512}, smemBytes{0};
  std::vector<int> members;  // indices into cfd_batch_t::handles
  cudaStream_t stream{nullptr};
  cudaEvent_t done{nullptr};
};

struct cfd_batch_t {
  std::vector<cfd_handle> handles;
  cfdb::Instance* dTable{nullptr};
  cudaStream_t stream{nullptr};
  cudaEvent_t fork{nullptr};
  std::vector<BatchGroup> groups;  // widest clusters first
  int clusterSize{1};              // the shape of the largest group (cfd_batch_shape)
  int threads{512};
  int lastIterations{0};
  cudaGraphExec_t graph{nullptr};  // the n-iteration launch, captured once
  int graphIterations{0};
};

namespace {
cfd_status refreshTable(cfd_batch b) {
  std::vector<cfdb::Instance> table;
  table.reserve(b->handles.size());
  for (const BatchGroup& g : b->groups) {
    for (int k : g.members) table.push_back(b->handles[static_cast<std::size_t>(k)]->solver->deviceView());
  }
  cudaError_t e = cudaMemcpyAsync(b->dTable, table.data(), table.size() * sizeof(cfdb::Instance),
                                  cudaMemcpyHostToDevice, b->stream);
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  return CFD_OK;
}

/// n iterations of every solve of the batch, ordered on `s`: one launch per
/// group, the groups forked from `s` onto their own streams and joined back,
/// so solves of different launch shapes run side by side (a group of small
/// clusters fills the SMs a group of wide ones leaves idle). Used directly
/// and under stream capture.
cfd_status launchGroups(cfd_batch b, int n, int stopStage, double tolerance, cudaStream_t s) {
  if (b->groups.size() == 1) {
    const BatchGroup& g = b->groups[0];
    return cfdb::launchSimple(b->dTable + g.offset, g.count, g.clusterSize, g.threads, n, stopStage, tolerance, s,
                              g.smemBytes);
  }
  cudaError_t e = cudaEventRecord(b->fork, s);
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  cfd_status st = CFD_OK;
  for (const BatchGroup& g : b->groups) {
    e = cudaStreamWaitEvent(g.stream, b->fork, 0);
    if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
    if (st == CFD_OK) {
      st = cfdb::launchSimple(b->dTable + g.offset, g.count, g.clusterSize, g.threads, n, stopStage, tolerance,
                              g.stream, g.smemBytes);
    }
    e = cudaEventRecord(g.done, g.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, g.done, 0);
    if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  }
  return st;
}
}  // namespace

extern "C" {

cfd_status cfd_batch_create(const cfd_handle* solvers, int count, cfd_batch* out) {
  if (solvers == nullptr || out == nullptr || count <= 0) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "a batch needs at least one solver");
  }
  auto* b = new cfd_batch_t;
  for (int k = 0; k < count; ++k) {
    if (solvers[k] == nullptr || solvers[k]->solver == nullptr) {
      delete b;
      return cfdb::fail(CFD_INVALID_ARGUMENT, "null solver in batch");
    }
    b->handles.push_back(solvers[k]);
  }
  // One group per launch shape (each solve keeps its own), widest first so
  // its clusters are placed before the narrower groups fill the gaps.
  for (int k = 0; k < count; ++k) {
    const cfdb::Solver& sv = *b->handles[static_cast<std::size_t>(k)]->solver;
    auto it = std::find_if(b->groups.begin(), b->groups.end(), [&](const BatchGroup& g) {
      return g.clusterSize == sv.clusterSize() && g.threads == sv.threads();
    });
    if (it == b->groups.end()) {
      BatchGroup g;
      g.clusterSize = sv.clusterSize();
      g.threads = sv.threads();
      b->groups.push_back(g);
      it = b->groups.end() - 1;
    }
    it->members.push_back(k);
    it->smemBytes = std::max(it->smemBytes, sv.launchSmemBytes(sv.clusterSize()));
  }
  std::stable_sort(b->groups.begin(), b->groups.end(),
                   [](const BatchGroup& a, const BatchGroup& c) { return a.clusterSize > c.clusterSize; });
  int offset = 0;
  std::size_t largest = 0;
  for (std::size_t g = 0; g < b->groups.size(); ++g) {
    b->groups[g].offset = offset;
    b->groups[g].count = static_cast<int>(b->groups[g].members.size());
    offset += b->groups[g].count;
    if (b->groups[g].count > b->groups[largest].count) largest = g;
  }
  b->clusterSize = b->groups[largest].clusterSize;
  b->threads = b->groups[largest].threads;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->dTable), count * sizeof(cfdb::Instance));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (BatchGroup& g : b->groups) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    cfd_batch_destroy(b);
    return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  }
  *out = b;
  return refreshTable(b);
}

cfd_status cfd_batch_launch(cfd_batch b, int n, void* stream) {
  if (b == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null batch");
  if (n < 1 || n > 256) return cfdb::fail(CFD_OUT_OF_RANGE, "a batch launch runs 1 to 256 iterations");
  for (cfd_handle h : b->handles) {
    if (!h->solver->initialised()) return cfdb::fail(CFD_INVALID_ARGUMENT, "a solver in the batch is not initialised");
  }
  cudaStream_t s = (stream != nullptr) ? static_cast<cudaStream_t>(stream) : b->stream;
  b->lastIterations = n;
  return launchGroups(b, n, cfdb::kStageEnd, -1.0, s);
}

cfd_status cfd_batch_graph_launch(cfd_batch b, int n, void* stream) {
  if (b == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null batch");
  if (n < 1 || n > 256) return cfdb::fail(CFD_OUT_OF_RANGE, "a batch launch runs 1 to 256 iterations");
  for (cfd_handle h : b->handles) {
    if (!h->solver->initialised()) return cfdb::fail(CFD_INVALID_ARGUMENT, "a solver in the batch is not initialised");
  }
  if (b->graph == nullptr || b->graphIterations != n) {
    if (b->graph != nullptr) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    if (cfd_status st = cfdb::prepareSimpleKernel(); st != CFD_OK) return st;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
    const cfd_status launched = launchGroups(b, n, cfdb::kStageEnd, -1.0, b->stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->stream, &g);
    if (launched != CFD_OK) {
      if (g != nullptr) cudaGraphDestroy(g);
      return launched;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
    if (g != nullptr) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->graph = nullptr;
      return cfdb::fail(CFD_INITIALIZATION_FAILURE, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    b->graphIterations = n;
  }
  cudaStream_t s = (stream != nullptr) ? static_cast<cudaStream_t>(stream) : b->stream;
  b->lastIterations = n;
  const cudaError_t e = cudaGraphLaunch(b->graph, s);
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  return CFD_OK;
}

cfd_status cfd_batch_monitors(cfd_batch b, int* taken, cfd_monitor* last) {
  if (b == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null batch");
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  for (std::size_t k = 0; k < b->handles.size(); ++k) {
    const cfdb::Instance& I = b->handles[k]->solver->deviceView();
    int words[2] = {0, 0};
    e = cudaMemcpy(words, I.iterations, sizeof(words), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
    if (words[1] != 0) return cfdb::launchFault(words[1]);
    const int ran = words[0];
    if (taken != nullptr) taken[k] = ran;
    if (last != nullptr && ran > 0) {
      double h[cfdb::kMonSlots];
      e = cudaMemcpy(h, I.history + static_cast<std::size_t>(ran - 1) * cfdb::kMonSlots, sizeof(h),
                     cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
      packMonitor(h, last + k);
    }
  }
  return CFD_OK;
}

cfd_status cfd_batch_iterate(cfd_batch b, int n, double tol, int* taken, cfd_monitor* last) {
  if (b == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null batch");
  if (cfd_status st = refreshTable(b); st != CFD_OK) return st;
  int done = 0;
  std::vector<int> total(b->handles.size(), 0);
  std::vector<int> ran(b->handles.size(), 0);
  while (done < n) {
    const int chunk = std::min(n - done, 256);
    for (cfd_handle h : b->handles) {
      if (!h->solver->initialised()) return cfdb::fail(CFD_INVALID_ARGUMENT, "a solver in the batch is not initialised");
    }
    if (cfd_status st = launchGroups(b, chunk, cfdb::kStageEnd, tol, b->stream); st != CFD_OK) {
      return st;
    }
    if (cfd_status st = cfd_batch_monitors(b, ran.data(), last); st != CFD_OK) return st;
    bool allStopped = true;
    for (std::size_t k = 0; k < ran.size(); ++k) {
      total[k] += ran[k];
      if (ran[k] == chunk) allStopped = false;
    }
    done += chunk;
    if (tol >= 0.0 && allStopped) break;
  }
  if (taken != nullptr) std::copy(total.begin(), total.end(), taken);
  return CFD_OK;
}

cfd_status cfd_batch_shape(cfd_batch b, int* clusterSize, int* threads) {
  if (b == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null batch");
  if (clusterSize != nullptr) *clusterSize = b->clusterSize;
  if (threads != nullptr) *threads = b->threads;
  return CFD_OK;
}

cfd_status cfd_batch_destroy(cfd_batch b) {
  if (b == nullptr) return CFD_OK;
  if (b->stream != nullptr) cudaStreamSynchronize(b->stream);
  for (BatchGroup& g : b->groups) {
    if (g.stream != nullptr) {
      cudaStreamSynchronize(g.stream);
      cudaStreamDestroy(g.stream);
    }
    if (g.done != nullptr) cudaEventDestroy(g.done);
  }
  if (b->graph != nullptr) cudaGraphExecDestroy(b->graph);
  if (b->dTable != nullptr) cudaFree(b->dTable);
  if (b->fork != nullptr) cudaEventDestroy(b->fork);
  if (b->stream != nullptr) cudaStreamDestroy(b->stream);
  delete b;
  return CFD_OK;
}

}  // extern "C"
