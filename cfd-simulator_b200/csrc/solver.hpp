// solver.hpp - host front end of one device-resident SIMPLE solve.
//
// Mirrors cfd::solver::SimpleSolver (include/cfd/solver/SimpleSolver.hpp:159-274):
// create / setTurbulenceModel / initialise / iterate / field / massFlux /
// divergence / setSettings, with the same validation and error codes. The
// one-time set-up steps (precomputeGeometry, initialise's dead band, flux
// seed and reference mass flow, KOmegaSST::initialise) run here on the host in
// the reference's order, so the state the device starts from is the
// reference's to the last bit. Everything per iteration runs on the device.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "common.hpp"
#include "forces.hpp"
#include "instance.hpp"
#include "streamlines.hpp"

namespace cfdb {

/// Set-up that must happen once on every CUDA device a process uses (kernel
/// attributes such as the dynamic shared-memory limit are per device), from
/// any host thread. run() calls `setup` with the device current the first
/// time it sees that device, under a lock, and remembers success.
class PerDeviceOnce {
 public:
  template <typename F>
  Status run(F&& setup) {
    int device = 0;
    const cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return fail(CFD_OUT_OF_RANGE, "device ordinal too large");
    std::lock_guard<std::mutex> lock(mutex_);
    if (done_[device]) return CFD_OK;
    const Status st = setup();
    if (st == CFD_OK) done_[device] = true;
    return st;
  }

 private:
  static constexpr int kMaxDevices = 64;
  std::mutex mutex_;
  bool done_[kMaxDevices] = {};
};

/// One cudaMalloc carved into aligned arrays; released as a whole.
class DeviceArena {
 public:
  DeviceArena() = default;
  DeviceArena(const DeviceArena&) = delete;
  DeviceArena& operator=(const DeviceArena&) = delete;
  ~DeviceArena();
  /// Reserve space for an array during sizing (pass 1) or hand it out (pass 2).
  template <typename T>
  T* take(std::size_t count) {
    const std::size_t bytes = (count * sizeof(T) + 255) & ~std::size_t{255};
    T* out = (base_ == nullptr) ? nullptr : reinterpret_cast<T*>(base_ + used_);
    used_ += bytes;
    return out;
  }
  Status allocate();  // after a sizing pass: one allocation, zero-filled
  void rewind() { used_ = 0; }
  std::size_t bytes() const { return used_; }

 private:
  char* base_{nullptr};
  std::size_t used_{0};
};

struct Settings {
  double velocityRelaxation{0.5};
  double pressureRelaxation{0.2};
  int momentumSweeps{3};
  int pressureIterations{200};
  double pressureTolerance{0.01};
  int scheme{0};
  double turbulenceRelaxation{0.5};
  double inflowIntensity{0.001};
  double inflowViscosityRatio{1.0};
  double inflowLengthScale{0.0};
  int nonOrthogonalCorrectors{1};
  double nonOrthogonalBlend{1.0};
  int precision{0};
  int innerIterations{16};
};

Settings fromC(const cfd_settings& s);
void toC(const Settings& s, cfd_settings* out);

class Solver {
 public:
  static Status create(const cfd_mesh_desc& mesh, const cfd_face_bc& bc, const Settings& s,
                       Solver** out);
  ~Solver();

  Status setTurbulence(int model);
  Status initialise(const double* u, const double* v, const double* p, const double* rho,
                    const double* mu);
  /// n iterations (stopStage = kStageEnd), or one partial one; tolerance < 0
  /// disables the convergence stop. history gets kMonSlots doubles per
  /// iteration run; *taken the number run.
  Status iterate(int n, int stopStage, double tolerance, std::vector<double>* history, int* taken);
  Status readField(int which, double* out);
  Status loadState(const double* u, const double* v, const double* p, const double* massFlux,
                   const double* k, const double* omega, const double* mut, const double* muEff);
  Status setSettings(const Settings& s);
  /// Surface data and forces of the current field (device, FP64). out gets
  /// the 10 values of launchForces; cp/cf (may be null) one per station in
  /// upper-then-lower order.
  Status forces(double speed, double alphaDeg, double density, double referencePressure,
                double chord, double* out, double* cp, double* cf, int* stations, int* leadingEdge);
  /// post::traceStreamlines on the current velocity field: lengths[s] points
  /// per seed (0: dropped), packed in `points` (2 doubles each) up to
  /// `capacity` points; *total gets the points needed.
  Status streamlines(const double* seeds, int count, const StreamlineSettings& o, int* lengths,
                     double* points, long long capacity, long long* total);

  int cellsI() const { return NI_; }
  int cellsJ() const { return NJ_; }
  int cells() const { return N_; }
  int faces() const { return F_; }
  double kInflow() const { return kIn_; }
  double omegaInflow() const { return wIn_; }
  double referenceMassFlow() const { return refMassFlow_; }
  int clusterSize() const { return clusterSize_; }
  bool initialised() const { return initialised_; }
  int threads() const { return threads_; }
  std::size_t deviceBytes() const { return arenaBytes_; }
  /// Rough device footprint of a solve of NI x NJ cells (the arena's layout).
  static std::size_t estimateBytes(int NI, int NJ);
  const Instance& deviceView() const { return view_; }
  /// Dynamic shared memory a launch of this solve needs on a cluster of
  /// `clusterSize` CTAs.
  int launchSmemBytes(int clusterSize) const;
  int precision() const { return settings_.precision; }
  int wallStations() const { return wall_.count(); }
  /// CTAs per cluster (1..16) and threads per CTA (multiple of 32, <= 512).
  Status setLaunchShape(int clusterSize, int threads);
  int multigridLevels() const { return static_cast<int>(mgShape_.size()); }
  cudaStream_t stream() const { return stream_; }

 private:
  Solver() = default;
  Status build(const cfd_mesh_desc& mesh, const cfd_face_bc& bc);
  Status sstInitialise();
  Status uploadSettings();
  Status download(const double* dev, std::size_t n, double* host);
  Status upload(double* dev, const double* host, std::size_t n);
  /// Levels of the mixed form's pressure multigrid (dimensions, wake maps,
  /// which run on rank 0 alone from shared memory).
  void planMultigrid(const std::vector<int>& wake0);
  /// Reference face f -> (family, index) of the device layout.
  int famOf(int f) const { return (f < jFaces_) ? 0 : 1; }
  int idxOf(int f) const;

  int NI_{0}, NJ_{0}, N_{0}, F_{0}, jFaces_{0};
  Settings settings_{};
  int model_{0};
  bool initialised_{false};
  bool hasPRef_{false};
  double refMassFlow_{1.0};
  double kIn_{0.0}, wIn_{0.0};

  // host copies of the metrics the one-time steps need (reference order)
  std::vector<double> centroid_, cellArea_, faceCentre_, faceNormal_, faceArea_;
  std::vector<int> owner_, neighbour_, boundary_, partner_;
  std::vector<int> kind_;
  std::vector<double> bcVel_, bcP_;
  std::vector<double> Sx_, Sy_, dx_, dy_, D_, w_;  // per reference face
  std::vector<int> across_;                          // oppositeCell per face
  std::vector<double> muMol_;
  std::vector<double> wallDist_;

  HostWallTable wall_;
  WallTable dWall_{};
  double* dStations_{nullptr};
  double* dFaceStage_{nullptr};  // a face field in reference order, on its way in
  double* dForces_{nullptr};

  DeviceArena arena_;
  std::size_t arenaBytes_{0};
  Instance view_{};
  Instance* dView_{nullptr};
  double* dHistory_{nullptr};
  int* dIterations_{nullptr};
  int historyCapacity_{0};
  double* dWallCentres_{nullptr};
  std::vector<double> nodes_;   // (x, y) per node, row by row, when the mesh gave them
  double* dNodes_{nullptr};
  double* dCentroids_{nullptr};
  cudaStream_t stream_{nullptr};
  int clusterSize_{8};
  int threads_{512};

  struct MgShape {
    int NI, NJ, smem, smemWake;
    std::vector<int> wake;
  };
  std::vector<MgShape> mgShape_;
  int mgDistributed_{0};
  int mgSmemBytes_{0};
};

/// Levels of the multigrid with at most this many cells run on one CTA from
/// shared memory (eight FP32 arrays per cell: ~130 KB for all of them).
constexpr int kMgSharedCells = 3072;

/// Launch the SIMPLE kernel over `count` instances (device array), one
/// cluster of `clusterSize` CTAs each.
Status launchWallDistance(int n, const double* centroid, int walls, const double* wallCentre,
                          double far, double* out, cudaStream_t stream);

Status launchSimple(const Instance* dInstances, int count, int clusterSize, int threads,
                    int iterations, int stopStage, double tolerance, cudaStream_t stream,
                    int smemBytes);

/// The error for a launch whose fault word (Instance::iterations[1]) is
/// nonzero: a bounded wait inside the kernel gave up, so its results are not
/// to be used.
Status launchFault(int word);

/// Dynamic shared memory of the chained k/omega sweeps on rows of NI cells
/// of `elemBytes` each (two rows, the scan's warp totals and the ring).
int chainSweepBytes(int NI, int elemBytes);

/// Dynamic shared memory the pressure CG needs to keep a solve's band on
/// chip (0: it does not fit and the CG runs from global memory).
int cgSharedBytes(int NI, int NJ, int clusterSize);
constexpr int kMaxCgSharedBytes = 210 * 1024;

/// Cluster size used for a solve of `cells` cells (power of two, 1..16).
int chooseClusterSize(int cells);

/// Set the kernel's launch attributes (once per process); must run before a
/// launch is captured into a CUDA graph.
Status prepareSimpleKernel();

/// Clusters of this shape the GPU holds at once (cudaOccupancyMaxActiveClusters).
int maxActiveClusters(int clusterSize, int threads, int smemBytes);

}  // namespace cfdb
