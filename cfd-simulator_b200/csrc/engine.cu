// engine.cu - continuous batching of many SIMPLE solves on one GPU.
//
// A request queue feeds a set of resident solves. Each step admits queued
// requests whose device footprint fits the memory budget, advances every
// resident solve by up to `chunk` iterations in as few launches as there are
// cluster shapes (one thread-block cluster per solve, each on its own
// descriptor), then reads all monitors back with one copy and retires the
// solves that finished. Retiring integrates the forces on the device and
// frees the solve's memory, so the queue can fill it on the next step.
//
// The stop rules are the reference worker's (src/app/SolverWorker.cpp:164-192):
// converged when worst() of the residuals drops below the tolerance,
// diverged on a non-finite residual, iteration limit at the cap. A diverged
// solve is restarted once from the freestream, as the polar sweep's
// RetryCold does (src/post/Polar.cpp:109-121).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "cfd_gpu.h"
#include "cfd_mesh.h"
#include "common.hpp"
#include "instance.hpp"
#include "solver.hpp"

namespace cfdb {

Status makeCGrid(const char* designation, const cfd_cgrid_options& o, HostMesh* out);

namespace {

constexpr double kPi = 3.14159265358979323846;  // the double std::numbers::pi rounds to
constexpr int kMaxSweepPoints = 400;               // post::kMaxSweepPoints (Polar.hpp)

/// A C-grid built for a request: the mesh, or the generator's refusal.
struct MeshResult {
  std::shared_ptr<const HostMesh> mesh;
  Status status{CFD_OK};
  std::string message;
  double seconds{0.0};  // generation time
};
using MeshFuture = std::shared_future<MeshResult>;

/// Host C-grid generation off the caller's thread. generateCGrid +
/// buildStructured (src/mesh/CGrid.cpp:98-399, src/mesh/Mesh.cpp:89-339) take
/// tens of milliseconds for a fine grid; a serving stream draws a new section,
/// Reynolds number and first-layer height per request, so most requests need
/// a grid of their own. Workers build them while the GPU runs, and a request
/// is admitted once its mesh is ready.
class MeshPool {
 public:
  explicit MeshPool(int threads) {
    for (int k = 0; k < threads; ++k) workers_.emplace_back([this] { run(); });
  }
  MeshPool(const MeshPool&) = delete;
  MeshPool& operator=(const MeshPool&) = delete;
  ~MeshPool() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stop_ = true;
    }
    wake_.notify_all();
    for (std::thread& t : workers_) t.join();
  }

  MeshFuture build(std::string designation, const cfd_cgrid_options& o) {
    std::packaged_task<MeshResult()> task([designation = std::move(designation), o] {
      MeshResult r;
      const auto t0 = std::chrono::steady_clock::now();
      auto m = std::make_shared<HostMesh>();
      r.status = makeCGrid(designation.c_str(), o, m.get());
      if (r.status == CFD_OK) {
        r.mesh = std::move(m);
      } else {
        r.message = cfd_last_error();  // the worker's own message
      }
      r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      return r;
    });
    MeshFuture f = task.get_future().share();
    {
      std::lock_guard<std::mutex> lock(mutex_);
      tasks_.push_back(std::move(task));
    }
    wake_.notify_one();
    return f;
  }

 private:
  void run() {
    for (;;) {
      std::packaged_task<MeshResult()> task;
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [this] { return stop_ || !tasks_.empty(); });
        if (tasks_.empty()) return;  // stopping, nothing left
        task = std::move(tasks_.front());
        tasks_.pop_front();
      }
      task();
    }
  }

  std::vector<std::thread> workers_;
  std::deque<std::packaged_task<MeshResult()>> tasks_;
  std::mutex mutex_;
  std::condition_variable wake_;
  bool stop_{false};
};

bool ready(const MeshFuture& f) {
  return f.wait_for(std::chrono::seconds(0)) == std::future_status::ready;
}

/// A start other than the freestream: the u, v and p a continued polar point
/// takes over from the previous point (src/app/Panels.cpp:1145-1156).
struct WarmStart {
  std::vector<double> u, v, p;
};

struct Slot {
  int id{0};
  cfd_request request{};
  std::unique_ptr<Solver> solver;
  std::shared_ptr<const HostMesh> mesh;
  int iterations{0};
  bool retried{false};
  bool continued{false};
  int sweep{-1};  // index of the sweep this point belongs to, or -1
  int point{0};   // its position in that sweep
  double meshSeconds{0.0};
  double submitted{0.0}, started{0.0};
  std::size_t bytes{0};
};

struct Pending {
  int id{0};
  cfd_request request{};
  std::shared_ptr<const HostMesh> mesh;  // set once the mesh is ready
  MeshFuture meshFuture;                 // the mesh being built, when not yet known
  bool builtMesh{false};                 // this request's submit started the build
  double meshSeconds{0.0};
  double submitted{0.0};
  int sweep{-1};
  int point{0};
  std::shared_ptr<const WarmStart> warm;  // null: start from the freestream
};

/// A polar sweep run point after point (the reference's sweep: startPolarSweep,
/// updatePolar, src/app/Panels.cpp:1601-1797): one request per angle of
/// sweepAngles, each started when the one before has retired, from its u and
/// p when the sweep is continued.
struct Sweep {
  cfd_request base{};
  std::vector<double> angles;
  int firstId{0};
  bool continued{false};
};

using MeshKey = std::tuple<std::string, int, int, int, double, double, double, double>;

MeshKey keyOf(const cfd_request& r) {
  return {std::string(r.designation, strnlen(r.designation, sizeof(r.designation))),
          r.grid_surface_points, r.grid_wake_points, r.grid_normal_points,
          r.grid_first_layer_height, r.grid_upstream_chords, r.grid_downstream_chords,
          r.grid_vertical_chords};
}

/// Tuned launch shapes per (cells I, cells J, model, precision), shared by
/// every engine of the process, so a grid runs with one shape (and one
/// reduction order) whichever engine it is submitted to.
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_shapes;
std::mutex g_shapesMutex;

}  // namespace

struct Engine {
  std::size_t budget{0};
  std::size_t used{0};
  bool tuned{false};  // launch shapes: by grid size (false) or the occupancy tuner (true)
  int chunk{32};
  int nextId{0};
  std::deque<Pending> queue;
  std::vector<Sweep> sweeps;
  std::vector<std::unique_ptr<Slot>> active;
  std::vector<cfd_result> done;
  std::map<int, std::vector<double>> surfaces;  // Cp per wall station of each finished solve
  std::map<MeshKey, MeshFuture> meshes;  // every grid requested so far, built or being built
  std::unique_ptr<MeshPool> pool;
  std::chrono::steady_clock::time_point t0{std::chrono::steady_clock::now()};
  // the chunk in flight: its launches run while step() returns to the caller
  bool inFlight{false};
  int inFlightSlots{0};
  std::vector<int> inFlightStreams;
  // device status area: per slot, chunk monitors then the iteration count
  double* dStatus{nullptr};
  int statusSlots{0};
  Instance* dTable{nullptr};
  int tableSlots{0};
  std::vector<cudaStream_t> streams;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  ~Engine() {
    waitForLaunches();
    active.clear();
    if (dStatus) cudaFree(dStatus);
    if (dTable) cudaFree(dTable);
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
  }

  Status reserve(int slots) {
    if (slots > statusSlots) {
      if (dStatus) cudaFree(dStatus);
      const int cap = std::max(slots, 2 * statusSlots);
      const std::size_t per = static_cast<std::size_t>(chunk) * kMonSlots + 1;
      if (cudaMalloc(reinterpret_cast<void**>(&dStatus), cap * per * sizeof(double)) != cudaSuccess) {
        dStatus = nullptr;
        statusSlots = 0;
        return fail(CFD_INITIALIZATION_FAILURE, "engine status allocation failed");
      }
      statusSlots = cap;
    }
    if (slots > tableSlots) {
      if (dTable) cudaFree(dTable);
      const int cap = std::max(slots, 2 * tableSlots);
      if (cudaMalloc(reinterpret_cast<void**>(&dTable), cap * sizeof(Instance)) != cudaSuccess) {
        dTable = nullptr;
        tableSlots = 0;
        return fail(CFD_INITIALIZATION_FAILURE, "engine table allocation failed");
      }
      tableSlots = cap;
    }
    return ok();
  }

  static void uniform(const cfd_request& r, int cells, std::vector<double>* u, std::vector<double>* v,
                      std::vector<double>* p, std::vector<double>* rho, std::vector<double>* mu) {
    // FlowField::uniform (FlowField.cpp:21-47) with chord 1
    const double alpha = r.alpha_deg * kPi / 180.0;
    u->assign(cells, r.speed * std::cos(alpha));
    v->assign(cells, r.speed * std::sin(alpha));
    p->assign(cells, 0.0);
    rho->assign(cells, r.density);
    mu->assign(cells, r.density * r.speed * 1.0 / r.reynolds);
  }

  Status start(const Pending& q, std::unique_ptr<Slot>* out) {
    std::unique_ptr<Solver> solver;
    if (Status st = makeSolver(q, &solver, q.warm.get()); st != CFD_OK) return st;
    std::pair<int, int> shape;
    if (Status st = tunedShape(q, *solver, &shape); st != CFD_OK) return st;
    if (Status st = solver->setLaunchShape(shape.first, shape.second); st != CFD_OK) return st;
    auto slot = std::make_unique<Slot>();
    slot->id = q.id;
    slot->request = q.request;
    slot->bytes = solver->deviceBytes();
    slot->solver = std::move(solver);
    slot->mesh = q.mesh;
    slot->continued = (q.warm != nullptr);
    slot->sweep = q.sweep;
    slot->point = q.point;
    slot->meshSeconds = q.meshSeconds;
    slot->submitted = q.submitted;
    slot->started = now();
    *out = std::move(slot);
    return ok();
  }

  /// The launch shape of a grid: among clusters of 4, 8 and 16 CTAs of 512
  /// threads, the one that gives the most solve-iterations per second on a
  /// full GPU. Each candidate is timed the way the engine runs it when busy:
  /// as many scratch solves of the grid (same model and precision, from their
  /// uniform start) as the GPU holds at once for that shape
  /// (cudaOccupancyMaxActiveClusters), in one launch over a descriptor table,
  /// so the shared L2 and HBM traffic of that many resident solves is in the
  /// measurement. Chosen once per (cells I, cells J, model, precision) and
  /// kept for the process, so a request runs with the same shape, and gives
  /// the same bits, whatever else is in the engine. CFD_ENGINE_TUNE=0 keeps the solver's
  /// default shape.
  Status tunedShape(const Pending& q, const Solver& s, std::pair<int, int>* out) {
    if (!tuned) {
      // By grid size as a lone solve runs, except that the mixed form takes
      // clusters of at most 8 CTAs: its cost per iteration falls less than
      // in proportion to the CTAs (the multigrid's coarse levels and its
      // barriers do not shrink), so smaller clusters fit more solves per GPU
      // (a 24-solve polar: 35 s on 8-CTA clusters, 37 s on 16, 43 s on 12),
      // while the plain form needs 16 for its on-chip CG band (104 s on 16,
      // 136 s on 12, 146 s on 8).
      int R = s.clusterSize();
      if (s.precision() == 1) R = std::min(R, 8);
      *out = {R, s.threads()};
      return ok();
    }
    const auto key = std::make_tuple(s.cellsI(), s.cellsJ(), q.request.model, s.precision());
    std::lock_guard<std::mutex> lock(g_shapesMutex);
    if (auto it = g_shapes.find(key); it != g_shapes.end()) {
      *out = it->second;
      return ok();
    }
    std::pair<int, int> best{s.clusterSize(), s.threads()};
    const char* env = std::getenv("CFD_ENGINE_TUNE");
    if (env == nullptr || std::atoi(env) != 0) {
      const int T = 512;
      std::vector<std::pair<int, int>> candidates;  // (R, resident clusters)
      int most = 0;
      for (int R : {4, 8, 16}) {
        if (R > s.cellsJ()) continue;
        const int resident = maxActiveClusters(R, T, s.launchSmemBytes(R));
        if (resident <= 0) continue;
        candidates.emplace_back(R, resident);
        most = std::max(most, resident);
      }
      // scratch solves, within a quarter of the engine's memory budget
      const std::size_t each = std::max<std::size_t>(s.deviceBytes(), 1);
      const int affordable = static_cast<int>(std::max<std::size_t>(1, budget / 4 / each));
      const int copies = std::min({most, affordable, 40});
      std::vector<std::unique_ptr<Solver>> probes;
      for (int k = 0; k < copies; ++k) {
        std::unique_ptr<Solver> p;
        if (makeSolver(q, &p) != CFD_OK) break;
        probes.push_back(std::move(p));
      }
      Instance* table = nullptr;
      if (!probes.empty() &&
          cudaMalloc(reinterpret_cast<void**>(&table), probes.size() * sizeof(Instance)) == cudaSuccess) {
        std::vector<Instance> rows;
        for (const auto& p : probes) rows.push_back(p->deviceView());
        double bestScore = -1.0;
        if (cudaMemcpy(table, rows.data(), rows.size() * sizeof(Instance), cudaMemcpyHostToDevice) ==
            cudaSuccess) {
          for (const auto& [R, resident] : candidates) {
            const int n = std::min<int>(resident, static_cast<int>(probes.size()));
            const int smem = probes[0]->launchSmemBytes(R);
            if (launchSimple(table, n, R, T, 2, kStageEnd, -1.0, nullptr, smem) != CFD_OK) continue;
            if (cudaDeviceSynchronize() != cudaSuccess) break;
            const auto t0 = std::chrono::steady_clock::now();
            if (launchSimple(table, n, R, T, 6, kStageEnd, -1.0, nullptr, smem) != CFD_OK) continue;
            if (cudaDeviceSynchronize() != cudaSuccess) break;
            const double perIteration =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / 6.0;
            // n solves advance one iteration per perIteration; a full GPU
            // holds `resident` of them (n < resident only when memory is short)
            const double score = n / perIteration * (static_cast<double>(resident) / n);
            if (score > bestScore) {
              bestScore = score;
              best = {R, T};
            }
          }
        }
        cudaFree(table);
      }
    }
    g_shapes[key] = best;
    *out = best;
    return ok();
  }

  Status makeSolver(const Pending& q, std::unique_ptr<Solver>* out, const WarmStart* warm = nullptr) {
    const HostMesh& m = *q.mesh;
    cfd_mesh_desc d;
    describe(m, &d);
    // buildFaceConditions with the default BoundaryConditions
    std::vector<int> kind(m.faces);
    std::vector<double> vel(2 * m.faces, 0.0), pres(m.faces, 0.0);
    const double alpha = q.request.alpha_deg * kPi / 180.0;
    const double ux = q.request.speed * std::cos(alpha), uy = q.request.speed * std::sin(alpha);
    for (int f = 0; f < m.faces; ++f) {
      int k = CFD_BC_INTERNAL;
      if (m.boundary[f] == CFD_FACE_WALL) k = CFD_BC_NOSLIP_WALL;
      else if (m.boundary[f] == CFD_FACE_FARFIELD) k = CFD_BC_FARFIELD;
      else if (m.boundary[f] == CFD_FACE_OUTLET) k = CFD_BC_OUTLET;
      kind[f] = k;
      if (k != CFD_BC_NOSLIP_WALL) {
        vel[2 * f] = ux;
        vel[2 * f + 1] = uy;
      }
    }
    cfd_face_bc bc{kind.data(), vel.data(), pres.data()};
    Solver* raw = nullptr;
    if (Status st = Solver::create(d, bc, fromC(q.request.settings), &raw); st != CFD_OK) return st;
    std::unique_ptr<Solver> solver(raw);
    if (Status st = solver->setTurbulence(q.request.model); st != CFD_OK) return st;
    // FlowField::uniform sets density and viscosity from the freestream; a
    // continued point then takes only velocity and pressure over
    // (Panels.cpp:1145-1156).
    std::vector<double> u, v, p, rho, mu;
    uniform(q.request, m.cells, &u, &v, &p, &rho, &mu);
    if (warm != nullptr && warm->u.size() == u.size()) {
      u = warm->u;
      v = warm->v;
      p = warm->p;
    }
    if (Status st = solver->initialise(u.data(), v.data(), p.data(), rho.data(), mu.data()); st != CFD_OK) {
      return st;
    }
    *out = std::move(solver);
    return ok();
  }

  /// The next point of a sweep once point `s` has retired with `status`:
  /// continued from s's u and p unless the sweep starts each point cold or
  /// s diverged even after its cold retry (Panels.cpp:1785-1796).
  void advanceSweep(const Slot& s, int status) {
    const Sweep& sw = sweeps[static_cast<std::size_t>(s.sweep)];
    const int next = s.point + 1;
    if (next >= static_cast<int>(sw.angles.size())) return;
    Pending q;
    q.id = sw.firstId + next;
    q.request = sw.base;
    q.request.alpha_deg = sw.angles[static_cast<std::size_t>(next)];
    q.mesh = s.mesh;
    q.submitted = now();
    q.sweep = s.sweep;
    q.point = next;
    const bool cold = !sw.continued || (s.retried && status == CFD_SOLVE_DIVERGED) || status == CFD_SOLVE_FAILED;
    if (!cold) {
      auto warm = std::make_shared<WarmStart>();
      const std::size_t n = static_cast<std::size_t>(s.solver->cells());
      warm->u.resize(n);
      warm->v.resize(n);
      warm->p.resize(n);
      if (s.solver->readField(CFD_FIELD_U, warm->u.data()) == CFD_OK &&
          s.solver->readField(CFD_FIELD_V, warm->v.data()) == CFD_OK &&
          s.solver->readField(CFD_FIELD_P, warm->p.data()) == CFD_OK) {
        q.warm = std::move(warm);
      }
    }
    queue.push_front(std::move(q));  // a sweep's next point goes ahead of new requests
  }

  /// A request that could not start (its solver failed to build or
  /// initialise): reported with CFD_SOLVE_FAILED and the library's status
  /// code, never as a physics outcome. A sweep stops there, as the
  /// reference's does (AbortFailed, Polar.cpp:95-98): its remaining points
  /// are reported failed too, so every id it was given gets a result.
  void failStart(const Pending& q, Status code) {
    cfd_result r{};
    r.id = q.id;
    r.status = CFD_SOLVE_FAILED;
    r.error = code;
    r.alpha_deg = q.request.alpha_deg;
    r.separation_upper_chord_fraction = r.separation_lower_chord_fraction = -1.0;
    r.submitted_s = q.submitted;
    r.started_s = r.finished_s = now();
    done.push_back(r);
    if (q.sweep < 0) return;
    const Sweep& sw = sweeps[static_cast<std::size_t>(q.sweep)];
    for (int k = q.point + 1; k < static_cast<int>(sw.angles.size()); ++k) {
      cfd_result rest = r;
      rest.id = sw.firstId + k;
      rest.alpha_deg = sw.angles[static_cast<std::size_t>(k)];
      done.push_back(rest);
    }
  }

  /// Start queued requests whose mesh is ready, in queue order, while they
  /// fit the memory budget, appending them to `into`; a request whose mesh is
  /// still being built keeps its place. An engine with nothing resident always
  /// takes one, so an oversized request cannot stall the queue.
  void admit(std::vector<std::unique_ptr<Slot>>& into, std::size_t resident) {
    for (auto it = queue.begin(); it != queue.end();) {
      Pending& q = *it;
      if (!q.mesh) {
        if (!ready(q.meshFuture)) {
          ++it;
          continue;
        }
        const MeshResult& m = q.meshFuture.get();
        if (m.status != CFD_OK) {
          failStart(q, m.status);
          it = queue.erase(it);
          continue;
        }
        q.mesh = m.mesh;
        if (q.builtMesh) q.meshSeconds = m.seconds;
      }
      const std::size_t need = Solver::estimateBytes(q.mesh->nodesI - 1, q.mesh->nodesJ - 1);
      if (resident + into.size() > 0 && used + need > budget) break;
      std::unique_ptr<Slot> slot;
      if (Status st = start(q, &slot); st != CFD_OK) {
        failStart(q, st);
        it = queue.erase(it);
        continue;
      }
      used += slot->bytes;
      into.push_back(std::move(slot));
      it = queue.erase(it);
    }
  }

  void finish(Slot& s, int status, const double* mon, Status error = CFD_OK) {
    cfd_result r{};
    r.id = s.id;
    r.status = status;
    r.error = error;
    r.iterations = s.iterations;
    r.retried_cold = s.retried ? 1 : 0;
    r.continued = s.continued ? 1 : 0;
    r.alpha_deg = s.request.alpha_deg;
    r.mesh_s = s.meshSeconds;
    r.cells = s.solver->cells();
    r.cluster_size = s.solver->clusterSize();
    r.continuity = mon[kMonContinuity];
    r.momentum_x = mon[kMonMomX];
    r.momentum_y = mon[kMonMomY];
    double f[12];
    r.separation_upper_chord_fraction = -1.0;
    r.separation_lower_chord_fraction = -1.0;
    std::vector<double> cp(static_cast<std::size_t>(std::max(s.solver->wallStations(), 1)));
    int stations = 0;
    if (status != CFD_SOLVE_DIVERGED && status != CFD_SOLVE_FAILED &&
        s.solver->forces(s.request.speed, s.request.alpha_deg, s.request.density, 0.0, 1.0, f, cp.data(),
                         nullptr, &stations, nullptr) == CFD_OK) {
      cp.resize(static_cast<std::size_t>(stations));
      surfaces[s.id] = std::move(cp);
      r.lift_coefficient = f[0];
      r.drag_coefficient = f[1];
      r.moment_coefficient = f[2];
      r.pressure_drag_coefficient = f[3];
      r.friction_drag_coefficient = f[4];
      r.separation_upper_chord_fraction = f[10];
      r.separation_lower_chord_fraction = f[11];
    }
    r.submitted_s = s.submitted;
    r.started_s = s.started;
    r.finished_s = now();
    done.push_back(r);
  }

  /// Launch `chunk` iterations of every resident solve, one launch per
  /// launch shape over a descriptor table, and return without waiting.
  Status launchChunk() {
    const int n = static_cast<int>(active.size());
    if (Status st = reserve(n); st != CFD_OK) return st;
    // group by launch shape; table rows in slot order within each group
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int k = 0; k < n; ++k) {
      const Solver& s = *active[k]->solver;
      groups[{s.clusterSize(), s.threads()}].push_back(k);
    }
    std::vector<Instance> table(n);
    std::vector<std::tuple<int, int, int, int, int>> launches;  // offset, count, R, T, smem
    const std::size_t per = static_cast<std::size_t>(chunk) * kMonSlots + 1;
    int offset = 0;
    for (const auto& [shape, members] : groups) {
      int smem = 0;
      for (std::size_t m = 0; m < members.size(); ++m) {
        const int k = members[m];
        Slot& s = *active[k];
        Instance I = s.solver->deviceView();
        double* status = dStatus + static_cast<std::size_t>(k) * per;
        I.history = status;
        I.iterations = reinterpret_cast<int*>(status + static_cast<std::size_t>(chunk) * kMonSlots);
        I.stopTol = s.request.tolerance;
        I.iterLimit = std::max(1, std::min(chunk, s.request.max_iterations - s.iterations));
        table[offset + static_cast<int>(m)] = I;
        smem = std::max(smem, s.solver->launchSmemBytes(shape.first));
      }
      launches.emplace_back(offset, static_cast<int>(members.size()), shape.first, shape.second, smem);
      offset += static_cast<int>(members.size());
    }
    if (cudaMemcpy(dTable, table.data(), n * sizeof(Instance), cudaMemcpyHostToDevice) != cudaSuccess) {
      return fail(CFD_INITIALIZATION_FAILURE, "engine table upload failed");
    }
    while (streams.size() < launches.size()) {
      cudaStream_t s;
      if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        return fail(CFD_INITIALIZATION_FAILURE, "engine stream creation failed");
      }
      streams.push_back(s);
    }
    inFlightStreams.clear();
    for (std::size_t g = 0; g < launches.size(); ++g) {
      const auto [off, count, R, T, smem] = launches[g];
      if (Status st = launchSimple(dTable + off, count, R, T, chunk, kStageEnd, -1.0, streams[g], smem);
          st != CFD_OK) {
        waitForLaunches();
        return st;
      }
      inFlightStreams.push_back(static_cast<int>(g));
    }
    inFlight = true;
    inFlightSlots = n;
    return ok();
  }

  /// Wait for the chunk in flight (its streams only, so the admission work
  /// queued meanwhile on the new solves' own streams is not waited for).
  Status waitForLaunches() {
    Status st = ok();
    for (int g : inFlightStreams) {
      if (cudaStreamSynchronize(streams[static_cast<std::size_t>(g)]) != cudaSuccess && st == CFD_OK) {
        st = fail(CFD_INITIALIZATION_FAILURE, "engine step failed on the device");
      }
    }
    inFlightStreams.clear();
    inFlight = false;
    return st;
  }

  /// Read every launched solve's monitors and iteration count, and retire
  /// the ones that converged, diverged (after one cold retry) or hit their cap.
  Status retire() {
    const int n = inFlightSlots;
    const std::size_t per = static_cast<std::size_t>(chunk) * kMonSlots + 1;
    std::vector<double> status(static_cast<std::size_t>(n) * per);
    if (cudaMemcpy(status.data(), dStatus, status.size() * sizeof(double), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
      return fail(CFD_INITIALIZATION_FAILURE, "engine status read failed");
    }
    std::vector<std::unique_ptr<Slot>> keep;
    for (int k = 0; k < n; ++k) {
      Slot& s = *active[k];
      const double* st = status.data() + static_cast<std::size_t>(k) * per;
      int words[2] = {0, 0};  // iterations, fault word
      std::memcpy(words, st + static_cast<std::size_t>(chunk) * kMonSlots, sizeof(words));
      const int ran = words[0];
      s.iterations += ran;
      const double* mon = st + static_cast<std::size_t>(std::max(ran, 1) - 1) * kMonSlots;
      const double a = mon[kMonContinuity], b = mon[kMonMomX], c = mon[kMonMomY];
      const bool finite = std::isfinite(a) && std::isfinite(b) && std::isfinite(c);
      int outcome = -1;
      Status error = CFD_OK;
      if (words[1] != 0) {
        // a bounded wait in the kernel gave up: the launch's values are not valid
        error = launchFault(words[1]);
        outcome = CFD_SOLVE_FAILED;
      } else if (!finite) {
        if (!s.retried) {
          // RetryCold: restart once from the freestream
          s.retried = true;
          std::vector<double> u, v, p, rho, mu;
          uniform(s.request, s.solver->cells(), &u, &v, &p, &rho, &mu);
          if (s.solver->initialise(u.data(), v.data(), p.data(), rho.data(), mu.data()) != CFD_OK) {
            outcome = CFD_SOLVE_DIVERGED;
          }
        } else {
          outcome = CFD_SOLVE_DIVERGED;
        }
      } else if (std::max({std::abs(a), std::abs(b), std::abs(c)}) < s.request.tolerance) {
        outcome = CFD_SOLVE_CONVERGED;
      } else if (s.iterations >= s.request.max_iterations) {
        outcome = CFD_SOLVE_ITERATION_LIMIT;
      }
      if (outcome >= 0) {
        finish(s, outcome, mon, error);
        if (s.sweep >= 0) advanceSweep(s, outcome);
        used -= s.bytes;
      } else {
        keep.push_back(std::move(active[k]));
      }
    }
    for (std::size_t k = static_cast<std::size_t>(n); k < active.size(); ++k) keep.push_back(std::move(active[k]));
    active = std::move(keep);
    return ok();
  }

  /// One engine step. While the chunk launched by the previous step runs,
  /// the requests that can join the next one are set up on the host (their
  /// solvers built, initialised and copied to the device on their own
  /// streams); then the step waits for the chunk, retires what finished,
  /// fills the memory that freed, launches the next chunk and returns with it
  /// running, so the caller's own work overlaps the GPU too.
  Status step(int* activeOut, int* queuedOut) {
    if (inFlight) {
      std::vector<std::unique_ptr<Slot>> staged;
      admit(staged, active.size());
      if (Status st = waitForLaunches(); st != CFD_OK) return st;
      if (Status st = retire(); st != CFD_OK) return st;
      for (auto& slot : staged) active.push_back(std::move(slot));
    }
    admit(active, active.size());
    if (!active.empty()) {
      if (Status st = launchChunk(); st != CFD_OK) return st;
    }
    if (activeOut) *activeOut = static_cast<int>(active.size());
    if (queuedOut) *queuedOut = static_cast<int>(queue.size());
    return ok();
  }
};

}  // namespace cfdb

struct cfd_engine_t {
  cfdb::Engine engine;
};

extern "C" {

cfd_status cfd_engine_create(unsigned long long budget, int chunk, cfd_engine* out) {
  if (out == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null output");
  if (chunk < 1 || chunk > 256) return cfdb::fail(CFD_OUT_OF_RANGE, "chunk must lie in 1..256");
  if (budget == 0) {
    std::size_t freeBytes = 0, total = 0;
    if (cudaMemGetInfo(&freeBytes, &total) != cudaSuccess) {
      return cfdb::fail(CFD_INITIALIZATION_FAILURE, "cannot query device memory");
    }
    budget = static_cast<unsigned long long>(0.8 * static_cast<double>(freeBytes));
  }
  auto* e = new cfd_engine_t;
  e->engine.budget = budget;
  e->engine.chunk = chunk;
  *out = e;
  return CFD_OK;
}

namespace {

cfd_status checkRequest(const cfd_request* r) {
  if (!(r->reynolds > 0.0) || !(r->speed > 0.0) || !(r->density > 0.0) || !(r->tolerance >= 0.0) ||
      r->max_iterations < 1 || (r->model != 0 && r->model != 1 && r->model != 2)) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "invalid request");
  }
  return CFD_OK;
}

/// The request's C-grid: from the engine's cache (built, or still being
/// built), else queued on the engine's mesh workers. *built tells whether
/// this call started the build.
cfdb::MeshFuture meshFor(cfdb::Engine& g, const cfd_request& r, bool* built) {
  const cfdb::MeshKey key = cfdb::keyOf(r);
  if (auto it = g.meshes.find(key); it != g.meshes.end()) {
    *built = false;
    return it->second;
  }
  if (!g.pool) {
    const unsigned cores = std::max(2u, std::thread::hardware_concurrency());
    g.pool = std::make_unique<cfdb::MeshPool>(static_cast<int>(std::min(8u, cores / 2)));
  }
  cfd_cgrid_options o;
  cfd_default_cgrid_options(&o);
  o.surface_points = r.grid_surface_points;
  o.wake_points = r.grid_wake_points;
  o.normal_points = r.grid_normal_points;
  o.first_layer_height = r.grid_first_layer_height;
  o.upstream_chords = r.grid_upstream_chords;
  o.downstream_chords = r.grid_downstream_chords;
  o.vertical_chords = r.grid_vertical_chords;
  const std::string name(r.designation, strnlen(r.designation, sizeof(r.designation)));
  cfdb::MeshFuture f = g.pool->build(name, o);
  g.meshes[key] = f;
  *built = true;
  return f;
}

}  // namespace

cfd_status cfd_engine_submit(cfd_engine e, const cfd_request* r, int* id) {
  if (e == nullptr || r == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  if (cfd_status st = checkRequest(r); st != CFD_OK) return st;
  cfdb::Engine& g = e->engine;
  cfdb::Pending q;
  q.id = g.nextId++;
  q.request = *r;
  q.meshFuture = meshFor(g, *r, &q.builtMesh);
  q.submitted = g.now();
  g.queue.push_back(q);
  if (id != nullptr) *id = q.id;
  return CFD_OK;
}

cfd_status cfd_sweep_angles(double start, double end, double step, double* out, int capacity, int* count) {
  if (count == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null count");
  if (!std::isfinite(start) || !std::isfinite(end) || !std::isfinite(step)) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "sweep bounds must be finite");
  }
  if (!(step > 0.0)) return cfdb::fail(CFD_INVALID_ARGUMENT, "the sweep step must be positive");
  // the step's sign comes from the direction of the sweep; the point count
  // is rounded when the step divides the range to within 1e-9 of a step
  const double signedStep = (end < start) ? -step : step;
  const double span = (end - start) / signedStep;
  const double rounded = std::round(span);
  const double intervals = (std::abs(span - rounded) < 1e-9) ? rounded : std::floor(span);
  if (intervals < 0.0) return cfdb::fail(CFD_INVALID_ARGUMENT, "the sweep covers no angles");
  const double points = intervals + 1.0;
  if (points > static_cast<double>(cfdb::kMaxSweepPoints)) {
    char message[160];
    std::snprintf(message, sizeof(message),
                  "a sweep of %.0f points is more than the %d allowed; every point is a full solve",
                  points, cfdb::kMaxSweepPoints);
    return cfdb::fail(CFD_INVALID_ARGUMENT, message);
  }
  const int n = static_cast<int>(points);
  *count = n;
  if (out == nullptr) return CFD_OK;
  if (capacity < n) return cfdb::fail(CFD_OUT_OF_RANGE, "angle buffer too small");
  // each angle computed from its index, so a long sweep does not drift
  for (int k = 0; k < n; ++k) out[k] = start + static_cast<double>(k) * signedStep;
  return CFD_OK;
}

cfd_status cfd_engine_submit_sweep(cfd_engine e, const cfd_request* base, double start, double end,
                                   double step, int continued, int* first_id, int* count) {
  if (e == nullptr || base == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  if (cfd_status st = checkRequest(base); st != CFD_OK) return st;
  int n = 0;
  if (cfd_status st = cfd_sweep_angles(start, end, step, nullptr, 0, &n); st != CFD_OK) return st;
  cfdb::Engine& g = e->engine;
  cfdb::Sweep sw;
  sw.base = *base;
  sw.angles.resize(static_cast<std::size_t>(n));
  if (cfd_status st = cfd_sweep_angles(start, end, step, sw.angles.data(), n, &n); st != CFD_OK) return st;
  sw.firstId = g.nextId;
  sw.continued = (continued != 0);
  g.nextId += n;
  cfdb::Pending q;
  q.id = sw.firstId;
  q.request = *base;
  q.request.alpha_deg = sw.angles.front();
  q.meshFuture = meshFor(g, *base, &q.builtMesh);
  q.submitted = g.now();
  q.sweep = static_cast<int>(g.sweeps.size());
  q.point = 0;
  g.sweeps.push_back(std::move(sw));
  g.queue.push_back(q);
  if (first_id != nullptr) *first_id = q.id;
  if (count != nullptr) *count = n;
  return CFD_OK;
}

cfd_status cfd_engine_step(cfd_engine e, int* active, int* queued) {
  if (e == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null engine");
  return e->engine.step(active, queued);
}

cfd_status cfd_engine_results(cfd_engine e, cfd_result* out, int capacity, int* count) {
  if (e == nullptr || count == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  cfdb::Engine& g = e->engine;
  const int n = std::min<int>(capacity, static_cast<int>(g.done.size()));
  for (int k = 0; k < n; ++k) out[k] = g.done[k];
  g.done.erase(g.done.begin(), g.done.begin() + n);
  *count = n;
  return CFD_OK;
}

cfd_status cfd_engine_surface(cfd_engine e, int id, double* cp, int capacity, int* stations) {
  if (e == nullptr || stations == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  cfdb::Engine& g = e->engine;
  auto it = g.surfaces.find(id);
  if (it == g.surfaces.end()) return cfdb::fail(CFD_INVALID_ARGUMENT, "no surface data for this request id");
  const int n = static_cast<int>(it->second.size());
  *stations = n;
  if (cp == nullptr) return CFD_OK;  // size query
  if (capacity < n) return cfdb::fail(CFD_INVALID_ARGUMENT, "cp buffer too small");
  std::copy(it->second.begin(), it->second.end(), cp);
  g.surfaces.erase(it);
  return CFD_OK;
}

cfd_status cfd_engine_set_shape_policy(cfd_engine e, int policy) {
  if (e == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null engine");
  if (policy != 0 && policy != 1) return cfdb::fail(CFD_INVALID_ARGUMENT, "policy must be 0 or 1");
  e->engine.tuned = (policy == 1);
  return CFD_OK;
}

double cfd_engine_clock(cfd_engine e) { return (e == nullptr) ? 0.0 : e->engine.now(); }

cfd_status cfd_engine_destroy(cfd_engine e) {
  delete e;
  return CFD_OK;
}

}  // extern "C"
