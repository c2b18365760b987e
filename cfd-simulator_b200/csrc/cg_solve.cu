// cg_solve.cu - the reference's Jacobi-preconditioned conjugate gradient
// (LinearSystem.cpp:118-210) as a device primitive on one thread-block
// cluster, for a symmetric five-point system on a structured block given in
// the reference's LDU layout (LinearSystem.hpp:29-71).
//
// The iteration is the reference's, with its L1 stopping rule and its
// breakdown guards; the dot products are summed in a fixed order (warp
// trees, then CTA ranks in order), so a solve is deterministic. One cluster
// barrier per iteration: the single-reduction arrangement described at
// cgSolveTeam.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "cfd_gpu.h"
#include "common.hpp"
#include "solver.hpp"
#include "team.cuh"

namespace cfdb {

/// A five-point symmetric system on an NI x NJ block, in the device layout:
/// per-face coefficients in N-face (j*NI + i) and E-face (j*(NI+1) + i) order.
struct CgView {
  int NI, NJ, N;
  const int* acrossJ0;
  const double* diag;
  const double* pN;
  const double* pE;
  const double* b;
  double *x, *r, *z, *q, *d0, *d1, *s1, *p;
  int maxIt;
  double tol;
  double* report;  // {iterations, initial, final, converged, bad wake map}: 8 words
};

namespace {

DEV double rowTimes(const CgView& V, int c, int i, int j, const double* v, double vc) {
  double y = V.diag[c] * vc;
  if (j > 0) y += V.pN[j * V.NI + i] * v[c - V.NI];
  else if (V.acrossJ0[i] >= 0) y += V.pN[i] * v[V.acrossJ0[i]];
  if (j < V.NJ - 1) y += V.pN[(j + 1) * V.NI + i] * v[c + V.NI];
  if (i > 0) y += V.pE[j * (V.NI + 1) + i] * v[c - 1];
  if (i < V.NI - 1) y += V.pE[j * (V.NI + 1) + i + 1] * v[c + 1];
  return y;
}

DEV double precondition(double rc, double dg) { return (fabs(dg) > 0.0) ? rc / dg : rc; }

}  // namespace

/// y = A v at cell c for a v given as a function of the cell (the matrix
/// row in multiply's face order).
template <typename F>
DEV double rowApply(const CgView& V, int c, int i, int j, double vc, F&& v) {
  double y = V.diag[c] * vc;
  if (j > 0) y += V.pN[j * V.NI + i] * v(c - V.NI);
  else if (V.acrossJ0[i] >= 0) y += V.pN[i] * v(V.acrossJ0[i]);
  if (j < V.NJ - 1) y += V.pN[(j + 1) * V.NI + i] * v(c + V.NI);
  if (i > 0) y += V.pE[j * (V.NI + 1) + i] * v(c - 1);
  if (i < V.NI - 1) y += V.pE[j * (V.NI + 1) + i + 1] * v(c + 1);
  return y;
}

/// The whole solve, run by every thread of the cluster: the reference's
/// Jacobi-PCG rearranged with one reduction per iteration (Chronopoulos and
/// Gear, 1989), as in the SIMPLE kernel's pressure solve: u = M^-1 r,
/// w = A u, one reduction of {r.u, w.u, sum |r|}; beta = gamma'/gamma,
/// d.Ad = delta' - beta gamma'/alpha, alpha = gamma'/d.Ad; p = u + beta p,
/// s = w + beta s, x += alpha p, r -= alpha s. The reference's L1 stopping
/// rule, cap and breakdown guards; the same iterates to rounding. r, w and s
/// are double-buffered ((r, z), (q, d0), (d1, s1)) so a cell can form its
/// neighbours' next u from their values of this iteration.
__device__ void cgSolveTeam(const CgView& V, Team& t, Shared& sh) {
  double* rB[2] = {V.r, V.z};
  double* wB[2] = {V.q, V.d0};
  double* sB[2] = {V.d1, V.s1};
  const int op1[1] = {kSum};
  const int op2[2] = {kSum, kSum};
  const int op3[3] = {kSum, kSum, kSum};
  double init[2] = {0.0, 0.0};
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % V.NI, j = c / V.NI;
    const double rc = V.b[c] - rowTimes(V, c, i, j, V.x, V.x[c]);
    rB[0][c] = rc;
    sB[0][c] = 0.0;
    V.p[c] = 0.0;
    init[0] += fabs(rc);
    init[1] += rc * precondition(rc, V.diag[c]);
  }
  teamReduce(t, sh, init, op2);
  const double initial = init[0];
  double finalResidual = initial;
  int iterations = 0;
  bool converged = false;
  if (initial <= 0.0) {
    converged = true;
  } else {
    // w0 = A u0: every r0 is in place since the reduction's barrier
    double acc[1] = {0.0};
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int i = c % V.NI, j = c / V.NI;
      const double un = precondition(rB[0][c], V.diag[c]);
      const double y = rowApply(V, c, i, j, un, [&](int n) { return precondition(rB[0][n], V.diag[n]); });
      wB[0][c] = y;
      acc[0] += y * un;
    }
    teamReduce(t, sh, acc, op1);
    if (fabs(acc[0]) > 0.0) {
      double gamma = init[1], alpha = gamma / acc[0], beta = 0.0;
      int cur = 0;
      for (int iter = 0; iter < V.maxIt; ++iter) {
        const double* r = rB[cur];
        const double* w = wB[cur];
        const double* sv = sB[cur];
        double* rn = rB[cur ^ 1];
        double* wn = wB[cur ^ 1];
        double* sn = sB[cur ^ 1];
        double sums[3] = {0.0, 0.0, 0.0};
        for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
          const int i = c % V.NI, j = c / V.NI;
          const double dg = V.diag[c];
          const double pc = precondition(r[c], dg) + beta * V.p[c];
          const double sc = w[c] + beta * sv[c];
          V.x[c] += alpha * pc;
          const double rc = r[c] - alpha * sc;
          const double un = precondition(rc, dg);
          const double y = rowApply(V, c, i, j, un, [&](int n) {
            const double s2 = w[n] + beta * sv[n];
            return precondition(r[n] - alpha * s2, V.diag[n]);
          });
          V.p[c] = pc;
          sn[c] = sc;
          rn[c] = rc;
          wn[c] = y;
          sums[0] += rc * un;
          sums[1] += y * un;
          sums[2] += fabs(rc);
        }
        cur ^= 1;
        teamReduce(t, sh, sums, op3);
        iterations = iter + 1;
        finalResidual = sums[2];
        if (sums[2] <= V.tol * initial) {
          converged = true;
          break;
        }
        if (!(fabs(gamma) > 0.0)) break;
        const double nextBeta = sums[0] / gamma;
        const double dAd = sums[1] - nextBeta * sums[0] / alpha;
        if (!(fabs(dAd) > 0.0)) break;
        beta = nextBeta;
        alpha = sums[0] / dAd;
        gamma = sums[0];
      }
    }
  }
  if (t.rank == 0 && t.tid == 0 && V.report != nullptr) {
    V.report[0] = static_cast<double>(iterations);
    V.report[1] = initial;
    V.report[2] = finalResidual;
    V.report[3] = converged ? 1.0 : 0.0;
  }
}

__global__ void __launch_bounds__(512, 1) cgSolveKernel(CgView V) {
  __shared__ Shared sh;
  Team t{cg::this_cluster(), 0, 0, 0, 0, 0, 0, 0};
  t.rank = t.cl.block_rank();
  t.R = t.cl.num_blocks();
  t.tid = threadIdx.x;
  t.T = blockDim.x;
  t.c0 = static_cast<int>((static_cast<long long>(V.N) * t.rank) / t.R);
  t.c1 = static_cast<int>((static_cast<long long>(V.N) * (t.rank + 1)) / t.R);
  if (V.report[4] != 0.0) return;  // a bad wake map (every CTA sees the same flag)
  cgSolveTeam(V, t, sh);
  t.cl.sync();  // no CTA leaves while a peer may still read its shared memory
}

/// Reference-order face coefficients -> device layout; missing wake map -> -1.
/// A wake-map entry that names no cell of the block (>= cells) would make the
/// solve read outside x: it is replaced by -1 and flagged in report[4], and the
/// solve kernel then leaves x untouched.
__global__ void cgLayoutKernel(int NI, int NJ, const double* upper, const int* across, double* pN,
                               double* pE, int* acrossOut, double* report) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int jFaces = NI * (NJ + 1);
  const int faces = jFaces + (NI + 1) * NJ;
  if (f < NI) {
    int a = (across != nullptr) ? across[f] : -1;
    if (a >= NI * NJ) {
      report[4] = 1.0;
      a = -1;
    }
    acrossOut[f] = (a >= 0) ? a : -1;
  }
  if (f >= faces) return;
  if (f < jFaces) {
    pN[f] = upper[f];
  } else {
    const int g = f - jFaces, i = g / NJ, j = g % NJ;
    pE[j * (NI + 1) + i] = upper[f];
  }
}

/// Validate a system's sizes; fills the view's dimensions.
Status cgCheck(const cfd_cg_system* s, const double* x, int maxIt, CgView* V) {
  if (s == nullptr || x == nullptr || s->diag == nullptr || s->upper == nullptr ||
      s->source == nullptr) {
    return fail(CFD_INVALID_ARGUMENT, "null system array");
  }
  if (s->cells_i < 1 || s->cells_j < 1) return fail(CFD_INVALID_ARGUMENT, "empty block");
  if (maxIt < 0) return fail(CFD_INVALID_ARGUMENT, "negative iteration cap");
  const long long cells = static_cast<long long>(s->cells_i) * s->cells_j;
  if (cells > (1LL << 30)) return fail(CFD_OUT_OF_RANGE, "block too large");
  V->NI = s->cells_i;
  V->NJ = s->cells_j;
  V->N = static_cast<int>(cells);
  return CFD_OK;
}

/// Lay out the coefficients, then solve on one cluster (two launches on `stream`).
Status cgRun(const cfd_cg_system* s, CgView V, cudaStream_t stream) {
  const int faces = V.NI * (V.NJ + 1) + (V.NI + 1) * V.NJ;
  const int block = 256;
  cudaError_t e = cudaMemsetAsync(V.report + 4, 0, sizeof(double), stream);
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  cgLayoutKernel<<<(faces + block - 1) / block, block, 0, stream>>>(
      V.NI, V.NJ, s->upper, s->across_j0, const_cast<double*>(V.pN), const_cast<double*>(V.pE),
      const_cast<int*>(V.acrossJ0), V.report);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  // the non-portable cluster size is a per-device kernel attribute
  static PerDeviceOnce configured;
  if (Status st = configured.run([]() -> Status {
        const cudaError_t a = cudaFuncSetAttribute(cgSolveKernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        return (a == cudaSuccess) ? ok() : fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(a));
      });
      st != CFD_OK) {
    return st;
  }
  const int R = chooseClusterSize(V.N);
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(static_cast<unsigned>(R), 1, 1);
  config.blockDim = dim3(512, 1, 1);
  config.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(R);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  config.attrs = attr;
  config.numAttrs = 1;
  e = cudaLaunchKernelEx(&config, cgSolveKernel, V);
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, std::string("CG launch: ") + cudaGetErrorString(e));
  return CFD_OK;
}

/// Wait for the solve on `stream`, then copy its report to the host (4
/// doubles, may be null); a wake map that names a cell outside the block is
/// an invalid argument (the solve did not run).
Status cgReport(const CgView& V, cudaStream_t stream, double* report) {
  double host[5];
  cudaError_t e = cudaMemcpyAsync(host, V.report, sizeof(host), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  if (host[4] != 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "across_j0 names a cell outside the block (entries must be < cells_i*cells_j)");
  }
  if (report != nullptr) for (int k = 0; k < 4; ++k) report[k] = host[k];
  return CFD_OK;
}

}  // namespace cfdb

extern "C" {

cfd_status cfd_cg_solve(const cfd_cg_system* system, double* x, double tolerance,
                        int max_iterations, double* report, void* stream) {
  cfdb::CgView V{};
  if (cfd_status st = cfdb::cgCheck(system, x, max_iterations, &V); st != CFD_OK) return st;
  const std::size_t N = V.N;
  const std::size_t FN = static_cast<std::size_t>(V.NI) * (V.NJ + 1);
  const std::size_t FE = static_cast<std::size_t>(V.NI + 1) * V.NJ;
  // Scratch for this call: both coefficient families, seven CG vectors, the
  // report (8 words) and the wake map.
  const std::size_t doubles = FN + FE + 7 * N + 8;
  char* scratch = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&scratch), doubles * sizeof(double) + V.NI * sizeof(int));
  if (e != cudaSuccess) return cfdb::fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  double* p = reinterpret_cast<double*>(scratch);
  V.pN = p; p += FN;
  V.pE = p; p += FE;
  V.r = p; p += N;
  V.z = p; p += N;
  V.q = p; p += N;
  V.d0 = p; p += N;
  V.d1 = p; p += N;
  V.s1 = p; p += N;
  V.p = p; p += N;
  V.report = p; p += 8;
  V.acrossJ0 = reinterpret_cast<const int*>(p);
  V.diag = system->diag;
  V.b = system->source;
  V.x = x;
  V.maxIt = max_iterations;
  V.tol = tolerance;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cfd_status st = cfdb::cgRun(system, V, s);
  if (st == CFD_OK) st = cfdb::cgReport(V, s, report);
  cudaFree(scratch);
  return st;
}

}  // extern "C"

// ---- the same solve without allocating ----------------------------------------------
//
// Some callers cannot call cudaMalloc: a host application whose memory manager
// has reserved the whole device up front (a cudaMalloc outside that manager
// fails or breaks its accounting), or a latency-critical loop that must not
// block on the implicit device-wide synchronisation cudaFree performs.
// cfd_cg_solve_noalloc serves them. Its scratch (both coefficient families,
// the seven CG vectors, the wake map and the report) is one file-scope device
// array of fixed size, so a call allocates nothing; the caller still provides
// the system and x in its own device memory.
//
// Limits and sharing:
//   * blocks of at most kNoAllocMaxNodes mesh nodes, (cells_i+1)*(cells_j+1)
//     <= 65,536 (the 384 x 96 medium C-grid has 37,345); larger blocks are
//     refused with CFD_OUT_OF_RANGE. The array is 4.75 MiB, held by every GPU
//     that loads this library until the process exits.
//   * every call shares the one array per device and it keeps the last
//     call's contents. Nothing in it needs clearing beforehand: each word a
//     solve reads is written earlier in the same call (coefficients and wake
//     map by the layout launch; the first residual, w and the zero p and s
//     at the start of the solve; each later half of the double-buffered r, w
//     and s in the iteration before it is read), and the error flag is
//     cleared by the call itself. Calls whose work overlaps on the GPU (other
//     host threads, or other streams of this one) race on the array and must
//     be serialised by the caller.
//   * the first call on each device resolves the array's device address with
//     cudaGetSymbolAddress, with that device current; make that first call
//     before any stream capture begins. Every call waits for its solve to
//     finish on its stream before returning.
//   * a wake-map entry that names no cell of the block is refused with
//     CFD_INVALID_ARGUMENT (the solve does not run; x is left as it was).

namespace cfdb {
namespace {

constexpr long long kNoAllocMaxNodes = 65536;
// 9 arrays of at most kNoAllocMaxNodes doubles (two face families and seven
// cell vectors, each at most (cells_i+1)*(cells_j+1) long), 8 report words,
// and the wake map (cells_i <= 32,767 ints) in the last kNoAllocMaxNodes/2
// doubles: 4.75 MiB.
constexpr std::size_t kNoAllocDoubles = 9 * kNoAllocMaxNodes + 8 + kNoAllocMaxNodes / 2;

static __device__ __align__(256) double g_noAllocScratch[kNoAllocDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_noAllocMutex;
double* g_noAllocAddress[kMaxDevices] = {};

/// Device address of g_noAllocScratch on the current device, resolved once.
Status noAllocScratch(double** out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  if (device < 0 || device >= kMaxDevices) return fail(CFD_OUT_OF_RANGE, "device ordinal too large");
  std::lock_guard<std::mutex> lock(g_noAllocMutex);
  if (g_noAllocAddress[device] == nullptr) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noAllocScratch);
    if (e != cudaSuccess) {
      return fail(CFD_INITIALIZATION_FAILURE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    g_noAllocAddress[device] = static_cast<double*>(ptr);
  }
  *out = g_noAllocAddress[device];
  return CFD_OK;
}

}  // namespace
}  // namespace cfdb

extern "C" {

cfd_status cfd_cg_solve_noalloc(const cfd_cg_system* system, double* x, double tolerance,
                                int max_iterations, double* report, void* stream) {
  cfdb::CgView V{};
  if (cfd_status st = cfdb::cgCheck(system, x, max_iterations, &V); st != CFD_OK) return st;
  const long long nodes = static_cast<long long>(V.NI + 1) * (V.NJ + 1);
  if (nodes > cfdb::kNoAllocMaxNodes) {
    return cfdb::fail(CFD_OUT_OF_RANGE,
                      "cfd_cg_solve_noalloc: block of " + std::to_string(nodes) +
                          " nodes exceeds the fixed scratch limit of 65536 nodes "
                          "((cells_i+1)*(cells_j+1)); use cfd_cg_solve");
  }
  double* base = nullptr;
  if (cfd_status st = cfdb::noAllocScratch(&base); st != CFD_OK) return st;
  const std::size_t slot = static_cast<std::size_t>(cfdb::kNoAllocMaxNodes);
  V.pN = base + 0 * slot;
  V.pE = base + 1 * slot;
  V.r = base + 2 * slot;
  V.z = base + 3 * slot;
  V.q = base + 4 * slot;
  V.d0 = base + 5 * slot;
  V.d1 = base + 6 * slot;
  V.s1 = base + 7 * slot;
  V.p = base + 8 * slot;
  V.report = base + 9 * slot;
  V.acrossJ0 = reinterpret_cast<const int*>(base + 9 * slot + 8);
  V.diag = system->diag;
  V.b = system->source;
  V.x = x;
  V.maxIt = max_iterations;
  V.tol = tolerance;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cfd_status st = cfdb::cgRun(system, V, s); st != CFD_OK) return st;
  return cfdb::cgReport(V, s, report);
}

}  // extern "C"
