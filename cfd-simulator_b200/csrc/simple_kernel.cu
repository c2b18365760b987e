// simple_kernel.cu - the SIMPLE outer iteration (laminar and k-omega SST) as
// one persistent kernel per launch, one thread-block cluster per solve.
//
// Why a cluster per solve
// -----------------------
// A SIMPLE iteration is ~15 dependent phases, and the pressure CG inside it
// adds two more per CG iteration (up to 200). Each phase is a 5-point stencil
// or a reduction over 1e4-1e5 cells: far too little work to hide a kernel
// launch or a grid-wide software barrier. A thread-block cluster gives the
// CTAs of one solve a hardware barrier (barrier.cluster) with release/acquire
// semantics, and distributed shared memory to exchange reduction partials,
// so a phase boundary costs a fraction of a microsecond and no spin loop.
// Independent solves occupy independent clusters; a batch of uneven solves is
// a longer grid, one instance descriptor per cluster.
//
// Arithmetic
// ----------
// The plain FP64 form is built with contraction off (no FMA) and evaluates
// every per-cell and per-face expression with the operands, association and
// accumulation order the reference uses, so each non-reduction stage gives
// the reference's values to the last bit. Face quantities are recomputed by
// every cell that touches the face (the owner and the neighbour compute the
// identical value) instead of being scattered, so no atomics are needed and
// a cell's sums are accumulated in the reference's face order:
//   Green-Gauss, assembly, net flux, divergence: S, N, W, E
//     (j-faces before i-faces, ascending index; Mesh.cpp:138-170)
//   Gauss-Seidel off-diagonal sum:               S, E, N, W
//     (Mesh::cellFaces order, Mesh.cpp:172-181; LinearSystem.cpp:94-112)
// Reductions (residual norms, CG dots, maxima) are deterministic: fixed-order
// warp trees, then rank order across the cluster; every CTA derives the same
// bits, so control flow that depends on them (CG exit, convergence) is
// uniform. Gauss-Seidel is red-black instead of lexicographic: exact with the
// wake cut because cellsI is even on a C-grid, so partners across the cut have
// opposite colours. It changes the iterate path but not the converged answer.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>

#include <string>

#include "common.hpp"
#include "instance.hpp"
#include "solver.hpp"
#include "team.cuh"

namespace cfdb {
namespace {

#define DEV __device__ __forceinline__

constexpr double kTinySolver = 1e-300;  // SimpleSolver.cpp:16
constexpr double kTinySst = 1.0e-30;    // KOmegaSST.cpp:22
constexpr double kMinOmega = 1.0e-10;   // KOmegaSST.cpp:20
// SSTConstants (KOmegaSST.hpp:147-171)
constexpr double kSigmaK1 = 0.85, kSigmaW1 = 0.5, kBeta1 = 0.075;
constexpr double kSigmaK2 = 1.0, kSigmaW2 = 0.856, kBeta2 = 0.0828;
constexpr double kBetaStar = 0.09, kKappa = 0.41, kA1 = 0.31, kProdLimit = 10.0;

// BoundaryKind values the kernel tests for (cfd_gpu.h CFD_BC_*; outlet and
// internal faces need no test of their own).
constexpr int kInlet = CFD_BC_INLET, kFarField = CFD_BC_FARFIELD, kWall = CFD_BC_NOSLIP_WALL;

// ---- faces of a cell ----------------------------------------------------------

struct Face {
  int fam;     // 0 N-face, 1 E-face
  int idx;     // index within its family
  int owner;   // owning cell
  int nb;      // neighbour cell of an interior face, else -1
  int other;   // nb, or the cell across the wake cut, else -1
  bool mine;   // the cell being processed owns this face
};

DEV Face faceS(const Instance& I, int c, int i, int j) {
  Face f;
  f.fam = 0;
  f.idx = j * I.NI + i;
  if (j > 0) {
    f.owner = c - I.NI; f.nb = c; f.other = c; f.mine = false;
  } else {
    f.owner = c; f.nb = -1; f.other = I.acrossJ0[i]; f.mine = true;
  }
  return f;
}
DEV Face faceN(const Instance& I, int c, int i, int j) {
  Face f;
  f.fam = 0;
  f.idx = (j + 1) * I.NI + i;
  f.owner = c;
  f.mine = true;
  f.nb = (j < I.NJ - 1) ? c + I.NI : -1;
  f.other = f.nb;
  return f;
}
DEV Face faceW(const Instance& I, int c, int i, int j) {
  Face f;
  f.fam = 1;
  f.idx = j * (I.NI + 1) + i;
  if (i > 0) {
    f.owner = c - 1; f.nb = c; f.mine = false;
  } else {
    f.owner = c; f.nb = -1; f.mine = true;
  }
  f.other = f.nb;
  return f;
}
DEV Face faceE(const Instance& I, int c, int i, int j) {
  Face f;
  f.fam = 1;
  f.idx = j * (I.NI + 1) + i + 1;
  f.owner = c;
  f.mine = true;
  f.nb = (i < I.NI - 1) ? c + 1 : -1;
  f.other = f.nb;
  return f;
}

DEV const FaceGeo& geo(const Instance& I, const Face& f) { return f.fam ? I.gE : I.gN; }
DEV double massFlux(const Instance& I, const Face& f) { return f.fam ? I.mfE[f.idx] : I.mfN[f.idx]; }
DEV double* massFluxPtr(const Instance& I, const Face& f) { return f.fam ? I.mfE + f.idx : I.mfN + f.idx; }
DEV int kindOf(const Instance& I, const Face& f) { return f.fam ? I.kindE[f.idx] : I.kindN[f.idx]; }
DEV double bcU(const Instance& I, const Face& f) { return f.fam ? I.bcuE[f.idx] : I.bcuN[f.idx]; }
DEV double bcV(const Instance& I, const Face& f) { return f.fam ? I.bcvE[f.idx] : I.bcvN[f.idx]; }
DEV double bcP(const Instance& I, const Face& f) { return f.fam ? I.bcpE[f.idx] : I.bcpN[f.idx]; }

/// SimpleSolver::imposesVelocity (SimpleSolver.cpp:247-262) for a boundary face.
DEV bool imposesVelocity(const Instance& I, const Face& f) {
  const int kind = kindOf(I, f);
  if (kind == kWall || kind == kInlet) return true;
  if (kind == kFarField) {
    const double dead = f.fam ? I.deadE[f.idx] : I.deadN[f.idx];
    return massFlux(I, f) < dead;
  }
  return false;
}

/// Accumulate a face's Green-Gauss contribution S*phi into the cell's sum:
/// added for the owner, subtracted for the neighbour (Gradient.cpp:29-40).
DEV void ggAdd(const Face& f, double Sx, double Sy, double phi, double& gx, double& gy) {
  const double cx = Sx * phi, cy = Sy * phi;
  if (f.mine) {
    gx += cx; gy += cy;
  } else {
    gx -= cx; gy -= cy;
  }
}

DEV void ggFinish(double vol, double& gx, double& gy) {
  if (vol > 0.0) {
    const double s = 1.0 / vol;
    gx *= s;
    gy *= s;
  }
}

/// Cell on the other side of face k (0 S, 1 N, 2 W, 3 E) of cell (i, j), or -1.
DEV int across(const Instance& I, int c, int i, int j, int k) {
  switch (k) {
    case 0: return (j > 0) ? c - I.NI : I.acrossJ0[i];
    case 1: return (j < I.NJ - 1) ? c + I.NI : -1;
    case 2: return (i > 0) ? c - 1 : -1;
    default: return (i < I.NI - 1) ? c + 1 : -1;
  }
}

// ---- phase: face values + Green-Gauss gradients of u, v, p ---------------------

/// interpolateFaceValues (SimpleSolver.cpp:268-304) for one face.
DEV void faceUVP(const Instance& I, const Face& f, double& fu, double& fv, double& fp) {
  const int o = f.owner;
  if (f.other >= 0) {
    const double w = geo(I, f).w[f.idx];
    const int n = f.other;
    fu = w * I.u[o] + (1.0 - w) * I.u[n];
    fv = w * I.v[o] + (1.0 - w) * I.v[n];
    fp = w * I.p[o] + (1.0 - w) * I.p[n];
    return;
  }
  if (imposesVelocity(I, f)) {
    fu = bcU(I, f);
    fv = bcV(I, f);
    fp = I.p[o];
  } else {
    fu = I.u[o];
    fv = I.v[o];
    fp = bcP(I, f);
  }
}

DEV void phaseGradients(const Instance& I, Team& t, double& speedMax) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0, px = 0.0, py = 0.0;
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      double fu, fv, fp;
      faceUVP(I, f, fu, fv, fp);
      const FaceGeo& g = geo(I, f);
      const double Sx = g.Sx[f.idx], Sy = g.Sy[f.idx];
      ggAdd(f, Sx, Sy, fu, ux, uy);
      ggAdd(f, Sx, Sy, fv, vx, vy);
      ggAdd(f, Sx, Sy, fp, px, py);
    }
    const double vol = I.vol[c];
    ggFinish(vol, ux, uy);
    ggFinish(vol, vx, vy);
    ggFinish(vol, px, py);
    I.gux[c] = ux; I.guy[c] = uy;
    I.gvx[c] = vx; I.gvy[c] = vy;
    I.gpx[c] = px; I.gpy[c] = py;
    speedMax = smax(speedMax, hypot(I.u[c], I.v[c]));
  }
}

// ---- phase: momentum assembly (u and v share the matrix), relaxation, residual --

DEV void phaseMomentum(const Instance& I, Team& t, double& resU, double& resV, double& diagL1) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double diag = 0.0, sU = 0.0, sV = 0.0;
    double off[4] = {0.0, 0.0, 0.0, 0.0};  // coefficient on the S, N, W, E cell
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      const FaceGeo& g = geo(I, f);
      const int o = f.owner;
      const double flux = massFlux(I, f);
      if (f.other >= 0) {
        const int n = f.other;
        const double w = g.w[f.idx];
        const double vis = w * I.mu[o] + (1.0 - w) * I.mu[n];
        const double dif = vis * g.D[f.idx];
        const double outward = smax(flux, 0.0);
        const double inward = smax(-flux, 0.0);
        const double Tx = g.Tx[f.idx], Ty = g.Ty[f.idx];
        const double fgux = I.gux[o] * w + I.gux[n] * (1.0 - w);
        const double fguy = I.guy[o] * w + I.guy[n] * (1.0 - w);
        const double fgvx = I.gvx[o] * w + I.gvx[n] * (1.0 - w);
        const double fgvy = I.gvy[o] * w + I.gvy[n] * (1.0 - w);
        const double cu = I.blend * vis * (fgux * Tx + fguy * Ty);
        const double cv = I.blend * vis * (fgvx * Tx + fgvy * Ty);
        if (f.nb >= 0) {
          double du = 0.0, dv = 0.0;
          if (I.sou) {
            const double uo = I.u[o], un = I.u[n], vo = I.v[o], vn = I.v[n];
            du = flux * ((w * uo + (1.0 - w) * un) - ((flux >= 0.0) ? uo : un));
            dv = flux * ((w * vo + (1.0 - w) * vn) - ((flux >= 0.0) ? vo : vn));
          }
          if (f.mine) {
            diag += outward + dif;
            off[k] = 0.0 + (-inward - dif);
            sU += cu; sV += cv;
            if (I.sou) { sU -= du; sV -= dv; }
          } else {
            diag += inward + dif;
            off[k] = 0.0 + (-outward - dif);
            sU -= cu; sV -= cv;
            if (I.sou) { sU += du; sV += dv; }
          }
        } else {
          // Wake cut: the owner's row only (SimpleSolver.cpp:379-398).
          diag += outward + dif;
          off[k] = 0.0 + (-inward - dif);
          sU += cu; sV += cv;
        }
        continue;
      }
      // Boundary face (SimpleSolver.cpp:400-416).
      const double vis = I.mu[o];
      const double dif = vis * g.D[f.idx];
      if (imposesVelocity(I, f)) {
        const double iu = bcU(I, f), iv = bcV(I, f);
        const double Tx = g.Tx[f.idx], Ty = g.Ty[f.idx];
        sU -= flux * iu; sV -= flux * iv;
        diag += dif;
        sU += dif * iu; sV += dif * iv;
        sU += I.blend * vis * (I.gux[o] * Tx + I.guy[o] * Ty);
        sV += I.blend * vis * (I.gvx[o] * Tx + I.gvy[o] * Ty);
      } else {
        diag += flux;
      }
    }
    const double vol = I.vol[c];
    sU -= I.gpx[c] * vol;
    sV -= I.gpy[c] * vol;
    // applyRelaxation (SimpleSolver.cpp:425-443).
    const double uc = I.u[c], vc = I.v[c];
    if (!(fabs(diag) > 0.0)) {
      diag = 1.0;
    } else {
      const double relaxed = diag / I.alphaU;
      sU += (relaxed - diag) * uc;
      sV += (relaxed - diag) * vc;
      diag = relaxed;
    }
    I.aD[c] = diag; I.aS[c] = off[0]; I.aN[c] = off[1]; I.aW[c] = off[2]; I.aE[c] = off[3];
    I.bU[c] = sU; I.bV[c] = sV;
    // residualL1 (LinearSystem.cpp:45-54): y = A x in multiply's face order.
    double yu = diag * uc, yv = diag * vc;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int n = across(I, c, i, j, k);
      if (n >= 0) {
        yu += off[k] * I.u[n];
        yv += off[k] * I.v[n];
      }
    }
    resU += fabs(sU - yu);
    resV += fabs(sV - yv);
    diagL1 += fabs(diag);
    if (I.precision == 1) {
      // FP32 rows and residuals for the correction-form sweeps.
      const Rows32& m = I.mom;
      m.D[c] = static_cast<float>(diag);
      m.S[c] = static_cast<float>(off[0]);
      m.N[c] = static_cast<float>(off[1]);
      m.W[c] = static_cast<float>(off[2]);
      m.E[c] = static_cast<float>(off[3]);
      m.r[c] = static_cast<float>(sU - yu);
      I.momRv[c] = static_cast<float>(sV - yv);
      m.x[c] = 0.0f;
      I.momXv[c] = 0.0f;
    }
  }
}

/// Mixed form: one red-black colour pass of the momentum corrections
/// (A du = ru, A dv = rv in FP32, shared rows). The last pass of the last
/// sweep also adds both corrections to the FP64 velocities of every own cell:
/// the other colour's corrections are final by then and no neighbour reads u
/// or v during the sweeps.
DEV void gsColourMixed(const Instance& I, Team& t, int colour, bool last) {
  const Rows32& m = I.mom;
  const float* __restrict__ D = m.D;
  const float* __restrict__ cS = m.S;
  const float* __restrict__ cN = m.N;
  const float* __restrict__ cW = m.W;
  const float* __restrict__ cE = m.E;
  const float* __restrict__ ru = m.r;
  const float* __restrict__ rv = I.momRv;
  float* __restrict__ xu = m.x;
  float* __restrict__ xv = I.momXv;
  const int NI = I.NI;
  const int H = (NI + 1) / 2;
  const int j0 = t.c0 / NI;
  const int slots = ((t.c1 - t.c0) / NI) * H;
  constexpr int kPair = 2;
  // only the colour's cells (i = 2k + ((j + colour) & 1)), two at a time,
  // every load first; missing neighbours are clamped to the cell and their
  // terms left out as before, so the sums are unchanged
  for (int q0 = t.tid; q0 < slots; q0 += kPair * t.T) {
    int cell[kPair], nb[kPair][4];
    bool ok[kPair];
    float d[kPair], a[kPair][4], b1[kPair], b2[kPair], x1[kPair][4], x2[kPair][4];
#pragma unroll
    for (int e = 0; e < kPair; ++e) {
      const int q = min(q0 + e * t.T, slots - 1);
      const int j = j0 + q / H;
      const int i = 2 * (q % H) + ((j + colour) & 1);
      ok[e] = (q0 + e * t.T < slots) && i < NI;
      const int ic = min(i, NI - 1);
      const int c = j * NI + ic;
      cell[e] = c;
      nb[e][0] = across(I, c, ic, j, 0);  // S
      nb[e][1] = across(I, c, ic, j, 3);  // E
      nb[e][2] = across(I, c, ic, j, 1);  // N
      nb[e][3] = across(I, c, ic, j, 2);  // W
      d[e] = D[c];
      a[e][0] = cS[c];
      a[e][1] = cE[c];
      a[e][2] = cN[c];
      a[e][3] = cW[c];
      b1[e] = ru[c];
      b2[e] = rv[c];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int n = (nb[e][k] >= 0) ? nb[e][k] : c;
        x1[e][k] = xu[n];
        x2[e][k] = xv[n];
      }
    }
#pragma unroll
    for (int e = 0; e < kPair; ++e) {
      if (!ok[e] || d[e] == 0.0f) continue;
      float ou = 0.0f, ov = 0.0f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (nb[e][k] >= 0) {
          ou += a[e][k] * x1[e][k];
          ov += a[e][k] * x2[e][k];
        }
      }
      xu[cell[e]] = (b1[e] - ou) / d[e];
      xv[cell[e]] = (b2[e] - ov) / d[e];
    }
  }
  if (last) {
    // the corrections of the whole band (this CTA wrote all of them) onto u, v
    __syncthreads();
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      I.u[c] += static_cast<double>(xu[c]);
      I.v[c] += static_cast<double>(xv[c]);
    }
  }
}

/// One colour of a red-black Gauss-Seidel sweep of the momentum system for u
/// and v together (one matrix, two right-hand sides; LinearSystem.cpp:77-116
/// per cell, off-diagonals summed S, E, N, W). Threads take only the cells of
/// the colour (a row holds ceil(NI/2) slots; i = 2k + ((j + colour) & 1)),
/// two at a time, and issue every load of both cells before the arithmetic:
/// a missing neighbour's index is clamped to the cell itself and its term is
/// left out exactly as before, so the sums and the bits are unchanged.
DEV void gsColour(const Instance& I, Team& t, int colour) {
  const double* __restrict__ D = I.aD;
  const double* __restrict__ cS = I.aS;
  const double* __restrict__ cN = I.aN;
  const double* __restrict__ cW = I.aW;
  const double* __restrict__ cE = I.aE;
  const double* __restrict__ bu = I.bU;
  const double* __restrict__ bv = I.bV;
  double* __restrict__ u = I.u;
  double* __restrict__ v = I.v;
  const int NI = I.NI;
  const int H = (NI + 1) / 2;
  const int j0 = t.c0 / NI;
  const int slots = ((t.c1 - t.c0) / NI) * H;
  constexpr int kPair = 2;
  for (int q0 = t.tid; q0 < slots; q0 += kPair * t.T) {
    int cell[kPair], nb[kPair][4];
    bool ok[kPair];
    double d[kPair], a[kPair][4], b1[kPair], b2[kPair], x1[kPair][4], x2[kPair][4];
#pragma unroll
    for (int e = 0; e < kPair; ++e) {
      const int q = min(q0 + e * t.T, slots - 1);
      const int j = j0 + q / H;
      const int i = 2 * (q % H) + ((j + colour) & 1);
      ok[e] = (q0 + e * t.T < slots) && i < NI;
      const int ic = min(i, NI - 1);
      const int c = j * NI + ic;
      cell[e] = c;
      nb[e][0] = across(I, c, ic, j, 0);  // S
      nb[e][1] = across(I, c, ic, j, 3);  // E
      nb[e][2] = across(I, c, ic, j, 1);  // N
      nb[e][3] = across(I, c, ic, j, 2);  // W
      d[e] = D[c];
      a[e][0] = cS[c];
      a[e][1] = cE[c];
      a[e][2] = cN[c];
      a[e][3] = cW[c];
      b1[e] = bu[c];
      b2[e] = bv[c];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int n = (nb[e][k] >= 0) ? nb[e][k] : c;
        x1[e][k] = u[n];
        x2[e][k] = v[n];
      }
    }
#pragma unroll
    for (int e = 0; e < kPair; ++e) {
      if (!ok[e] || !(fabs(d[e]) > 0.0)) continue;
      double o1 = 0.0, o2 = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (nb[e][k] >= 0) {
          o1 += a[e][k] * x1[e][k];
          o2 += a[e][k] * x2[e][k];
        }
      }
      u[cell[e]] = (b1[e] - o1) / d[e];
      v[cell[e]] = (b2[e] - o2) / d[e];
    }
  }
}

/// Lexicographic Gauss-Seidel, executed as wavefronts: cells with i + j = d
/// for d = 0, 1, ... Within a wavefront no cell depends on another; every
/// cell sees its S and W neighbours already updated and its N and E
/// neighbours not yet, exactly as in cell-index order. Across the wake cut,
/// the partner (NI-1-i, 0) of (i, 0) lies on an earlier wavefront exactly when
/// its cell index is smaller, so that coupling is reproduced too. The result
/// is the reference's sweep (LinearSystem.cpp:77-116) to the last bit.
///
/// One CTA runs one system: rank 0 sweeps x1, rank 1 (or rank 0 again when
/// the cluster has one CTA) sweeps x2. The caller ends with a cluster barrier.
DEV void gsWavefrontSweeps(const Instance& I, Team& t, int sweeps, const double* D,
                           const double* cS, const double* cN, const double* cW,
                           const double* cE, const double* b1, double* x1, const double* D2,
                           const double* cS2, const double* cN2, const double* cW2,
                           const double* cE2, const double* b2, double* x2) {
  const bool one = (t.R == 1);
  if (!one && t.rank > 1) return;
  const int fronts = I.NI + I.NJ - 1;
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (int d = 0; d < fronts; ++d) {
      const int jLo = (d - (I.NI - 1) > 0) ? d - (I.NI - 1) : 0;
      const int jHi = (d < I.NJ - 1) ? d : I.NJ - 1;
      const int count = jHi - jLo + 1;
      const int work = one ? 2 * count : count;
      for (int k = t.tid; k < work; k += t.T) {
        const bool second = one ? (k >= count) : (t.rank == 1);
        const int j = jLo + (one ? (k % count) : k);
        const int i = d - j;
        const int c = j * I.NI + i;
        const double* Dv = second ? D2 : D;
        const double dd = Dv[c];
        if (!(fabs(dd) > 0.0)) continue;
        const double* aS = second ? cS2 : cS;
        const double* aN = second ? cN2 : cN;
        const double* aW = second ? cW2 : cW;
        const double* aE = second ? cE2 : cE;
        double* x = second ? x2 : x1;
        const double* b = second ? b2 : b1;
        const int nS = across(I, c, i, j, 0), nE = across(I, c, i, j, 3);
        const int nN = across(I, c, i, j, 1), nW = across(I, c, i, j, 2);
        double off = 0.0;
        if (nS >= 0) off += aS[c] * x[nS];
        if (nE >= 0) off += aE[c] * x[nE];
        if (nN >= 0) off += aN[c] * x[nN];
        if (nW >= 0) off += aW[c] * x[nW];
        x[c] = (b[c] - off) / dd;
      }
      __syncthreads();
    }
  }
}

/// Block-wide exclusive scan of affine maps x -> p + q x composed in thread
/// order: each thread passes the composition (p, q) of its own elements
/// (identity (0, 1) if none) and receives the composition of all elements of
/// lower threads. Uses sc[0 .. 2*warps) of shared memory; two __syncthreads.
template <typename T>
DEV void blockAffineExclusiveScan(T& p, T& q, T* sc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  // inclusive scan within the warp (later maps applied after earlier ones)
  T ip = p, iq = q;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T pp = __shfl_up_sync(0xffffffffu, ip, off);
    const T qq = __shfl_up_sync(0xffffffffu, iq, off);
    if (lane >= off) {
      ip = ip + iq * pp;
      iq = iq * qq;
    }
  }
  // exclusive within the warp
  T ep = __shfl_up_sync(0xffffffffu, ip, 1);
  T eq = __shfl_up_sync(0xffffffffu, iq, 1);
  if (lane == 0) {
    ep = T(0);
    eq = T(1);
  }
  if (lane == 31) {
    sc[2 * warp] = ip;
    sc[2 * warp + 1] = iq;
  }
  __syncthreads();
  if (warp == 0) {
    T wp = (lane < nwarps) ? sc[2 * lane] : T(0);
    T wq = (lane < nwarps) ? sc[2 * lane + 1] : T(1);
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const T pp = __shfl_up_sync(0xffffffffu, wp, off);
      const T qq = __shfl_up_sync(0xffffffffu, wq, off);
      if (lane >= off) {
        wp = wp + wq * pp;
        wq = wq * qq;
      }
    }
    T xp = __shfl_up_sync(0xffffffffu, wp, 1);
    T xq = __shfl_up_sync(0xffffffffu, wq, 1);
    if (lane == 0) {
      xp = T(0);
      xq = T(1);
    }
    if (lane < nwarps) {
      sc[2 * lane] = xp;
      sc[2 * lane + 1] = xq;
    }
  }
  __syncthreads();
  // earlier warps first, then the earlier lanes of this warp
  const T wp = sc[2 * warp], wq = sc[2 * warp + 1];
  p = ep + eq * wp;
  q = eq * wq;
}

/// One row of a lexicographic Gauss-Seidel sweep (LinearSystem.cpp:77-116).
/// With row j-1 already updated and row j+1 and the east neighbours still
/// holding their old values, the cell-order update of row j is the
/// first-order recurrence x_i = p_i + q_i x_{i-1},
///   p_i = (b_i - aS x_S - aE x_E - aN x_N) / a_P,  q_i = -aW / a_P,
/// solved by a block-wide scan. Row 0 is split in two: the wake-cut partner
/// (NI-1-i, 0) of (i, 0) comes later in the row for i < NI/2 (old value) and
/// earlier for i >= NI/2 (new value), so the second half is solved after the
/// first. A cell with a_P = 0 keeps its value (p = x, q = 0). This is the
/// reference's sweep map; only the rounding differs from cell-by-cell order.
///
/// Run by every thread of one CTA; rowPrev holds row j-1's new values,
/// oldRow and northRow rows j and j+1 as the previous sweep left them (the
/// unknowns themselves, or a copy). Needs NI <= 8 * blockDim.x. Leaves row
/// j's new values in rowNew and ends with a barrier; the caller publishes.
template <typename T>
struct SysView {
  const T *D, *S, *N, *W, *E, *b;
  T* x;
};

/// The row solve for any cells per thread (up to 8), loading as it goes.
template <typename T>
DEV void gsRowSolveAny(const Instance& I, int j, const SysView<T>& y, const T* oldRow, const T* northRow, T* rowNew,
                       const T* rowPrev, T* sc) {
  const T *D = y.D, *cS = y.S, *cN = y.N, *cW = y.W, *cE = y.E, *b = y.b;
  const int NI = I.NI, NJ = I.NJ;
  const int nt = blockDim.x;
  const int per = (NI + nt - 1) / nt;  // contiguous cells per thread
  const int i0 = threadIdx.x * per;
  const int segments = (j == 0) ? 2 : 1;
  T carry = T(0);
  for (int seg = 0; seg < segments; ++seg) {
    const int lo = (segments == 1) ? 0 : (seg == 0 ? 0 : NI / 2);
    const int hi = (segments == 1) ? NI : (seg == 0 ? NI / 2 : NI);
    T pv[8], qv[8];
    T P = T(0), Q = T(1);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      pv[e] = T(0);
      qv[e] = T(1);
      const int i = i0 + e;
      if (e >= per || i < lo || i >= hi) continue;
      const int c = j * NI + i;
      const T d = D[c];
      if (!(fabs(d) > T(0))) {
        pv[e] = oldRow[i];
        qv[e] = T(0);
      } else {
        T off = T(0);
        if (j > 0) {
          off += cS[c] * rowPrev[i];
        } else {
          const int a = I.acrossJ0[i];
          if (a >= 0) off += cS[c] * ((a < i) ? rowNew[a] : oldRow[a]);
        }
        if (i < NI - 1) off += cE[c] * oldRow[i + 1];
        if (j < NJ - 1) off += cN[c] * northRow[i];
        pv[e] = (b[c] - off) / d;
        qv[e] = (i > 0) ? -cW[c] / d : T(0);
      }
      P = pv[e] + qv[e] * P;
      Q = qv[e] * Q;
    }
    blockAffineExclusiveScan(P, Q, sc);
    T xv = P + Q * carry;  // value entering this thread's chunk
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int i = i0 + e;
      if (e >= per || i < lo || i >= hi) continue;
      xv = pv[e] + qv[e] * xv;
      rowNew[i] = xv;
    }
    __syncthreads();
    if (hi > lo) carry = rowNew[hi - 1];
  }
}

/// The row solve for at most MAXPER cells per thread. Every operand of the
/// thread's cells is loaded before any is used (indices clamped into the row;
/// values of cells outside it are never used), so the loads overlap instead
/// of waiting behind the branch on the diagonal.
template <typename T, int MAXPER>
DEV void gsRowSolveN(const Instance& I, int j, const SysView<T>& y, const T* oldRow, const T* northRow, T* rowNew,
                     const T* rowPrev, T* sc) {
  const T* __restrict__ D = y.D;
  const T* __restrict__ cS = y.S;
  const T* __restrict__ cN = y.N;
  const T* __restrict__ cW = y.W;
  const T* __restrict__ cE = y.E;
  const T* __restrict__ b = y.b;
  const int NI = I.NI, NJ = I.NJ;
  const int nt = blockDim.x;
  const int per = (NI + nt - 1) / nt;  // contiguous cells per thread
  const int i0 = threadIdx.x * per;
  const bool hasNorth = j < NJ - 1;
  const long long rowBase = static_cast<long long>(j) * NI;
  T dv[MAXPER], sv[MAXPER], ev[MAXPER], nv[MAXPER], wv[MAXPER], bv[MAXPER];
  T oldI[MAXPER], oldE[MAXPER], northI[MAXPER], prevI[MAXPER];
  int wake[MAXPER];
#pragma unroll
  for (int e = 0; e < MAXPER; ++e) {
    const int i = min(i0 + e, NI - 1);
    const long long c = rowBase + i;
    dv[e] = D[c];
    sv[e] = cS[c];
    ev[e] = cE[c];
    nv[e] = cN[c];
    wv[e] = cW[c];
    bv[e] = b[c];
    oldI[e] = oldRow[i];
    oldE[e] = oldRow[min(i + 1, NI - 1)];
    northI[e] = hasNorth ? northRow[i] : T(0);
    prevI[e] = (j > 0) ? rowPrev[i] : T(0);
    wake[e] = (j == 0) ? I.acrossJ0[i] : -1;
  }
  const int segments = (j == 0) ? 2 : 1;
  T carry = T(0);
  for (int seg = 0; seg < segments; ++seg) {
    const int lo = (segments == 1) ? 0 : (seg == 0 ? 0 : NI / 2);
    const int hi = (segments == 1) ? NI : (seg == 0 ? NI / 2 : NI);
    T pv[MAXPER], qv[MAXPER];
    T P = T(0), Q = T(1);
#pragma unroll
    for (int e = 0; e < MAXPER; ++e) {
      pv[e] = T(0);
      qv[e] = T(1);
      const int i = i0 + e;
      if (e >= per || i < lo || i >= hi) continue;
      const T d = dv[e];
      if (!(fabs(d) > T(0))) {
        pv[e] = oldI[e];
        qv[e] = T(0);
      } else {
        T off = T(0);
        if (j > 0) {
          off += sv[e] * prevI[e];
        } else {
          const int a = wake[e];
          if (a >= 0) off += sv[e] * ((a < i) ? rowNew[a] : oldRow[a]);
        }
        if (i < NI - 1) off += ev[e] * oldE[e];
        if (hasNorth) off += nv[e] * northI[e];
        pv[e] = (bv[e] - off) / d;
        qv[e] = (i > 0) ? -wv[e] / d : T(0);
      }
      P = pv[e] + qv[e] * P;
      Q = qv[e] * Q;
    }
    blockAffineExclusiveScan(P, Q, sc);
    T xv = P + Q * carry;  // value entering this thread's chunk
#pragma unroll
    for (int e = 0; e < MAXPER; ++e) {
      const int i = i0 + e;
      if (e >= per || i < lo || i >= hi) continue;
      xv = pv[e] + qv[e] * xv;
      rowNew[i] = xv;
    }
    __syncthreads();
    if (hi > lo) carry = rowNew[hi - 1];
  }
}

template <typename T>
DEV void gsRowSolve(const Instance& I, int j, const SysView<T>& y, const T* oldRow, const T* northRow, T* rowNew,
                    const T* rowPrev, T* sc) {
  if (I.NI <= 2 * static_cast<int>(blockDim.x)) {
    gsRowSolveN<T, 2>(I, j, y, oldRow, northRow, rowNew, rowPrev, sc);
  } else {
    gsRowSolveAny(I, j, y, oldRow, northRow, rowNew, rowPrev, sc);
  }
}

/// One row of the sweep on the unknowns in place: solve from the unknowns,
/// then publish row j to global memory (east/north reads of later rows and
/// the next sweep) and to rowPrev (the south values of row j + 1). Every
/// read of this row's old values and of rowPrev happened before the scan's
/// barriers. Ends without a barrier (the caller synchronises before the
/// next row).
template <typename T>
DEV void gsRow(const Instance& I, int j, const SysView<T>& y, T* rowNew, T* rowPrev, T* sc) {
  T* x = y.x;
  const int NI = I.NI;
  gsRowSolve(I, j, y, x + static_cast<long long>(j) * NI, x + static_cast<long long>(j + 1) * NI, rowNew, rowPrev,
             sc);
  for (int i = threadIdx.x; i < NI; i += blockDim.x) {
    x[j * NI + i] = rowNew[i];
    rowPrev[i] = rowNew[i];
  }
}

/// `sweeps` lexicographic sweeps of one system by one CTA, row after row.
/// Needs 2 * NI + 2 * warps doubles of shared memory.
template <typename T>
DEV void gsRowScanSweeps(const Instance& I, int sweeps, const SysView<T>& y, T* smem) {
  T* rowNew = smem;          // row j, new values
  T* rowPrev = smem + I.NI;  // row j - 1, new values
  T* sc = smem + 2 * I.NI;
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (int j = 0; j < I.NJ; ++j) {
      gsRow(I, j, y, rowNew, rowPrev, sc);
      prefetchRow(I, (j + 1 < I.NJ) ? j + 1 : 0, y);
      __syncthreads();
    }
  }
}

/// The k and omega sweeps as a software pipeline over 2 * sweeps CTAs: CTA
/// (eq, s) runs sweep s of equation eq (0: k, 1: omega) and at step t updates
/// row t - 2s. Sweep s reads row j+1 as left by sweep s-1 (done at step t-1),
/// row j as left by sweep s-1 (step t-2) and row j-1 from its own previous
/// step, so every value is the one the sequential order would use, and no row
/// is written at the step it is read by another sweep (sweep s-1 writes row
/// j+2, sweep s+1 row j-2). Every CTA of the cluster joins each step's
/// barrier. Same arithmetic as gsRowScanSweeps, NJ + 2 (sweeps - 1) steps
/// instead of sweeps * NJ.
/// Bring row j's coefficients and right-hand side (fixed during the sweeps)
/// towards this SM's L1 ahead of its scan, one prefetch per 128-byte line,
/// spread over the CTA's threads. A hint only: it changes no value.
template <typename T>
DEV void prefetchRow(const Instance& I, int j, const SysView<T>& y) {
  if (j < 0 || j >= I.NJ) return;
  constexpr int perLine = 128 / static_cast<int>(sizeof(T));
  const int lines = (I.NI + perLine - 1) / perLine;
  const T* arrays[6] = {y.D, y.S, y.N, y.W, y.E, y.b};
  for (int q = threadIdx.x; q < 6 * lines; q += blockDim.x) {
    const T* line = arrays[q / lines] + static_cast<long long>(j) * I.NI + (q % lines) * perLine;
    asm volatile("prefetch.global.L1 [%0];" ::"l"(line));
  }
}

template <typename T>
DEV void gsRowScanPipelined(const Instance& I, Team& t, int sweeps, const SysView<T>& kSys,
                            const SysView<T>& wSys, T* smem) {
  const int role = static_cast<int>(t.rank);
  const bool active = role < 2 * sweeps;
  const bool omega = active && role >= sweeps;
  const int s = active ? role % sweeps : 0;
  const SysView<T>& y = omega ? wSys : kSys;
  T* rowNew = smem;
  T* rowPrev = smem + I.NI;
  T* sc = smem + 2 * I.NI;
  const int steps = I.NJ + 2 * (sweeps - 1);
  if (active) prefetchRow(I, -2 * s, y);
  for (int step = 0; step < steps; ++step) {
    const int j = step - 2 * s;
    if (active && j >= 0 && j < I.NJ) gsRow(I, j, y, rowNew, rowPrev, sc);
    if (active) prefetchRow(I, j + 1, y);  // the next step's row, over the barrier
    t.cl.sync();
  }
}

// ---- the chained k/omega sweeps: rows pushed to the next stage ------------------

constexpr int kChainSlots = 4;                    // ring rows per stage (Shared::chainBar)
constexpr long long kChainSpinLimit = 1LL << 24;  // polls before a wait gives up (~0.3 s)

/// Shared memory of gsRowScanChained, in elements of T.
__host__ __device__ inline long long chainSmemElems(int NI) { return (2LL + kChainSlots) * NI + 64; }

DEV unsigned smemAddr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
/// The shared::cluster address of this CTA's shared-memory address `a` in CTA `rank`.
DEV unsigned clusterAddr(unsigned a, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
DEV void mbarInit(unsigned long long* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(b)) : "memory");
}
/// This CTA's one arrival on the barrier's current phase, expecting `bytes`.
DEV void mbarArm(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(b)), "r"(bytes) : "memory");
}
/// Whether the phase of parity `parity` has completed (acquire, cluster scope).
DEV bool mbarDone(const unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smemAddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
/// Store v into another CTA's shared memory; its mbarrier counts the bytes.
DEV void pushRemote(unsigned dst, double v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(dst), "d"(v),
               "r"(bar)
               : "memory");
}
DEV void pushRemote(unsigned dst, float v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];" ::"r"(dst), "f"(v),
               "r"(bar)
               : "memory");
}
DEV unsigned loadRelaxedCluster(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
DEV void storeRelaxedCluster(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

/// Kernel start: the ring barriers armed for the first kChainSlots rows (of
/// `rowBytes` each), the release count at zero, and the split CG's halo
/// barrier armed for the bytes the neighbouring CTAs push each iteration. Made visible to the peers and
/// the async proxy before the kernel's first cluster barrier.
DEV void chainSetup(Shared& sh, unsigned rowBytes, unsigned haloBytes) {
  if (threadIdx.x == 0) {
    // cgGlobalSplit's halo barrier, armed for its first iteration
    mbarInit(&sh.haloBar);
    mbarArm(&sh.haloBar, haloBytes);
    sh.haloPhase = 0u;
    sh.haloBytes = haloBytes;
    for (int k = 0; k < kChainSlots; ++k) {
      mbarInit(&sh.chainBar[k]);
      mbarArm(&sh.chainBar[k], rowBytes);
    }
    sh.chainAck = 0u;
    sh.chainNever = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
}

/// The k and omega sweeps as a chain of 2 * sweeps CTAs, CTA (eq, s) running
/// sweep s of equation eq (0: k, 1: omega), without cluster-wide barriers.
/// Row g (counted over the launch: g = base + j, base = calls so far x NJ)
/// travels through ring slot g % kChainSlots: as a stage finishes a row it
/// pushes the values into the next stage's slot with st.async, whose bytes
/// complete that slot's mbarrier; the next stage waits for rows j and j+1
/// (its old own-row and north values), reads them from its own shared
/// memory, and when done with row j re-arms the slot for row g + kChainSlots
/// and writes g + 1 into its producer's release count, which the producer
/// waits for before pushing into that slot again. The first stage reads the
/// unknowns, the last writes them, so the values and the arithmetic are
/// those of gsRowScanSweeps (the same bits). A wait that gives up sets
/// kFaultChainWait in the launch's fault word and the call waits no more, so
/// the launch always ends (and reports the fault). With `waitTest` the second
/// stage also waits once per call for a count nothing sets, which gives up
/// and reports the fault while the rows still flow as usual.
template <typename T>
DEV void gsRowScanChained(const Instance& I, Team& t, Shared& sh, int sweeps, const SysView<T>& kSys,
                          const SysView<T>& wSys, T* smem, unsigned base, bool waitTest) {
  const int role = static_cast<int>(t.rank);
  if (role >= 2 * sweeps) return;
  const int s = role % sweeps;
  const bool hasProducer = s > 0, hasConsumer = s < sweeps - 1;
  const SysView<T>& y = (role >= sweeps) ? wSys : kSys;
  const int NI = I.NI, NJ = I.NJ;
  const unsigned rowBytes = static_cast<unsigned>(NI * sizeof(T));
  T* rowNew = smem;
  T* rowPrev = smem + NI;
  T* sc = smem + 2 * NI;
  T* ring = smem + 2 * NI + 64;
  const unsigned nextRing = hasConsumer ? clusterAddr(smemAddr(ring), role + 1) : 0u;
  const unsigned nextBar = hasConsumer ? clusterAddr(smemAddr(&sh.chainBar[0]), role + 1) : 0u;
  unsigned* producerAck = hasProducer ? t.cl.map_shared_rank(&sh.chainAck, role - 1) : nullptr;
  T* x = y.x;
  bool faulted = false;  // a wait of this call gave up: the call waits no more
  prefetchRow(I, 0, y);
  for (int j = 0; j < NJ; ++j) {
    const unsigned g = base + static_cast<unsigned>(j);
    const unsigned slot = g % kChainSlots, slotN = (g + 1) % kChainSlots;
    if (threadIdx.x == 0 && waitTest && s == 1 && j == 0) {
      // test: once per call the second stage waits for a count nothing sets
      long long spins = 0;
      while (loadRelaxedCluster(&sh.chainNever) == 0u && ++spins <= kChainSpinLimit) {
      }
      if (spins > kChainSpinLimit) atomicOr(I.iterations + 1, kFaultChainWait);
    }
    if (threadIdx.x == 0 && !faulted) {
      long long spins = 0;
      for (;;) {
        bool ready = true;
        if (hasProducer) {
          ready = mbarDone(&sh.chainBar[slot], (g / kChainSlots) & 1u) &&
                  (j + 1 >= NJ || mbarDone(&sh.chainBar[slotN], ((g + 1) / kChainSlots) & 1u));
        }
        // the next stage has released the row this slot held (g - kChainSlots)
        if (ready && hasConsumer && g + 1 >= kChainSlots) {
          ready = loadRelaxedCluster(&sh.chainAck) >= g + 1 - kChainSlots;
        }
        if (ready) break;
        if (++spins > kChainSpinLimit) {
          atomicOr(I.iterations + 1, kFaultChainWait);
          faulted = true;
          break;
        }
      }
    }
    __syncthreads();
    const long long row = static_cast<long long>(j) * NI;
    const T* oldRow = hasProducer ? ring + slot * NI : x + row;
    const T* northRow = hasProducer ? ring + slotN * NI : x + row + NI;
    gsRowSolve(I, j, y, oldRow, northRow, rowNew, rowPrev, sc);
    // every read of ring slot `slot` happened before gsRowSolve's barriers
    if (threadIdx.x == 0 && hasProducer) {
      mbarArm(&sh.chainBar[slot], rowBytes);  // for row g + kChainSlots
      storeRelaxedCluster(producerAck, g + 1);
    }
    for (int i = threadIdx.x; i < NI; i += blockDim.x) {
      const T v = rowNew[i];
      rowPrev[i] = v;
      if (hasConsumer) {
        pushRemote(nextRing + (slot * NI + i) * static_cast<unsigned>(sizeof(T)), v, nextBar + slot * 8u);
      } else {
        x[row + i] = v;
      }
    }
    prefetchRow(I, j + 1, y);
    if (!hasProducer && j + 2 < NJ) {
      // the first stage's next north row (the unknowns, fixed until the last stage writes them)
      constexpr int perLine = 128 / static_cast<int>(sizeof(T));
      for (int q = threadIdx.x; q * perLine < NI; q += blockDim.x) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(x + row + 2 * NI + q * perLine));
      }
    }
    // the next row's wait ends in a barrier, which orders these rowPrev
    // writes and rowNew reads before the next row's use of them
  }
}

DEV SysView<double> kSystem(const Instance& I) { return SysView<double>{I.kD, I.kS, I.kN, I.kW, I.kE, I.kB, I.k}; }
DEV SysView<double> omegaSystem(const Instance& I) {
  return SysView<double>{I.wD, I.wS, I.wN, I.wW, I.wE, I.wB, I.om};
}
DEV SysView<float> correctionSystem(const Rows32& r) { return SysView<float>{r.D, r.S, r.N, r.W, r.E, r.r, r.x}; }

// ---- phase: Rhie-Chow face fluxes (SimpleSolver.cpp:445-496) -------------------

DEV void rhieChowFace(const Instance& I, const Face& f) {
  const FaceGeo& g = geo(I, f);
  const int o = f.owner;
  const double Sx = g.Sx[f.idx], Sy = g.Sy[f.idx], D = g.D[f.idx];
  double* mf = massFluxPtr(I, f);
  if (f.other >= 0) {
    const int n = f.other;
    const double w = g.w[f.idx];
    const double ix = I.u[o] * w + I.u[n] * (1.0 - w);
    const double iy = I.v[o] * w + I.v[n] * (1.0 - w);
    const double dens = w * I.rho[o] + (1.0 - w) * I.rho[n];
    const double mob = w * (I.vol[o] / I.aD[o]) + (1.0 - w) * (I.vol[n] / I.aD[n]);
    const double sgx = I.gpx[o] * w + I.gpx[n] * (1.0 - w);
    const double sgy = I.gpy[o] * w + I.gpy[n] * (1.0 - w);
    const double compact = (I.p[n] - I.p[o]) * D;
    const double smooth = sgx * Sx + sgy * Sy;
    *mf = dens * (ix * Sx + iy * Sy) - dens * mob * (compact - smooth);
    return;
  }
  const double dens = I.rho[o];
  if (imposesVelocity(I, f)) {
    *mf = dens * (bcU(I, f) * Sx + bcV(I, f) * Sy);
  } else {
    const double mob = I.vol[o] / I.aD[o];
    const double compact = (bcP(I, f) - I.p[o]) * D;
    const double smooth = I.gpx[o] * Sx + I.gpy[o] * Sy;
    *mf = dens * (I.u[o] * Sx + I.v[o] * Sy) - dens * mob * (compact - smooth);
  }
}

DEV void phaseRhieChow(const Instance& I, Team& t) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    if (j == 0) rhieChowFace(I, faceS(I, c, i, j));
    rhieChowFace(I, faceN(I, c, i, j));
    if (i == 0) rhieChowFace(I, faceW(I, c, i, j));
    rhieChowFace(I, faceE(I, c, i, j));
  }
}

// ---- phase: pressure-correction assembly (SimpleSolver.cpp:498-580) ------------

/// rho_f * mobility_f * D for a face with a cell on each side (the same
/// coefficient the flux correction uses).
DEV double pressureCoefficient(const Instance& I, const Face& f, int n) {
  const FaceGeo& g = geo(I, f);
  const int o = f.owner;
  const double w = g.w[f.idx];
  const double dens = w * I.rho[o] + (1.0 - w) * I.rho[n];
  const double mob = w * (I.vol[o] / I.aD[o]) + (1.0 - w) * (I.vol[n] / I.aD[n]);
  return dens * mob * g.D[f.idx];
}

DEV void phasePressureAssembly(const Instance& I, Team& t, double& netL1, double& bSum) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double net = 0.0, diag = 0.0;
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      const double flux = massFlux(I, f);
      if (f.mine) net += flux; else net -= flux;
      if (f.other >= 0) {
        const double coef = pressureCoefficient(I, f, f.other);
        diag += coef;
        if (f.mine) {
          double* slot = f.fam ? I.pE + f.idx : I.pN + f.idx;
          *slot = 0.0 + (-coef);
        }
        continue;
      }
      if (imposesVelocity(I, f)) continue;
      const double mob = I.vol[c] / I.aD[c];
      diag += I.rho[c] * mob * geo(I, f).D[f.idx];
    }
    I.net[c] = net;
    I.pD[c] = diag;
    I.pB[c] = -net;
    netL1 += fabs(net);
    bSum += -net;
  }
}

/// y = A x for the pressure-correction matrix, in multiply's face order.
DEV double pressureRow(const Instance& I, int c, int i, int j, const double* xv, double xc) {
  double y = I.pD[c] * xc;
  if (j > 0) y += I.pN[j * I.NI + i] * xv[c - I.NI];
  else if (I.acrossJ0[i] >= 0) y += I.pN[i] * xv[I.acrossJ0[i]];
  if (j < I.NJ - 1) y += I.pN[(j + 1) * I.NI + i] * xv[c + I.NI];
  if (i > 0) y += I.pE[j * (I.NI + 1) + i] * xv[c - 1];
  if (i < I.NI - 1) y += I.pE[j * (I.NI + 1) + i + 1] * xv[c + 1];
  return y;
}

// ---- phase: correction (SimpleSolver.cpp:582-660) ------------------------------

DEV void correctFace(const Instance& I, const Face& f) {
  const FaceGeo& g = geo(I, f);
  const int o = f.owner;
  double* mf = massFluxPtr(I, f);
  if (f.other >= 0) {
    const int n = f.other;
    const double w = g.w[f.idx];
    const double dens = w * I.rho[o] + (1.0 - w) * I.rho[n];
    const double mob = w * (I.vol[o] / I.aD[o]) + (1.0 - w) * (I.vol[n] / I.aD[n]);
    *mf -= dens * mob * g.D[f.idx] * (I.x[n] - I.x[o]);
    return;
  }
  if (imposesVelocity(I, f)) return;
  const double mob = I.vol[o] / I.aD[o];
  *mf -= I.rho[o] * mob * g.D[f.idx] * (0.0 - I.x[o]);
}

DEV void phaseCorrect(const Instance& I, Team& t) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double gx = 0.0, gy = 0.0;
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      const FaceGeo& g = geo(I, f);
      double fc;
      if (f.other >= 0) {
        const double w = g.w[f.idx];
        fc = w * I.x[f.owner] + (1.0 - w) * I.x[f.other];
      } else if (imposesVelocity(I, f)) {
        fc = I.x[f.owner];
      } else {
        fc = 0.0;
      }
      ggAdd(f, g.Sx[f.idx], g.Sy[f.idx], fc, gx, gy);
    }
    ggFinish(I.vol[c], gx, gy);
    I.p[c] += I.alphaP * I.x[c];
    const double mob = I.vol[c] / I.aD[c];
    I.u[c] -= gx * mob;
    I.v[c] -= gy * mob;
    if (j == 0) correctFace(I, fs[0]);
    correctFace(I, fs[1]);
    if (i == 0) correctFace(I, fs[2]);
    correctFace(I, fs[3]);
  }
}

// ---- divergence (SimpleSolver.cpp:796-817) -------------------------------------

DEV double cellDivergence(const Instance& I, int c, int i, int j) {
  double net = 0.0;
  const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const Face& f = fs[k];
    const double dens = smax(I.rho[f.owner], kTinySolver);
    const double vf = massFlux(I, f) / dens;
    if (f.mine) net += vf; else net -= vf;
  }
  const double area = I.vol[c];
  return (area > 0.0) ? net / area : 0.0;
}

// ---- k-omega SST (KOmegaSST.cpp) -----------------------------------------------

/// Face value of k or omega (KOmegaSST.cpp:26-68, with the no-slip override
/// of :236-241 for omega). isOmega selects the wall treatment.
DEV double sstFaceValue(const Instance& I, const Face& f, const double* phi, bool isOmega) {
  const int o = f.owner;
  if (f.nb >= 0) {
    const double w = geo(I, f).w[f.idx];
    return w * phi[o] + (1.0 - w) * phi[f.nb];
  }
  if (f.other >= 0) {
    const double w = 1.0;  // ownerWeight() of a face without a neighbour
    return w * phi[o] + (1.0 - w) * phi[f.other];
  }
  const double inflow = isOmega ? I.wIn : I.kIn;
  switch (kindOf(I, f)) {
    case kWall: return isOmega ? phi[o] : 0.0;
    case kInlet: return inflow;
    case kFarField: return (massFlux(I, f) < 0.0) ? inflow : phi[o];
    default: return phi[o];
  }
}

DEV void phaseSstBlending(const Instance& I, Team& t, double& divMax) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    divMax = smax(divMax, fabs(cellDivergence(I, c, i, j)));
    // computeStrain (:202-216), gradients from the start of the iteration.
    const double s11 = I.gux[c], s22 = I.gvy[c];
    const double s12 = 0.5 * (I.guy[c] + I.gvx[c]);
    const double S = sqrt(2.0 * (s11 * s11 + s22 * s22 + 2.0 * s12 * s12));
    I.strain[c] = S;
    // Green-Gauss gradients of k and omega (:224-244).
    double kx = 0.0, ky = 0.0, wx = 0.0, wy = 0.0;
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      const FaceGeo& g = geo(I, f);
      const double Sx = g.Sx[f.idx], Sy = g.Sy[f.idx];
      ggAdd(f, Sx, Sy, sstFaceValue(I, f, I.k, false), kx, ky);
      ggAdd(f, Sx, Sy, sstFaceValue(I, f, I.om, true), wx, wy);
    }
    const double vol = I.vol[c];
    ggFinish(vol, kx, ky);
    ggFinish(vol, wx, wy);
    I.gkx[c] = kx; I.gky[c] = ky; I.gwx[c] = wx; I.gwy[c] = wy;
    // Cross-diffusion and the blending functions (:247-286).
    const double d = smax(I.wallDist[c], kTinySst);
    const double rho = I.rho[c];
    const double nu = I.muMol[c] / smax(rho, kTinySst);
    const double omega = smax(I.om[c], kMinOmega);
    const double energy = smax(I.k[c], 0.0);
    const double cdv = 2.0 * rho * kSigmaW2 * (kx * wx + ky * wy) / omega;
    const double cdp = smax(cdv, 1.0e-10);
    const double term1 = sqrt(smax(energy, 0.0)) / (kBetaStar * omega * d);
    const double term2 = 500.0 * nu / (d * d * omega);
    const double term3 = 4.0 * rho * kSigmaW2 * energy / (cdp * d * d);
    const double arg1 = smin(smax(term1, term2), term3);
    const double F1 = tanh(sclamp(arg1 * arg1 * arg1 * arg1, 0.0, 50.0));
    const double arg2 = smax(2.0 * term1, term2);
    const double F2 = tanh(sclamp(arg2 * arg2, 0.0, 50.0));
    I.cd[c] = cdv;
    I.f1[c] = F1;
    I.f2[c] = F2;
    // Limited production (:362-368).
    const double raw = I.mut[c] * S * S;
    const double ceiling = kProdLimit * kBetaStar * rho * smax(I.k[c], 0.0) * smax(I.om[c], kMinOmega);
    I.prod[c] = smin(raw, ceiling);
  }
}

DEV double blendF1(double f1, double nearValue, double farValue) { return f1 * nearValue + (1.0 - f1) * farValue; }

/// Assemble, relax and measure one row of the k and of the omega equation
/// (KOmegaSST.cpp:378-466); both equations in one pass over the faces.
DEV void phaseSstAssembly(const Instance& I, Team& t, double (&acc)[4]) {
  const double relax = sclamp(I.alphaT, 0.05, 1.0);
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double dK = 0.0, bK = 0.0, dW = 0.0, bW = 0.0;
    double oK[4] = {0.0, 0.0, 0.0, 0.0}, oW[4] = {0.0, 0.0, 0.0, 0.0};
    const Face fs[4] = {faceS(I, c, i, j), faceN(I, c, i, j), faceW(I, c, i, j), faceE(I, c, i, j)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Face& f = fs[k];
      const FaceGeo& g = geo(I, f);
      const int o = f.owner;
      const double flux = massFlux(I, f);
      const double Dt = g.Dt[f.idx];
      if (f.other >= 0) {
        const int n = f.other;
        const double w = (f.nb >= 0) ? g.w[f.idx] : 1.0;
        const double f1o = I.f1[o], f1n = I.f1[n];
        const double sko = blendF1(f1o, kSigmaK1, kSigmaK2), skn = blendF1(f1n, kSigmaK1, kSigmaK2);
        const double swo = blendF1(f1o, kSigmaW1, kSigmaW2), swn = blendF1(f1n, kSigmaW1, kSigmaW2);
        const double muo = I.muMol[o], mun = I.muMol[n], mto = I.mut[o], mtn = I.mut[n];
        const double difK = (w * (muo + sko * mto) + (1.0 - w) * (mun + skn * mtn)) * Dt;
        const double difW = (w * (muo + swo * mto) + (1.0 - w) * (mun + swn * mtn)) * Dt;
        const double outward = smax(flux, 0.0);
        const double inward = smax(-flux, 0.0);
        if (f.mine) {
          dK += outward + difK;
          dW += outward + difW;
          oK[k] = 0.0 + (-inward - difK);
          oW[k] = 0.0 + (-inward - difW);
        } else {
          dK += inward + difK;
          dW += inward + difW;
          oK[k] = 0.0 + (-outward - difK);
          oW[k] = 0.0 + (-outward - difW);
        }
        continue;
      }
      const double f1o = I.f1[o];
      const double difK = (I.muMol[o] + blendF1(f1o, kSigmaK1, kSigmaK2) * I.mut[o]) * Dt;
      const double difW = (I.muMol[o] + blendF1(f1o, kSigmaW1, kSigmaW2) * I.mut[o]) * Dt;
      const int kind = kindOf(I, f);
      const bool imposed = kind == kWall || kind == kInlet || (kind == kFarField && flux < 0.0);
      if (imposed) {
        const double valK = (kind == kWall) ? 0.0 : I.kIn;
        const double valW = I.wIn;  // the omega equation's wall value is its inflow value
        dK += difK + smax(flux, 0.0);
        bK += (difK - smin(flux, 0.0)) * valK;
        dW += difW + smax(flux, 0.0);
        bW += (difW - smin(flux, 0.0)) * valW;
      } else {
        dK += smax(flux, 0.0);
        dW += smax(flux, 0.0);
      }
    }
    // Sources (:446-453): explicit production, implicit destruction.
    const double vol = I.vol[c];
    const double rho = I.rho[c];
    const double F1 = I.f1[c];
    const double omPos = smax(I.om[c], kMinOmega);
    const double S = I.strain[c];
    bK += I.prod[c] * vol;
    dK += kBetaStar * rho * omPos * vol;
    const double gamma = blendF1(F1, I.gamma1, I.gamma2);
    const double beta = blendF1(F1, kBeta1, kBeta2);
    double wProd = gamma * rho * S * S;
    wProd += (1.0 - F1) * I.cd[c];
    bW += wProd * vol;
    dW += beta * rho * omPos * vol;
    // Implicit under-relaxation (:455-463).
    const double kc = I.k[c], wc = I.om[c];
    if (fabs(dK) > kTinySst) {
      const double relaxed = dK / relax;
      bK += (relaxed - dK) * kc;
      dK = relaxed;
    }
    if (fabs(dW) > kTinySst) {
      const double relaxed = dW / relax;
      bW += (relaxed - dW) * wc;
      dW = relaxed;
    }
    I.kD[c] = dK; I.kS[c] = oK[0]; I.kN[c] = oK[1]; I.kW[c] = oK[2]; I.kE[c] = oK[3]; I.kB[c] = bK;
    I.wD[c] = dW; I.wS[c] = oW[0]; I.wN[c] = oW[1]; I.wW[c] = oW[2]; I.wE[c] = oW[3]; I.wB[c] = bW;
    double yk = dK * kc, yw = dW * wc;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int n = across(I, c, i, j, k);
      if (n >= 0) {
        yk += oK[k] * I.k[n];
        yw += oW[k] * I.om[n];
      }
    }
    acc[0] += fabs(bK - yk);
    acc[1] += fabs(dK);
    acc[2] += fabs(bW - yw);
    acc[3] += fabs(dW);
    if (I.precision == 1) {
      const Rows32& a = I.tk;
      a.D[c] = static_cast<float>(dK); a.S[c] = static_cast<float>(oK[0]);
      a.N[c] = static_cast<float>(oK[1]); a.W[c] = static_cast<float>(oK[2]);
      a.E[c] = static_cast<float>(oK[3]); a.r[c] = static_cast<float>(bK - yk); a.x[c] = 0.0f;
      const Rows32& b = I.tw;
      b.D[c] = static_cast<float>(dW); b.S[c] = static_cast<float>(oW[0]);
      b.N[c] = static_cast<float>(oW[1]); b.W[c] = static_cast<float>(oW[2]);
      b.E[c] = static_cast<float>(oW[3]); b.r[c] = static_cast<float>(bW - yw); b.x[c] = 0.0f;
    }
  }
}

/// wallOmega (KOmegaSST.cpp:86-92).
DEV double wallOmega(const Instance& I, double nu, double distance, double energy) {
  const double d = smax(distance, kTinySst);
  const double viscous = 6.0 * nu / (kBeta1 * d * d);
  const double logarithmic = sqrt(smax(energy, 0.0)) / (I.betaStarQuarter * kKappa * d);
  return sqrt(viscous * viscous + logarithmic * logarithmic);
}

/// Floors, wall conditions, eddy viscosity, ranges (KOmegaSST.cpp:289-345,
/// :469-471, :513-529; SimpleSolver.cpp:232-245, :782-790).
DEV void phaseSstFinish(const Instance& I, Team& t, double (&mx)[8]) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % I.NI, j = c / I.NI;
    double kRaw = I.k[c], wRaw = I.om[c];
    if (I.precision == 1) {
      kRaw += static_cast<double>(I.tk.x[c]);
      wRaw += static_cast<double>(I.tw.x[c]);
    }
    double kc = smax(kRaw, 0.0);
    double wc = smax(wRaw, kMinOmega);
    const uint8_t mask = I.wallMask[c];
    if (mask != 0) {
      const double d = smax(I.wallDist[c], kTinySst);
      const double rho = smax(I.rho[c], kTinySst);
      const double mu = I.muMol[c];
      const double nu = mu / rho;
      wc = wallOmega(I, nu, d, kc);
      const double uc = I.u[c], vc = I.v[c];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (!(mask & (1u << k))) continue;
        const Face f = (k == 0) ? faceS(I, c, i, j) : (k == 1) ? faceN(I, c, i, j)
                                 : (k == 2) ? faceW(I, c, i, j) : faceE(I, c, i, j);
        const FaceGeo& g = geo(I, f);
        const double nX = g.nx[f.idx] * -1.0, nY = g.ny[f.idx] * -1.0;
        const double dn = uc * nX + vc * nY;
        const double px = uc - nX * dn, py = vc - nY * dn;
        const double tangential = hypot(px, py);
        const double shear = mu * tangential / d;
        const double fv = sqrt(shear / rho);
        mx[5] = smax(mx[5], fv * d / smax(nu, kTinySst));
      }
    }
    I.k[c] = kc;
    I.om[c] = wc;
    const double denom = smax(kA1 * smax(wc, kMinOmega), I.strain[c] * I.f2[c]);
    const double mut = I.rho[c] * kA1 * smax(kc, 0.0) / smax(denom, kTinySst);
    I.mut[c] = mut;
    I.mu[c] = I.muMol[c] + mut;
    // ranges: max of (k, omega, mut) and of their negatives (for the minima)
    mx[0] = smax(mx[0], kc); mx[1] = smax(mx[1], -kc);
    mx[2] = smax(mx[2], wc); mx[3] = smax(mx[3], -wc);
    mx[4] = smax(mx[4], mut); mx[6] = smax(mx[6], -mut);
    const double muMol = I.muMol[c];
    if (muMol > 0.0) mx[7] = smax(mx[7], mut / muMol);
  }
}

// ---- pressure CG: one reduction per iteration ----------------------------------
//
// The reference's Jacobi-PCG (LinearSystem.cpp:118-210) needs two global
// reductions per iteration (d.Ad, then r.z and sum |r|): two cluster barriers.
// Here it is rearranged as Chronopoulos and Gear's single-reduction PCG
// (J. Comput. Appl. Math. 25, 1989), which computes the same iterates in
// exact arithmetic with one reduction of three sums per iteration:
//
//   u = M^-1 r,  w = A u,  gamma = r.u,  delta = w.u,  rho = sum |r|
//   beta_k = gamma_k / gamma_(k-1),  d.Ad_k = delta_k - beta_k gamma_k / alpha_(k-1),
//   alpha_k = gamma_k / d.Ad_k
//   p = u + beta p,  s = w + beta s (= A p),  x += alpha p,  r -= alpha s
//
// with the reference's stopping rule (rho <= tolerance * rho_0, tested after
// each update), its cap, and its breakdown guards (d.Ad = 0 before an update,
// r.z = 0 before forming beta). One launch phase per iteration: each cell
// forms its own p, s, x, r and u' = M^-1 r', and w' = A u' from its
// neighbours' u', which it recomputes from their r, w and s of the previous
// iteration (read from the other half of double-buffered r, w and s, so no
// neighbour's update can race with the read). Every cell's u' is the same
// expression in every thread that forms it, so the bits agree.
//
// Rounding: the iterates differ from the reference's two-reduction form only
// in the last bits (~1e-13 relative after 200 iterations on the 384x96 and
// 768x192 pressure systems, the same order as summing the dot products in
// another order), checked by the parity tests after the pressure solve.

DEV double precondition(double rc, double dg) { return (fabs(dg) > 0.0) ? rc / dg : rc; }

/// The three reduced sums of one iteration, and the scalars they give.
struct CgScalars {
  double alpha{0.0}, beta{0.0}, gamma{0.0};
};

/// After a reduction of {gamma', delta', rho'}: the reference's stop tests and
/// the next alpha and beta. Returns false when the solve stops.
DEV bool cgNext(const Instance& I, CgScalars& k, const double (&acc)[3], double initial) {
  if (acc[2] <= I.cgTol * initial) return false;  // converged
  if (!(fabs(k.gamma) > 0.0)) return false;        // r.z vanished
  const double beta = acc[0] / k.gamma;
  const double dAd = acc[1] - beta * acc[0] / k.alpha;  // p.Ap of the next direction
  if (!(fabs(dAd) > 0.0)) return false;
  k.beta = beta;
  k.alpha = acc[0] / dAd;
  k.gamma = acc[0];
  return true;
}

/// Band layout of the shared-memory CG: per CTA, 9 cell arrays of `stride`
/// doubles (stride = the largest band's cells, so a neighbour's value sits at
/// the same offset in its CTA) and the band's face coefficients: north-family
/// faces of rows j0 .. j1 (stride + NI) and east-family faces (stride + rows).
enum CgSmemArray : int { kSD = 0, kSX, kSP, kSR0, kSR1, kSW0, kSW1, kSS0, kSS1, kCgCellArrays };

__host__ __device__ inline int cgRowsMax(int NJ, int R) { return (NJ + R - 1) / R; }
__host__ __device__ inline int cgSmemStride(int NI, int NJ, int R) { return cgRowsMax(NJ, R) * NI; }
__host__ __device__ inline long long cgSmemDoubles(int NI, int NJ, int R) {
  const long long stride = cgSmemStride(NI, NJ, R);
  return kCgCellArrays * stride + (stride + NI) + (stride + cgRowsMax(NJ, R));
}

DEV int bandFirstCell(int NI, int NJ, int R, int r) { return NI * ((NJ * r) / R); }

/// The single-reduction PCG with the band in shared memory: vectors, the
/// diagonal and the face coefficients stay on chip; a neighbour in the band
/// below or above is read from that CTA's shared memory (DSMEM). On entry
/// I.r = b (x = 0); `initial` = sum |b|, `gamma` = b.M^-1 b. Returns the
/// iterations run; x is written to global memory at the end.
DEV int cgShared(const Instance& I, Team& t, Shared& sh, double* dyn, double initial, double gamma) {
  const int NI = I.NI, NJ = I.NJ;
  const int R = static_cast<int>(t.R), rank = static_cast<int>(t.rank);
  const int stride = cgSmemStride(NI, NJ, R);
  double* a[kCgCellArrays];
#pragma unroll
  for (int k = 0; k < kCgCellArrays; ++k) a[k] = dyn + k * stride;
  double* fN = dyn + kCgCellArrays * stride;  // face row j0 + lj at lj * NI
  double* fE = fN + stride + NI;              // row j0 + lj at lj * (NI + 1)
  const int j0 = t.c0 / NI;
  const int cBelow = (rank > 0) ? bandFirstCell(NI, NJ, R, rank - 1) : 0;
  const int cAbove = t.c1;
  // remote views of the neighbouring bands' diagonal, r, w and s
  double* below[kCgCellArrays] = {};
  double* above[kCgCellArrays] = {};
#pragma unroll
  for (int k = 0; k < kCgCellArrays; ++k) {
    if (rank > 0) below[k] = t.cl.map_shared_rank(a[k], rank - 1);
    if (rank < R - 1) above[k] = t.cl.map_shared_rank(a[k], rank + 1);
  }
  // load the band: diagonal, b, zero x, p and s; the face coefficients with
  // the boundary faces' zeros (the wake cut's j = 0 faces keep theirs)
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int m = c - t.c0;
    a[kSD][m] = I.pD[c];
    a[kSX][m] = 0.0;
    a[kSP][m] = 0.0;
    a[kSR0][m] = I.r[c];
    a[kSS0][m] = 0.0;
  }
  const int rows = (t.c1 - t.c0) / NI;
  for (int k = t.tid; k < (rows + 1) * NI; k += t.T) {
    const int lj = k / NI, i = k % NI, j = j0 + lj;
    double v = 0.0;
    if (j > 0 && j < NJ) v = I.pN[j * NI + i];
    else if (j == 0 && I.acrossJ0[i] >= 0) v = I.pN[i];
    fN[k] = v;
  }
  for (int k = t.tid; k < rows * (NI + 1); k += t.T) {
    const int lj = k / (NI + 1), i = k % (NI + 1), j = j0 + lj;
    fE[k] = (i > 0 && i < NI) ? I.pE[j * (NI + 1) + i] : 0.0;
  }
  t.cl.sync();  // every band loaded before anyone reads a neighbour's

  // where cell n's array k lives: this band, the band below, or above
  auto at = [&](int k, int n) -> double {
    if (n >= t.c0 && n < t.c1) return a[k][n - t.c0];
    if (n < t.c0) return below[k][n - cBelow];
    return above[k][n - cAbove];
  };
  // w0 = A u0 and delta0 = w0.u0
  {
    double acc[1] = {0.0};
    const int op1[1] = {kSum};
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int m = c - t.c0, i = c % NI, j = c / NI, lj = j - j0;
      auto uAt = [&](int n) { return precondition(at(kSR0, n), at(kSD, n)); };
      const double un = precondition(a[kSR0][m], a[kSD][m]);
      double y = a[kSD][m] * un;
      const int nS = (j > 0) ? c - NI : I.acrossJ0[i];
      if (nS >= 0) y += fN[lj * NI + i] * uAt(nS);
      if (j < NJ - 1) y += fN[(lj + 1) * NI + i] * uAt(c + NI);
      if (i > 0) y += fE[lj * (NI + 1) + i] * uAt(c - 1);
      if (i < NI - 1) y += fE[lj * (NI + 1) + i + 1] * uAt(c + 1);
      a[kSW0][m] = y;
      acc[0] += y * un;
    }
    teamReduce(t, sh, acc, op1);
    if (!(fabs(acc[0]) > 0.0)) {
      for (int c = t.c0 + t.tid; c < t.c1; c += t.T) I.x[c] = 0.0;
      t.cl.sync();
      return 0;
    }
    CgScalars k0;
    k0.alpha = gamma / acc[0];
    k0.gamma = gamma;
    int iterations = 0;
    int cur = 0;
    const int op3[3] = {kSum, kSum, kSum};
    CgScalars k = k0;
    for (int iter = 0; iter < I.cgMax; ++iter) {
      const int rC = cur ? kSR1 : kSR0, rN = cur ? kSR0 : kSR1;
      const int wC = cur ? kSW1 : kSW0, wN = cur ? kSW0 : kSW1;
      const int sC = cur ? kSS1 : kSS0, sN = cur ? kSS0 : kSS1;
      const double alpha = k.alpha, beta = k.beta;
      double sums[3] = {0.0, 0.0, 0.0};
      for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
        const int m = c - t.c0, i = c % NI, j = c / NI, lj = j - j0;
        // the next u of a cell from its r, w and s of this iteration
        auto uAt = [&](int n) {
          const double sn = at(wC, n) + beta * at(sC, n);
          return precondition(at(rC, n) - alpha * sn, at(kSD, n));
        };
        const double dg = a[kSD][m];
        const double pc = precondition(a[rC][m], dg) + beta * a[kSP][m];
        const double sc = a[wC][m] + beta * a[sC][m];
        a[kSX][m] += alpha * pc;
        const double rc = a[rC][m] - alpha * sc;
        const double un = precondition(rc, dg);
        double y = dg * un;
        const int nS = (j > 0) ? c - NI : I.acrossJ0[i];
        if (nS >= 0) y += fN[lj * NI + i] * uAt(nS);
        if (j < NJ - 1) y += fN[(lj + 1) * NI + i] * uAt(c + NI);
        if (i > 0) y += fE[lj * (NI + 1) + i] * uAt(c - 1);
        if (i < NI - 1) y += fE[lj * (NI + 1) + i + 1] * uAt(c + 1);
        a[kSP][m] = pc;
        a[sN][m] = sc;
        a[rN][m] = rc;
        a[wN][m] = y;
        sums[0] += rc * un;
        sums[1] += y * un;
        sums[2] += fabs(rc);
      }
      cur ^= 1;
      teamReduce(t, sh, sums, op3);
      iterations = iter + 1;
      if (!cgNext(I, k, sums, initial)) break;
    }
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) I.x[c] = a[kSX][c - t.c0];
    t.cl.sync();  // x visible to the correction; no peer still reads this band
    return iterations;
  }
}

/// The same single-reduction PCG with the vectors in global memory (bands
/// too large for shared memory): x, p, and r, w, s double-buffered as
/// (r, z), (q, d0), (d1, s1). Same arithmetic, cell order and reduction
/// order as cgShared, so both give the same bits.
DEV int cgGlobal(const Instance& I, Team& t, Shared& sh, double initial, double gamma) {
  const int NI = I.NI, NJ = I.NJ;
  double* rB[2] = {I.r, I.z};
  double* wB[2] = {I.q, I.d0};
  double* sB[2] = {I.d1, I.s1};
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    I.cgp[c] = 0.0;
    sB[0][c] = 0.0;
  }
  // w0 = A u0 (u0 from b, stable since the start's reduction)
  double acc[1] = {0.0};
  const int op1[1] = {kSum};
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % NI, j = c / NI;
    auto uAt = [&](int n) { return precondition(rB[0][n], I.pD[n]); };
    const double un = precondition(rB[0][c], I.pD[c]);
    double y = I.pD[c] * un;
    const int nS = (j > 0) ? c - NI : I.acrossJ0[i];
    if (nS >= 0) y += I.pN[j * NI + i] * uAt(nS);
    if (j < NJ - 1) y += I.pN[(j + 1) * NI + i] * uAt(c + NI);
    if (i > 0) y += I.pE[j * (NI + 1) + i] * uAt(c - 1);
    if (i < NI - 1) y += I.pE[j * (NI + 1) + i + 1] * uAt(c + 1);
    wB[0][c] = y;
    acc[0] += y * un;
  }
  teamReduce(t, sh, acc, op1);
  if (!(fabs(acc[0]) > 0.0)) return 0;
  CgScalars k;
  k.alpha = gamma / acc[0];
  k.gamma = gamma;
  int iterations = 0;
  int cur = 0;
  const int op3[3] = {kSum, kSum, kSum};
  // Restrict-qualified views: no store of the loop below can alias a load of
  // it, so the loads of the next cells may be issued ahead of the stores of
  // the current ones (the loop is latency-bound without that).
  const double* __restrict__ pD = I.pD;
  const double* __restrict__ pN = I.pN;
  const double* __restrict__ pE = I.pE;
  const int* __restrict__ wake = I.acrossJ0;
  double* __restrict__ xv = I.x;
  double* __restrict__ pv = I.cgp;
  for (int iter = 0; iter < I.cgMax; ++iter) {
    const double* __restrict__ r = rB[cur];
    const double* __restrict__ w = wB[cur];
    const double* __restrict__ sv = sB[cur];
    double* __restrict__ rn = rB[cur ^ 1];
    double* __restrict__ wn = wB[cur ^ 1];
    double* __restrict__ sn = sB[cur ^ 1];
    const double alpha = k.alpha, beta = k.beta;
    double sums[3] = {0.0, 0.0, 0.0};
    // the next u of a cell from its r, w and s of this iteration
    auto uAt = [&](int n) {
      const double s2 = w[n] + beta * sv[n];
      return precondition(r[n] - alpha * s2, pD[n]);
    };
#pragma unroll 2
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int i = c % NI, j = c / NI;
      const double dg = pD[c];
      const double pc = precondition(r[c], dg) + beta * pv[c];
      const double sc = w[c] + beta * sv[c];
      xv[c] += alpha * pc;
      const double rc = r[c] - alpha * sc;
      const double un = precondition(rc, dg);
      double y = dg * un;
      const int nS = (j > 0) ? c - NI : wake[i];
      if (nS >= 0) y += pN[j * NI + i] * uAt(nS);
      if (j < NJ - 1) y += pN[(j + 1) * NI + i] * uAt(c + NI);
      if (i > 0) y += pE[j * (NI + 1) + i] * uAt(c - 1);
      if (i < NI - 1) y += pE[j * (NI + 1) + i + 1] * uAt(c + 1);
      pv[c] = pc;
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
    if (!cgNext(I, k, sums, initial)) break;
  }
  return iterations;
}

/// Cells per software-pipeline group in cgGlobalSplit's passes.
constexpr int kCgPair = 2;

/// Shared memory of cgGlobalSplit, in doubles: the u of the two rows
/// bordering the band, pushed there by the neighbouring CTAs (2 x NI), and
/// the u of its own band (the largest band's cells). At 768x192 on 16 CTAs
/// this is 84 KB, inside the SM's 100 KB shared-memory carve-out, which
/// leaves the rest of the SM's 256 KB to the L1 cache: a larger carve-out
/// measured slower in every phase.
__host__ __device__ inline long long cgSplitSmemDoubles(int NI, int NJ, int R) {
  return 2LL * NI + cgSmemStride(NI, NJ, R);
}

/// The single-reduction PCG of cgGlobal in two passes per iteration, for
/// bands in global memory, with r, w and s held once. The first pass forms
/// each own cell's p, s, x, r and next u in place, keeps u in shared memory,
/// and pushes the u of the band's first and last rows into the halo of the
/// CTA below and above (st.async, completing that CTA's halo mbarrier); after
/// waiting for its own halo rows and a block barrier, the second pass forms
/// w' = A u'. A CTA's pushes for the next iteration follow the iteration's
/// reduction, which the receiver reaches only after its second pass, so one
/// halo buffer suffices. Each pass has few independent loads per cell, so
/// they overlap across cells; the one-pass form's neighbour recomputation
/// (four loads per neighbour, three vectors double-buffered) leaves it
/// latency-bound and 30 % larger in L2. The same expressions in the same cell
/// order as cgGlobal and cgShared, so the same bits. A halo wait that gives
/// up sets kFaultHaloWait in the launch's fault word and the solve carries
/// on without waiting again.
DEV int cgGlobalSplit(const Instance& I, Team& t, Shared& sh, double* dyn, double initial, double gamma,
                      bool waitTest) {
  const int NI = I.NI, NJ = I.NJ;
  const int R = static_cast<int>(t.R), rank = static_cast<int>(t.rank);
  const double* __restrict__ pD = I.pD;
  const double* __restrict__ pN = I.pN;
  const double* __restrict__ pE = I.pE;
  const int* __restrict__ wake = I.acrossJ0;
  double* __restrict__ xv = I.x;
  double* __restrict__ pv = I.cgp;
  double* __restrict__ rv = I.r;
  double* __restrict__ wv = I.q;
  double* __restrict__ sv = I.d1;
  // the u of the rows bordering the band, pushed here by the neighbouring
  // CTAs ([0, NI): row j0 - 1; [NI, 2 NI): row j1), then the band's own u
  double* halo = dyn;
  double* __restrict__ ub = dyn + 2 * NI;  // cell c at ub[c - c0]
  const int c0 = t.c0;
  // cells of this thread in the band: c0 + tid + k T, k < own
  const int own = (t.c1 - t.c0 > t.tid) ? (t.c1 - t.c0 - t.tid + t.T - 1) / t.T : 0;
  // (i, j) of this thread's first cell and of the band's last, and the step
  // between a thread's consecutive cells
  const int firstI = (t.c0 + t.tid) % NI, firstJ = (t.c0 + t.tid) / NI;
  const int lastI = (t.c1 - 1) % NI, lastJ = (t.c1 - 1) / NI;
  const int stepI = t.T % NI, stepJ = t.T / NI;
  const int j0 = t.c0 / NI, j1 = t.c1 / NI;
  // where this band's first row goes (the halo's upper half in the CTA
  // below) and its last row (the lower half in the CTA above), with their
  // barriers; 0 where there is no neighbour
  const bool hasBelow = rank > 0, hasAbove = rank < R - 1;
  const unsigned toBelow = hasBelow ? clusterAddr(smemAddr(halo + NI), rank - 1) : 0u;
  const unsigned toAbove = hasAbove ? clusterAddr(smemAddr(halo), rank + 1) : 0u;
  const unsigned belowBar = hasBelow ? clusterAddr(smemAddr(&sh.haloBar), rank - 1) : 0u;
  const unsigned aboveBar = hasAbove ? clusterAddr(smemAddr(&sh.haloBar), rank + 1) : 0u;
  const int lastRow = t.c1 - NI;  // first cell of the band's last row
  bool haloFaulted = false;
  // w0 = A u0 (u0 from b, stable since the start's reduction); p = s = 0
  double acc[1] = {0.0};
  const int op1[1] = {kSum};
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % NI, j = c / NI;
    auto uAt = [&](int n) { return precondition(rv[n], pD[n]); };
    const double un = precondition(rv[c], pD[c]);
    double y = pD[c] * un;
    const int nS = (j > 0) ? c - NI : wake[i];
    if (nS >= 0) y += pN[j * NI + i] * uAt(nS);
    if (j < NJ - 1) y += pN[(j + 1) * NI + i] * uAt(c + NI);
    if (i > 0) y += pE[j * (NI + 1) + i] * uAt(c - 1);
    if (i < NI - 1) y += pE[j * (NI + 1) + i + 1] * uAt(c + 1);
    acc[0] += y * un;
    wv[c] = y;
    pv[c] = 0.0;
    sv[c] = 0.0;
    ub[c - c0] = un;  // u0: pass 1 of the first iteration takes M^-1 r from here
  }
  teamReduce(t, sh, acc, op1);
  if (!(fabs(acc[0]) > 0.0)) return 0;
  CgScalars k;
  k.alpha = gamma / acc[0];
  k.gamma = gamma;
  int iterations = 0;
  const int op3[3] = {kSum, kSum, kSum};
  for (int iter = 0; iter < I.cgMax; ++iter) {
    const double alpha = k.alpha, beta = k.beta;
    double sums[3] = {0.0, 0.0, 0.0};
    // pass 1: own cells. Software-pipelined by hand: the next pair of cells'
    // loads are issued before this pair's arithmetic (the division's slow
    // path otherwise keeps the compiler from hoisting them), so two pairs of
    // loads are in flight per thread. Indices past the band are clamped to its
    // last cell and their values discarded; cells keep their order per thread.
    {
      double nD[kCgPair], nR[kCgPair], nP[kCgPair], nW[kCgPair], nS[kCgPair], nX[kCgPair];
      auto load = [&](int k, int u) {
        const int c = min(t.c0 + t.tid + k * t.T, t.c1 - 1);
        nD[u] = pD[c]; nR[u] = rv[c]; nP[u] = pv[c]; nW[u] = wv[c]; nS[u] = sv[c]; nX[u] = xv[c];
      };
#pragma unroll
      for (int u = 0; u < kCgPair; ++u) load(u, u);
      for (int k = 0; k < own; k += kCgPair) {
        double cD[kCgPair], cR[kCgPair], cP[kCgPair], cW[kCgPair], cS[kCgPair], cX[kCgPair];
#pragma unroll
        for (int u = 0; u < kCgPair; ++u) {
          cD[u] = nD[u]; cR[u] = nR[u]; cP[u] = nP[u]; cW[u] = nW[u]; cS[u] = nS[u]; cX[u] = nX[u];
        }
        if (k + kCgPair < own) {
#pragma unroll
          for (int u = 0; u < kCgPair; ++u) load(k + kCgPair + u, u);
        }
#pragma unroll
        for (int u = 0; u < kCgPair; ++u) {
          if (k + u >= own) break;
          const int c = t.c0 + t.tid + (k + u) * t.T;
          const double dg = cD[u];
          const double rc0 = cR[u];
          // M^-1 r of the previous iteration: the u this thread stored for
          // the cell then (the same operation on the same r, so the same bits)
          const double pc = ub[c - c0] + beta * cP[u];
          const double sc = cW[u] + beta * cS[u];
          xv[c] = cX[u] + alpha * pc;
          const double rc = rc0 - alpha * sc;
          const double un = precondition(rc, dg);
          pv[c] = pc;
          sv[c] = sc;
          rv[c] = rc;
          ub[c - c0] = un;
          // the band's first and last rows are the neighbours' halo rows
          if (hasBelow && c < c0 + NI) pushRemote(toBelow + 8u * static_cast<unsigned>(c - c0), un, belowBar);
          if (hasAbove && c >= lastRow) pushRemote(toAbove + 8u * static_cast<unsigned>(c - lastRow), un, aboveBar);
          sums[0] += rc * un;
          sums[2] += fabs(rc);
        }
      }
    }
    // the neighbours' rows of this iteration (pushed in their pass 1); then
    // the barrier is armed for the next iteration's, before this CTA can
    // reach the reduction after which the neighbours push them
    if (threadIdx.x == 0 && waitTest && iter == 0) {
      // test: the first iteration also waits for a count nothing sets
      long long spins = 0;
      while (loadRelaxedCluster(&sh.chainNever) == 0u && ++spins <= kChainSpinLimit) {
      }
      if (spins > kChainSpinLimit) atomicOr(I.iterations + 1, kFaultHaloWait);
    }
    if (threadIdx.x == 0) {
      long long spins = 0;
      while (!haloFaulted && !mbarDone(&sh.haloBar, sh.haloPhase & 1u)) {
        if (++spins > kChainSpinLimit) {
          atomicOr(I.iterations + 1, kFaultHaloWait);
          haloFaulted = true;
        }
      }
      if (!haloFaulted) {
        sh.haloPhase += 1u;
        mbarArm(&sh.haloBar, sh.haloBytes);
      }
    }
    __syncthreads();
    // pass 2: w' = A u'; the coefficient loads pipelined as in pass 1 (every
    // face index is in range for any cell, so they are loaded unconditionally).
    {
      // the cell of the next load as (i, j), stepped by T cells per load
      // (no integer division per cell); past the band, loads repeat its
      // last cell and their values are not used
      int li = firstI, lj = firstJ;
      double nD[kCgPair], nNs[kCgPair], nNn[kCgPair], nEw[kCgPair], nEe[kCgPair];
      int nI[kCgPair], nJ[kCgPair], nWk[kCgPair];
      auto load = [&](int kk, int u) {
        const bool in = kk < own;
        const int i = in ? li : lastI, j = in ? lj : lastJ;
        const int c = j * NI + i;
        nI[u] = i;
        nJ[u] = j;
        nD[u] = pD[c];
        nNs[u] = pN[c];           // face (i, j): south
        nNn[u] = pN[c + NI];      // face (i, j + 1): north
        nEw[u] = pE[c + j];       // face j (NI + 1) + i: west
        nEe[u] = pE[c + j + 1];   // east
        nWk[u] = (j == 0) ? wake[i] : -1;
        li += stepI;
        lj += stepJ;
        if (li >= NI) {
          li -= NI;
          lj += 1;
        }
      };
#pragma unroll
      for (int u = 0; u < kCgPair; ++u) load(u, u);
      for (int k = 0; k < own; k += kCgPair) {
        double cD[kCgPair], cNs[kCgPair], cNn[kCgPair], cEw[kCgPair], cEe[kCgPair];
        int cI[kCgPair], cJ[kCgPair], cWk[kCgPair];
#pragma unroll
        for (int u = 0; u < kCgPair; ++u) {
          cD[u] = nD[u]; cNs[u] = nNs[u]; cNn[u] = nNn[u]; cEw[u] = nEw[u]; cEe[u] = nEe[u];
          cI[u] = nI[u]; cJ[u] = nJ[u]; cWk[u] = nWk[u];
        }
        if (k + kCgPair < own) {
#pragma unroll
          for (int u = 0; u < kCgPair; ++u) load(k + kCgPair + u, u);
        }
#pragma unroll
        for (int u = 0; u < kCgPair; ++u) {
          if (k + u >= own) break;
          const int i = cI[u], j = cJ[u];
          const int c = j * NI + i;
          const int m = c - c0;
          const double un = ub[m];
          double y = cD[u] * un;
          if (j > 0) y += cNs[u] * ((j == j0) ? halo[i] : ub[m - NI]);
          else if (cWk[u] >= 0) y += cNs[u] * ub[cWk[u] - c0];
          if (j < NJ - 1) y += cNn[u] * ((j + 1 == j1) ? halo[NI + i] : ub[m + NI]);
          if (i > 0) y += cEw[u] * ub[m - 1];
          if (i < NI - 1) y += cEe[u] * ub[m + 1];
          wv[c] = y;
          sums[1] += y * un;
        }
      }
    }
    teamReduce(t, sh, sums, op3);
    iterations = iter + 1;
    if (!cgNext(I, k, sums, initial)) break;
  }
  return iterations;
}

/// The reference's two-reduction Jacobi-PCG with the vectors in global memory
/// (kernel flag bit 3; kept to compare with): the next direction d' = z +
/// beta d is formed redundantly for each neighbour from z and d, which are
/// both stable across the barrier, so A d' needs no extra exchange.
DEV int cgTwoReductions(const Instance& I, Team& t, Shared& sh, double initial, double rz) {
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const double zc = precondition(I.r[c], I.pD[c]);
    I.z[c] = zc;
    I.d0[c] = zc;
  }
  t.cl.sync();
  const int op2[2] = {kSum, kSum};
  int cgIters = 0;
  double* dCur = I.d0;
  double* dNext = I.d1;
  double beta = 0.0;
  for (int iter = 0; iter < I.cgMax; ++iter) {
    double dAd[1] = {0.0};
    const int opS[1] = {kSum};
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int i = c % I.NI, j = c / I.NI;
      double dc;
      if (iter == 0) {
        dc = dCur[c];
        I.q[c] = pressureRow(I, c, i, j, dCur, dc);
      } else {
        dc = I.z[c] + beta * dCur[c];
        dNext[c] = dc;
        double y = I.pD[c] * dc;
        int n = (j > 0) ? c - I.NI : I.acrossJ0[i];
        if (n >= 0) y += I.pN[j * I.NI + i] * (I.z[n] + beta * dCur[n]);
        if (j < I.NJ - 1) { n = c + I.NI; y += I.pN[(j + 1) * I.NI + i] * (I.z[n] + beta * dCur[n]); }
        if (i > 0) { n = c - 1; y += I.pE[j * (I.NI + 1) + i] * (I.z[n] + beta * dCur[n]); }
        if (i < I.NI - 1) { n = c + 1; y += I.pE[j * (I.NI + 1) + i + 1] * (I.z[n] + beta * dCur[n]); }
        I.q[c] = y;
      }
      dAd[0] += dc * I.q[c];
    }
    if (iter > 0) { double* tmp = dCur; dCur = dNext; dNext = tmp; }
    teamReduce(t, sh, dAd, opS);
    if (!(fabs(dAd[0]) > 0.0)) break;
    const double step = rz / dAd[0];
    double rr[2] = {0.0, 0.0};
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const double dc = dCur[c];
      I.x[c] += step * dc;
      const double rc = I.r[c] - step * I.q[c];
      I.r[c] = rc;
      const double zc = precondition(rc, I.pD[c]);
      I.z[c] = zc;
      rr[0] += fabs(rc);
      rr[1] += rc * zc;
    }
    teamReduce(t, sh, rr, op2);
    cgIters = iter + 1;
    if (rr[0] <= I.cgTol * initial) break;
    if (!(fabs(rz) > 0.0)) break;
    beta = rr[1] / rz;
    rz = rr[1];
  }
  return cgIters;
}

#include "pressure_mg.cuh"

}  // namespace

// ---- the kernel -----------------------------------------------------------------

/// Run `iterations` outer iterations (or fewer: `stopStage` ends the first
/// iteration early; `tolerance` >= 0 stops at convergence or divergence as
/// SolverWorker does, SolverWorker.cpp:164-185). One cluster per instance.
__global__ void __launch_bounds__(512, 1)
simpleKernel(const Instance* __restrict__ instances, int iterations, int stopStage, double tolerance,
             int smemBytes, int flags) {
  __shared__ Shared sh;
  extern __shared__ double dyn[];
  Team t{cg::this_cluster(), 0, 0, 0, 0, 0, 0, 0};
  t.rank = t.cl.block_rank();
  t.R = t.cl.num_blocks();
  t.tid = threadIdx.x;
  t.T = blockDim.x;
  const Instance& I = instances[blockIdx.x / t.R];
  // Each CTA owns a band of whole rows; the same split in every phase.
  t.c0 = I.NI * ((I.NJ * static_cast<int>(t.rank)) / static_cast<int>(t.R));
  t.c1 = I.NI * ((I.NJ * (static_cast<int>(t.rank) + 1)) / static_cast<int>(t.R));
  const bool sst = (I.model == 2);
  // With kernel flag bit 7 the pressure CG keeps its band in shared memory
  // when every band has a row and the largest band's arrays fit in what the
  // launch provides. By default it runs from global memory in two passes
  // (cgGlobalSplit), which measured faster on every benchmark grid (384x96
  // on 16 CTAs: 1.98 against 2.54 ms per iteration; 192x48: 1.08 against
  // 1.28 ms) and leaves most of the SM's shared memory to the L1 cache.
  const bool cgInShared = (flags & kFlagSharedCg) && !(flags & kFlagTwoReductionCg) &&
                          I.NJ >= static_cast<int>(t.R) &&
                          cgSmemDoubles(I.NI, I.NJ, static_cast<int>(t.R)) * 8 <= smemBytes;
  const bool leader = (t.rank == 0 && t.tid == 0);
  // Ordered before any peer's access by the first cluster barrier below.
  chainSetup(sh, static_cast<unsigned>(I.NI) * ((I.precision == 1) ? 4u : 8u),
             static_cast<unsigned>(I.NI) * 8u * ((t.rank > 0 ? 1u : 0u) + (t.rank + 1 < t.R ? 1u : 0u)));
  if (leader) I.iterations[1] = 0;

  int done = 0;
  const int limit = (I.iterLimit < iterations) ? I.iterLimit : iterations;
  const double stopTol = (tolerance >= 0.0) ? tolerance : I.stopTol;
  for (int it = 0; it < limit; ++it) {
    double mon[kMonSlots];
#pragma unroll
    for (int s = 0; s < kMonSlots; ++s) mon[s] = 0.0;

    // 1. face values and gradients; velocity scale.
    {
      double v1[1] = {0.0};
      const int op[1] = {kMax};
      phaseGradients(I, t, v1[0]);
      teamReduce(t, sh, v1, op);
      double scale = smax(0.0, v1[0]);
      if (!(scale > 0.0)) scale = 1.0;
      mon[kMonMomX] = scale;  // held until the residuals are known
    }
    if (stopStage == kStageGradients) { done = it + 1; break; }

    // 2. momentum assembly + relaxation + residuals (u and v together).
    {
      double v3[3] = {0.0, 0.0, 0.0};
      const int op[3] = {kSum, kSum, kSum};
      phaseMomentum(I, t, v3[0], v3[1], v3[2]);
      teamReduce(t, sh, v3, op);
      const double scale = v3[2] * mon[kMonMomX];
      mon[kMonMomX] = v3[0] / smax(scale, kTinySolver);
      mon[kMonMomY] = v3[1] / smax(scale, kTinySolver);
    }
    if (stopStage == kStageMomentumAssembly) { done = it + 1; break; }

    // 3. Gauss-Seidel sweeps, red-black, u and v together.
    for (int sweep = 0; sweep < I.sweeps && I.precision == 1; ++sweep) {
      for (int colour = 0; colour < 2; ++colour) {
        gsColourMixed(I, t, colour, sweep == I.sweeps - 1 && colour == 1);
        t.cl.sync();
      }
    }
    for (int sweep = 0; sweep < I.sweeps && I.precision == 0; ++sweep) {
      for (int colour = 0; colour < 2; ++colour) {
        gsColour(I, t, colour);
        t.cl.sync();
      }
    }
    if (stopStage == kStageMomentumSolve) { done = it + 1; break; }

    // 4. Rhie-Chow face fluxes.
    phaseRhieChow(I, t);
    t.cl.sync();
    if (stopStage == kStageRhieChow) { done = it + 1; break; }

    bool stopped = false;
    const int passes = (I.nCorr > 1) ? I.nCorr : 1;
    for (int pass = 0; pass < passes && !stopped; ++pass) {
      // 5. pressure-correction assembly; CG start (x = 0, r = b, d = z = M^-1 r).
      double v2[2] = {0.0, 0.0};
      const int op2[2] = {kSum, kSum};
      phasePressureAssembly(I, t, v2[0], v2[1]);
      teamReduce(t, sh, v2, op2);
      if (pass == 0) {
        mon[kMonMassImbalance] = v2[0];
        mon[kMonContinuity] = v2[0] / I.refMassFlow;
      }
      const double mean = I.hasPRef ? 0.0 : v2[1] / static_cast<double>(I.N);
      double init[2] = {0.0, 0.0};
      for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
        double b = I.pB[c];
        if (!I.hasPRef) { b -= mean; I.pB[c] = b; }
        I.x[c] = 0.0;
        I.r[c] = b;
        init[0] += fabs(b);
        init[1] += b * precondition(b, I.pD[c]);
      }
      teamReduce(t, sh, init, op2);
      if (stopStage == kStagePressureAssembly) { stopped = true; break; }

      // 6. the pressure correction: Jacobi-preconditioned CG (LinearSystem.cpp:
      // 118-210) with one reduction per iteration (cgShared / cgGlobal), or
      // the mixed form's multigrid CG.
      const double initial = init[0];
      const double rz = init[1];
      int cgIters = 0;
      if (initial > 0.0 && I.precision == 1) {
        cgIters = pressureMixed(I, t, sh, dyn, initial);
      } else if (initial > 0.0 && (flags & kFlagTwoReductionCg)) {
        cgIters = cgTwoReductions(I, t, sh, initial, rz);
      } else if (initial > 0.0 && cgInShared) {
        cgIters = cgShared(I, t, sh, dyn, initial, rz);
      } else if (initial > 0.0 && !(flags & kFlagOnePassCg) && I.NJ >= static_cast<int>(t.R) &&
                 cgSplitSmemDoubles(I.NI, I.NJ, static_cast<int>(t.R)) * 8 <= smemBytes) {
        cgIters = cgGlobalSplit(I, t, sh, dyn, initial, rz, (flags & kFlagHaloWaitTest) != 0);
      } else if (initial > 0.0) {
        cgIters = cgGlobal(I, t, sh, initial, rz);
      }
      mon[kMonPressureIterations] += static_cast<double>(cgIters);
      if (!I.hasPRef) {
        double sx[1] = {0.0};
        const int opS[1] = {kSum};
        for (int c = t.c0 + t.tid; c < t.c1; c += t.T) sx[0] += I.x[c];
        teamReduce(t, sh, sx, opS);
        const double m = sx[0] / static_cast<double>(I.N);
        for (int c = t.c0 + t.tid; c < t.c1; c += t.T) I.x[c] -= m;
        t.cl.sync();
      }
      if (stopStage == kStagePressureSolve) { stopped = true; break; }

      // 7. correct p, u, v and the face fluxes.
      phaseCorrect(I, t);
      t.cl.sync();
      if (stopStage == kStageCorrect) { stopped = true; break; }
    }
    if (stopped) {
      if (leader) {
        for (int s = 0; s < kMonSlots; ++s) I.history[it * kMonSlots + s] = mon[s];
      }
      done = it + 1;
      break;
    }

    // 8. divergence (+ SST strain, gradients of k and omega, blending, production).
    if (sst) {
      double v1[1] = {0.0};
      const int op[1] = {kMax};
      phaseSstBlending(I, t, v1[0]);
      teamReduce(t, sh, v1, op);
      mon[kMonMaxDivergence] = smax(0.0, v1[0]);
      if (stopStage == kStageSstBlending) { done = it + 1; break; }

      double a4[4] = {0.0, 0.0, 0.0, 0.0};
      const int op4[4] = {kSum, kSum, kSum, kSum};
      phaseSstAssembly(I, t, a4);
      teamReduce(t, sh, a4, op4);
      mon[kMonTurbFirst] = a4[0] / smax(a4[1] * smax(I.kIn, kTinySst), kTinySst);
      mon[kMonTurbSecond] = a4[2] / smax(a4[3] * smax(I.wIn, kTinySst), kTinySst);
      if (stopStage == kStageSstAssembly) { done = it + 1; break; }

      // k and omega sweep in the reference's cell order: their floors and
      // the wall-cell omega override act after the sweeps, so the converged
      // state depends on the order (a colouring would move it by ~1e-3).
      const bool chained = t.R >= 6 && !(flags & (kFlagSequentialRows | kFlagBarrierSweeps));
      const unsigned chainBase = static_cast<unsigned>(it) * static_cast<unsigned>(I.NJ);
      const bool waitTest = (flags & kFlagChainWaitTest) != 0;
      if (!(flags & kFlagPlainWavefront) && I.NI <= 8 * t.T &&
          (2 * I.NI + 64) * 8 <= smemBytes) {
        if (I.precision == 1) {
          // mixed form: the same sweep map on the FP32 corrections
          float* fs = reinterpret_cast<float*>(dyn);
          const SysView<float> ks = correctionSystem(I.tk), ws = correctionSystem(I.tw);
          if (chained && chainSmemElems(I.NI) * 4 <= smemBytes) {
            gsRowScanChained(I, t, sh, 3, ks, ws, fs, chainBase, waitTest);
          } else if (t.R >= 6 && !(flags & kFlagSequentialRows)) {
            gsRowScanPipelined(I, t, 3, ks, ws, fs);
          } else if (t.R == 1) {
            gsRowScanSweeps(I, 3, ks, fs);
            gsRowScanSweeps(I, 3, ws, fs);
          } else if (t.rank == 0) {
            gsRowScanSweeps(I, 3, ks, fs);
          } else if (t.rank == 1) {
            gsRowScanSweeps(I, 3, ws, fs);
          }
        } else if (chained && chainSmemElems(I.NI) * 8 <= smemBytes) {
          gsRowScanChained(I, t, sh, 3, kSystem(I), omegaSystem(I), dyn, chainBase, waitTest);
        } else if (t.R >= 6 && !(flags & kFlagSequentialRows)) {
          gsRowScanPipelined(I, t, 3, kSystem(I), omegaSystem(I), dyn);
        } else if (t.R == 1) {
          // one CTA: k, then omega
          gsRowScanSweeps(I, 3, kSystem(I), dyn);
          gsRowScanSweeps(I, 3, omegaSystem(I), dyn);
        } else if (t.rank == 0) {
          // rank 0 sweeps k, rank 1 omega
          gsRowScanSweeps(I, 3, kSystem(I), dyn);
        } else if (t.rank == 1) {
          gsRowScanSweeps(I, 3, omegaSystem(I), dyn);
        }
      } else {
        gsWavefrontSweeps(I, t, 3, I.kD, I.kS, I.kN, I.kW, I.kE, I.kB, I.k, I.wD, I.wS, I.wN,
                          I.wW, I.wE, I.wB, I.om);
      }
      t.cl.sync();
      if (stopStage == kStageSstSolve) { done = it + 1; break; }

      double m8[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) m8[s] = -INFINITY;
      m8[5] = 0.0;
      m8[7] = 0.0;
      const int op8[8] = {kMax, kMax, kMax, kMax, kMax, kMax, kMax, kMax};
      phaseSstFinish(I, t, m8);
      teamReduce(t, sh, m8, op8);
      mon[kMonMaxK] = m8[0]; mon[kMonMinK] = -m8[1];
      mon[kMonMaxW] = m8[2]; mon[kMonMinW] = -m8[3];
      mon[kMonMaxMut] = m8[4]; mon[kMonMinMut] = -m8[6];
      mon[kMonMaxYPlus] = m8[5];
      mon[kMonMaxRatio] = m8[7];
    } else {
      double v1[1] = {0.0};
      const int op[1] = {kMax};
      for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
        v1[0] = smax(v1[0], fabs(cellDivergence(I, c, c % I.NI, c / I.NI)));
      }
      teamReduce(t, sh, v1, op);
      mon[kMonMaxDivergence] = smax(0.0, v1[0]);
    }

    if (leader) {
      for (int s = 0; s < kMonSlots; ++s) I.history[it * kMonSlots + s] = mon[s];
    }
    done = it + 1;
    if (stopTol >= 0.0) {
      const double a = mon[kMonContinuity], b = mon[kMonMomX], cc = mon[kMonMomY];
      if (!isfinite(a) || !isfinite(b) || !isfinite(cc)) break;
      if (smax(smax(fabs(a), fabs(b)), fabs(cc)) < stopTol) break;
    }
  }
  if (leader) *I.iterations = done;
  // No CTA may exit while a peer can still read its shared memory.
  t.cl.sync();
}

/// Brute-force distance from each cell centroid to the nearest no-slip wall
/// face centre (TurbulenceModel.cpp:28-65). One thread per cell.
__global__ void wallDistanceKernel(int n, const double* __restrict__ centroid,
                                   int walls, const double* __restrict__ wallCentre,
                                   double far, double* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (walls == 0) {
    out[c] = far;
    return;
  }
  const double cx = centroid[2 * c], cy = centroid[2 * c + 1];
  double best = 1.7976931348623157e308;
  for (int w = 0; w < walls; ++w) {
    const double dx = cx - wallCentre[2 * w];
    const double dy = cy - wallCentre[2 * w + 1];
    const double sq = dx * dx + dy * dy;
    best = smin(best, sq);
  }
  out[c] = sqrt(best);
}

}  // namespace cfdb

// ---- launch helpers ---------------------------------------------------------------

namespace cfdb {

int chooseClusterSize(int cells) {
  // About four cells per thread at 512 threads per CTA before another CTA is
  // added; 16 is the largest (non-portable) cluster.
  int r = 1;
  while (r < 16 && cells > r * 512 * 4) r *= 2;
  return r;
}

int kernelFlags() {
  // Implementation choices for tuning comparisons: bit 7 keeps the pressure
  // CG's band in shared memory where it fits (bit 0, global memory, is the
  // default now), bit 1 uses the plain wavefront sweeps, bit 2 runs
  // the k/omega row sweeps one after another instead of pipelined across
  // CTAs, bit 4 runs the global-memory CG in one pass per iteration
  // instead of two, bit 5 pipelines the k/omega row sweeps with a cluster
  // barrier per row instead of chaining them through DSMEM (these five give
  // identical results); bit 3 runs the reference's two-reduction CG instead
  // of the single-reduction one (the same to rounding). Bit 6 is for tests:
  // a chained k/omega stage also waits for a count that nothing sets, so
  // that wait gives up and the launch reports its fault word; bit 8 does the
  // same for the two-pass pressure CG's halo wait.
  const char* env = std::getenv("CFD_KERNEL_FLAGS");
  return (env != nullptr) ? std::atoi(env) : 0;
}

int chainSweepBytes(int NI, int elemBytes) { return static_cast<int>(chainSmemElems(NI) * elemBytes); }

int cgSharedBytes(int NI, int NJ, int clusterSize) {
  // The chained k/omega row sweeps keep two rows, the scan's warp totals and
  // a ring of rows; the pressure CG the exported boundary rows and the
  // band's u of the two-pass global-memory form, or with kernel flag bit 7
  // its whole band (cgShared) where that fits.
  const long long wave = chainSmemElems(NI) * 8;
  long long bytes = 0;
  if (NJ >= clusterSize && (kernelFlags() & kFlagSharedCg)) bytes = cgSmemDoubles(NI, NJ, clusterSize) * 8;
  if (bytes > kMaxCgSharedBytes) bytes = 0;
  if (bytes == 0 && NJ >= clusterSize && cgSplitSmemDoubles(NI, NJ, clusterSize) * 8 <= kMaxCgSharedBytes) {
    bytes = cgSplitSmemDoubles(NI, NJ, clusterSize) * 8;
  }
  if (bytes < wave && wave <= kMaxCgSharedBytes) bytes = wave;
  return static_cast<int>(bytes);
}

namespace {

PerDeviceOnce g_simpleKernelConfigured;

/// The non-portable cluster size (16) and the dynamic shared-memory limit
/// are attributes of the kernel on each device: set them on every device
/// this process launches on.
Status configureSimpleKernel() {
  return g_simpleKernelConfigured.run([]() -> Status {
    cudaError_t e = cudaFuncSetAttribute(simpleKernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) {
      e = cudaFuncSetAttribute(simpleKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxCgSharedBytes);
    }
    if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
    return ok();
  });
}

}  // namespace

Status prepareSimpleKernel() { return configureSimpleKernel(); }

int maxActiveClusters(int clusterSize, int threads, int smemBytes) {
  if (configureSimpleKernel() != CFD_OK) return 0;
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(static_cast<unsigned>(clusterSize * 64), 1, 1);
  config.blockDim = dim3(static_cast<unsigned>(threads), 1, 1);
  config.dynamicSmemBytes = static_cast<size_t>(smemBytes);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(clusterSize);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  config.attrs = attr;
  config.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, simpleKernel, &config) != cudaSuccess) return 0;
  return clusters;
}

Status launchSimple(const Instance* dInstances, int count, int clusterSize, int threads,
                    int iterations, int stopStage, double tolerance, cudaStream_t stream,
                    int smemBytes) {
  if (Status st = configureSimpleKernel(); st != CFD_OK) return st;
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(static_cast<unsigned>(count * clusterSize), 1, 1);
  config.blockDim = dim3(static_cast<unsigned>(threads), 1, 1);
  config.dynamicSmemBytes = static_cast<size_t>(smemBytes);
  config.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(clusterSize);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  config.attrs = attr;
  config.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&config, simpleKernel, dInstances, iterations, stopStage, tolerance,
                                     smemBytes, kernelFlags());
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, std::string("SIMPLE kernel launch: ") + cudaGetErrorString(e));
  return CFD_OK;
}

Status launchWallDistance(int n, const double* centroid, int walls, const double* wallCentre,
                          double far, double* out, cudaStream_t stream) {
  const int block = 256;
  wallDistanceKernel<<<(n + block - 1) / block, block, 0, stream>>>(n, centroid, walls, wallCentre, far, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CFD_INITIALIZATION_FAILURE, cudaGetErrorString(e));
  return CFD_OK;
}

}  // namespace cfdb
