// instance.hpp - the device-side descriptor of one SIMPLE solve.
//
// One solve ("instance") is a structured block of NI x NJ cells, cell
// c = j*NI + i. Every field lives in HBM as structure-of-arrays over c.
// Face fields come in two families laid out so a warp reads them along i:
//   N-faces (the reference's j-faces, Mesh.cpp:138-151): index j*NI + i,
//            j = 0..NJ; face (i, j) is the south face of cell (i, j) and the
//            north face of cell (i, j-1). Same index as the reference.
//   E-faces (the reference's i-faces, Mesh.cpp:153-170): index j*(NI+1) + i,
//            i = 0..NI; face (i, j) is the west face of cell (i, j) and the
//            east face of cell (i-1, j). The reference numbers these
//            offset + i*NJ + j; the host permutes on the way in and out.
// The wake cut is a map acrossJ0[i]: the cell on the far side of the j = 0
// face of column i, or -1 (Mesh.cpp:78-87 oppositeCell).
//
// Matrices are stored by row: diag plus one coefficient per neighbour (S, N,
// W, E), so a row is read with five coalesced loads. The symmetric pressure-
// correction matrix is stored per face instead (pN, pE), one coefficient for
// both rows, which is what its CG inner loop streams.
#pragma once

#include <cstdint>

namespace cfdb {

struct FaceGeo {
  const double* Sx;  // area vector S = n * |f|, out of the owner
  const double* Sy;
  const double* D;   // |S|^2 / (S.d), over-relaxed orthogonal factor (0 if degenerate)
  const double* Tx;  // T = S - d * D
  const double* Ty;
  const double* w;   // interpolation weight of the owner
  const double* Dt;  // |geometric| as the SST transport forms it (1e-30 guard)
  const double* nx;  // unit normal (wall faces: y+ only)
  const double* ny;
};

// Stop points (cfd_gpu.h CFD_STAGE_*), repeated here for device code.
enum Stage : int {
  kStageGradients = 0,
  kStageMomentumAssembly,
  kStageMomentumSolve,
  kStageRhieChow,
  kStagePressureAssembly,
  kStagePressureSolve,
  kStageCorrect,
  kStageSstBlending,
  kStageSstAssembly,
  kStageSstSolve,
  kStageEnd
};

// Kernel implementation flags (bit mask).
constexpr int kFlagGlobalCg = 1;
constexpr int kFlagPlainWavefront = 2;
constexpr int kFlagSequentialRows = 4;

// Layout of one monitor record (cfd_monitor), in doubles.
enum MonitorSlot : int {
  kMonContinuity = 0, kMonMomX, kMonMomY, kMonMassImbalance, kMonMaxDivergence,
  kMonPressureIterations, kMonTurbFirst, kMonTurbSecond, kMonMinK, kMonMaxK, kMonMinW,
  kMonMaxW, kMonMinMut, kMonMaxMut, kMonMaxRatio, kMonMaxYPlus, kMonSlots
};

struct Instance {
  int NI, NJ, N;
  int model;  // 0 none, 1 laminar closure, 2 k-omega SST

  // ---- settings (SimpleSettings) ----
  double alphaU, alphaP, blend, alphaT;
  int sweeps, cgMax, sou, nCorr;
  double cgTol;
  int hasPRef;
  double refMassFlow;
  // SST constants (SSTConstants, KOmegaSST.hpp:147-171) and freestream
  double kIn, wIn, gamma1, gamma2, betaStarQuarter;

  // ---- geometry (read-only during a launch) ----
  const double* vol;
  FaceGeo gN, gE;
  const int* acrossJ0;
  const int8_t* kindN;
  const int8_t* kindE;
  const double *bcuN, *bcvN, *bcpN, *bcuE, *bcvE, *bcpE;
  const double *deadN, *deadE;
  const double* wallDist;
  const uint8_t* wallMask;  // bit 0 S, 1 N, 2 W, 3 E: that face is a no-slip wall owned by the cell

  // ---- flow state ----
  double *u, *v, *p, *rho, *mu, *muMol;
  double *mfN, *mfE;
  double *gux, *guy, *gvx, *gvy, *gpx, *gpy;
  // momentum system (shared by u and v), relaxed; aD doubles as momentumDiagonal
  double *aD, *aS, *aN, *aW, *aE, *bU, *bV;
  // pressure correction
  double *pD, *pN, *pE, *pB, *net;
  double *x, *r, *z, *q, *d0, *d1;
  double* div;

  // ---- SST ----
  double *k, *om, *mut, *strain, *f1, *f2, *cd, *prod, *gkx, *gky, *gwx, *gwy;
  double *kD, *kS, *kN, *kW, *kE, *kB;
  double *wD, *wS, *wN, *wW, *wE, *wB;

  // ---- outputs ----
  double* history;   // kMonSlots doubles per iteration of the launch
  int* iterations;   // iterations completed by the launch

  // ---- per-solve limits of a launch (batches and the engine) ----
  double stopTol;    // convergence tolerance when the launch gives none (< 0: none)
  int iterLimit;     // at most this many iterations in a launch
};

}  // namespace cfdb
