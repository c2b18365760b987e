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
constexpr int kFlagGlobalCg = 1;    // the default now; kept so the flag value stays accepted
constexpr int kFlagPlainWavefront = 2;
constexpr int kFlagSequentialRows = 4;
constexpr int kFlagTwoReductionCg = 8;
constexpr int kFlagOnePassCg = 16;
constexpr int kFlagBarrierSweeps = 32;
constexpr int kFlagSharedCg = 128;  // the pressure CG's band in shared memory where it fits
constexpr int kFlagChainWaitTest = 64;  // tests only: a chained stage also waits for a count nothing sets
constexpr int kFlagHaloWaitTest = 256;  // tests only: the split CG also waits once for a count nothing sets

// Fault codes a launch leaves in iterations[1] (bits, or-ed together).
constexpr int kFaultChainWait = 1;  // a chained k/omega sweep stage gave up waiting for its neighbour
constexpr int kFaultHaloWait = 2;   // the pressure CG gave up waiting for a neighbour's halo row

// Layout of one monitor record (cfd_monitor), in doubles.
enum MonitorSlot : int {
  kMonContinuity = 0, kMonMomX, kMonMomY, kMonMassImbalance, kMonMaxDivergence,
  kMonPressureIterations, kMonTurbFirst, kMonTurbSecond, kMonMinK, kMonMaxK, kMonMinW,
  kMonMaxW, kMonMinMut, kMonMaxMut, kMonMaxRatio, kMonMaxYPlus, kMonSlots
};

// ---- mixed form: the pressure-correction multigrid -----------------------------

constexpr int kMaxMgLevels = 12;

/// One level of the pressure-correction multigrid: a cellsI x cellsJ block
/// with a five-point row per cell, cell c = j*NI + i as on the fine grid.
/// Level l+1 aggregates 2 x 2 cells of level l (the top row alone when NJ is
/// odd) and its rows are the Galerkin sums of the fine rows. The wake cut
/// carries over: on every level column i at j = 0 couples to wake[i].
struct MgLevel {
  int NI, NJ;
  float *D, *S, *N, *W, *E;  // row coefficients (global memory)
  float* inv;                // 1 / D (0 where D = 0)
  float *x, *b;              // iterate and right-hand side (global memory)
  const int* wake;           // partner column across j = 0, or -1
  int smem;                  // byte offset of the level in shared memory when rank 0 runs it alone
  int smemWake;              // byte offset of its wake map there
};

struct Multigrid {
  int levels;       // >= 1
  int distributed;  // levels 0 .. distributed-1 are split over the cluster in row bands
  int warpFrom;     // levels warpFrom .. levels-1 (64 cells or fewer) run on rank 0's warp 0
  int pre, post, coarse;  // Gauss-Seidel sweeps (red-black) per level and on the coarsest
  int smemBytes;    // shared memory of the levels rank 0 runs alone
  MgLevel lv[kMaxMgLevels];
  // inner flexible-CG vectors, FP32, fine-grid layout
  float *r, *q, *e, *z0, *z1, *d0, *d1;
};

/// FP32 rows of one system in correction form, A delta = r: the mixed form
/// sweeps delta in FP32 from zero and adds it to the FP64 unknowns.
struct Rows32 {
  float *D, *S, *N, *W, *E;  // row coefficients
  float *r, *x;              // residual b - A phi (from FP64) and the correction
};

struct Instance {
  int NI, NJ, N;
  int model;  // 0 none, 1 laminar closure, 2 k-omega SST
  int precision;  // 0 plain FP64, 1 mixed FP32/FP64
  int mgCap;      // mixed form: multigrid-CG iterations per pressure correction

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
  // pressure correction; the single-reduction CG double-buffers r in (r, z),
  // w = A u in (q, d0) and s = A p in (d1, s1), with the direction in cgp
  double *pD, *pN, *pE, *pB, *net;
  double *x, *r, *z, *q, *d0, *d1, *s1, *cgp;
  double* div;

  // ---- SST ----
  double *k, *om, *mut, *strain, *f1, *f2, *cd, *prod, *gkx, *gky, *gwx, *gwy;
  double *kD, *kS, *kN, *kW, *kE, *kB;
  double *wD, *wS, *wN, *wW, *wE, *wB;

  // ---- outputs ----
  double* history;   // kMonSlots doubles per iteration of the launch
  int* iterations;   // iterations completed by the launch, then the launch's fault
                     // word (iterations[1]: nonzero when a bounded wait gave up)

  // ---- mixed form ----
  Multigrid mg;
  Rows32 mom;          // momentum rows (shared by u and v); r, x belong to u
  float *momRv, *momXv;  // v's residual and correction
  Rows32 tk, tw;       // k and omega

  // ---- per-solve limits of a launch (batches and the engine) ----
  double stopTol;    // convergence tolerance when the launch gives none (< 0: none)
  int iterLimit;     // at most this many iterations in a launch
};

}  // namespace cfdb
