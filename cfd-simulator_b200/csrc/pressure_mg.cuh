// pressure_mg.cuh - the mixed form's pressure-correction solve (included by
// simple_kernel.cu inside its anonymous namespace).
//
// The plain form runs the reference's Jacobi-PCG (LinearSystem.cpp:118-210)
// and, at its cap of 200 iterations, reduces the L1 residual of the p'
// system by only ~2.5x on a 384x96 C-grid (it would need ~1000 iterations
// for the reference's 1% target). The mixed form solves the same system to
// the same stopping rule (sum |r| <= tol * sum |r0|) with a stronger inner
// solver, at most `mgCap` iterations (the settings' inner_iterations):
//
//   outer (FP64):  x = 0, r = b;  repeat: inner solve A e = r in FP32,
//                  x += e, r = b - A x (FP64 rows), stop on the L1 rule.
//   inner (FP32):  flexible CG (Polak-Ribiere beta, dot products and norms
//                  accumulated in FP64) preconditioned by one multigrid
//                  V-cycle per iteration.
//   V-cycle:       2x2 aggregation with Galerkin rows, so every level is a
//                  five-point block with the wake-cut map carried over;
//                  red-black Gauss-Seidel (red then black going down, black
//                  then red coming up, so the cycle is symmetric); the
//                  fine levels are split over the cluster in row bands with a
//                  cluster barrier per half sweep, the coarse levels (a few
//                  thousand cells) run on rank 0 alone from shared memory
//                  with __syncthreads only, and the last few (64 cells or
//                  fewer) on its warp 0 with __syncwarp.
//
// Fusions that save barriers: the red half sweep of a level from a zero
// start is x = b / D and is written by whatever phase produced b; the
// prolongation is folded into the first post-smoothing half sweep (a black
// cell needs only its red neighbours' corrected values, and every red value
// is recomputed by the following red half sweep); the last red half sweep on
// the fine level is fused with the CG's reduction.

/// A level as the code sees it: coefficient and vector pointers in global or
/// shared memory.
struct Lv {
  int NI, NJ;
  float *D, *S, *N, *W, *E, *inv, *x, *b;
  const int* wake;
};

/// The rows [j0, j1) of a level that one worker set covers: a row band of
/// the cluster, all of a level for the CTA that runs it alone, or all of it
/// for one warp.
struct Span {
  int j0, j1, tid, T;
};

DEV Lv globalLevel(const MgLevel& M) {
  return Lv{M.NI, M.NJ, M.D, M.S, M.N, M.W, M.E, M.inv, M.x, M.b, M.wake};
}

/// Eight arrays of the level in shared memory from byte offset M.smem, each
/// rounded up to 4 floats, and its wake map from M.smemWake.
DEV Lv sharedLevel(const MgLevel& M, char* smem) {
  float* p = reinterpret_cast<float*>(smem + M.smem);
  const int n = (M.NI * M.NJ + 3) & ~3;
  return Lv{M.NI, M.NJ, p, p + n, p + 2 * n, p + 3 * n, p + 4 * n, p + 5 * n, p + 6 * n, p + 7 * n,
            reinterpret_cast<const int*>(smem + M.smemWake)};
}

DEV Lv levelView(const Multigrid& G, int l, char* smem) {
  const MgLevel& M = G.lv[l];
  return (l < G.distributed) ? globalLevel(M) : sharedLevel(M, smem);
}

DEV Span bandOf(const Lv& L, const Team& t) {
  const int R = static_cast<int>(t.R), r = static_cast<int>(t.rank);
  return Span{(L.NJ * r) / R, (L.NJ * (r + 1)) / R, t.tid, t.T};
}
DEV Span wholeOf(const Lv& L) { return Span{0, L.NJ, static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)}; }
DEV Span warpOf(const Lv& L) { return Span{0, L.NJ, static_cast<int>(threadIdx.x & 31), 32}; }

/// f(c, i, j) for every cell of the span.
template <typename F>
DEV void forCells(const Lv& L, const Span& s, F&& f) {
  const int count = (s.j1 - s.j0) * L.NI;
  for (int m = s.tid; m < count; m += s.T) {
    const int jj = m / L.NI;
    const int i = m - jj * L.NI, j = s.j0 + jj;
    f(j * L.NI + i, i, j);
  }
}

/// Neighbour indices of cell (i, j) for branch-free row products: a missing
/// neighbour is replaced by the cell itself, whose coefficient on that side
/// is zero on every level (the fine rows are built that way and the Galerkin
/// sums only ever add existing couplings), so every load can be issued
/// unconditionally and together.
struct Nbrs {
  int s, n, w, e;
};
DEV Nbrs neighbours(const int* wake, int NI, int NJ, int c, int i, int j) {
  const int a = wake[i];
  Nbrs q;
  q.s = (j > 0) ? c - NI : ((a >= 0) ? a : c);
  q.n = (j < NJ - 1) ? c + NI : c;
  q.w = (i > 0) ? c - 1 : c;
  q.e = (i < NI - 1) ? c + 1 : c;
  return q;
}

/// Off-diagonal part of row c applied to x (S, N, W, E).
DEV float offSum(const Lv& L, const float* x, int c, int i, int j) {
  const Nbrs q = neighbours(L.wake, L.NI, L.NJ, c, i, j);
  return L.S[c] * x[q.s] + L.N[c] * x[q.n] + L.W[c] * x[q.w] + L.E[c] * x[q.e];
}

/// The same with every neighbour's value corrected by its aggregate's value
/// on the next coarser level (piecewise-constant prolongation). The
/// aggregates follow from (i, j) directly; a missing neighbour (the cell
/// itself, zero coefficient) uses the cell's own aggregate.
DEV float offSumProlonged(const Lv& L, const float* ec, int NIc, int c, int i, int j) {
  const Nbrs q = neighbours(L.wake, L.NI, L.NJ, c, i, j);
  const int own = (j >> 1) * NIc + (i >> 1);
  const int a = L.wake[i];
  const int gS = (j > 0) ? ((j - 1) >> 1) * NIc + (i >> 1) : ((a >= 0) ? (a >> 1) : own);
  const int gN = (j < L.NJ - 1) ? ((j + 1) >> 1) * NIc + (i >> 1) : own;
  const int gW = (i > 0) ? (j >> 1) * NIc + ((i - 1) >> 1) : own;
  const int gE = (i < L.NI - 1) ? (j >> 1) * NIc + ((i + 1) >> 1) : own;
  return L.S[c] * (L.x[q.s] + ec[gS]) + L.N[c] * (L.x[q.n] + ec[gN]) +
         L.W[c] * (L.x[q.w] + ec[gW]) + L.E[c] * (L.x[q.e] + ec[gE]);
}

/// Gauss-Seidel half sweep over the cells of one colour. The new values are
/// written through a pointer declared not to alias the one the neighbours
/// are read through (they never touch the same cells: a colour's neighbours
/// are all of the other colour), so consecutive cells' loads can overlap.
template <bool kProlonged>
DEV void sweepCells(const Lv& L, const Span& s, int colour, const float* ec, int NIc) {
  const int rows = s.j1 - s.j0;
  if ((L.NI & 1) != 0) {
    // the coarsest level may have an odd width: plain loop
    forCells(L, s, [&](int c, int i, int j) {
      if (((i + j) & 1) != colour) return;
      const float off = kProlonged ? offSumProlonged(L, ec, NIc, c, i, j) : offSum(L, L.x, c, i, j);
      L.x[c] = (L.b[c] - off) * L.inv[c];
    });
    return;
  }
  const int half = L.NI >> 1;
  const int count = rows * half;
  auto cellOf = [&](int m, int& c, int& i, int& j) {
    const int jj = m / half;
    j = s.j0 + jj;
    i = 2 * (m - jj * half) + ((colour + j) & 1);
    c = j * L.NI + i;
  };
  auto value = [&](int c, int i, int j) {
    const float off = kProlonged ? offSumProlonged(L, ec, NIc, c, i, j) : offSum(L, L.x, c, i, j);
    return (L.b[c] - off) * L.inv[c];
  };
  // two cells per step, both computed before either is stored, so their
  // loads overlap (a store to x could alias the other cell's loads)
  for (int m = s.tid; m < count; m += 2 * s.T) {
    int cA, iA, jA;
    cellOf(m, cA, iA, jA);
    const float vA = value(cA, iA, jA);
    const int mB = m + s.T;
    if (mB < count) {
      int cB, iB, jB;
      cellOf(mB, cB, iB, jB);
      const float vB = value(cB, iB, jB);
      L.x[cA] = vA;
      L.x[cB] = vB;
    } else {
      L.x[cA] = vA;
    }
  }
}

DEV void colourSweep(const Lv& L, const Span& s, int colour) { sweepCells<false>(L, s, colour, nullptr, 0); }

/// The black half sweep that opens post-smoothing, with the coarse
/// correction ec (level above, NIc columns) added to the neighbours on the fly.
DEV void colourSweepProlonged(const Lv& L, const Span& s, const float* ec, int NIc) {
  sweepCells<true>(L, s, 1, ec, NIc);
}

/// Sum of the fine residual b - A x over the aggregate of coarse cell (I, J).
DEV float aggregateResidual(const Lv& F, int I, int J) {
  float sum = 0.0f;
  for (int bj = 0; bj < 2; ++bj) {
    const int jf = 2 * J + bj;
    if (jf >= F.NJ) break;
#pragma unroll
    for (int ai = 0; ai < 2; ++ai) {
      const int fi = 2 * I + ai, f = jf * F.NI + fi;
      sum += F.b[f] - F.D[f] * F.x[f] - offSum(F, F.x, f, fi, jf);
    }
  }
  return sum;
}

/// Restrict the fine residual b - A x to the coarse right-hand side (sum over
/// each aggregate). With `start`, also begin the coarse level: red cells
/// b / D, black 0.
template <bool kStart>
DEV void restrictCells(const Lv& F, const Lv& C, const Span& s) {
  float* __restrict__ bw = C.b;
  float* __restrict__ xw = C.x;
  const int count = (s.j1 - s.j0) * C.NI;
#pragma unroll 2
  for (int m = s.tid; m < count; m += s.T) {
    const int jj = m / C.NI;
    const int I = m - jj * C.NI, J = s.j0 + jj;
    const int cc = J * C.NI + I;
    const float val = aggregateResidual(F, I, J);
    bw[cc] = val;
    if (kStart) xw[cc] = (((I + J) & 1) == 0) ? val * C.inv[cc] : 0.0f;
  }
}

DEV void restrictInto(const Lv& F, const Lv& C, const Span& s) { restrictCells<true>(F, C, s); }

/// Galerkin rows of the coarse level: P^T A P with P the 2x2 aggregation.
/// Couplings inside an aggregate join the diagonal; the others are summed
/// per side. Row 0's S couplings cross the wake cut to the partner aggregate.
DEV void galerkin(const Lv& F, const Lv& C, const Span& s) {
  forCells(C, s, [&](int cc, int I, int J) {
    float D = 0.0f, S = 0.0f, N = 0.0f, W = 0.0f, E = 0.0f;
    for (int bj = 0; bj < 2; ++bj) {
      const int jf = 2 * J + bj;
      if (jf >= F.NJ) break;
#pragma unroll
      for (int ai = 0; ai < 2; ++ai) {
        const int fi = 2 * I + ai, f = jf * F.NI + fi;
        D += F.D[f];
        if (jf > 0) {
          if (bj == 1) D += F.S[f]; else S += F.S[f];
        } else if (F.wake[fi] >= 0) {
          S += F.S[f];
        }
        if (jf < F.NJ - 1) {
          if (bj == 0) D += F.N[f]; else N += F.N[f];
        }
        if (fi > 0) {
          if (ai == 1) D += F.W[f]; else W += F.W[f];
        }
        if (fi < F.NI - 1) {
          if (ai == 0) D += F.E[f]; else E += F.E[f];
        }
      }
    }
    C.D[cc] = D; C.S[cc] = S; C.N[cc] = N; C.W[cc] = W; C.E[cc] = E;
    C.inv[cc] = (D != 0.0f) ? 1.0f / D : 0.0f;
  });
}

/// The levels below `first` down to the coarsest, then back up to `first`,
/// by one worker set that synchronises with `sync` (a CTA or a warp). On
/// entry level `first` holds its right-hand side and its red start; on exit
/// its x is final.
template <typename Sync, typename SpanOf>
DEV void localCycle(const Multigrid& G, char* smem, int first, Sync sync, SpanOf spanOf) {
  const int L = G.levels;
  int l = first;
  for (; l < L; ++l) {
    const Lv A = sharedLevel(G.lv[l], smem);
    const Span s = spanOf(A);
    const bool coarsest = (l == L - 1);
    const int sweeps = coarsest ? G.coarse : G.pre;
    sync();
    colourSweep(A, s, 1);
    for (int k = 1; k < sweeps; ++k) {
      sync();
      colourSweep(A, s, 0);
      sync();
      colourSweep(A, s, 1);
    }
    if (coarsest) break;
    sync();
    const Lv C = sharedLevel(G.lv[l + 1], smem);
    restrictInto(A, C, spanOf(C));
  }
  for (l = L - 2; l >= first; --l) {
    const Lv A = sharedLevel(G.lv[l], smem);
    const Lv C = sharedLevel(G.lv[l + 1], smem);
    const Span s = spanOf(A);
    for (int h = 0; h < 2 * G.post; ++h) {
      sync();
      if (h == 0) colourSweepProlonged(A, s, C.x, C.NI);
      else colourSweep(A, s, (h & 1) ? 0 : 1);
    }
  }
  sync();
}

/// Rank 0 alone: take the first shared-memory level's right-hand side (the
/// cluster restricted it into global memory), run the V-cycle below it
/// (levels of at most 64 cells on warp 0 alone), and publish that level's x
/// to global memory for the cluster's prolongation.
DEV void sharedCycle(const Multigrid& G, char* smem) {
  const int L = G.levels, m = G.distributed, w = G.warpFrom;
  {
    // the cluster restricted into level m's global right-hand side
    const Lv C = sharedLevel(G.lv[m], smem);
    const float* bg = G.lv[m].b;
    forCells(C, wholeOf(C), [&](int c, int i, int j) {
      const float b = bg[c];
      C.b[c] = b;
      C.x[c] = (((i + j) & 1) == 0) ? b * C.inv[c] : 0.0f;
    });
  }
  auto warp = [] { __syncwarp(); };
  if (w == m) {
    // every shared level is small: warp 0 runs them all
    __syncthreads();
    if (threadIdx.x < 32) localCycle(G, smem, m, warp, [](const Lv& A) { return warpOf(A); });
  } else {
    // block levels [m, w), then warp levels [w, L)
    int l = m;
    for (; l < w; ++l) {
      const Lv A = sharedLevel(G.lv[l], smem);
      const Span s = wholeOf(A);
      const bool coarsest = (l == L - 1);
      const int sweeps = coarsest ? G.coarse : G.pre;
      __syncthreads();
      colourSweep(A, s, 1);
      for (int k = 1; k < sweeps; ++k) {
        __syncthreads();
        colourSweep(A, s, 0);
        __syncthreads();
        colourSweep(A, s, 1);
      }
      if (coarsest) break;
      __syncthreads();
      const Lv C = sharedLevel(G.lv[l + 1], smem);
      restrictInto(A, C, wholeOf(C));
    }
    if (w < L) {
      __syncthreads();
      if (threadIdx.x < 32) localCycle(G, smem, w, warp, [](const Lv& A) { return warpOf(A); });
    }
    for (l = ((w < L) ? w : L - 1) - 1; l >= m; --l) {
      const Lv A = sharedLevel(G.lv[l], smem);
      const Lv C = sharedLevel(G.lv[l + 1], smem);
      const Span s = wholeOf(A);
      for (int h = 0; h < 2 * G.post; ++h) {
        __syncthreads();
        if (h == 0) colourSweepProlonged(A, s, C.x, C.NI);
        else colourSweep(A, s, (h & 1) ? 0 : 1);
      }
    }
  }
  __syncthreads();
  const Lv A = sharedLevel(G.lv[m], smem);
  float* out = G.lv[m].x;
  for (int c = threadIdx.x; c < A.NI * A.NJ; c += blockDim.x) out[c] = A.x[c];
}

/// z = M r, one V-cycle. On entry the fine level's red cells of z hold r / D
/// and its black cells 0 (written by the caller's previous loop, before any
/// barrier). On exit, after a cluster barrier, z is complete except for the
/// last red half sweep on the fine level, which the caller fuses with its
/// reduction.
DEV void vcycle(const Multigrid& G, Team& t, char* smem, float* z) {
  const int L = G.levels, Ld = G.distributed;
  auto view = [&](int l) {
    Lv v = levelView(G, l, smem);
    if (l == 0) {
      v.x = z;
      v.b = G.r;
    }
    return v;
  };
  for (int l = 0; l < Ld; ++l) {
    const Lv F = view(l);
    const Span s = bandOf(F, t);
    const bool coarsest = (l == L - 1);
    const int sweeps = coarsest ? G.coarse : G.pre;
    t.cl.sync();
    colourSweep(F, s, 1);
    for (int k = 1; k < sweeps; ++k) {
      t.cl.sync();
      colourSweep(F, s, 0);
      t.cl.sync();
      colourSweep(F, s, 1);
    }
    if (coarsest) break;
    t.cl.sync();
    if (l + 1 < Ld) {
      const Lv C = view(l + 1);
      restrictInto(F, C, bandOf(C, t));
    } else {
      // every CTA restricts its band into the first shared level's global
      // right-hand side; rank 0 then runs the levels below on its own
      const Lv C = globalLevel(G.lv[l + 1]);
      restrictCells<false>(F, C, bandOf(C, t));
      t.cl.sync();
      if (t.rank == 0) sharedCycle(G, smem);
    }
  }
  for (int l = (Ld < L) ? Ld - 1 : L - 2; l >= 0; --l) {
    const Lv F = view(l);
    const Span s = bandOf(F, t);
    const float* ec = G.lv[l + 1].x;  // coarse correction, global memory on every level
    const int NIc = G.lv[l + 1].NI;
    int halves = 2 * G.post;
    if (l == 0) --halves;  // the caller's last red half sweep
    for (int h = 0; h < halves; ++h) {
      t.cl.sync();
      if (h == 0) colourSweepProlonged(F, s, ec, NIc);
      else colourSweep(F, s, (h & 1) ? 0 : 1);
    }
  }
  t.cl.sync();
}

/// The pressure-correction solve of the mixed form. On entry I.x = 0 and
/// I.r = I.pB (the caller's start of the CG); `initial` = sum |b|. Returns
/// the inner iterations run (the monitor's pressure iterations).
__device__ __noinline__ int pressureMixed(const Instance& I, Team& t, Shared& sh, double* dyn,
                                          double initial) {
  // The multigrid descriptor is read at every phase: keep a copy on chip.
  __shared__ Multigrid mgs;
  {
    const int* src = reinterpret_cast<const int*>(&I.mg);
    int* dst = reinterpret_cast<int*>(&mgs);
    for (int k = t.tid; k < static_cast<int>(sizeof(Multigrid) / sizeof(int)); k += t.T) dst[k] = src[k];
    __syncthreads();
  }
  const Multigrid& G = mgs;
  char* smem = reinterpret_cast<char*>(dyn);
  const int NI = I.NI, NJ = I.NJ;
  const int op1[1] = {kSum};
  const int op3[3] = {kSum, kSum, kSum};

  // ---- set-up: the fine rows in FP32, then the Galerkin levels ----
  const Lv F0 = globalLevel(G.lv[0]);
  for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
    const int i = c % NI, j = c / NI;
    F0.D[c] = static_cast<float>(I.pD[c]);
    F0.S[c] = static_cast<float>((j > 0) ? I.pN[j * NI + i] : ((I.acrossJ0[i] >= 0) ? I.pN[i] : 0.0));
    F0.N[c] = static_cast<float>((j < NJ - 1) ? I.pN[(j + 1) * NI + i] : 0.0);
    F0.W[c] = static_cast<float>((i > 0) ? I.pE[j * (NI + 1) + i] : 0.0);
    F0.E[c] = static_cast<float>((i < NI - 1) ? I.pE[j * (NI + 1) + i + 1] : 0.0);
    F0.inv[c] = (F0.D[c] != 0.0f) ? 1.0f / F0.D[c] : 0.0f;
  }
  for (int l = 1; l < G.distributed; ++l) {
    t.cl.sync();
    const Lv C = levelView(G, l, smem);
    galerkin(levelView(G, l - 1, smem), C, bandOf(C, t));
  }
  t.cl.sync();
  if (G.distributed < G.levels && t.rank == 0) {
    for (int l = G.distributed; l < G.levels; ++l) {
      int* w = reinterpret_cast<int*>(smem + G.lv[l].smemWake);
      for (int i = t.tid; i < G.lv[l].NI; i += t.T) w[i] = G.lv[l].wake[i];
    }
    __syncthreads();
    for (int l = G.distributed; l < G.levels; ++l) {
      if (l > G.distributed) __syncthreads();
      const Lv C = sharedLevel(G.lv[l], smem);
      galerkin(levelView(G, l - 1, smem), C, wholeOf(C));
    }
    // the first V-cycle's barriers order these rows before their use
  }

  const double tolAbs = I.cgTol * initial;
  float* r = G.r;
  float* q = G.q;
  float* e = G.e;
  int total = 0;
  for (int refine = 0; refine < 3 && total < I.mgCap; ++refine) {
    // ---- inner solve of A e = r in FP32 ----
    float* zc = G.z0;
    float* zp = G.z1;
    float* dc = G.d0;
    float* dn = G.d1;
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int i = c % NI, j = c / NI;
      const float rc = static_cast<float>(I.r[c]);
      r[c] = rc;
      e[c] = 0.0f;
      zc[c] = (((i + j) & 1) == 0) ? rc * F0.inv[c] : 0.0f;
    }
    vcycle(G, t, smem, zc);
    double rz;
    {
      Lv Z = F0;
      Z.x = zc;
      Z.b = r;
      double v1[1] = {0.0};
      for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
        const int i = c % NI, j = c / NI;
        if (((i + j) & 1) == 0) zc[c] = (r[c] - offSum(Z, zc, c, i, j)) * Z.inv[c];
        v1[0] += static_cast<double>(r[c]) * static_cast<double>(zc[c]);
      }
      teamReduce(t, sh, v1, op1);
      rz = v1[0];
    }
    double beta = 0.0;
    for (int it = 0; total < I.mgCap; ++it) {
      // q = A d' with d' = z + beta d, formed for each cell and its neighbours.
      double dq[1] = {0.0};
      const float fb = static_cast<float>(beta);
      {
        auto dir = [&](int n) { return (it == 0) ? zc[n] : zc[n] + fb * dc[n]; };
        auto row = [&](int c, float& dv) {
          const int j = c / NI, i = c - j * NI;
          const Nbrs nb = neighbours(F0.wake, NI, NJ, c, i, j);
          dv = dir(c);
          return F0.D[c] * dv + F0.S[c] * dir(nb.s) + F0.N[c] * dir(nb.n) + F0.W[c] * dir(nb.w) +
                 F0.E[c] * dir(nb.e);
        };
        // two cells per step, loads before stores
        for (int c = t.c0 + t.tid; c < t.c1; c += 2 * t.T) {
          float dvA, dvB = 0.0f;
          const float yA = row(c, dvA);
          const int cB = c + t.T;
          const bool hasB = cB < t.c1;
          const float yB = hasB ? row(cB, dvB) : 0.0f;
          dn[c] = dvA;
          q[c] = yA;
          dq[0] += static_cast<double>(dvA) * static_cast<double>(yA);
          if (hasB) {
            dn[cB] = dvB;
            q[cB] = yB;
            dq[0] += static_cast<double>(dvB) * static_cast<double>(yB);
          }
        }
      }
      {
        float* tmp = dc;
        dc = dn;
        dn = tmp;
      }
      teamReduce(t, sh, dq, op1);
      if (!(fabs(dq[0]) > 0.0) || !isfinite(dq[0])) break;
      const float alpha = static_cast<float>(rz / dq[0]);
      double v3[3] = {0.0, 0.0, 0.0};
      {
        // e += alpha d, r -= alpha q, and the next V-cycle's red start
        // z = r / D; two cells per step, loads before stores
        auto upd = [&](int c, float& ev, float& rv, float& zv) {
          const int j = c / NI, i = c - j * NI;
          ev = e[c] + alpha * dc[c];
          rv = r[c] - alpha * q[c];
          zv = (((i + j) & 1) == 0) ? rv * F0.inv[c] : 0.0f;
        };
        for (int c = t.c0 + t.tid; c < t.c1; c += 2 * t.T) {
          float eA, rA, zA, eB = 0.0f, rB = 0.0f, zB = 0.0f;
          upd(c, eA, rA, zA);
          const int cB = c + t.T;
          const bool hasB = cB < t.c1;
          if (hasB) upd(cB, eB, rB, zB);
          e[c] = eA; r[c] = rA; zp[c] = zA;
          v3[2] += fabs(static_cast<double>(rA));
          if (hasB) {
            e[cB] = eB; r[cB] = rB; zp[cB] = zB;
            v3[2] += fabs(static_cast<double>(rB));
          }
        }
      }
      ++total;
      vcycle(G, t, smem, zp);
      {
        Lv Z = F0;
        Z.x = zp;
        Z.b = r;
        // the last red half sweep of the V-cycle, fused with r.z_new and
        // r.z_old: red cells first (with their update), then black ones, so
        // no warp diverges on the colour
        const Span band = bandOf(Z, t);
        sweepCells<false>(Z, band, 0, nullptr, 0);
        __syncthreads();  // the dot products read every red cell of the band
        for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
          const double rc = static_cast<double>(r[c]);
          v3[0] += rc * static_cast<double>(zp[c]);
          v3[1] += rc * static_cast<double>(zc[c]);
        }
      }
      teamReduce(t, sh, v3, op3);
      if (v3[2] <= tolAbs) break;
      if (!(fabs(rz) > 0.0) || !isfinite(v3[0])) break;
      beta = (v3[0] - v3[1]) / rz;  // Polak-Ribiere: stays a CG for a varying preconditioner
      rz = v3[0];
      float* tmp = zc;
      zc = zp;
      zp = tmp;
    }
    // ---- outer refinement in FP64: x += e, r = b - A x ----
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) I.x[c] += static_cast<double>(e[c]);
    t.cl.sync();
    double l1[1] = {0.0};
    for (int c = t.c0 + t.tid; c < t.c1; c += t.T) {
      const int i = c % NI, j = c / NI;
      const double rc = I.pB[c] - pressureRow(I, c, i, j, I.x, I.x[c]);
      I.r[c] = rc;
      l1[0] += fabs(rc);
    }
    teamReduce(t, sh, l1, op1);
    if (l1[0] <= tolAbs) break;
  }
  return total;
}
