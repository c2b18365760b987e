/* cfd_oracle.c - CPU restatement of the reference's SIMPLE solve.
 *
 * TEST INFRASTRUCTURE ONLY (see cfd_oracle.h). Plain C, FP64, contraction
 * off, single thread; it restates the reference loop for loop in its own
 * face-loop form so that, on the reference's mesh and inputs, it reproduces
 * the reference's numbers: tests pin it against golden vectors produced by
 * the reference itself (tests/golden/). Citations are to the reference tree.
 *
 * One deliberate regrouping, exact by construction: the u and v momentum
 * systems are assembled together before either is solved. In the reference
 * (SimpleSolver.cpp:685-710) v is assembled after u's Gauss-Seidel, but v's
 * assembly reads only gradV, gradP, the fluxes, the viscosity and v itself,
 * none of which u's solve writes, so both orders give identical bits.
 */
#include "cfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { K_INTERNAL = 0, K_INLET = 1, K_OUTLET = 2, K_FARFIELD = 3, K_WALL = 4 };
enum { B_INTERIOR = 0, B_WALL = 1, B_FARFIELD = 2, B_OUTLET = 3, B_WAKECUT = 4 };
enum {
  ST_GRADIENTS = 0, ST_MOM_ASSEMBLY, ST_MOM_SOLVE, ST_RHIE_CHOW, ST_P_ASSEMBLY, ST_P_SOLVE,
  ST_CORRECT, ST_SST_BLENDING, ST_SST_ASSEMBLY, ST_SST_SOLVE, ST_END
};
enum {
  F_U = 0, F_V, F_P, F_RHO, F_MU_EFF, F_MASS_FLUX, F_DIVERGENCE, F_MU_MOL, F_GRAD_U, F_GRAD_V,
  F_GRAD_P, F_MOM_DIAG, F_MOM_SRC_U, F_MOM_SRC_V, F_MOM_UPPER, F_MOM_LOWER, F_MOM_DIAGONAL,
  F_P_DIAG, F_P_SOURCE, F_P_UPPER, F_NET_FLUX, F_P_CORRECTION, F_K, F_OMEGA, F_MUT,
  F_WALL_DIST, F_STRAIN, F_F1, F_F2, F_CD, F_PROD, F_GRAD_K, F_GRAD_OMEGA, F_T_DIAG_K,
  F_T_SRC_K, F_T_DIAG_W, F_T_SRC_W
};

static const double kTiny = 1e-300;   /* SimpleSolver.cpp:16 */
static const double kTinyT = 1.0e-30; /* KOmegaSST.cpp:22 */
static const double kMinOmega = 1.0e-10;
static const double SK1 = 0.85, SW1 = 0.5, B1 = 0.075, SK2 = 1.0, SW2 = 0.856, B2 = 0.0828;
static const double BSTAR = 0.09, KAPPA = 0.41, A1 = 0.31, PLIM = 10.0;

static char g_err[256];
const char* or_last_error(void) { return g_err; }

/* std::max / std::min / std::clamp, NaN behaviour included */
static double mx(double a, double b) { return (a < b) ? b : a; }
static double mn(double a, double b) { return (b < a) ? b : a; }
static double clampd(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

typedef struct { double* diag; double* source; double* upper; double* lower; } ldu;

struct or_solver {
  or_mesh m;
  int NI, NJ, N, F;
  int* cellFaces; /* 4 per cell: below, right, above, left (Mesh.cpp:172-181) */
  int* across;    /* oppositeCell per face (Mesh.cpp:78-87) */
  const int* kind;
  const double* bcVel;
  const double* bcP;
  double alphaU, alphaP, cgTol, alphaT, intensity, ratio, lengthScale, blend;
  int sweeps, cgMax, sou, nCorr, model, gsOrder;
  /* geometry (SimpleSolver.hpp:203-209) */
  double *Sx, *Sy, *dX, *dY, *Tx, *Ty, *D, *w;
  /* state */
  double *u, *v, *p, *rho, *mu, *muMol, *mf, *dead;
  double *fu, *fv, *fp, *gu, *gv, *gp;
  ldu mom; double* srcV; double* momDiag;
  ldu pres; double* net; double* corr;
  int hasPRef; double refMassFlow;
  /* SST */
  double *k, *om, *mut, *wd, *S, *f1, *f2, *cd, *cdp, *prod, *gk, *gw;
  ldu tk, tw;
  double kIn, wIn, resK, resW, maxYPlus;
  int initialised;
};

static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
static double length2(double x, double y) { return hypot(x, y); }

static void ldu_alloc(ldu* s, int n, int f) {
  s->diag = zalloc(n); s->source = zalloc(n); s->upper = zalloc(f); s->lower = zalloc(f);
}
static void ldu_free(ldu* s) { free(s->diag); free(s->source); free(s->upper); free(s->lower); }
static void ldu_clear(ldu* s, int n, int f) {
  memset(s->diag, 0, sizeof(double) * n); memset(s->source, 0, sizeof(double) * n);
  memset(s->upper, 0, sizeof(double) * f); memset(s->lower, 0, sizeof(double) * f);
}

static int opposite(const or_mesh* m, int f) {
  if (m->neighbour[f] >= 0) return m->neighbour[f];
  if (m->boundary[f] == B_WAKECUT && m->partner[f] >= 0) return m->owner[m->partner[f]];
  return -1;
}

/* ---- LinearSystem (LinearSystem.cpp) -------------------------------------- */

static void multiply(const or_mesh* m, const double* diag, const double* upper,
                     const double* lower, const double* x, double* y) {
  for (int c = 0; c < m->cells; ++c) y[c] = diag[c] * x[c];
  for (int f = 0; f < m->faces; ++f) {
    const int o = m->owner[f], n = m->neighbour[f];
    if (n >= 0) {
      y[o] += upper[f] * x[n];
      y[n] += lower[f] * x[o];
      continue;
    }
    const int a = opposite(m, f);
    if (a >= 0) y[o] += upper[f] * x[a];
  }
}

static double residualL1(const or_mesh* m, const ldu* s, const double* x, double* scratch) {
  multiply(m, s->diag, s->upper, s->lower, x, scratch);
  double total = 0.0;
  for (int c = 0; c < m->cells; ++c) total += fabs(s->source[c] - scratch[c]);
  return total;
}

static double diagonalL1(const or_mesh* m, const ldu* s) {
  double total = 0.0;
  for (int c = 0; c < m->cells; ++c) total += fabs(s->diag[c]);
  return total;
}

static void build_cell_faces(const or_mesh* m, int* cf) {
  const int NI = m->nodes_i - 1, NJ = m->nodes_j - 1, jFaces = NI * m->nodes_j;
  for (int j = 0; j < NJ; ++j)
    for (int i = 0; i < NI; ++i) {
      int* q = cf + 4 * (j * NI + i);
      q[0] = j * NI + i;                       /* below */
      q[1] = jFaces + (i + 1) * NJ + j;        /* right */
      q[2] = (j + 1) * NI + i;                 /* above */
      q[3] = jFaces + i * NJ + j;              /* left  */
    }
}

static void gs_cell(const or_mesh* m, const int* cf, const double* diag, const double* source,
                    const double* upper, const double* lower, double* x, int c) {
  const double d = diag[c];
  if (!(fabs(d) > 0.0)) return;
  double off = 0.0;
  for (int q = 0; q < 4; ++q) {
    const int f = cf[4 * c + q];
    const int o = m->owner[f], n = m->neighbour[f];
    if (n >= 0) {
      if (o == c) off += upper[f] * x[n]; else off += lower[f] * x[o];
      continue;
    }
    const int a = opposite(m, f);
    if (a >= 0 && o == c) off += upper[f] * x[a];
  }
  x[c] = (source[c] - off) / d;
}

/* gaussSeidel (LinearSystem.cpp:77-116); gsOrder 1 visits the (i+j) even
 * cells, then the odd ones, in each sweep. */
static void gauss_seidel(const or_mesh* m, const int* cf, const double* diag, const double* source,
                         const double* upper, const double* lower, double* x, int sweeps, int order) {
  const int NI = m->nodes_i - 1;
  for (int s = 0; s < sweeps; ++s) {
    if (order == 0) {
      for (int c = 0; c < m->cells; ++c) gs_cell(m, cf, diag, source, upper, lower, x, c);
    } else {
      for (int colour = 0; colour < 2; ++colour)
        for (int c = 0; c < m->cells; ++c)
          if ((((c % NI) + (c / NI)) & 1) == colour) gs_cell(m, cf, diag, source, upper, lower, x, c);
    }
  }
}

/* conjugateGradient (LinearSystem.cpp:118-210) */
static void conjugate_gradient(const or_mesh* m, const double* diag, const double* source,
                               const double* upper, const double* lower, double* x, double tol,
                               int maxIt, double* report) {
  const int n = m->cells;
  report[0] = 0; report[1] = 0; report[2] = 0; report[3] = 0;
  if (n == 0) return;
  double* r = zalloc(n); double* d = zalloc(n); double* z = zalloc(n); double* q = zalloc(n);
  multiply(m, diag, upper, lower, x, q);
  for (int c = 0; c < n; ++c) r[c] = source[c] - q[c];
  double init = 0.0;
  for (int c = 0; c < n; ++c) init += fabs(r[c]);
  report[1] = init; report[2] = init;
  if (init <= 0.0) { report[3] = 1; goto done; }
  for (int c = 0; c < n; ++c) z[c] = (fabs(diag[c]) > 0.0) ? r[c] / diag[c] : r[c];
  memcpy(d, z, sizeof(double) * n);
  double rz = 0.0;
  for (int c = 0; c < n; ++c) rz += r[c] * z[c];
  for (int it = 0; it < maxIt; ++it) {
    multiply(m, diag, upper, lower, d, q);
    double dAd = 0.0;
    for (int c = 0; c < n; ++c) dAd += d[c] * q[c];
    if (!(fabs(dAd) > 0.0)) break;
    const double step = rz / dAd;
    for (int c = 0; c < n; ++c) { x[c] += step * d[c]; r[c] -= step * q[c]; }
    report[0] = it + 1;
    double fin = 0.0;
    for (int c = 0; c < n; ++c) fin += fabs(r[c]);
    report[2] = fin;
    if (fin <= tol * init) { report[3] = 1; break; }
    for (int c = 0; c < n; ++c) z[c] = (fabs(diag[c]) > 0.0) ? r[c] / diag[c] : r[c];
    double rzn = 0.0;
    for (int c = 0; c < n; ++c) rzn += r[c] * z[c];
    if (!(fabs(rz) > 0.0)) break;
    const double beta = rzn / rz;
    rz = rzn;
    for (int c = 0; c < n; ++c) d[c] = z[c] + beta * d[c];
  }
done:
  free(r); free(d); free(z); free(q);
}

/* greenGaussGradient (Gradient.cpp:20-50); out (x, y) per cell */
static void green_gauss(const or_mesh* m, const double* fv, double* g) {
  memset(g, 0, sizeof(double) * 2 * m->cells);
  for (int f = 0; f < m->faces; ++f) {
    const double ax = m->face_normal[2 * f] * m->face_area[f];
    const double ay = m->face_normal[2 * f + 1] * m->face_area[f];
    const double cx = ax * fv[f], cy = ay * fv[f];
    const int o = m->owner[f], n = m->neighbour[f];
    g[2 * o] += cx; g[2 * o + 1] += cy;
    if (n >= 0) { g[2 * n] -= cx; g[2 * n + 1] -= cy; }
  }
  for (int c = 0; c < m->cells; ++c) {
    const double vol = m->cell_area[c];
    if (vol > 0.0) { const double s = 1.0 / vol; g[2 * c] *= s; g[2 * c + 1] *= s; }
  }
}

/* ownerWeight (Gradient.cpp:7-18) */
static double owner_weight(const or_mesh* m, int f) {
  const int n = m->neighbour[f];
  if (n < 0) return 1.0;
  const int o = m->owner[f];
  const double cx = m->face_centre[2 * f], cy = m->face_centre[2 * f + 1];
  const double to = length2(m->centroid[2 * o] - cx, m->centroid[2 * o + 1] - cy);
  const double tn = length2(m->centroid[2 * n] - cx, m->centroid[2 * n + 1] - cy);
  const double total = to + tn;
  return (total > 0.0) ? tn / total : 0.5;
}

/* ---- SimpleSolver ----------------------------------------------------------- */

or_solver* or_create(const or_mesh* mesh, const int* kind, const double* velocity,
                     const double* pressure, const double* st, int model, int gs_order) {
  if (mesh->cells <= 0) { strcpy(g_err, "cannot solve on an empty mesh"); return NULL; }
  if (!(st[0] > 0.0) || st[0] > 1.0 || !(st[1] > 0.0) || st[1] > 1.0) {
    strcpy(g_err, "relaxation factors must lie in (0, 1]");
    return NULL;
  }
  or_solver* s = (or_solver*)calloc(1, sizeof(or_solver));
  s->m = *mesh;
  const or_mesh* m = &s->m;
  s->NI = m->nodes_i - 1; s->NJ = m->nodes_j - 1; s->N = m->cells; s->F = m->faces;
  const int N = s->N, F = s->F;
  s->kind = kind; s->bcVel = velocity; s->bcP = pressure;
  s->alphaU = st[0]; s->alphaP = st[1]; s->sweeps = (int)st[2]; s->cgMax = (int)st[3];
  s->cgTol = st[4]; s->sou = (st[5] != 0.0); s->alphaT = st[6]; s->intensity = st[7];
  s->ratio = st[8]; s->lengthScale = st[9]; s->nCorr = (int)st[10]; s->blend = st[11];
  s->model = model; s->gsOrder = gs_order;
  s->cellFaces = (int*)calloc(4 * (size_t)N, sizeof(int));
  build_cell_faces(m, s->cellFaces);
  s->across = (int*)calloc(F, sizeof(int));
  for (int f = 0; f < F; ++f) s->across[f] = opposite(m, f);
  s->Sx = zalloc(F); s->Sy = zalloc(F); s->dX = zalloc(F); s->dY = zalloc(F);
  s->Tx = zalloc(F); s->Ty = zalloc(F); s->D = zalloc(F); s->w = zalloc(F);
  s->u = zalloc(N); s->v = zalloc(N); s->p = zalloc(N); s->rho = zalloc(N); s->mu = zalloc(N);
  s->muMol = zalloc(N); s->mf = zalloc(F); s->dead = zalloc(F);
  s->fu = zalloc(F); s->fv = zalloc(F); s->fp = zalloc(F);
  s->gu = zalloc(2 * N); s->gv = zalloc(2 * N); s->gp = zalloc(2 * N);
  ldu_alloc(&s->mom, N, F); s->srcV = zalloc(N); s->momDiag = zalloc(N);
  for (int c = 0; c < N; ++c) s->momDiag[c] = 1.0;
  ldu_alloc(&s->pres, N, F); s->net = zalloc(N); s->corr = zalloc(N);
  s->k = zalloc(N); s->om = zalloc(N); s->mut = zalloc(N); s->wd = zalloc(N); s->S = zalloc(N);
  s->f1 = zalloc(N); s->f2 = zalloc(N); s->cd = zalloc(N); s->cdp = zalloc(N); s->prod = zalloc(N);
  s->gk = zalloc(2 * N); s->gw = zalloc(2 * N);
  ldu_alloc(&s->tk, N, F); ldu_alloc(&s->tw, N, F);

  /* precomputeGeometry (SimpleSolver.cpp:82-131) */
  for (int f = 0; f < F; ++f) {
    const double ax = m->face_normal[2 * f] * m->face_area[f];
    const double ay = m->face_normal[2 * f + 1] * m->face_area[f];
    s->Sx[f] = ax; s->Sy[f] = ay;
    const int o = m->owner[f], a = s->across[f];
    const double ox = m->centroid[2 * o], oy = m->centroid[2 * o + 1];
    const double fx = m->face_centre[2 * f], fy = m->face_centre[2 * f + 1];
    double dx, dy, w;
    if (m->neighbour[f] >= 0) {
      dx = m->centroid[2 * a] - ox; dy = m->centroid[2 * a + 1] - oy;
      w = owner_weight(m, f);
    } else if (a >= 0) {
      const double axc = m->centroid[2 * a], ayc = m->centroid[2 * a + 1];
      dx = axc - ox; dy = ayc - oy;
      const double to = length2(ox - fx, oy - fy), ta = length2(axc - fx, ayc - fy);
      const double span = to + ta;
      w = (span > 0.0) ? ta / span : 0.5;
    } else {
      dx = fx - ox; dy = fy - oy; w = 1.0;
    }
    s->dX[f] = dx; s->dY[f] = dy; s->w[f] = w;
    const double sd = ax * dx + ay * dy, ss = ax * ax + ay * ay;
    if (fabs(sd) > kTiny) {
      s->D[f] = ss / sd;
      s->Tx[f] = ax - dx * s->D[f];
      s->Ty[f] = ay - dy * s->D[f];
    }
  }
  s->hasPRef = 0;
  for (int f = 0; f < F; ++f)
    if (kind[f] == K_OUTLET || kind[f] == K_FARFIELD) { s->hasPRef = 1; break; }
  s->refMassFlow = 1.0;
  return s;
}

static int imposes(const or_solver* s, int f) {
  switch (s->kind[f]) {
    case K_WALL: case K_INLET: return 1;
    case K_FARFIELD: return s->mf[f] < s->dead[f];
    default: return 0;
  }
}

/* interpolateFaceValues (SimpleSolver.cpp:268-304) */
static void interpolate_faces(or_solver* s) {
  const or_mesh* m = &s->m;
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], a = s->across[f];
    if (a >= 0) {
      const double w = s->w[f];
      s->fu[f] = w * s->u[o] + (1.0 - w) * s->u[a];
      s->fv[f] = w * s->v[o] + (1.0 - w) * s->v[a];
      s->fp[f] = w * s->p[o] + (1.0 - w) * s->p[a];
    } else if (imposes(s, f)) {
      s->fu[f] = s->bcVel[2 * f]; s->fv[f] = s->bcVel[2 * f + 1]; s->fp[f] = s->p[o];
    } else {
      s->fu[f] = s->u[o]; s->fv[f] = s->v[o]; s->fp[f] = s->bcP[f];
    }
  }
}

/* wallDistances (TurbulenceModel.cpp:28-65) */
static void wall_distances(or_solver* s) {
  const or_mesh* m = &s->m;
  int walls = 0;
  for (int f = 0; f < s->F; ++f) walls += (s->kind[f] == K_WALL);
  if (walls == 0) {
    double total = 0.0;
    for (int c = 0; c < s->N; ++c) total += m->cell_area[c];
    const double far = 1.0e6 * sqrt(fabs(total) + 1.0);
    for (int c = 0; c < s->N; ++c) s->wd[c] = far;
    return;
  }
  /* the wall faces in ascending order, then the same scan over them */
  int* wall = (int*)malloc(sizeof(int) * (size_t)walls);
  int n = 0;
  for (int f = 0; f < s->F; ++f) {
    if (s->kind[f] == K_WALL) wall[n++] = f;
  }
  for (int c = 0; c < s->N; ++c) {
    const double cx = m->centroid[2 * c], cy = m->centroid[2 * c + 1];
    double best = 1.7976931348623157e308;
    for (int k = 0; k < walls; ++k) {
      const int f = wall[k];
      const double dx = cx - m->face_centre[2 * f], dy = cy - m->face_centre[2 * f + 1];
      best = mn(best, dx * dx + dy * dy);
    }
    s->wd[c] = sqrt(best);
  }
  free(wall);
}

static double wall_omega(double nu, double distance, double energy) {
  const double d = mx(distance, kTinyT);
  const double viscous = 6.0 * nu / (B1 * d * d);
  const double logarithmic = sqrt(mx(energy, 0.0)) / (pow(BSTAR, 0.25) * KAPPA * d);
  return sqrt(viscous * viscous + logarithmic * logarithmic);
}

/* KOmegaSST::initialise (KOmegaSST.cpp:104-200) */
static int sst_initialise(or_solver* s) {
  if (!isfinite(s->intensity) || s->intensity < 0.0 || !isfinite(s->ratio) || s->ratio <= 0.0 ||
      !isfinite(s->lengthScale) || s->lengthScale < 0.0) {
    strcpy(g_err, "invalid turbulence inflow");
    return 1;
  }
  wall_distances(s);
  double U = 0.0, R = 0.0, M = 0.0;
  for (int c = 0; c < s->N; ++c) {
    const double sp = length2(s->u[c], s->v[c]);
    if (sp > U) U = sp;
    R = mx(R, s->rho[c]);
    M = mx(M, s->mu[c]);
  }
  if (!(U > 0.0) || !(R > 0.0) || !(M > 0.0)) {
    strcpy(g_err, "the starting field has no scale to set freestream turbulence from");
    return 1;
  }
  const double I = mx(s->intensity, 1.0e-8);
  s->kIn = 1.5 * (I * U) * (I * U);
  if (s->lengthScale > 0.0) {
    s->wIn = mx(sqrt(s->kIn) / (pow(BSTAR, 0.25) * s->lengthScale), kMinOmega);
  } else {
    const double eddy = s->ratio * M;
    s->wIn = mx(R * s->kIn / eddy, kMinOmega);
  }
  for (int c = 0; c < s->N; ++c) {
    s->k[c] = s->kIn;
    const double d = mx(s->wd[c], kTinyT);
    const double nu = s->mu[c] / mx(s->rho[c], kTinyT);
    s->om[c] = mx(s->wIn, wall_omega(nu, d, s->k[c]));
    s->mut[c] = s->rho[c] * s->k[c] / s->om[c];
  }
  s->resK = s->resW = 0.0;
  s->maxYPlus = 0.0;
  return 0;
}

static void apply_eddy_viscosity(or_solver* s) {
  if (s->model == 0) return;
  for (int c = 0; c < s->N; ++c) s->mu[c] = s->muMol[c] + ((s->model == 2) ? s->mut[c] : 0.0);
}

int or_initialise(or_solver* s, const double* u, const double* v, const double* p,
                  const double* rho, const double* mu) {
  const or_mesh* m = &s->m;
  const int N = s->N, F = s->F;
  memcpy(s->u, u, sizeof(double) * N); memcpy(s->v, v, sizeof(double) * N);
  memcpy(s->p, p, sizeof(double) * N); memcpy(s->rho, rho, sizeof(double) * N);
  memcpy(s->mu, mu, sizeof(double) * N); memcpy(s->muMol, mu, sizeof(double) * N);
  double speed = 0.0;
  for (int c = 0; c < N; ++c) speed = mx(speed, length2(s->u[c], s->v[c]));
  for (int f = 0; f < F; ++f) {
    s->dead[f] = 0.0;
    if (s->kind[f] != K_FARFIELD) continue;
    s->dead[f] = 1.0e-3 * s->rho[m->owner[f]] * speed * length2(s->Sx[f], s->Sy[f]);
  }
  interpolate_faces(s);
  for (int f = 0; f < F; ++f) {
    const int o = m->owner[f];
    const double w = s->w[f];
    double dens = s->rho[o];
    if (m->neighbour[f] >= 0) dens = w * s->rho[o] + (1.0 - w) * s->rho[m->neighbour[f]];
    s->mf[f] = dens * (s->fu[f] * s->Sx[f] + s->fv[f] * s->Sy[f]);
  }
  s->refMassFlow = 0.0;
  for (int f = 0; f < F; ++f) {
    if (m->boundary[f] == B_INTERIOR || s->kind[f] == K_INTERNAL) continue;
    s->refMassFlow += mx(-s->mf[f], 0.0);
  }
  if (!(s->refMassFlow > 0.0)) s->refMassFlow = 1.0;
  if (s->model == 2 && sst_initialise(s) != 0) return 1;
  apply_eddy_viscosity(s);
  s->initialised = 1;
  return 0;
}

/* assembleMomentum for both components (SimpleSolver.cpp:319-423) */
static void assemble_momentum(or_solver* s) {
  const or_mesh* m = &s->m;
  ldu* A = &s->mom;
  ldu_clear(A, s->N, s->F);
  memset(s->srcV, 0, sizeof(double) * s->N);
  double* bU = A->source;
  double* bV = s->srcV;
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], other = s->across[f], n = m->neighbour[f];
    const double flux = s->mf[f];
    const double Tx = s->Tx[f], Ty = s->Ty[f];
    if (other >= 0) {
      const double w = s->w[f];
      const double vis = w * s->mu[o] + (1.0 - w) * s->mu[other];
      const double dif = vis * s->D[f];
      const double out = mx(flux, 0.0), in = mx(-flux, 0.0);
      const double gux = s->gu[2 * o] * w + s->gu[2 * other] * (1.0 - w);
      const double guy = s->gu[2 * o + 1] * w + s->gu[2 * other + 1] * (1.0 - w);
      const double gvx = s->gv[2 * o] * w + s->gv[2 * other] * (1.0 - w);
      const double gvy = s->gv[2 * o + 1] * w + s->gv[2 * other + 1] * (1.0 - w);
      const double cu = s->blend * vis * (gux * Tx + guy * Ty);
      const double cv = s->blend * vis * (gvx * Tx + gvy * Ty);
      if (n >= 0) {
        A->diag[o] += out + dif;
        A->upper[f] += -in - dif;
        A->diag[n] += in + dif;
        A->lower[f] += -out - dif;
        bU[o] += cu; bU[n] -= cu;
        bV[o] += cv; bV[n] -= cv;
        if (s->sou) {
          const double uo = s->u[o], un = s->u[n], vo = s->v[o], vn = s->v[n];
          const double du = flux * ((w * uo + (1.0 - w) * un) - ((flux >= 0.0) ? uo : un));
          const double dv = flux * ((w * vo + (1.0 - w) * vn) - ((flux >= 0.0) ? vo : vn));
          bU[o] -= du; bU[n] += du;
          bV[o] -= dv; bV[n] += dv;
        }
      } else {
        A->diag[o] += out + dif;
        A->upper[f] += -in - dif;
        bU[o] += cu;
        bV[o] += cv;
      }
      continue;
    }
    const double vis = s->mu[o];
    const double dif = vis * s->D[f];
    if (imposes(s, f)) {
      const double iu = s->bcVel[2 * f], iv = s->bcVel[2 * f + 1];
      bU[o] -= flux * iu; bV[o] -= flux * iv;
      A->diag[o] += dif;
      bU[o] += dif * iu; bV[o] += dif * iv;
      bU[o] += s->blend * vis * (s->gu[2 * o] * Tx + s->gu[2 * o + 1] * Ty);
      bV[o] += s->blend * vis * (s->gv[2 * o] * Tx + s->gv[2 * o + 1] * Ty);
    } else {
      A->diag[o] += flux;
    }
  }
  for (int c = 0; c < s->N; ++c) {
    bU[c] -= s->gp[2 * c] * m->cell_area[c];
    bV[c] -= s->gp[2 * c + 1] * m->cell_area[c];
  }
  /* applyRelaxation (SimpleSolver.cpp:425-443) */
  for (int c = 0; c < s->N; ++c) {
    const double un = A->diag[c];
    if (!(fabs(un) > 0.0)) { A->diag[c] = 1.0; continue; }
    const double rel = un / s->alphaU;
    A->diag[c] = rel;
    bU[c] += (rel - un) * s->u[c];
    bV[c] += (rel - un) * s->v[c];
  }
}

/* computeRhieChowFluxes (SimpleSolver.cpp:445-496) */
static void rhie_chow(or_solver* s) {
  const or_mesh* m = &s->m;
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], a = s->across[f];
    const double Sx = s->Sx[f], Sy = s->Sy[f];
    if (a >= 0) {
      const double w = s->w[f];
      const double ix = s->u[o] * w + s->u[a] * (1.0 - w);
      const double iy = s->v[o] * w + s->v[a] * (1.0 - w);
      const double dens = w * s->rho[o] + (1.0 - w) * s->rho[a];
      const double mob = w * (m->cell_area[o] / s->momDiag[o]) + (1.0 - w) * (m->cell_area[a] / s->momDiag[a]);
      const double sgx = s->gp[2 * o] * w + s->gp[2 * a] * (1.0 - w);
      const double sgy = s->gp[2 * o + 1] * w + s->gp[2 * a + 1] * (1.0 - w);
      const double compact = (s->p[a] - s->p[o]) * s->D[f];
      const double smooth = sgx * Sx + sgy * Sy;
      s->mf[f] = dens * (ix * Sx + iy * Sy) - dens * mob * (compact - smooth);
      continue;
    }
    const double dens = s->rho[o];
    if (imposes(s, f)) {
      s->mf[f] = dens * (s->bcVel[2 * f] * Sx + s->bcVel[2 * f + 1] * Sy);
    } else {
      const double mob = m->cell_area[o] / s->momDiag[o];
      const double compact = (s->bcP[f] - s->p[o]) * s->D[f];
      const double smooth = s->gp[2 * o] * Sx + s->gp[2 * o + 1] * Sy;
      s->mf[f] = dens * (s->u[o] * Sx + s->v[o] * Sy) - dens * mob * (compact - smooth);
    }
  }
}

/* rho_f * mobility_f * D of a face with a cell on both sides */
static double p_coefficient(const or_solver* s, int f, int o, int n) {
  const or_mesh* m = &s->m;
  const double w = s->w[f];
  const double dens = w * s->rho[o] + (1.0 - w) * s->rho[n];
  const double mob = w * (m->cell_area[o] / s->momDiag[o]) + (1.0 - w) * (m->cell_area[n] / s->momDiag[n]);
  return dens * mob * s->D[f];
}

/* assemblePressureCorrection (SimpleSolver.cpp:498-580) */
static void assemble_pressure(or_solver* s) {
  const or_mesh* m = &s->m;
  ldu* A = &s->pres;
  ldu_clear(A, s->N, s->F);
  memset(s->net, 0, sizeof(double) * s->N);
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], n = m->neighbour[f];
    s->net[o] += s->mf[f];
    if (n >= 0) s->net[n] -= s->mf[f];
    if (n >= 0) {
      const double coef = p_coefficient(s, f, o, n);
      A->diag[o] += coef; A->upper[f] += -coef; A->diag[n] += coef; A->lower[f] += -coef;
      continue;
    }
    const int a = s->across[f];
    if (a >= 0) {
      const double coef = p_coefficient(s, f, o, a);
      A->diag[o] += coef; A->upper[f] += -coef;
      continue;
    }
    if (imposes(s, f)) continue;
    const double mob = m->cell_area[o] / s->momDiag[o];
    A->diag[o] += s->rho[o] * mob * s->D[f];
  }
  for (int c = 0; c < s->N; ++c) A->source[c] = -s->net[c];
  if (!s->hasPRef) {
    double mean = 0.0;
    for (int c = 0; c < s->N; ++c) mean += A->source[c];
    mean /= (double)s->N;
    for (int c = 0; c < s->N; ++c) A->source[c] -= mean;
  }
}

/* correct (SimpleSolver.cpp:582-660) */
static void correct(or_solver* s) {
  const or_mesh* m = &s->m;
  const double* pc = s->corr;
  double* fc = zalloc(s->F);
  double* g = zalloc(2 * s->N);
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], a = s->across[f];
    if (a >= 0) fc[f] = s->w[f] * pc[o] + (1.0 - s->w[f]) * pc[a];
    else if (imposes(s, f)) fc[f] = pc[o];
    else fc[f] = 0.0;
  }
  green_gauss(m, fc, g);
  for (int c = 0; c < s->N; ++c) {
    s->p[c] += s->alphaP * pc[c];
    const double mob = m->cell_area[c] / s->momDiag[c];
    s->u[c] -= g[2 * c] * mob;
    s->v[c] -= g[2 * c + 1] * mob;
  }
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], a = s->across[f];
    if (a >= 0) {
      const double w = s->w[f];
      const double dens = w * s->rho[o] + (1.0 - w) * s->rho[a];
      const double mob = w * (m->cell_area[o] / s->momDiag[o]) + (1.0 - w) * (m->cell_area[a] / s->momDiag[a]);
      s->mf[f] -= dens * mob * s->D[f] * (pc[a] - pc[o]);
      continue;
    }
    if (imposes(s, f)) continue;
    const double mob = m->cell_area[o] / s->momDiag[o];
    s->mf[f] -= s->rho[o] * mob * s->D[f] * (0.0 - pc[o]);
  }
  free(fc);
  free(g);
}

static void divergence(const or_solver* s, double* net) {
  const or_mesh* m = &s->m;
  memset(net, 0, sizeof(double) * s->N);
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f], n = m->neighbour[f];
    const double vf = s->mf[f] / mx(s->rho[o], kTiny);
    net[o] += vf;
    if (n >= 0) net[n] -= vf;
  }
  for (int c = 0; c < s->N; ++c) {
    const double a = m->cell_area[c];
    net[c] = (a > 0.0) ? net[c] / a : 0.0;
  }
}

/* ---- k-omega SST (KOmegaSST.cpp) ---------------------------------------------- */

/* interpolate (KOmegaSST.cpp:26-68) */
static void sst_face_values(const or_solver* s, const double* phi, double wallValue, double inflow,
                            double* out) {
  const or_mesh* m = &s->m;
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f];
    if (m->neighbour[f] >= 0) {
      const double w = owner_weight(m, f);
      out[f] = w * phi[o] + (1.0 - w) * phi[m->neighbour[f]];
      continue;
    }
    const int a = s->across[f];
    if (a >= 0) {
      const double w = owner_weight(m, f);
      out[f] = w * phi[o] + (1.0 - w) * phi[a];
      continue;
    }
    switch (s->kind[f]) {
      case K_WALL: out[f] = wallValue; break;
      case K_INLET: out[f] = inflow; break;
      case K_FARFIELD: out[f] = (s->mf[f] < 0.0) ? inflow : phi[o]; break;
      default: out[f] = phi[o]; break;
    }
  }
}

static double blendf(double f1, double a, double b) { return f1 * a + (1.0 - f1) * b; }

static void sst_blending(or_solver* s) {
  const or_mesh* m = &s->m;
  const int N = s->N;
  /* computeStrain (:202-216) */
  for (int c = 0; c < N; ++c) {
    const double s11 = s->gu[2 * c], s22 = s->gv[2 * c + 1];
    const double s12 = 0.5 * (s->gu[2 * c + 1] + s->gv[2 * c]);
    s->S[c] = sqrt(2.0 * (s11 * s11 + s22 * s22 + 2.0 * s12 * s12));
  }
  /* computeBlending (:218-287) */
  double* fv = zalloc(s->F);
  sst_face_values(s, s->k, 0.0, s->kIn, fv);
  green_gauss(m, fv, s->gk);
  sst_face_values(s, s->om, s->om[0], s->wIn, fv);
  for (int f = 0; f < s->F; ++f)
    if (m->neighbour[f] < 0 && s->across[f] < 0 && s->kind[f] == K_WALL) fv[f] = s->om[m->owner[f]];
  green_gauss(m, fv, s->gw);
  free(fv);
  for (int c = 0; c < N; ++c) {
    const double d = mx(s->wd[c], kTinyT);
    const double rho = s->rho[c];
    const double nu = s->muMol[c] / mx(rho, kTinyT);
    const double omega = mx(s->om[c], kMinOmega);
    const double energy = mx(s->k[c], 0.0);
    s->cd[c] = 2.0 * rho * SW2 * (s->gk[2 * c] * s->gw[2 * c] + s->gk[2 * c + 1] * s->gw[2 * c + 1]) / omega;
    s->cdp[c] = mx(s->cd[c], 1.0e-10);
    const double t1 = sqrt(mx(energy, 0.0)) / (BSTAR * omega * d);
    const double t2 = 500.0 * nu / (d * d * omega);
    const double t3 = 4.0 * rho * SW2 * energy / (s->cdp[c] * d * d);
    const double arg1 = mn(mx(t1, t2), t3);
    s->f1[c] = tanh(clampd(arg1 * arg1 * arg1 * arg1, 0.0, 50.0));
    const double arg2 = mx(2.0 * t1, t2);
    s->f2[c] = tanh(clampd(arg2 * arg2, 0.0, 50.0));
  }
  /* production (:362-368) */
  for (int c = 0; c < N; ++c) {
    const double raw = s->mut[c] * s->S[c] * s->S[c];
    const double ceiling = PLIM * BSTAR * s->rho[c] * mx(s->k[c], 0.0) * mx(s->om[c], kMinOmega);
    s->prod[c] = mn(raw, ceiling);
  }
}

/* the `solve` lambda of solveTransport up to (not including) the sweeps */
static double sst_assemble(or_solver* s, ldu* A, const double* phi, double wallValue, double inflow,
                           const double* sigma, const double* sExp, const double* sImp, double* scratch) {
  const or_mesh* m = &s->m;
  ldu_clear(A, s->N, s->F);
  for (int f = 0; f < s->F; ++f) {
    const int o = m->owner[f];
    const int other = (m->neighbour[f] >= 0) ? m->neighbour[f] : s->across[f];
    const double ax = m->face_normal[2 * f] * m->face_area[f];
    const double ay = m->face_normal[2 * f + 1] * m->face_area[f];
    const double flux = s->mf[f];
    if (other >= 0) {
      const double w = owner_weight(m, f);
      const double dfv = w * (s->muMol[o] + sigma[o] * s->mut[o]) + (1.0 - w) * (s->muMol[other] + sigma[other] * s->mut[other]);
      const double dx = m->centroid[2 * other] - m->centroid[2 * o];
      const double dy = m->centroid[2 * other + 1] - m->centroid[2 * o + 1];
      const double sd = ax * dx + ay * dy;
      const double geometric = (fabs(sd) > kTinyT) ? (ax * ax + ay * ay) / sd : 0.0;
      const double dif = dfv * fabs(geometric);
      const double out = mx(flux, 0.0), in = mx(-flux, 0.0);
      A->diag[o] += out + dif;
      A->upper[f] += -in - dif;
      if (m->neighbour[f] >= 0) {
        A->diag[other] += in + dif;
        A->lower[f] += -out - dif;
      }
      continue;
    }
    const double dfv = s->muMol[o] + sigma[o] * s->mut[o];
    const double dx = m->face_centre[2 * f] - m->centroid[2 * o];
    const double dy = m->face_centre[2 * f + 1] - m->centroid[2 * o + 1];
    const double sd = ax * dx + ay * dy;
    const double geometric = (fabs(sd) > kTinyT) ? (ax * ax + ay * ay) / sd : 0.0;
    const double dif = dfv * fabs(geometric);
    const int kind = s->kind[f];
    const int imposed = kind == K_WALL || kind == K_INLET || (kind == K_FARFIELD && flux < 0.0);
    if (imposed) {
      const double value = (kind == K_WALL) ? wallValue : inflow;
      A->diag[o] += dif + mx(flux, 0.0);
      A->source[o] += (dif - mn(flux, 0.0)) * value;
    } else {
      A->diag[o] += mx(flux, 0.0);
    }
  }
  for (int c = 0; c < s->N; ++c) {
    const double vol = m->cell_area[c];
    A->source[c] += sExp[c] * vol;
    A->diag[c] += sImp[c] * vol;
  }
  const double relax = clampd(s->alphaT, 0.05, 1.0);
  for (int c = 0; c < s->N; ++c) {
    if (fabs(A->diag[c]) > kTinyT) {
      const double rel = A->diag[c] / relax;
      A->source[c] += (rel - A->diag[c]) * phi[c];
      A->diag[c] = rel;
    }
  }
  return residualL1(m, A, phi, scratch) / mx(diagonalL1(m, A) * mx(inflow, kTinyT), kTinyT);
}

static void sst_assemble_both(or_solver* s) {
  const int N = s->N;
  double* sigma = zalloc(N); double* sExp = zalloc(N); double* sImp = zalloc(N); double* scratch = zalloc(N);
  const double g1 = B1 / BSTAR - SW1 * KAPPA * KAPPA / sqrt(BSTAR);
  const double g2 = B2 / BSTAR - SW2 * KAPPA * KAPPA / sqrt(BSTAR);
  for (int c = 0; c < N; ++c) {
    sigma[c] = blendf(s->f1[c], SK1, SK2);
    sExp[c] = s->prod[c];
    sImp[c] = BSTAR * s->rho[c] * mx(s->om[c], kMinOmega);
  }
  s->resK = sst_assemble(s, &s->tk, s->k, 0.0, s->kIn, sigma, sExp, sImp, scratch);
  for (int c = 0; c < N; ++c) {
    sigma[c] = blendf(s->f1[c], SW1, SW2);
    const double gamma = blendf(s->f1[c], g1, g2);
    const double beta = blendf(s->f1[c], B1, B2);
    const double rho = s->rho[c];
    sExp[c] = gamma * rho * s->S[c] * s->S[c];
    sExp[c] += (1.0 - s->f1[c]) * s->cd[c];
    sImp[c] = beta * rho * mx(s->om[c], kMinOmega);
  }
  s->resW = sst_assemble(s, &s->tw, s->om, s->wIn, s->wIn, sigma, sExp, sImp, scratch);
  free(sigma); free(sExp); free(sImp); free(scratch);
}

/* floors, applyWallConditions, updateEddyViscosity, updateRanges (:289-345, :469-471, :513-529) */
static void sst_finish(or_solver* s, double* mon) {
  const or_mesh* m = &s->m;
  const int N = s->N;
  for (int c = 0; c < N; ++c) { s->k[c] = mx(s->k[c], 0.0); s->om[c] = mx(s->om[c], kMinOmega); }
  s->maxYPlus = 0.0;
  for (int f = 0; f < s->F; ++f) {
    if (s->kind[f] != K_WALL) continue;
    const int o = m->owner[f];
    const double d = mx(s->wd[o], kTinyT);
    const double rho = mx(s->rho[o], kTinyT);
    const double nu = s->muMol[o] / rho;
    s->om[o] = wall_omega(nu, d, s->k[o]);
    const double nX = m->face_normal[2 * f] * -1.0, nY = m->face_normal[2 * f + 1] * -1.0;
    const double dn = s->u[o] * nX + s->v[o] * nY;
    const double tang = length2(s->u[o] - nX * dn, s->v[o] - nY * dn);
    const double shear = s->muMol[o] * tang / d;
    const double fv = sqrt(shear / rho);
    s->maxYPlus = mx(s->maxYPlus, fv * d / mx(nu, kTinyT));
  }
  for (int c = 0; c < N; ++c) {
    const double energy = mx(s->k[c], 0.0);
    const double omega = mx(s->om[c], kMinOmega);
    const double den = mx(A1 * omega, s->S[c] * s->f2[c]);
    s->mut[c] = s->rho[c] * A1 * energy / mx(den, kTinyT);
  }
  double kmin = s->k[0], kmax = s->k[0], wmin = s->om[0], wmax = s->om[0], tmin = s->mut[0], tmax = s->mut[0];
  for (int c = 1; c < N; ++c) {
    kmin = mn(kmin, s->k[c]); kmax = mx(kmax, s->k[c]);
    wmin = mn(wmin, s->om[c]); wmax = mx(wmax, s->om[c]);
    tmin = mn(tmin, s->mut[c]); tmax = mx(tmax, s->mut[c]);
  }
  apply_eddy_viscosity(s);
  double ratio = 0.0;
  for (int c = 0; c < N; ++c)
    if (s->muMol[c] > 0.0) ratio = mx(ratio, s->mut[c] / s->muMol[c]);
  mon[6] = s->resK; mon[7] = s->resW;
  mon[8] = kmin; mon[9] = kmax; mon[10] = wmin; mon[11] = wmax; mon[12] = tmin; mon[13] = tmax;
  mon[14] = ratio; mon[15] = s->maxYPlus;
}

/* ---- iterate (SimpleSolver.cpp:662-794) -------------------------------------------- */

static int iterate_once(or_solver* s, int stop, double* mon) {
  const or_mesh* m = &s->m;
  const int N = s->N;
  for (int q = 0; q < 16; ++q) mon[q] = 0.0;
  interpolate_faces(s);
  green_gauss(m, s->fu, s->gu);
  green_gauss(m, s->fv, s->gv);
  green_gauss(m, s->fp, s->gp);
  if (stop == ST_GRADIENTS) return 1;

  double scale = 0.0;
  for (int c = 0; c < N; ++c) scale = mx(scale, length2(s->u[c], s->v[c]));
  if (!(scale > 0.0)) scale = 1.0;
  assemble_momentum(s);
  double* scratch = zalloc(N);
  ldu vsys = s->mom;
  vsys.source = s->srcV;
  const double rU = residualL1(m, &s->mom, s->u, scratch);
  const double rV = residualL1(m, &vsys, s->v, scratch);
  const double dl = diagonalL1(m, &s->mom) * scale;
  mon[1] = rU / mx(dl, kTiny);
  mon[2] = rV / mx(dl, kTiny);
  memcpy(s->momDiag, s->mom.diag, sizeof(double) * N);
  if (stop == ST_MOM_ASSEMBLY) { free(scratch); return 1; }

  gauss_seidel(m, s->cellFaces, s->mom.diag, s->mom.source, s->mom.upper, s->mom.lower, s->u, s->sweeps, s->gsOrder & 1);
  gauss_seidel(m, s->cellFaces, s->mom.diag, s->srcV, s->mom.upper, s->mom.lower, s->v, s->sweeps, s->gsOrder & 1);
  if (stop == ST_MOM_SOLVE) { free(scratch); return 1; }

  rhie_chow(s);
  if (stop == ST_RHIE_CHOW) { free(scratch); return 1; }

  const int passes = (s->nCorr > 1) ? s->nCorr : 1;
  for (int pass = 0; pass < passes; ++pass) {
    assemble_pressure(s);
    if (pass == 0) {
      double imb = 0.0;
      for (int c = 0; c < N; ++c) imb += fabs(s->net[c]);
      mon[3] = imb;
      mon[0] = imb / s->refMassFlow;
    }
    memset(s->corr, 0, sizeof(double) * N);
    if (stop == ST_P_ASSEMBLY) { free(scratch); return 1; }
    double rep[4];
    conjugate_gradient(m, s->pres.diag, s->pres.source, s->pres.upper, s->pres.lower, s->corr,
                       s->cgTol, s->cgMax, rep);
    mon[5] += rep[0];
    if (!s->hasPRef) {
      double mean = 0.0;
      for (int c = 0; c < N; ++c) mean += s->corr[c];
      mean /= (double)N;
      for (int c = 0; c < N; ++c) s->corr[c] -= mean;
    }
    if (stop == ST_P_SOLVE) { free(scratch); return 1; }
    correct(s);
    if (stop == ST_CORRECT) { free(scratch); return 1; }
  }
  divergence(s, scratch);
  for (int c = 0; c < N; ++c) mon[4] = mx(mon[4], fabs(scratch[c]));
  free(scratch);

  if (s->model == 2) {
    sst_blending(s);
    if (stop == ST_SST_BLENDING) return 1;
    sst_assemble_both(s);
    mon[6] = s->resK; mon[7] = s->resW;
    if (stop == ST_SST_ASSEMBLY) return 1;
    gauss_seidel(m, s->cellFaces, s->tk.diag, s->tk.source, s->tk.upper, s->tk.lower, s->k, 3, (s->gsOrder >> 1) & 1);
    gauss_seidel(m, s->cellFaces, s->tw.diag, s->tw.source, s->tw.upper, s->tw.lower, s->om, 3, (s->gsOrder >> 1) & 1);
    if (stop == ST_SST_SOLVE) return 1;
    sst_finish(s, mon);
  } else if (s->model == 1) {
    apply_eddy_viscosity(s);
  }
  return 0;
}

int or_iterate(or_solver* s, int n, int stop_stage, double* monitor) {
  double local[16];
  for (int it = 0; it < n; ++it) {
    double* mon = monitor ? monitor + 16 * it : local;
    if (iterate_once(s, (it == 0) ? stop_stage : ST_END, mon)) return it + 1;
  }
  return n;
}

void or_load_state(or_solver* s, const double* u, const double* v, const double* p,
                   const double* mass_flux, const double* k, const double* omega, const double* mut,
                   const double* mu_eff) {
  const int N = s->N;
  if (u) memcpy(s->u, u, sizeof(double) * N);
  if (v) memcpy(s->v, v, sizeof(double) * N);
  if (p) memcpy(s->p, p, sizeof(double) * N);
  if (mass_flux) memcpy(s->mf, mass_flux, sizeof(double) * s->F);
  if (k) memcpy(s->k, k, sizeof(double) * N);
  if (omega) memcpy(s->om, omega, sizeof(double) * N);
  if (mut) memcpy(s->mut, mut, sizeof(double) * N);
  if (mu_eff) memcpy(s->mu, mu_eff, sizeof(double) * N);
}

void or_scalars(or_solver* s, double* out3) {
  out3[0] = s->kIn; out3[1] = s->wIn; out3[2] = s->refMassFlow;
}

int or_read(or_solver* s, int which, double* out) {
  const int N = s->N, F = s->F;
  const size_t cb = sizeof(double) * N, fb = sizeof(double) * F;
  switch (which) {
    case F_U: memcpy(out, s->u, cb); return 0;
    case F_V: memcpy(out, s->v, cb); return 0;
    case F_P: memcpy(out, s->p, cb); return 0;
    case F_RHO: memcpy(out, s->rho, cb); return 0;
    case F_MU_EFF: memcpy(out, s->mu, cb); return 0;
    case F_MASS_FLUX: memcpy(out, s->mf, fb); return 0;
    case F_DIVERGENCE: divergence(s, out); return 0;
    case F_MU_MOL: memcpy(out, s->muMol, cb); return 0;
    case F_GRAD_U: memcpy(out, s->gu, 2 * cb); return 0;
    case F_GRAD_V: memcpy(out, s->gv, 2 * cb); return 0;
    case F_GRAD_P: memcpy(out, s->gp, 2 * cb); return 0;
    case F_MOM_DIAG: case F_MOM_DIAGONAL: memcpy(out, s->mom.diag, cb); return 0;
    case F_MOM_SRC_U: memcpy(out, s->mom.source, cb); return 0;
    case F_MOM_SRC_V: memcpy(out, s->srcV, cb); return 0;
    case F_MOM_UPPER: memcpy(out, s->mom.upper, fb); return 0;
    case F_MOM_LOWER: memcpy(out, s->mom.lower, fb); return 0;
    case F_P_DIAG: memcpy(out, s->pres.diag, cb); return 0;
    case F_P_SOURCE: memcpy(out, s->pres.source, cb); return 0;
    case F_P_UPPER: memcpy(out, s->pres.upper, fb); return 0;
    case F_NET_FLUX: memcpy(out, s->net, cb); return 0;
    case F_P_CORRECTION: memcpy(out, s->corr, cb); return 0;
    case F_K: memcpy(out, s->k, cb); return 0;
    case F_OMEGA: memcpy(out, s->om, cb); return 0;
    case F_MUT: memcpy(out, s->mut, cb); return 0;
    case F_WALL_DIST: memcpy(out, s->wd, cb); return 0;
    case F_STRAIN: memcpy(out, s->S, cb); return 0;
    case F_F1: memcpy(out, s->f1, cb); return 0;
    case F_F2: memcpy(out, s->f2, cb); return 0;
    case F_CD: memcpy(out, s->cd, cb); return 0;
    case F_PROD: memcpy(out, s->prod, cb); return 0;
    case F_GRAD_K: memcpy(out, s->gk, 2 * cb); return 0;
    case F_GRAD_OMEGA: memcpy(out, s->gw, 2 * cb); return 0;
    case F_T_DIAG_K: memcpy(out, s->tk.diag, cb); return 0;
    case F_T_SRC_K: memcpy(out, s->tk.source, cb); return 0;
    case F_T_DIAG_W: memcpy(out, s->tw.diag, cb); return 0;
    case F_T_SRC_W: memcpy(out, s->tw.source, cb); return 0;
    default: return 1;
  }
}

void or_free(or_solver* s) {
  if (!s) return;
  double* arrays[] = {s->Sx, s->Sy, s->dX, s->dY, s->Tx, s->Ty, s->D, s->w, s->u, s->v, s->p,
                      s->rho, s->mu, s->muMol, s->mf, s->dead, s->fu, s->fv, s->fp, s->gu, s->gv,
                      s->gp, s->srcV, s->momDiag, s->net, s->corr, s->k, s->om, s->mut, s->wd,
                      s->S, s->f1, s->f2, s->cd, s->cdp, s->prod, s->gk, s->gw};
  for (size_t q = 0; q < sizeof(arrays) / sizeof(arrays[0]); ++q) free(arrays[q]);
  ldu_free(&s->mom); ldu_free(&s->pres); ldu_free(&s->tk); ldu_free(&s->tw);
  free(s->cellFaces); free(s->across);
  free(s);
}

/* ---- primitives ---------------------------------------------------------------- */

void or_ldu_multiply(const or_mesh* m, const double* diag, const double* upper,
                     const double* lower, const double* x, double* y) {
  multiply(m, diag, upper, lower, x, y);
}

void or_ldu_gauss_seidel(const or_mesh* m, const double* diag, const double* source,
                         const double* upper, const double* lower, double* x, int sweeps,
                         int gs_order) {
  int* cf = (int*)calloc(4 * (size_t)m->cells, sizeof(int));
  build_cell_faces(m, cf);
  gauss_seidel(m, cf, diag, source, upper, lower, x, sweeps, gs_order);
  free(cf);
}

void or_ldu_cg(const or_mesh* m, const double* diag, const double* source, const double* upper,
               const double* lower, double* x, double tolerance, int max_iterations, double* report) {
  conjugate_gradient(m, diag, source, upper, lower, x, tolerance, max_iterations, report);
}

void or_green_gauss(const or_mesh* m, const double* face_values, double* out) {
  green_gauss(m, face_values, out);
}
