// mesh.cpp - host generation of structured meshes (C-grid, box) and their
// finite-volume metrics.
//
// The arithmetic follows the reference step for step, because the solver's
// parity contract is stated on the reference's own meshes: a different
// rounding anywhere here would move every downstream number. The pieces:
//   NACA 4-digit section        src/geom/Naca4.cpp:65-132, src/geom/Airfoil.cpp:37-149
//   node distributions          src/mesh/Distribution.cpp:7-109
//   C-grid node placement       src/mesh/CGrid.cpp:98-382
//   structured block metrics    src/mesh/Mesh.cpp:89-339
//   Cartesian box               src/mesh/BoxGrid.cpp:7-65
// Only what the solver consumes is built: no quality report, no logging.

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <numbers>
#include <string>
#include <vector>

#include "cfd_mesh.h"
#include "common.hpp"

namespace cfdb {
namespace {

struct P2 {
  double x{0.0};
  double y{0.0};
};
inline P2 operator+(P2 a, P2 b) { return {a.x + b.x, a.y + b.y}; }
inline P2 operator-(P2 a, P2 b) { return {a.x - b.x, a.y - b.y}; }
inline P2 operator*(P2 a, double s) { return {a.x * s, a.y * s}; }
inline double dotp(P2 a, P2 b) { return a.x * b.x + a.y * b.y; }
inline double crossp(P2 a, P2 b) { return a.x * b.y - a.y * b.x; }
inline double lenp(P2 a) { return std::hypot(a.x, a.y); }
inline double distp(P2 a, P2 b) { return lenp(b - a); }
inline P2 unit(P2 v) {
  const double l = lenp(v);
  return (l > 0.0) ? v * (1.0 / l) : P2{0.0, 0.0};
}
inline P2 quarterLeft(P2 v) { return {-v.y, v.x}; }
inline P2 quarterRight(P2 v) { return {v.y, -v.x}; }

// ---- one-dimensional node distributions (Distribution.cpp) ----------------

std::vector<double> evenStations(int intervals) {
  std::vector<double> t(static_cast<std::size_t>(intervals) + 1);
  for (int k = 0; k <= intervals; ++k) t[k] = static_cast<double>(k) / static_cast<double>(intervals);
  t.back() = 1.0;
  return t;
}

/// Growth ratio r with first*(r^n-1)/(r-1) = total, by 200 bisection steps on
/// [1, 3] (Distribution.cpp:23-53).
double growthRatio(double first, double total, int n) {
  if (n <= 1 || first <= 0.0 || total <= 0.0) return 1.0;
  if (first * static_cast<double>(n) >= total) return 1.0;
  auto series = [&](double r) {
    if (std::abs(r - 1.0) < 1e-12) return first * static_cast<double>(n);
    return first * (std::pow(r, static_cast<double>(n)) - 1.0) / (r - 1.0);
  };
  double lo = 1.0, hi = 3.0;
  if (series(hi) < total) return hi;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (series(mid) < total) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

std::vector<double> graded(double first, double total, int n) {
  std::vector<double> t(static_cast<std::size_t>(n) + 1, 0.0);
  const double r = growthRatio(first, total, n);
  double step = first, sum = 0.0;
  for (int k = 1; k <= n; ++k) {
    sum += step;
    t[k] = sum;
    step *= r;
  }
  if (sum > 0.0) for (double& v : t) v /= sum;
  t.front() = 0.0;
  t.back() = 1.0;
  return t;
}

std::vector<double> gradedBothEnds(double first, double total, int n) {
  if (n < 2) return evenStations(n);
  const int half = n / 2;
  const std::vector<double> low = graded(first, 0.5 * total, half);
  std::vector<double> t(static_cast<std::size_t>(n) + 1, 0.0);
  for (int k = 0; k <= half; ++k) t[k] = 0.5 * low[k];
  for (int k = 0; k <= half; ++k) t[n - k] = 1.0 - 0.5 * low[k];
  if (n % 2 != 0) t[half + 1] = 0.5 * (t[half] + t[half + 2]);
  t.front() = 0.0;
  t.back() = 1.0;
  return t;
}

// ---- NACA 4-digit wall contour (Naca4.cpp, Airfoil.cpp) ------------------

struct Naca {
  int m{0}, p{0}, tt{12};
};

Status parseNaca(const char* text, Naca* out) {
  std::string s;
  for (const char* q = text; q != nullptr && *q != '\0'; ++q) {
    if (!std::isspace(static_cast<unsigned char>(*q))) s.push_back(static_cast<char>(std::toupper(*q)));
  }
  if (s.rfind("NACA", 0) == 0) s.erase(0, 4);
  if (s.size() != 4) return fail(CFD_INVALID_ARGUMENT, "a four-digit NACA designation is required");
  for (char c : s) {
    if (!std::isdigit(static_cast<unsigned char>(c))) return fail(CFD_INVALID_ARGUMENT, "designation contains a non-digit");
  }
  Naca n{s[0] - '0', s[1] - '0', (s[2] - '0') * 10 + (s[3] - '0')};
  if (n.m > 0 && n.p == 0) return fail(CFD_INVALID_ARGUMENT, "camber position digit must be non-zero when camber is");
  if (n.m == 0 && n.p > 0) return fail(CFD_INVALID_ARGUMENT, "zero camber with a camber position");
  if (n.tt == 0) return fail(CFD_INVALID_ARGUMENT, "zero thickness");
  if (n.tt > 40) return fail(CFD_INVALID_ARGUMENT, "four-digit family is defined up to 40% thickness");
  *out = n;
  return ok();
}

/// Half thickness with the closed-trailing-edge last coefficient -0.1036.
double halfThickness(double x, double t) {
  if (!(x > 0.0)) return 0.0;
  const double xc = std::min(x, 1.0);
  const double x2 = xc * xc, x3 = x2 * xc, x4 = x3 * xc;
  return 5.0 * t * (0.2969 * std::sqrt(xc) + -0.1260 * xc + -0.3516 * x2 + 0.2843 * x3 + -0.1036 * x4);
}

double meanLine(double x, double m, double p) {
  if (m == 0.0 || p <= 0.0 || p >= 1.0) return 0.0;
  const double xc = std::clamp(x, 0.0, 1.0);
  if (xc <= p) return (m / (p * p)) * (2.0 * p * xc - xc * xc);
  const double q = 1.0 - p;
  return (m / (q * q)) * ((1.0 - 2.0 * p) + 2.0 * p * xc - xc * xc);
}

double meanLineSlope(double x, double m, double p) {
  if (m == 0.0 || p <= 0.0 || p >= 1.0) return 0.0;
  const double xc = std::clamp(x, 0.0, 1.0);
  const double den = (xc <= p) ? (p * p) : ((1.0 - p) * (1.0 - p));
  return (2.0 * m / den) * (p - xc);
}

/// Closed contour for chord 1: upper surface from trailing to leading edge,
/// then lower back to the trailing edge, closed on its first point.
/// Returns also the trailing-edge point.
std::vector<P2> nacaContour(const Naca& n, int perSurface, P2* trailing) {
  const double m = n.m / 100.0, p = n.p / 10.0, t = n.tt / 100.0;
  const std::size_t count = static_cast<std::size_t>(perSurface);
  std::vector<double> xs(count);
  const double last = static_cast<double>(perSurface - 1);
  for (std::size_t i = 0; i < count; ++i) {
    xs[i] = 0.5 * (1.0 - std::cos(std::numbers::pi * static_cast<double>(i) / last));
  }
  xs.front() = 0.0;
  xs.back() = 1.0;
  std::vector<P2> upper(count), lower(count), camber(count);
  for (std::size_t i = 0; i < count; ++i) {
    const double x = xs[i];
    const double yc = meanLine(x, m, p);
    const double yt = halfThickness(x, t);
    const double theta = std::atan(meanLineSlope(x, m, p));
    const double s = std::sin(theta), c = std::cos(theta);
    camber[i] = P2{x * 1.0, yc * 1.0};
    upper[i] = P2{(x - yt * s) * 1.0, (yc + yt * c) * 1.0};
    lower[i] = P2{(x + yt * s) * 1.0, (yc - yt * c) * 1.0};
  }
  upper.front() = camber.front();
  lower.front() = camber.front();
  upper.back() = camber.back();
  lower.back() = camber.back();
  std::vector<P2> contour;
  contour.reserve(2 * count);
  for (std::size_t i = count; i-- > 0;) contour.push_back(upper[i]);
  for (std::size_t i = 1; i < count - 1; ++i) contour.push_back(lower[i]);
  contour.push_back(contour.front());
  *trailing = (upper.back() + lower.back()) * 0.5;
  return contour;
}

}  // namespace

// ---- structured block -> face-based metrics (Mesh.cpp:89-339) -------------

Status buildBlock(int ni, int nj, std::vector<double> nodesXY, const std::vector<int>& jMinType,
                  int jMaxType, int iMinType, int iMaxType, const std::vector<int>& jMinPartner,
                  HostMesh* out) {
  if (ni < 2 || nj < 2) return fail(CFD_INVALID_ARGUMENT, "a structured block needs at least 2x2 nodes");
  const int NI = ni - 1, NJ = nj - 1;
  HostMesh& g = *out;
  g = HostMesh{};
  g.nodesI = ni;
  g.nodesJ = nj;
  g.nodes = std::move(nodesXY);
  const std::size_t cells = static_cast<std::size_t>(NI) * NJ;
  const std::size_t jFaces = static_cast<std::size_t>(NI) * nj;
  const std::size_t iFaces = static_cast<std::size_t>(ni) * NJ;
  const std::size_t faces = jFaces + iFaces;
  g.cells = static_cast<int>(cells);
  g.faces = static_cast<int>(faces);
  auto node = [&](int i, int j) { return P2{g.nodes[2 * (static_cast<std::size_t>(j) * ni + i)], g.nodes[2 * (static_cast<std::size_t>(j) * ni + i) + 1]}; };

  g.owner.assign(faces, -1);
  g.neighbour.assign(faces, -1);
  g.boundary.assign(faces, CFD_FACE_INTERIOR);
  g.partner.assign(faces, -1);
  std::vector<int> faceNodeA(faces), faceNodeB(faces);
  for (int j = 0; j < nj; ++j) {
    for (int i = 0; i < NI; ++i) {
      const std::size_t f = static_cast<std::size_t>(j) * NI + i;
      faceNodeA[f] = j * ni + i;
      faceNodeB[f] = j * ni + i + 1;
      if (j == 0) {
        g.owner[f] = i;
        g.boundary[f] = jMinType[i];
        if (!jMinPartner.empty()) {
          const int q = jMinPartner[i];
          g.partner[f] = (q >= 0 && q < NI) ? q : -1;
        }
      } else if (j == nj - 1) {
        g.owner[f] = (NJ - 1) * NI + i;
        g.boundary[f] = jMaxType;
      } else {
        g.owner[f] = (j - 1) * NI + i;
        g.neighbour[f] = j * NI + i;
      }
    }
  }
  for (int i = 0; i < ni; ++i) {
    for (int j = 0; j < NJ; ++j) {
      const std::size_t f = jFaces + static_cast<std::size_t>(i) * NJ + j;
      faceNodeA[f] = j * ni + i;
      faceNodeB[f] = (j + 1) * ni + i;
      if (i == 0) {
        g.owner[f] = j * NI;
        g.boundary[f] = iMinType;
      } else if (i == ni - 1) {
        g.owner[f] = j * NI + NI - 1;
        g.boundary[f] = iMaxType;
      } else {
        g.owner[f] = j * NI + i - 1;
        g.neighbour[f] = j * NI + i;
      }
    }
  }

  // Cells: anticlockwise corners, shoelace area and first-moment centroid.
  g.cellArea.assign(cells, 0.0);
  g.centroid.assign(2 * cells, 0.0);
  for (int j = 0; j < NJ; ++j) {
    for (int i = 0; i < NI; ++i) {
      const P2 q[4] = {node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)};
      double twice = 0.0, cx = 0.0, cy = 0.0;
      for (int k = 0; k < 4; ++k) {
        const P2 a = q[k], b = q[(k + 1) % 4];
        const double w = crossp(a, b);
        twice += w;
        cx += (a.x + b.x) * w;
        cy += (a.y + b.y) * w;
      }
      const std::size_t c = static_cast<std::size_t>(j) * NI + i;
      g.cellArea[c] = 0.5 * twice;
      P2 centre;
      if (std::abs(twice) > 0.0) {
        centre = P2{cx / (3.0 * twice), cy / (3.0 * twice)};
      } else {
        centre = (q[0] + q[1] + q[2] + q[3]) * 0.25;
      }
      g.centroid[2 * c] = centre.x;
      g.centroid[2 * c + 1] = centre.y;
    }
  }

  // Faces: centre, length, unit normal out of the owner.
  g.faceCentre.assign(2 * faces, 0.0);
  g.faceNormal.assign(2 * faces, 0.0);
  g.faceArea.assign(faces, 0.0);
  for (std::size_t f = 0; f < faces; ++f) {
    const P2 a{g.nodes[2 * faceNodeA[f]], g.nodes[2 * faceNodeA[f] + 1]};
    const P2 b{g.nodes[2 * faceNodeB[f]], g.nodes[2 * faceNodeB[f] + 1]};
    const P2 tangent = b - a;
    const double len = lenp(tangent);
    const P2 mid = (a + b) * 0.5;
    g.faceCentre[2 * f] = mid.x;
    g.faceCentre[2 * f + 1] = mid.y;
    g.faceArea[f] = len;
    P2 normal{0.0, 0.0};
    if (len > 0.0) {
      if (f < jFaces) {
        const int j = static_cast<int>(f / static_cast<std::size_t>(NI));
        normal = (j == 0) ? quarterRight(tangent) : quarterLeft(tangent);
      } else {
        const int i = static_cast<int>((f - jFaces) / static_cast<std::size_t>(NJ));
        normal = (i == 0) ? quarterLeft(tangent) : quarterRight(tangent);
      }
      normal = normal * (1.0 / len);
    }
    g.faceNormal[2 * f] = normal.x;
    g.faceNormal[2 * f + 1] = normal.y;
  }
  double total = 0.0;
  for (double a : g.cellArea) total += a;
  g.totalArea = total;
  return ok();
}

Status makeCGrid(const char* designation, const cfd_cgrid_options& o, HostMesh* out) {
  Naca naca;
  if (Status s = parseNaca(designation, &naca); s != CFD_OK) return s;
  if (o.surface_points < 8) return fail(CFD_INVALID_ARGUMENT, "surfacePoints must be at least 8");
  if (o.wake_points < 2) return fail(CFD_INVALID_ARGUMENT, "wakePoints must be at least 2");
  if (o.normal_points < 3) return fail(CFD_INVALID_ARGUMENT, "normalPoints must be at least 3");
  if (!(o.upstream_chords > 0.5) || !(o.downstream_chords > 0.5) || !(o.vertical_chords > 0.5)) {
    return fail(CFD_INVALID_ARGUMENT, "domain extents must each be more than half a chord");
  }
  if (!(o.first_layer_height > 0.0) || o.first_layer_height > 0.1) {
    return fail(CFD_INVALID_ARGUMENT, "firstLayerHeight must lie in (0, 0.1] chords");
  }
  if (o.surface_points > 100000) return fail(CFD_INVALID_ARGUMENT, "surfacePoints must be at most 100000");
  const double chord = 1.0;

  P2 trailing;
  std::vector<P2> wall = nacaContour(naca, o.surface_points, &trailing);
  std::reverse(wall.begin(), wall.end());  // clockwise: the wall normal is a left turn

  const int wallNodes = static_cast<int>(wall.size());
  const int wakeNodes = o.wake_points;
  const int ni = 2 * wakeNodes + wallNodes;
  const int nj = o.normal_points;
  const int firstWall = wakeNodes;
  const int lastWall = wakeNodes + wallNodes - 1;

  const double xTE = trailing.x;
  const double wakeLength = o.downstream_chords * chord;
  const double teSpacing = std::max(distp(wall[0], wall[1]), 1e-9 * chord);
  const std::vector<double> innerWake = graded(teSpacing, wakeLength, wakeNodes);
  const double outerSpacing = wakeLength / (2.0 * static_cast<double>(wakeNodes));
  const std::vector<double> outerWake = graded(outerSpacing, wakeLength, wakeNodes);
  const double halfHeight = o.vertical_chords * chord;
  const double noseRadius = xTE + o.upstream_chords * chord;

  std::vector<P2> inner(ni), outer(ni);
  for (int i = 0; i < wakeNodes; ++i) {
    const double x = xTE + innerWake[wakeNodes - i] * wakeLength;
    const double xo = xTE + outerWake[wakeNodes - i] * wakeLength;
    inner[i] = P2{x, 0.0};
    outer[i] = P2{xo, -halfHeight};
    inner[ni - 1 - i] = P2{x, 0.0};
    outer[ni - 1 - i] = P2{xo, halfHeight};
  }
  for (int k = 0; k < wallNodes; ++k) {
    inner[firstWall + k] = wall[k];
    const double phi = std::numbers::pi * static_cast<double>(k) / static_cast<double>(wallNodes - 1);
    outer[firstWall + k] = P2{xTE - noseRadius * std::sin(phi), -halfHeight * std::cos(phi)};
  }

  // Wall-normal directions along the inner curve, then smoothing passes with
  // the two outflow ends held.
  std::vector<P2> dir(ni);
  for (int i = 0; i < ni; ++i) {
    P2 t;
    if (i == 0) t = inner[1] - inner[0];
    else if (i == ni - 1) t = inner[i] - inner[i - 1];
    else t = inner[i + 1] - inner[i - 1];
    dir[i] = quarterLeft(unit(t));
  }
  for (int pass = 0; pass < o.normal_smoothing_passes; ++pass) {
    std::vector<P2> next = dir;
    for (int i = 1; i < ni - 1; ++i) next[i] = unit(dir[i - 1] + dir[i] * 2.0 + dir[i + 1]);
    dir.swap(next);
  }

  // Depth of the wall-normal zone: capped by 0.3/curvature where the inner
  // curve is concave, then a forward/backward sweep bounding its growth.
  std::vector<double> curvature(ni, 0.0);
  for (int i = 1; i + 1 < ni; ++i) {
    const P2 back = inner[i] - inner[i - 1];
    const P2 fwd = inner[i + 1] - inner[i];
    const double lb = lenp(back), lf = lenp(fwd);
    if (lb <= 0.0 || lf <= 0.0) continue;
    const P2 tb = back * (1.0 / lb), tf = fwd * (1.0 / lf);
    curvature[i] = std::atan2(crossp(tb, tf), dotp(tb, tf)) / (0.5 * (lb + lf));
  }
  const double zoneCap = o.normal_blend_length * chord;
  std::vector<double> zone(ni, zoneCap);
  for (int i = 0; i < ni; ++i) {
    if (curvature[i] > 0.0) zone[i] = std::min(zoneCap, 0.3 / curvature[i]);
  }
  for (int pass = 0; pass < 2; ++pass) {
    for (int i = 1; i < ni; ++i) zone[i] = std::min(zone[i], zone[i - 1] + 0.25 * distp(inner[i], inner[i - 1]));
    for (int i = ni - 2; i >= 0; --i) zone[i] = std::min(zone[i], zone[i + 1] + 0.25 * distp(inner[i], inner[i + 1]));
  }

  // March each grid line from the wall to its far-field node, turning at a
  // smooth-step rate in log distance.
  const double firstLayer = o.first_layer_height * chord;
  const double orthoZone = 5.0 * firstLayer;
  std::vector<double> xy(2 * static_cast<std::size_t>(ni) * nj);
  for (int i = 0; i < ni; ++i) {
    const P2 start = inner[i];
    const P2 span = outer[i] - start;
    const double reachMax = lenp(span);
    const P2 straight = unit(span);
    const P2 n0 = dir[i];
    const double turn = std::atan2(crossp(n0, straight), dotp(n0, straight));
    const double needSpan = std::max(1.5, 2.5 * std::abs(turn));
    const double outerBlend = std::max(zone[i], 1e-9 * chord);
    const double innerBlend = std::min(orthoZone, outerBlend * std::exp(-needSpan));
    const double logSpan = std::log(outerBlend / innerBlend);
    const std::vector<double> t = graded(firstLayer, reachMax, nj - 1);
    for (int j = 0; j < nj; ++j) {
      const double reach = t[j] * reachMax;
      double w = 1.0;
      if (reach <= innerBlend) {
        w = 0.0;
      } else if (reach < outerBlend) {
        const double s = std::clamp(std::log(reach / innerBlend) / logSpan, 0.0, 1.0);
        w = s * s * (3.0 - 2.0 * s);
      }
      const double ang = w * turn;
      const double sn = std::sin(ang), cs = std::cos(ang);
      const P2 d{n0.x * cs - n0.y * sn, n0.x * sn + n0.y * cs};
      const P2 at = start + d * reach;
      const std::size_t k = static_cast<std::size_t>(j) * ni + i;
      xy[2 * k] = at.x;
      xy[2 * k + 1] = at.y;
    }
  }

  std::vector<int> jMin(ni - 1, CFD_FACE_WALL), partner(ni - 1, -1);
  for (int k = 0; k < ni - 1; ++k) {
    if (!(k >= firstWall && k < lastWall)) {
      jMin[k] = CFD_FACE_WAKECUT;
      partner[k] = ni - 2 - k;
    }
  }
  return buildBlock(ni, nj, std::move(xy), jMin, CFD_FACE_FARFIELD, CFD_FACE_OUTLET,
                    CFD_FACE_OUTLET, partner, out);
}

Status makeBox(double ox, double oy, double length, double height, int cx, int cy, int grading,
               double firstCell, int left, int right, int lower, int upper, HostMesh* out) {
  if (cx < 1 || cy < 1) return fail(CFD_INVALID_ARGUMENT, "a box needs at least one cell per direction");
  if (!std::isfinite(length) || length <= 0.0 || !std::isfinite(height) || height <= 0.0) {
    return fail(CFD_INVALID_ARGUMENT, "box extents must be positive and finite");
  }
  if (grading != 0 && (!(firstCell > 0.0) || firstCell >= 0.5)) {
    return fail(CFD_INVALID_ARGUMENT, "firstCellHeight must lie in (0, 0.5)");
  }
  const std::vector<double> xf = evenStations(cx);
  std::vector<double> yf;
  if (grading == 0) yf = evenStations(cy);
  else if (grading == 1) yf = graded(firstCell, 1.0, cy);
  else yf = gradedBothEnds(firstCell, 1.0, cy);
  const int ni = cx + 1, nj = cy + 1;
  std::vector<double> xy;
  xy.reserve(2 * static_cast<std::size_t>(ni) * nj);
  for (int j = 0; j < nj; ++j) {
    const double y = oy + height * yf[j];
    for (int i = 0; i < ni; ++i) {
      xy.push_back(ox + length * xf[i]);
      xy.push_back(y);
    }
  }
  std::vector<int> jMin(ni - 1, lower);
  return buildBlock(ni, nj, std::move(xy), jMin, upper, left, right, {}, out);
}

}  // namespace cfdb

// ---- C ABI -----------------------------------------------------------------

struct cfd_mesh_t {
  cfdb::HostMesh mesh;
};

extern "C" {

void cfd_default_cgrid_options(cfd_cgrid_options* o) {
  o->upstream_chords = 12.0;
  o->downstream_chords = 25.0;
  o->vertical_chords = 12.0;
  o->surface_points = 160;
  o->wake_points = 56;
  o->normal_points = 72;
  o->first_layer_height = 3e-4;
  o->normal_blend_length = 0.06;
  o->normal_smoothing_passes = 6;
}

cfd_status cfd_mesh_cgrid(const char* designation, const cfd_cgrid_options* options, cfd_mesh* out) {
  if (out == nullptr || designation == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  cfd_cgrid_options o;
  if (options != nullptr) o = *options; else cfd_default_cgrid_options(&o);
  auto* m = new cfd_mesh_t;
  if (cfdb::Status s = cfdb::makeCGrid(designation, o, &m->mesh); s != CFD_OK) {
    delete m;
    return s;
  }
  *out = m;
  return CFD_OK;
}

cfd_status cfd_mesh_box(double ox, double oy, double length, double height, int cx, int cy,
                        int grading, double firstCell, int left, int right, int lower, int upper,
                        cfd_mesh* out) {
  if (out == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  auto* m = new cfd_mesh_t;
  if (cfdb::Status s = cfdb::makeBox(ox, oy, length, height, cx, cy, grading, firstCell, left,
                                     right, lower, upper, &m->mesh);
      s != CFD_OK) {
    delete m;
    return s;
  }
  *out = m;
  return CFD_OK;
}

cfd_status cfd_mesh_describe(cfd_mesh m, cfd_mesh_desc* d) {
  if (m == nullptr || d == nullptr) return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  cfdb::describe(m->mesh, d);
  return CFD_OK;
}

const double* cfd_mesh_nodes(cfd_mesh m) { return (m == nullptr) ? nullptr : m->mesh.nodes.data(); }

cfd_status cfd_mesh_face_conditions(cfd_mesh m, double speed, double alphaDeg, int* kind,
                                    double* velocity, double* pressure) {
  if (m == nullptr || kind == nullptr || velocity == nullptr || pressure == nullptr) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "null argument");
  }
  if (!std::isfinite(speed) || speed <= 0.0) return cfdb::fail(CFD_INVALID_ARGUMENT, "freestream speed must be positive");
  if (!std::isfinite(alphaDeg) || std::abs(alphaDeg) > 90.0) {
    return cfdb::fail(CFD_INVALID_ARGUMENT, "angle of attack must lie within +/-90 degrees");
  }
  // FreestreamConditions::velocity (Freestream.cpp:11-14).
  const double alpha = alphaDeg * std::numbers::pi / 180.0;
  const double ux = speed * std::cos(alpha), uy = speed * std::sin(alpha);
  const cfdb::HostMesh& g = m->mesh;
  for (int f = 0; f < g.faces; ++f) {
    int k = CFD_BC_INTERNAL;
    switch (g.boundary[f]) {
      case CFD_FACE_WALL: k = CFD_BC_NOSLIP_WALL; break;
      case CFD_FACE_FARFIELD: k = CFD_BC_FARFIELD; break;
      case CFD_FACE_OUTLET: k = CFD_BC_OUTLET; break;
      default: k = CFD_BC_INTERNAL; break;
    }
    kind[f] = k;
    pressure[f] = 0.0;
    velocity[2 * f] = (k == CFD_BC_NOSLIP_WALL) ? 0.0 : ux;
    velocity[2 * f + 1] = (k == CFD_BC_NOSLIP_WALL) ? 0.0 : uy;
  }
  return CFD_OK;
}

void cfd_mesh_free(cfd_mesh m) { delete m; }

}  // extern "C"
