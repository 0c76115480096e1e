// Sibson (natural-neighbour) coordinates for the drivers' fill of bad points, host code:
// MATLAB's scatteredInterpolant(..., 'natural') is native host code in the reference's
// fill (func/LocalICGN.m:199-220, func_quadtree/LocalICGNQuadtree.m:212-325,
// func_quadtree/Subpb1Quadtree.m:188-254) and so is this.
//
// Watson's construction on a Delaunay triangulation of the source points (the caller's:
// simplices, their neighbours and circumcircles): the query's cavity is the connected set of
// triangles whose circumcircle holds it, starting at the triangle that contains it; walking
// the cavity's boundary ring counter-clockwise, the query's new Voronoi vertices are the
// circumcentres of (q, b_i, b_i+1); the area the query takes from ring vertex b_i is the
// polygon of the two new vertices at b_i and the circumcentres of the cavity triangles at
// b_i in fan order.  The weights are those areas over their sum.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/aldic_b200.h"

namespace {

inline void circumcentre(const double* a, const double* b, const double* c, double* o) {
  const double d = 2.0 * (a[0] * (b[1] - c[1]) + b[0] * (c[1] - a[1]) + c[0] * (a[1] - b[1]));
  const double a2 = a[0] * a[0] + a[1] * a[1], b2 = b[0] * b[0] + b[1] * b[1], c2 = c[0] * c[0] + c[1] * c[1];
  o[0] = (a2 * (b[1] - c[1]) + b2 * (c[1] - a[1]) + c2 * (a[1] - b[1])) / d;
  o[1] = (a2 * (c[0] - b[0]) + b2 * (a[0] - c[0]) + c2 * (b[0] - a[0])) / d;
}

double shoelace(const std::vector<double>& xy) {
  const size_t n = xy.size() / 2;
  if (n < 3) return 0.0;
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const size_t j = (i + 1) % n;
    s += xy[2 * i] * xy[2 * j + 1] - xy[2 * j] * xy[2 * i + 1];
  }
  return 0.5 * std::fabs(s);
}

}  // namespace

int aldic_sibson_weights(int64_t k, const double* P, int64_t ntri, const int32_t* simplices, const int32_t* neighbors,
                         const double* cc, const double* r2, double scale, int64_t m, const double* Q,
                         const int32_t* qsimplex, int32_t cap, int32_t* idx, double* w, int32_t* count) {
  if (k < 3 || ntri < 1 || m < 0 || cap < 3 || !P || !simplices || !neighbors || !cc || !r2 || (m > 0 && (!Q ||
      !qsimplex || !idx || !w || !count)))
    return ALDIC_ERR_ARG;
  const double tol = 1e-10;
  std::vector<int64_t> stamp((size_t)ntri, -1);  // query whose BFS saw the triangle
  std::vector<char> in((size_t)ntri, 0);          // ... and whether it is in that cavity
  std::vector<int64_t> vstamp((size_t)k, -1);
  std::vector<int32_t> nxt((size_t)k), from((size_t)k);
  std::vector<int32_t> cav, stack, ring;
  std::vector<double> newv, poly;
  for (int64_t qi = 0; qi < m; ++qi) {
    const double* q = Q + 2 * qi;
    int32_t* oi = idx + qi * cap;
    double* ow = w + qi * cap;
    const int32_t s = qsimplex[qi];
    if (s < 0 || s >= ntri) {  // outside the hull (or on it): the caller decides
      count[qi] = -2;
      continue;
    }
    // the cavity
    cav.clear();
    stack.assign(1, s);
    stamp[(size_t)s] = qi;
    bool ok = true;
    while (!stack.empty()) {
      const int32_t t = stack.back();
      stack.pop_back();
      const double dx = q[0] - cc[2 * t], dy = q[1] - cc[2 * t + 1];
      const bool inside = dx * dx + dy * dy <= r2[t] * (1 + tol) + (tol * scale) * (tol * scale);
      in[(size_t)t] = inside ? 1 : 0;
      if (!inside) continue;
      cav.push_back(t);
      for (int e = 0; e < 3; ++e) {
        const int32_t u = neighbors[3 * t + e];
        if (u >= 0 && stamp[(size_t)u] != qi) {
          stamp[(size_t)u] = qi;
          stack.push_back(u);
        }
      }
    }
    // the boundary ring, counter-clockwise: one outgoing edge per ring vertex
    int32_t start = -1, nedge = 0;
    for (int32_t t : cav) {
      const int32_t* v = simplices + 3 * t;
      const double* a = P + 2 * v[0];
      const double* b = P + 2 * v[1];
      const double* c = P + 2 * v[2];
      const bool ccw = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]) > 0;
      for (int e = 0; e < 3 && ok; ++e) {
        const int32_t u = neighbors[3 * t + e];
        if (u >= 0 && stamp[(size_t)u] == qi && in[(size_t)u]) continue;
        if (u < 0) {
          ok = false;  // the cavity reaches the hull
          break;
        }
        int32_t p0 = v[(e + 1) % 3], p1 = v[(e + 2) % 3];
        if (!ccw) std::swap(p0, p1);
        if (vstamp[(size_t)p0] == qi) {
          ok = false;  // not a simple ring
          break;
        }
        vstamp[(size_t)p0] = qi;
        nxt[(size_t)p0] = p1;
        from[(size_t)p0] = t;
        start = p0;
        ++nedge;
      }
      if (!ok) break;
    }
    if (!ok || start < 0 || nedge > cap) {
      count[qi] = -1;
      continue;
    }
    ring.clear();
    ring.push_back(start);
    for (;;) {
      const int32_t v = nxt[(size_t)ring.back()];
      if (vstamp[(size_t)v] != qi) {
        ok = false;
        break;
      }
      if (v == start) break;
      ring.push_back(v);
      if ((int32_t)ring.size() > nedge) {
        ok = false;
        break;
      }
    }
    if (!ok || (int32_t)ring.size() != nedge) {
      count[qi] = -1;
      continue;
    }
    const int32_t nr = (int32_t)ring.size();
    newv.assign(2 * (size_t)nr, 0.0);
    for (int32_t i = 0; i < nr; ++i)
      circumcentre(q, P + 2 * ring[i], P + 2 * ring[(i + 1) % nr], &newv[2 * (size_t)i]);
    double tot = 0.0;
    for (int32_t i = 0; i < nr && ok; ++i) {
      const int32_t bi = ring[i], prev = ring[(i + nr - 1) % nr];
      int32_t t = from[(size_t)prev], came = -1;
      const int32_t end = from[(size_t)bi];
      poly.assign(newv.begin() + 2 * (size_t)((i + nr - 1) % nr), newv.begin() + 2 * (size_t)((i + nr - 1) % nr) + 2);
      bool closed = false;
      for (size_t guard = 0; guard <= cav.size(); ++guard) {  // the fan of cavity triangles at bi
        poly.push_back(cc[2 * t]);
        poly.push_back(cc[2 * t + 1]);
        if (t == end) {
          closed = true;
          break;
        }
        const int32_t* v = simplices + 3 * t;
        int32_t step = -1;
        for (int e = 0; e < 3; ++e) {
          if (v[e] == bi) continue;
          const int32_t u = neighbors[3 * t + e];
          if (u >= 0 && stamp[(size_t)u] == qi && in[(size_t)u] && u != came) {
            step = u;
            break;
          }
        }
        if (step < 0) break;
        came = t;
        t = step;
      }
      if (!closed) {
        ok = false;
        break;
      }
      poly.push_back(newv[2 * (size_t)i]);
      poly.push_back(newv[2 * (size_t)i + 1]);
      const double a = shoelace(poly);
      oi[i] = bi;
      ow[i] = a;
      tot += a;
    }
    if (!ok || !(tot > 0.0)) {
      count[qi] = -1;
      continue;
    }
    for (int32_t i = 0; i < nr; ++i) ow[i] /= tot;
    count[qi] = nr;
  }
  return ALDIC_OK;
}
