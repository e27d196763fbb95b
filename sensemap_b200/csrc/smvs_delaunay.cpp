// smvs_delaunay.cpp — 2-D Delaunay triangulation of integer pixel positions
// (host), for the Delaunay initial map (InitDepthMapFromDelaunay,
// patch_match_controller.cc:398-474, which triangulates the projected sparse
// points with CGAL's Delaunay_triangulation_2 over their (u, v) coordinates).
//
// Incremental Bowyer-Watson insertion with an infinite vertex: each point
// removes the triangles whose circumcircle strictly contains it (for a hull
// triangle: the point lies strictly outside its hull edge, or on the edge's
// interior) and is joined to the boundary of that cavity. Predicates are exact
// (64-bit orientation, 128-bit in-circle determinant), so the result is a true
// Delaunay triangulation for any input: unique wherever no four points are
// co-circular; on co-circular points the insertion order (Z-order of the
// positions) decides the diagonal. A point whose position repeats an earlier
// one is skipped, as CGAL returns the existing vertex for it.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <utility>
#include <vector>

#include "../../include/smvs.h"
#include "../../include/smvs_testing.h"

namespace smvs {

namespace {

constexpr int kInf = -1;  // the infinite vertex

struct Tri {
  int v[3];  // counter-clockwise (positive orientation in (x, y)); kInf at most once
  int n[3];  // n[i]: the triangle across the edge opposite v[i]
  bool alive;
};

struct Mesh {
  const int64_t* x;
  const int64_t* y;
  std::vector<Tri> t;
  std::vector<int> stack, cavity, mark;
  int stamp = 0;
  int last = 0;

  int64_t Orient(int a, int b, int c) const {
    return (x[b] - x[a]) * (y[c] - y[a]) - (y[b] - y[a]) * (x[c] - x[a]);
  }
  // > 0 when d lies strictly inside the circumcircle of the counter-clockwise (a, b, c).
  int InCircle(int a, int b, int c, int d) const {
    const __int128 adx = x[a] - x[d], ady = y[a] - y[d];
    const __int128 bdx = x[b] - x[d], bdy = y[b] - y[d];
    const __int128 cdx = x[c] - x[d], cdy = y[c] - y[d];
    const __int128 det = (adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) -
                         (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady) +
                         (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady);
    return det > 0 ? 1 : (det < 0 ? -1 : 0);
  }
  bool Conflict(int ti, int p) const {
    const Tri& T = t[ti];
    int k = -1;
    for (int i = 0; i < 3; ++i)
      if (T.v[i] == kInf) k = i;
    if (k < 0) return InCircle(T.v[0], T.v[1], T.v[2], p) > 0;
    // Hull triangle (a, b, inf): the half-plane left of a -> b, open, plus the
    // open segment ab itself.
    const int a = T.v[(k + 1) % 3], b = T.v[(k + 2) % 3];
    const int64_t o = Orient(a, b, p);
    if (o > 0) return true;
    if (o < 0) return false;
    const int64_t dot = (x[p] - x[a]) * (x[b] - x[a]) + (y[p] - y[a]) * (y[b] - y[a]);
    const int64_t len = (x[b] - x[a]) * (x[b] - x[a]) + (y[b] - y[a]) * (y[b] - y[a]);
    return dot > 0 && dot < len;
  }
  int Add(int a, int b, int c) {
    t.push_back({{a, b, c}, {-1, -1, -1}, true});
    return (int)t.size() - 1;
  }
  // A triangle in conflict with p: walk from the last triangle towards p across
  // edges p lies strictly right of; fall back to a scan of all triangles.
  int Locate(int p) {
    int cur = last;
    if (!t[cur].alive) cur = -1;
    for (int steps = 0; cur >= 0 && steps < (int)t.size() + 8; ++steps) {
      const Tri& T = t[cur];
      bool hull = false;
      for (int i = 0; i < 3; ++i) hull |= (T.v[i] == kInf);
      if (hull) {
        if (Conflict(cur, p)) return cur;
        break;
      }
      int next = -1;
      for (int i = 0; i < 3 && next < 0; ++i) {
        const int a = T.v[(i + 1) % 3], b = T.v[(i + 2) % 3];
        if (Orient(a, b, p) < 0) next = T.n[i];
      }
      if (next < 0) {
        if (Conflict(cur, p)) return cur;
        break;
      }
      cur = next;
    }
    for (int i = (int)t.size() - 1; i >= 0; --i)
      if (t[i].alive && Conflict(i, p)) return i;
    return -1;
  }
  void Insert(int p) {
    const int start = Locate(p);
    if (start < 0) return;  // cannot happen for a new position
    ++stamp;
    cavity.clear();
    stack.assign(1, start);
    mark[start] = stamp;
    while (!stack.empty()) {
      const int c = stack.back();
      stack.pop_back();
      cavity.push_back(c);
      for (int i = 0; i < 3; ++i) {
        const int nb = t[c].n[i];
        if (nb >= 0 && mark[nb] != stamp && Conflict(nb, p)) {
          mark[nb] = stamp;
          stack.push_back(nb);
        }
      }
    }
    // Boundary edges of the cavity, each with the triangle outside it, and the
    // new triangles (edge a -> b, then p), linked to those outside triangles.
    struct Edge { int a, b, out, tri; };
    std::vector<Edge> edges;
    for (int c : cavity) {
      for (int i = 0; i < 3; ++i) {
        const int nb = t[c].n[i];
        if (nb >= 0 && mark[nb] == stamp) continue;
        edges.push_back({t[c].v[(i + 1) % 3], t[c].v[(i + 2) % 3], nb, -1});
      }
    }
    for (int c : cavity) t[c].alive = false;
    for (auto& e : edges) {
      e.tri = Add(e.a, e.b, p);
      if ((int)mark.size() < (int)t.size()) mark.resize(t.size() * 2, 0);
      Tri& T = t[e.tri];
      T.n[2] = e.out;  // across a -> b
      if (e.out >= 0) {
        Tri& O = t[e.out];
        for (int j = 0; j < 3; ++j) {
          const int oa = O.v[(j + 1) % 3], ob = O.v[(j + 2) % 3];
          if (oa == e.b && ob == e.a) O.n[j] = e.tri;
        }
      }
    }
    // Neighbours among the new triangles: triangle (a, b, p) meets the one
    // that starts at b across its edge b -> p (n[0]) and the one that ends at
    // a across p -> a (n[1]).
    for (auto& e : edges)
      for (auto& f : edges) {
        if (f.a == e.b) t[e.tri].n[0] = f.tri;
        if (f.b == e.a) t[e.tri].n[1] = f.tri;
      }
    last = edges.empty() ? last : edges.back().tri;
    for (auto& e : edges) {
      bool hull = (e.a == kInf || e.b == kInf);
      if (!hull) { last = e.tri; break; }
    }
  }
};

}  // namespace

// Triangles (counter-clockwise vertex index triples into xy) of the Delaunay
// triangulation of the n points xy[2i], xy[2i + 1]; fewer than three distinct
// non-collinear points give none.
int DelaunayTriangulate(const int32_t* xy, int n, std::vector<int32_t>& tris) {
  tris.clear();
  if (n < 3) return SMVS_OK;
  std::vector<int64_t> X(n), Y(n);
  for (int i = 0; i < n; ++i) { X[i] = xy[2 * i]; Y[i] = xy[2 * i + 1]; }
  Mesh m;
  m.x = X.data();
  m.y = Y.data();
  // Distinct positions in input order (the first of a repeated position wins).
  std::vector<int> order;
  order.reserve(n);
  {
    std::vector<std::pair<uint64_t, int>> keys(n);
    for (int i = 0; i < n; ++i) keys[i] = {((uint64_t)(uint32_t)xy[2 * i] << 32) | (uint32_t)xy[2 * i + 1], i};
    std::vector<std::pair<uint64_t, int>> sorted = keys;
    std::sort(sorted.begin(), sorted.end());
    std::vector<char> dup(n, 0);
    for (int i = 1; i < n; ++i)
      if (sorted[i].first == sorted[i - 1].first) dup[sorted[i].second] = 1;
    for (int i = 0; i < n; ++i)
      if (!dup[i]) order.push_back(i);
  }
  // Insertion in Z-order of the positions (ties by input order): each walk to
  // the next point's triangle stays short. The order only decides the
  // diagonal of co-circular points.
  {
    auto spread = [](uint64_t v) {
      v &= 0xffffffffull;
      v = (v | (v << 16)) & 0x0000ffff0000ffffull;
      v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
      v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
      v = (v | (v << 2)) & 0x3333333333333333ull;
      v = (v | (v << 1)) & 0x5555555555555555ull;
      return v;
    };
    int64_t mx = 0, my = 0;
    for (int i : order) { mx = std::min(mx, X[i]); my = std::min(my, Y[i]); }
    std::vector<std::pair<uint64_t, int>> z;
    z.reserve(order.size());
    for (int i : order) z.push_back({spread((uint64_t)(X[i] - mx)) | (spread((uint64_t)(Y[i] - my)) << 1), i});
    std::sort(z.begin(), z.end());
    for (size_t k = 0; k < z.size(); ++k) order[k] = z[k].second;
  }
  // The first triangle: the first point, the next one, and the first point
  // not collinear with them.
  if (order.size() < 3) return SMVS_OK;
  const int a = order[0], b = order[1];
  int ci = -1;
  for (size_t k = 2; k < order.size(); ++k)
    if (m.Orient(a, b, order[k]) != 0) { ci = (int)k; break; }
  if (ci < 0) return SMVS_OK;
  const int c = order[ci];
  int p0 = a, p1 = b, p2 = c;
  if (m.Orient(p0, p1, p2) < 0) std::swap(p1, p2);
  m.t.reserve(order.size() * 6 + 16);
  m.mark.assign(order.size() * 6 + 16, 0);
  const int f = m.Add(p0, p1, p2);
  const int h0 = m.Add(p2, p1, kInf);  // across p1 -> p2
  const int h1 = m.Add(p0, p2, kInf);  // across p2 -> p0
  const int h2 = m.Add(p1, p0, kInf);  // across p0 -> p1
  m.t[f].n[0] = h0; m.t[f].n[1] = h1; m.t[f].n[2] = h2;
  // Hull triangle (a, b, inf): n[2] = across a -> b (the finite one); n[0]
  // across b -> inf, n[1] across inf -> a.
  m.t[h0].n[2] = f; m.t[h0].n[0] = h2; m.t[h0].n[1] = h1;
  m.t[h1].n[2] = f; m.t[h1].n[0] = h0; m.t[h1].n[1] = h2;
  m.t[h2].n[2] = f; m.t[h2].n[0] = h1; m.t[h2].n[1] = h0;
  m.last = f;
  for (size_t k = 2; k < order.size(); ++k)
    if ((int)k != ci) m.Insert(order[k]);
  for (const Tri& T : m.t) {
    if (!T.alive || T.v[0] == kInf || T.v[1] == kInf || T.v[2] == kInf) continue;
    tris.push_back(T.v[0]);
    tris.push_back(T.v[1]);
    tris.push_back(T.v[2]);
  }
  return SMVS_OK;
}

}  // namespace smvs

extern "C" int smvs_test_delaunay(const int32_t* xy, int n, int32_t* tris, int capacity, int* num_tris) {
  if (!num_tris || n < 0 || (n && !xy)) return SMVS_EINVAL;
  std::vector<int32_t> out;
  const int st = smvs::DelaunayTriangulate(xy, n, out);
  if (st) return st;
  *num_tris = (int)(out.size() / 3);
  if (tris && capacity > 0) {
    const int m = *num_tris < capacity ? *num_tris : capacity;
    for (int i = 0; i < 3 * m; ++i) tris[i] = out[i];
  }
  return SMVS_OK;
}
