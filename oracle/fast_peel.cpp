// CPU baseline: a dependency-free restatement of the reference's finite
// precision `fast-bvh-peel` (test and benchmark infrastructure only; the
// product never links it).
//
// Follows, in the reference checkout:
//   src/fast_peel.cpp:26-104   integer side/area, ring cleanup with convex-hull
//                              repair, area and one-cell-ribbon rejection
//   src/fast_peel.cpp:152-315  scene import on a 2^bits grid (here from arrays
//                              instead of JSON), near clip, depth plane fit,
//                              window clip, mesh contour topology
//   src/fast_peel.cpp:316-456  grid boxes, split with rounded constructions,
//                              separating axes, cut with the binary64 tie band
//   src/fast_peel.cpp:457-623  conforming mesh and the FastPolicy predicates
//   src/peel_common.h:20-460   median-split BVH (leaf <= 4), contour topology,
//                              whole-source classification, near-first query
//                              with rank-mask pruning, mesh noding and the
//                              all-layer scheduler
// Boost small_vector and nlohmann::json are replaced by std::vector and plain
// structs, OpenMP by a std::thread dynamic-schedule loop.  Timing covers the extraction (classification, every layer's
// clipping and meshing), as the reference's `algorithm_seconds` does
// (fast_peel.cpp:659-664); import, projection and topology are excluded.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <numeric>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

// Dynamic-schedule parallel loop over [0, n) in chunks (the reference uses
// OpenMP `schedule(dynamic, chunk)`; this image ships no OpenMP runtime).
template <class Fn>
void parallel_for(int64_t n, int threads, int64_t chunk, Fn &&fn) {
  if (threads <= 1 || n <= chunk) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (int64_t begin; (begin = next.fetch_add(chunk)) < n;)
      for (int64_t i = begin, end = std::min(n, begin + chunk); i < end; ++i) fn(i);
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
}

struct Point {
  int32_t x = 0, y = 0;
  bool operator==(Point b) const { return x == b.x && y == b.y; }
  bool operator!=(Point b) const { return !(*this == b); }
  bool operator<(Point b) const { return x == b.x ? y < b.y : x < b.x; }
};
using Ring = std::vector<Point>;
using V3 = std::array<double, 3>;

int64_t side(Point a, Point b, Point p) {
  return int64_t(b.x - a.x) * (p.y - a.y) - int64_t(b.y - a.y) * (p.x - a.x);
}
int64_t area2(const Ring &r) {
  int64_t a = 0;
  for (size_t j = 1; j + 1 < r.size(); ++j) a += side(r[0], r[j], r[j + 1]);
  return a;
}

struct Counts {
  uint64_t candidates = 0, nodes = 0, cuts = 0, rejected = 0, repairs = 0, collapsed = 0,
           ties = 0;
};

// Remove repeats, repair non-convex rounding with a monotone-chain hull, drop
// polygons of at most one grid cell of area and one-cell-wide ribbons.
void clean(Ring &r, Counts &c) {
  r.erase(std::unique(r.begin(), r.end()), r.end());
  if (r.size() > 1 && r.front() == r.back()) r.pop_back();
  if (r.size() < 3) {
    if (!r.empty()) ++c.collapsed;
    r.clear();
    return;
  }
  bool convex = true;
  for (size_t i = 0; i < r.size() && convex; ++i)
    if (side(r[i], r[(i + 1) % r.size()], r[(i + 2) % r.size()]) < 0) convex = false;
  if (!convex) {
    ++c.repairs;
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    Ring hull;
    for (Point p : r) {
      while (hull.size() > 1 && side(hull[hull.size() - 2], hull.back(), p) <= 0) hull.pop_back();
      hull.push_back(p);
    }
    size_t lower = hull.size();
    for (auto it = r.rbegin() + 1; it != r.rend(); ++it) {
      while (hull.size() > lower && side(hull[hull.size() - 2], hull.back(), *it) <= 0)
        hull.pop_back();
      hull.push_back(*it);
    }
    hull.pop_back();
    r = std::move(hull);
  }
  if (r.size() < 3 || area2(r) <= 2) {
    ++c.collapsed;
    r.clear();
    return;
  }
  for (size_t i = 0; i < r.size(); ++i) {
    Point a = r[i], b = r[(i + 1) % r.size()];
    int64_t threshold = 2 * (int64_t(std::abs(b.x - a.x)) + std::abs(b.y - a.y));
    if (threshold == 0) continue;
    int64_t widest = 0;
    for (Point p : r) widest = std::max(widest, side(a, b, p));
    if (widest <= threshold) {
      ++c.collapsed;
      r.clear();
      return;
    }
  }
}

template <class V, class F>
std::vector<V> clip_float(const std::vector<V> &p, F f) {
  std::vector<V> out;
  for (size_t i = 0; i < p.size(); ++i) {
    V a = p[i], b = p[(i + 1) % p.size()];
    double da = f(a), db = f(b);
    if (da >= 0) out.push_back(a);
    if ((da < 0 && db > 0) || (da > 0 && db < 0)) {
      double t = da / (da - db);
      V q;
      for (size_t k = 0; k < q.size(); ++k) q[k] = a[k] + t * (b[k] - a[k]);
      out.push_back(q);
    }
  }
  return out;
}

struct Source {
  int id;
  std::array<double, 3> score;
  Ring initial;
};

struct Scene {
  bool perspective = false;
  int bits = 30;
  double near = 0.01;
  std::vector<Source> sources;
  std::vector<std::array<Point, 2>> contours;
  bool resolved = true;
  int collapsed = 0;
};

// Scene import from arrays (fast_peel.cpp:152-315) with the contour topology
// of peel_common.h:88-124.
Scene read(const double *V, const int *F, int64_t nf, const double *camera, const double *st,
           int bits, bool resolved) {
  Scene s;
  s.bits = bits;
  s.resolved = resolved;
  s.perspective = st[4] != 0.0;
  s.near = st[5];
  const double grid = double(int64_t(1) << bits);
  const double w[4] = {st[0], st[1], st[2], st[3]};
  struct Incident {
    int direction, facing;
    std::array<Point, 2> projected;
  };
  std::map<V3, int> vertex_ids;
  std::map<std::pair<int, int>, std::vector<Incident>> edges;
  for (int64_t f = 0; f < nf; ++f) {
    std::vector<V3> vertices;
    std::array<int, 3> conn{};
    bool clipped = false;
    for (int k = 0; k < 3; ++k) {
      const double *p = V + 3 * int64_t(F[3 * f + k]);
      V3 world{p[0], p[1], p[2]};
      if (resolved) conn[k] = vertex_ids.emplace(world, int(vertex_ids.size())).first->second;
      V3 c;
      for (int r = 0; r < 3; ++r)
        c[r] = camera[4 * r] * p[0] + camera[4 * r + 1] * p[1] + camera[4 * r + 2] * p[2] +
               camera[4 * r + 3];
      vertices.push_back(c);
      clipped |= s.perspective && c[2] < s.near;
    }
    if (s.perspective) vertices = clip_float(vertices, [&](V3 v) { return v[2] - s.near; });
    if (vertices.size() < 3) {
      ++s.collapsed;
      continue;
    }
    std::vector<std::array<double, 2>> p;
    std::vector<double> depths;
    for (auto v : vertices) {
      double q = s.perspective ? 1 / v[2] : 1;
      p.push_back({(v[0] * q - w[0]) * grid / (w[2] - w[0]), (v[1] * q - w[1]) * grid / (w[3] - w[1])});
      depths.push_back(s.perspective ? -q : v[2]);
    }
    size_t k = 2;
    double det = 0;
    for (; k < p.size(); ++k) {
      det = (p[1][0] - p[0][0]) * (p[k][1] - p[0][1]) - (p[1][1] - p[0][1]) * (p[k][0] - p[0][0]);
      if (det != 0) break;
    }
    if (k == p.size()) {
      ++s.collapsed;
      continue;
    }
    double x1 = p[1][0] - p[0][0], y1 = p[1][1] - p[0][1], x2 = p[k][0] - p[0][0],
           y2 = p[k][1] - p[0][1];
    Source src;
    src.id = int(f);
    src.score = {((depths[1] - depths[0]) * y2 - (depths[k] - depths[0]) * y1) / det,
                 (x1 * (depths[k] - depths[0]) - x2 * (depths[1] - depths[0])) / det, 0};
    src.score[2] = depths[0] - src.score[0] * p[0][0] - src.score[1] * p[0][1];
    for (double v : src.score)
      if (!std::isfinite(v)) throw std::runtime_error("Unrepresentable depth plane");
    for (auto v : p) clipped |= v[0] < 0 || v[0] > grid || v[1] < 0 || v[1] > grid;
    std::array<Point, 3> original{};
    if (!clipped)
      for (int i = 0; i < 3; ++i)
        original[i] = {int32_t(std::llround(p[i][0])), int32_t(std::llround(p[i][1]))};
    for (int axis = 0; axis < 2; ++axis) {
      p = clip_float(p, [&](std::array<double, 2> v) { return v[axis]; });
      p = clip_float(p, [&](std::array<double, 2> v) { return grid - v[axis]; });
    }
    for (auto v : p)
      src.initial.push_back({int32_t(std::llround(std::clamp(v[0], 0., grid))),
                             int32_t(std::llround(std::clamp(v[1], 0., grid)))});
    if (src.initial.size() > 2 && area2(src.initial) < 0)
      std::reverse(src.initial.begin(), src.initial.end());
    Counts c;
    clean(src.initial, c);
    if (src.initial.empty()) {
      ++s.collapsed;
      continue;
    }
    if (resolved) {
      if (clipped) {
        for (size_t i = 0; i < src.initial.size(); ++i)
          s.contours.push_back({src.initial[i], src.initial[(i + 1) % src.initial.size()]});
      } else {
        for (int i = 0; i < 3; ++i) {
          int a = conn[i], b = conn[(i + 1) % 3];
          edges[{std::min(a, b), std::max(a, b)}].push_back(
              {a < b ? 1 : -1, det > 0 ? 1 : -1, {original[i], original[(i + 1) % 3]}});
        }
      }
    }
    s.sources.push_back(std::move(src));
  }
  for (auto &e : edges) {
    auto &g = e.second;
    if (g.size() == 2 && g[0].direction != g[1].direction && g[0].facing == g[1].facing) continue;
    s.contours.push_back(g.front().projected);
  }
  return s;
}

struct Box {
  int32_t lo[2] = {INT32_MAX, INT32_MAX}, hi[2] = {INT32_MIN, INT32_MIN};
  double near = INFINITY, far = -INFINITY;
  int64_t center(int axis) const { return int64_t(lo[axis]) + hi[axis]; }
  void add(Point p) {
    lo[0] = std::min(lo[0], p.x);
    lo[1] = std::min(lo[1], p.y);
    hi[0] = std::max(hi[0], p.x);
    hi[1] = std::max(hi[1], p.y);
  }
  void add(const Box &b) {
    for (int k = 0; k < 2; ++k) {
      lo[k] = std::min(lo[k], b.lo[k]);
      hi[k] = std::max(hi[k], b.hi[k]);
    }
    near = std::min(near, b.near);
    far = std::max(far, b.far);
  }
};
bool overlap(const Box &a, const Box &b) {
  return a.lo[0] <= b.hi[0] && b.lo[0] <= a.hi[0] && a.lo[1] <= b.hi[1] && b.lo[1] <= a.hi[1];
}
Box bound(const Ring &r) {
  Box b;
  for (Point p : r) b.add(p);
  return b;
}

// Median-split hierarchy over boxes, leaves of at most four items.
struct BVH {
  struct Node {
    Box box;
    int left = -1, right = -1, begin = 0, end = 0;
  };
  std::vector<Node> nodes;
  std::vector<int> ids, max_rank;
  const std::vector<Box> &boxes;
  explicit BVH(const std::vector<Box> &b) : boxes(b) {
    ids.resize(b.size());
    std::iota(ids.begin(), ids.end(), 0);
    nodes.reserve(2 * b.size() / 4 + 2);
    if (!b.empty()) build(0, int(b.size()));
  }
  int build(int begin, int end) {
    int i = int(nodes.size());
    nodes.emplace_back();
    Box box;
    for (int j = begin; j < end; ++j) box.add(boxes[ids[j]]);
    nodes[i].box = box;
    if (end - begin <= 4) {
      nodes[i].begin = begin;
      nodes[i].end = end;
      return i;
    }
    int axis = box.hi[1] - box.lo[1] > box.hi[0] - box.lo[0], mid = (begin + end) / 2;
    std::nth_element(ids.begin() + begin, ids.begin() + mid, ids.begin() + end, [&](int a, int b) {
      auto x = boxes[a].center(axis), y = boxes[b].center(axis);
      return x == y ? a < b : x < y;
    });
    int a = build(begin, mid), b = build(mid, end);
    nodes[i].left = a;
    nodes[i].right = b;
    return i;
  }
  void summarize_ranks(const std::vector<int> &ranks) {
    max_rank.assign(nodes.size(), -1);
    for (size_t i = nodes.size(); i-- > 0;) {
      const Node &n = nodes[i];
      if (n.left < 0) {
        for (int j = n.begin; j < n.end; ++j) max_rank[i] = std::max(max_rank[i], ranks[ids[j]]);
      } else {
        max_rank[i] = std::max(max_rank[n.left], max_rank[n.right]);
      }
    }
  }
  template <class Fn>
  void visit(const Box &b, Fn &&f, int i = 0) const {
    if (nodes.empty() || !overlap(nodes[i].box, b)) return;
    const Node &n = nodes[i];
    if (n.left < 0) {
      for (int j = n.begin; j < n.end; ++j)
        if (overlap(boxes[ids[j]], b)) f(ids[j]);
    } else {
      visit(b, f, n.left);
      visit(b, f, n.right);
    }
  }
};

template <class Fn>
std::pair<Ring, Ring> split(const Ring &r, Fn eval, Counts &c) {
  double d[64];
  std::vector<double> big;
  double *dv = r.size() <= 64 ? d : (big.resize(r.size()), big.data());
  bool pos = false, neg = false;
  for (size_t i = 0; i < r.size(); ++i) {
    dv[i] = eval(r[i]);
    pos |= dv[i] > 0;
    neg |= dv[i] < 0;
  }
  if (!neg) return {r, {}};
  if (!pos) return {{}, r};
  Ring in, out;
  for (size_t i = 0; i < r.size(); ++i) {
    size_t j = (i + 1) % r.size();
    if (dv[i] >= 0) in.push_back(r[i]);
    if (dv[i] <= 0) out.push_back(r[i]);
    if ((dv[i] > 0 && dv[j] < 0) || (dv[i] < 0 && dv[j] > 0)) {
      double t = dv[i] / (dv[i] - dv[j]);
      Point p{int32_t(std::llround(r[i].x + t * (r[j].x - r[i].x))),
              int32_t(std::llround(r[i].y + t * (r[j].y - r[i].y)))};
      in.push_back(p);
      out.push_back(p);
    }
  }
  clean(in, c);
  clean(out, c);
  return {std::move(in), std::move(out)};
}

bool separated(const Ring &a, const Ring &b) {
  for (size_t i = 0; i < a.size(); ++i) {
    bool pos = false;
    for (Point p : b)
      if (side(a[i], a[(i + 1) % a.size()], p) > 0) {
        pos = true;
        break;
      }
    if (!pos) return true;
  }
  return false;
}

double at(const std::array<double, 3> &s, Point p) { return s[0] * p.x + s[1] * p.y + s[2]; }

struct Patch {
  int source;
  Ring points;
};
struct Work {
  std::vector<Ring> visible, hidden;
  Counts counts;
};
struct Face {
  int source;
  std::array<std::array<double, 2>, 3> points;
};

void cut(Work &w, const Ring &candidate, const Source &target, const Source &other) {
  Box cb = bound(candidate);
  std::vector<Ring> next;
  std::array<double, 3> d;
  for (int k = 0; k < 3; ++k) d[k] = target.score[k] - other.score[k];
  double tol = 32 * std::numeric_limits<double>::epsilon() *
               std::max({std::abs(target.score[2]), std::abs(other.score[2]), 1e-300});
  for (auto &p : w.visible) {
    if (!overlap(bound(p), cb) || separated(p, candidate) || separated(candidate, p)) {
      next.push_back(std::move(p));
      continue;
    }
    bool pos = false, neg = false;
    for (Point v : p) {
      double x = at(d, v);
      pos |= x > tol;
      neg |= x < -tol;
    }
    if (!pos && !neg) {
      ++w.counts.ties;
      pos = target.id > other.id;
    }
    if (!pos) {
      next.push_back(std::move(p));
      continue;
    }
    Ring inside = p;
    std::vector<Ring> outside;
    if (neg) {
      auto parts = split(inside, [&](Point v) { return at(d, v); }, w.counts);
      inside = std::move(parts.first);
      if (!parts.second.empty()) outside.push_back(std::move(parts.second));
    }
    for (size_t j = 0; j < candidate.size() && !inside.empty(); ++j) {
      Point a = candidate[j], b = candidate[(j + 1) % candidate.size()];
      auto parts = split(inside, [&](Point v) { return double(side(a, b, v)); }, w.counts);
      inside = std::move(parts.first);
      if (!parts.second.empty()) outside.push_back(std::move(parts.second));
    }
    if (inside.empty()) {
      next.push_back(std::move(p));
    } else {
      ++w.counts.cuts;
      w.hidden.push_back(std::move(inside));
      for (auto &v : outside) next.push_back(std::move(v));
    }
  }
  w.visible = std::move(next);
}

struct Policy {
  const Scene &s;
  std::vector<Box> boxes(const std::vector<Patch> &patches) const {
    std::vector<Box> out(patches.size());
    for (size_t i = 0; i < patches.size(); ++i) {
      out[i] = bound(patches[i].points);
      const auto &score = s.sources[patches[i].source].score;
      for (Point p : patches[i].points) {
        double z = at(score, p);
        double err = 64 * std::numeric_limits<double>::epsilon() *
                     (std::abs(score[0] * p.x) + std::abs(score[1] * p.y) + std::abs(score[2]));
        out[i].near = std::min(out[i].near, z - err);
        out[i].far = std::max(out[i].far, z + err);
      }
    }
    return out;
  }
  bool touches_contour(int i, int j) const {
    const auto &src = s.sources[i];
    auto e = s.contours[j];
    for (size_t k = 0; k < src.initial.size(); ++k) {
      Point a = src.initial[k], b = src.initial[(k + 1) % src.initial.size()];
      int64_t margin = 4 * (int64_t(std::abs(b.x - a.x)) + std::abs(b.y - a.y));
      if (side(a, b, e[0]) < -margin && side(a, b, e[1]) < -margin) return false;
    }
    bool positive = false, negative = false;
    int64_t margin = 4 * (int64_t(std::abs(e[1].x - e[0].x)) + std::abs(e[1].y - e[0].y));
    for (Point p : src.initial) {
      int64_t v = side(e[0], e[1], p);
      positive |= v >= -margin;
      negative |= v <= margin;
    }
    return positive && negative;
  }
  int ray_order(int i, int j, int64_t px, int64_t py) const {
    const auto &src = s.sources[i];
    double target = src.score[0] * (px / 3.) + src.score[1] * (py / 3.) + src.score[2];
    const auto &other = s.sources[j];
    bool edge = false;
    for (size_t k = 0; k < other.initial.size(); ++k) {
      Point a = other.initial[k], b = other.initial[(k + 1) % other.initial.size()];
      int64_t cross = int64_t(b.x - a.x) * (py - 3 * int64_t(a.y)) -
                      int64_t(b.y - a.y) * (px - 3 * int64_t(a.x));
      if (cross < 0) return 0;
      edge |= cross == 0;
    }
    if (edge) return -1;
    double z = other.score[0] * (px / 3.) + other.score[1] * (py / 3.) + other.score[2];
    double tol = 64 * std::numeric_limits<double>::epsilon() *
                 std::max({std::abs(z), std::abs(target), 1e-300});
    if (std::abs(z - target) <= tol) return -1;
    return int(z < target);
  }
};

std::vector<int> classify(const Policy &p, const BVH &sources, int threads) {
  const Scene &s = p.s;
  std::vector<int> ranks(sources.boxes.size(), -1);
  if (!s.resolved) return ranks;
  std::vector<Box> edges;
  for (auto e : s.contours) {
    Box b;
    b.add(e[0]);
    b.add(e[1]);
    for (int d = 0; d < 2; ++d) {
      b.lo[d] -= 4;
      b.hi[d] += 4;
    }
    edges.push_back(b);
  }
  BVH contours(edges);
  parallel_for(int64_t(ranks.size()), threads, 64, [&](int64_t i) {
    bool boundary = false;
    contours.visit(sources.boxes[i], [&](int j) {
      if (!boundary) boundary = p.touches_contour(int(i), j);
    });
    if (boundary || s.sources[i].initial.size() != 3) return;
    int64_t px = 0, py = 0;
    for (Point q : s.sources[i].initial) {
      px += q.x;
      py += q.y;
    }
    Box point;
    point.add(Point{int32_t(px / 3), int32_t(py / 3)});
    point.add(Point{int32_t((px + 2) / 3), int32_t((py + 2) / 3)});
    int rank = 0;
    bool ambiguous = false;
    sources.visit(point, [&](int j) {
      if (j == int(i)) return;
      int hit = p.ray_order(int(i), j, px, py);
      ambiguous |= hit < 0;
      rank += hit > 0;
    });
    if (!ambiguous) ranks[i] = rank;
  });
  return ranks;
}

void query(const Policy &p, const std::vector<Patch> &input, const BVH &tree, const Patch &target,
           const Box &box, Work &w, const std::vector<int> *ranks, int layer, int i = 0) {
  if (w.visible.empty() || tree.nodes.empty()) return;
  const auto &node = tree.nodes[i];
  ++w.counts.nodes;
  if (ranks && !tree.max_rank.empty() && tree.max_rank[i] < layer) return;
  if (!overlap(node.box, box) || node.box.near > box.far) return;
  if (node.left < 0) {
    for (int j = node.begin; j < node.end && !w.visible.empty(); ++j) {
      int c = tree.ids[j];
      if (input[c].source == target.source || (ranks && (*ranks)[c] < layer) ||
          !overlap(tree.boxes[c], box) || tree.boxes[c].near > box.far)
        continue;
      ++w.counts.candidates;
      cut(w, input[c].points, p.s.sources[target.source], p.s.sources[input[c].source]);
    }
  } else {
    int a = node.left, b = node.right;
    if (tree.nodes[a].box.near > tree.nodes[b].box.near) std::swap(a, b);
    query(p, input, tree, target, box, w, ranks, layer, a);
    query(p, input, tree, target, box, w, ranks, layer, b);
  }
}

// Conforming boundary noding and centroid fans (peel_common.h:202-258,
// fast_peel.cpp:457-478).
std::vector<Face> mesh(const std::vector<Patch> &patches, int threads) {
  std::vector<Point> points;
  for (auto &p : patches) points.insert(points.end(), p.points.begin(), p.points.end());
  std::sort(points.begin(), points.end());
  points.erase(std::unique(points.begin(), points.end()), points.end());
  std::vector<Box> boxes(points.size());
  for (size_t i = 0; i < points.size(); ++i) boxes[i].add(points[i]);
  BVH tree(boxes);
  std::vector<std::vector<Face>> output(patches.size());
  parallel_for(int64_t(patches.size()), threads, 32, [&](int64_t k) {
    const auto &patch = patches[k];
    Ring ring;
    for (size_t i = 0; i < patch.points.size(); ++i) {
      Point a = patch.points[i], b = patch.points[(i + 1) % patch.points.size()];
      Box box;
      box.add(a);
      box.add(b);
      Ring along;
      tree.visit(box, [&](int j) {
        Point v = points[j];
        if (v != b && side(a, b, v) == 0) along.push_back(v);
      });
      std::sort(along.begin(), along.end());
      if (b < a) std::reverse(along.begin(), along.end());
      ring.insert(ring.end(), along.begin(), along.end());
    }
    auto pt = [](Point v) { return std::array<double, 2>{double(v.x), double(v.y)}; };
    auto &out = output[k];
    if (ring.size() == 3) {
      out.push_back({patch.source, {pt(ring[0]), pt(ring[1]), pt(ring[2])}});
    } else if (ring.size() > 3) {
      std::array<double, 2> center{};
      for (Point v : ring) {
        center[0] += v.x;
        center[1] += v.y;
      }
      for (auto &v : center) v /= double(ring.size());
      for (size_t i = 0; i < ring.size(); ++i)
        out.push_back({patch.source, {center, pt(ring[i]), pt(ring[(i + 1) % ring.size()])}});
    }
  });
  std::vector<Face> all;
  for (auto &v : output) all.insert(all.end(), v.begin(), v.end());
  return all;
}

struct Totals {
  int64_t layers = 0, patches = 0, faces = 0, residual = 0;
};

// One output region: its layer, the input face it comes from, and its ring
// on the 2^bits grid.
struct Region {
  int layer, face;
  Ring ring;
};

// The all-layer scheduler (peel_common.h:341-460) with the accelerated path.
// With `regions`, every layer's convex regions are also collected.
Totals extract(const Scene &s, int layers, int threads, std::vector<Region> *regions = nullptr) {
  Policy p{s};
  std::vector<Patch> originals;
  for (size_t i = 0; i < s.sources.size(); ++i) originals.push_back({int(i), s.sources[i].initial});
  auto original_boxes = s.resolved ? p.boxes(originals) : std::vector<Box>{};
  BVH original_tree(original_boxes);
  std::vector<int> ranks =
      s.resolved ? classify(p, original_tree, threads) : std::vector<int>(originals.size(), -1);
  if (s.resolved) original_tree.summarize_ranks(ranks);
  std::vector<Patch> residual;
  std::vector<std::vector<int>> direct;
  for (size_t i = 0; i < originals.size(); ++i) {
    if (ranks[i] < 0) {
      residual.push_back(originals[i]);
    } else {
      if (direct.size() <= size_t(ranks[i])) direct.resize(ranks[i] + 1);
      direct[ranks[i]].push_back(int(i));
    }
  }
  Totals t;
  const int limit = layers ? layers : int(originals.size());
  for (int k = 0; k < limit && (!residual.empty() || size_t(k) < direct.size()); ++k) {
    auto boxes = p.boxes(residual);
    BVH tree(boxes);
    std::vector<Work> work(residual.size());
    parallel_for(int64_t(residual.size()), threads, 32, [&](int64_t i) {
      Work &w = work[i];
      const Patch &target = residual[i];
      w.visible.push_back(target.points);
      if (s.resolved) query(p, originals, original_tree, target, boxes[i], w, &ranks, k);
      query(p, residual, tree, target, boxes[i], w, nullptr, 0);
      if (w.visible.empty()) {
        w.hidden.clear();
        w.hidden.push_back(target.points);
        ++w.counts.rejected;
      }
    });
    std::vector<Patch> layer;
    if (size_t(k) < direct.size())
      for (int i : direct[k]) layer.push_back(originals[i]);
    std::vector<Patch> next;
    for (size_t i = 0; i < work.size(); ++i) {
      for (auto &r : work[i].visible) layer.push_back({residual[i].source, std::move(r)});
      for (auto &r : work[i].hidden) next.push_back({residual[i].source, std::move(r)});
    }
    if (layer.empty()) throw std::runtime_error("BVH peeling made no progress");
    if (regions)
      for (const Patch &patch : layer)
        regions->push_back({k, s.sources[patch.source].id, patch.points});
    auto faces = mesh(layer, threads);
    t.layers += 1;
    t.patches += int64_t(layer.size());
    t.faces += int64_t(faces.size());
    residual = std::move(next);
  }
  if (!layers && !residual.empty()) throw std::runtime_error("Peeling exceeded source-count layer limit");
  t.residual = int64_t(residual.size());
  return t;
}

}  // namespace

extern "C" {

// Import once, then time `repeat` extractions.  seconds[repeat] receives each
// extraction's wall time; out[4] = layers, convex patches, triangles, residual
// patches of the last run.  Returns 0, or -1 on an algorithm error.
int fastpeel_run(const double *vertices, const int32_t *faces, int64_t nf, const double *camera,
                 const double *settings, int32_t threads, int32_t repeat, int32_t bits,
                 int32_t resolved, int32_t layers, double *seconds, int64_t *out) {
  try {
    Scene s = read(vertices, faces, nf, camera, settings, bits, resolved != 0);
    Totals t;
    for (int r = 0; r < repeat; ++r) {
      auto start = std::chrono::steady_clock::now();
      t = extract(s, layers, threads);
      seconds[r] = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    }
    out[0] = t.layers;
    out[1] = t.patches;
    out[2] = t.faces;
    out[3] = t.residual;
    return 0;
  } catch (const std::exception &) {
    return -1;
  }
}

// One extraction that also returns its regions: meta[3 * i] = layer, input
// face and vertex count of region i, coords[2 * j] the grid coordinates of
// its vertices (region after region).  out[0..1] receive the region and
// vertex counts; when either exceeds its capacity nothing is written to meta
// or coords and the call returns 1 (call again with larger buffers).  out[2]
// receives the layer count.  Returns 0, 1, or -1 on an algorithm error.
int fastpeel_regions(const double *vertices, const int32_t *faces, int64_t nf,
                     const double *camera, const double *settings, int32_t threads, int32_t bits,
                     int32_t resolved, int32_t layers, int64_t region_capacity,
                     int64_t vertex_capacity, int64_t *meta, int64_t *coords, int64_t *out) {
  try {
    Scene s = read(vertices, faces, nf, camera, settings, bits, resolved != 0);
    std::vector<Region> regions;
    Totals t = extract(s, layers, threads, &regions);
    int64_t count = 0;
    for (const Region &r : regions) count += int64_t(r.ring.size());
    out[0] = int64_t(regions.size());
    out[1] = count;
    out[2] = t.layers;
    if (out[0] > region_capacity || count > vertex_capacity) return 1;
    int64_t j = 0;
    for (size_t i = 0; i < regions.size(); ++i) {
      meta[3 * i] = regions[i].layer;
      meta[3 * i + 1] = regions[i].face;
      meta[3 * i + 2] = int64_t(regions[i].ring.size());
      for (Point v : regions[i].ring) {
        coords[2 * j] = v.x;
        coords[2 * j + 1] = v.y;
        ++j;
      }
    }
    return 0;
  } catch (const std::exception &) {
    return -1;
  }
}

int fastpeel_max_threads(void) {
  unsigned n = std::thread::hardware_concurrency();
  return n ? int(n) : 1;
}

}  // extern "C"
