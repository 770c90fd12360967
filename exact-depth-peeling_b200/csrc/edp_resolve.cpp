// Exact intersection splitting of a binary64 triangle scene, on the host
// cores (include/edp_resolve.h).  The peelers take resolved meshes: no two
// triangles may cross.  This is the preprocessing step of
// src/resolve_intersections.cpp:19-105 in the reference (CGAL autorefine with
// provenance), built on this library's own construction, which the Python
// module peel_b200/resolve.py also implements (for rational inputs):
//
// 1. Candidate pairs: boxes padded by 1e-9 (1 + max |coordinate|) that
//    overlap, found by a sweep in increasing padded-box x (ties by index).
// 2. Each pair's exact contact: the points of each triangle on the other's
//    plane, intersected along the planes' common line (a segment, a point or
//    nothing); coplanar pairs give their touching points and are an error
//    when they overlap with positive area.
// 3. A triangle whose interior a contact segment crosses is cut by the
//    segment's supporting line (in pair order, one cut per distinct line), so
//    every piece is convex.
// 4. Every point created by a contact or a cut is inserted into every piece
//    edge it lies strictly inside, so pieces along a crossing share edges.
// 5. A piece that is still a triangle is written as is; any other is written
//    as a fan from a corner with no inserted point beside it, or else around
//    the centroid of its first three corners.
//
// Arithmetic.  Input coordinates are binary64, so every one is an integer
// multiple of 2^-E for the scene's finest exponent E: the resolver works on
// the integers x 2^E, exactly, with homogeneous points (X, Y, Z, W), W > 0.
// A point made by a construction is the intersection of two lines through
// input vertices or contact points (never of lines through earlier
// constructions), which bounds the size of every number.  Outputs are the
// exact homogeneous points and their correctly rounded binary64 values.
#include "../../include/edp_resolve.h"

#include <algorithm>
#include <array>
#include <exception>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

namespace {

using u64 = uint64_t;
using u128 = unsigned __int128;

// Numbers above this many 64-bit limbs are refused (the caller falls back to
// the arbitrary-precision Python construction).
constexpr int kMaxLimbs = 1024;
struct TooLarge {};
struct BadInput {};
struct CoplanarOverlap {
  int64_t a, b;
};

// ---------------------------------------------------------------- integers

// Signed integer: magnitude in little-endian 64-bit limbs with a small
// inline buffer (most input-level numbers fit in it).
class Int {
 public:
  Int() = default;
  explicit Int(int64_t v) {
    if (v != 0) {
      reserve(1);
      neg_ = v < 0;
      p_[0] = neg_ ? u64(0) - u64(v) : u64(v);
      n_ = 1;
    }
  }
  Int(const Int &o) { assign(o); }
  Int(Int &&o) noexcept { take(std::move(o)); }
  Int &operator=(const Int &o) {
    if (this != &o) assign(o);
    return *this;
  }
  Int &operator=(Int &&o) noexcept {
    if (this != &o) {
      release();
      take(std::move(o));
    }
    return *this;
  }
  ~Int() { release(); }

  int size() const { return n_; }
  bool negative() const { return neg_; }
  int sign() const { return n_ == 0 ? 0 : neg_ ? -1 : 1; }
  const u64 *limbs() const { return p_; }
  u64 *limbs() { return p_; }

  // Room for `n` limbs (contents kept up to size()).
  void reserve(int n) {
    if (n <= cap_) return;
    if (n > kMaxLimbs) throw TooLarge{};
    int cap = std::max(n, 2 * cap_);
    u64 *q = new u64[cap];
    std::memcpy(q, p_, sizeof(u64) * n_);
    if (p_ != inline_) delete[] p_;
    p_ = q;
    cap_ = cap;
  }
  void set_size(int n, bool neg) {
    n_ = n;
    while (n_ > 0 && p_[n_ - 1] == 0) --n_;
    neg_ = n_ > 0 && neg;
  }
  void negate() { neg_ = n_ > 0 && !neg_; }
  int bits() const {
    if (n_ == 0) return 0;
    return 64 * (n_ - 1) + (64 - __builtin_clzll(p_[n_ - 1]));
  }

 private:
  static constexpr int kInline = 4;
  void assign(const Int &o) {
    n_ = 0;
    reserve(o.n_);
    std::memcpy(p_, o.p_, sizeof(u64) * o.n_);
    n_ = o.n_;
    neg_ = o.neg_;
  }
  void take(Int &&o) {
    if (o.p_ == o.inline_) {
      p_ = inline_;
      cap_ = kInline;
      std::memcpy(inline_, o.inline_, sizeof(u64) * o.n_);
    } else {
      p_ = o.p_;
      cap_ = o.cap_;
      o.p_ = o.inline_;
      o.cap_ = kInline;
    }
    n_ = o.n_;
    neg_ = o.neg_;
    o.n_ = 0;
    o.neg_ = false;
  }
  void release() {
    if (p_ != inline_) delete[] p_;
    p_ = inline_;
    cap_ = kInline;
  }
  int n_ = 0;
  bool neg_ = false;
  int cap_ = kInline;
  u64 *p_ = inline_;
  u64 inline_[kInline];
};

int cmp_mag(const Int &a, const Int &b) {
  if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
  for (int i = a.size() - 1; i >= 0; --i)
    if (a.limbs()[i] != b.limbs()[i]) return a.limbs()[i] < b.limbs()[i] ? -1 : 1;
  return 0;
}

// |a| + |b| with the given sign.
Int add_mag(const Int &a, const Int &b, bool neg) {
  const Int &x = a.size() >= b.size() ? a : b, &y = a.size() >= b.size() ? b : a;
  Int r;
  r.reserve(x.size() + 1);
  u64 carry = 0;
  for (int i = 0; i < x.size(); ++i) {
    u128 s = u128(x.limbs()[i]) + (i < y.size() ? y.limbs()[i] : 0) + carry;
    r.limbs()[i] = u64(s);
    carry = u64(s >> 64);
  }
  r.limbs()[x.size()] = carry;
  r.set_size(x.size() + 1, neg);
  return r;
}

// |a| - |b| (|a| >= |b|) with the given sign.
Int sub_mag(const Int &a, const Int &b, bool neg) {
  Int r;
  r.reserve(a.size());
  u64 borrow = 0;
  for (int i = 0; i < a.size(); ++i) {
    const u64 bi = i < b.size() ? b.limbs()[i] : 0;
    const u64 d = a.limbs()[i] - bi - borrow;
    borrow = (a.limbs()[i] < bi || (a.limbs()[i] == bi && borrow)) ? 1 : 0;
    r.limbs()[i] = d;
  }
  r.set_size(a.size(), neg);
  return r;
}

Int operator+(const Int &a, const Int &b) {
  if (a.sign() == 0) return b;
  if (b.sign() == 0) return a;
  if (a.negative() == b.negative()) return add_mag(a, b, a.negative());
  const int c = cmp_mag(a, b);
  if (c == 0) return Int();
  return c > 0 ? sub_mag(a, b, a.negative()) : sub_mag(b, a, b.negative());
}

Int operator-(const Int &a, const Int &b) {
  if (b.sign() == 0) return a;
  Int nb = b;
  nb.negate();
  return a + nb;
}

Int operator*(const Int &a, const Int &b) {
  if (a.sign() == 0 || b.sign() == 0) return Int();
  const int n = a.size() + b.size();
  Int r;
  r.reserve(n);
  u64 *out = r.limbs();
  std::memset(out, 0, sizeof(u64) * n);
  for (int i = 0; i < a.size(); ++i) {
    u64 carry = 0;
    const u128 ai = a.limbs()[i];
    for (int j = 0; j < b.size(); ++j) {
      u128 t = ai * b.limbs()[j] + out[i + j] + carry;
      out[i + j] = u64(t);
      carry = u64(t >> 64);
    }
    out[i + b.size()] = carry;
  }
  r.set_size(n, a.negative() != b.negative());
  return r;
}

int cmp(const Int &a, const Int &b) {
  if (a.sign() != b.sign()) return a.sign() < b.sign() ? -1 : 1;
  const int m = cmp_mag(a, b);
  return a.negative() ? -m : m;
}

bool operator!=(const Int &a, const Int &b) { return cmp(a, b) != 0; }

// a * 2^k (k >= 0).
Int shl(const Int &a, int k) {
  if (a.sign() == 0 || k == 0) return a;
  const int words = k / 64, bits = k % 64;
  Int r;
  r.reserve(a.size() + words + 1);
  u64 *out = r.limbs();
  std::memset(out, 0, sizeof(u64) * (a.size() + words + 1));
  for (int i = 0; i < a.size(); ++i) {
    out[i + words] |= a.limbs()[i] << bits;
    if (bits) out[i + words + 1] |= a.limbs()[i] >> (64 - bits);
  }
  r.set_size(a.size() + words + 1, a.negative());
  return r;
}

// Hexadecimal text of a (with a leading '-' when negative).
std::string hex(const Int &a) {
  if (a.sign() == 0) return "0";
  static const char *digits = "0123456789abcdef";
  std::string s;
  for (int i = a.size() - 1; i >= 0; --i)
    for (int k = 60; k >= 0; k -= 4) s.push_back(digits[(a.limbs()[i] >> k) & 15]);
  const size_t first = s.find_first_not_of('0');
  s = s.substr(first);
  return a.negative() ? "-" + s : s;
}

// In place: r -= t (|r| >= |t|, both non-negative).
void sub_in_place(Int &r, const Int &t) {
  u64 borrow = 0;
  u64 *a = r.limbs();
  const u64 *b = t.limbs();
  for (int i = 0; i < r.size(); ++i) {
    const u64 bi = i < t.size() ? b[i] : 0;
    const u64 d = a[i] - bi - borrow;
    borrow = (a[i] < bi || (a[i] == bi && borrow)) ? 1 : 0;
    a[i] = d;
  }
  r.set_size(r.size(), false);
}

// In place: r >>= 1 (r non-negative).
void shr1_in_place(Int &r) {
  u64 *a = r.limbs();
  for (int i = 0; i < r.size(); ++i) a[i] = (a[i] >> 1) | (i + 1 < r.size() ? a[i + 1] << 63 : 0);
  r.set_size(r.size(), false);
}

// The leading 64 bits of |a| (a != 0) as m 2^e, m in [2^63, 2^64), truncated:
// |a| = m 2^e (1 + t) with 0 <= t < 2^-63.
long double leading(const Int &a, int &e) {
  const int n = a.size(), top = a.bits() - 64 * (n - 1);  // bits in the top limb
  const u64 hi = a.limbs()[n - 1];
  u64 m = top == 64 ? hi : (hi << (64 - top)) | (n > 1 ? a.limbs()[n - 2] >> top : 0);
  e = a.bits() - 64;
  return static_cast<long double>(m);
}

// Correctly rounded binary64 value of num / (den * 2^scale), den > 0 (round
// to nearest, ties to even); results outside the normal range are refused.
// Most values are settled by the leading bits: the quotient of the truncated
// leading 64 bits (x87 extended precision) is within 2^-61 of the exact
// value, and when both ends of that interval round to the same binary64 value
// it is the answer; otherwise binary long division decides.
double to_double(const Int &num, const Int &den, int scale) {
  if (num.sign() == 0) return 0.0;
  if (den.size() == 1 && den.limbs()[0] == 1 && num.bits() <= 53) {
    // An integer of at most 53 bits: exact in binary64.
    const double v = std::ldexp(double(num.limbs()[0]), -scale);
    if (!(v >= 0x1p-1022) || !std::isfinite(v)) throw TooLarge{};
    return num.negative() ? -v : v;
  }
  {
    int en, ed;
    const long double mn = leading(num, en), md = leading(den, ed);
    const long double q = std::ldexp(mn / md, en - ed - scale);
    const long double eps = 0x1p-60L;
    const double lo = static_cast<double>(q * (1.0L - eps));
    const double hi = static_cast<double>(q * (1.0L + eps));
    if (lo == hi && std::isfinite(lo) && lo >= 0x1p-1022) return num.negative() ? -lo : lo;
  }
  Int a = num;
  if (a.negative()) a.negate();
  // Quotient a 2^s / den with 55 or 56 bits, by binary long division.
  const int s = 55 - (a.bits() - den.bits());
  Int rem = s >= 0 ? shl(a, s) : a;
  const Int d = s >= 0 ? den : shl(den, -s);
  const int qbits = rem.bits() - d.bits() + 1;
  Int t = shl(d, qbits - 1);
  u64 q = 0;
  for (int b = qbits - 1; b >= 0; --b) {
    if (cmp_mag(rem, t) >= 0) {
      sub_in_place(rem, t);
      q |= u64(1) << b;
    }
    shr1_in_place(t);
  }
  const bool sticky = rem.sign() != 0;
  // Keep 53 bits of q and round.
  const int extra = (64 - __builtin_clzll(q)) - 53;
  u64 mant = q >> extra;
  const u64 half = u64(1) << (extra - 1);
  const u64 low = q & ((u64(1) << extra) - 1);
  if (low > half || (low == half && (sticky || (mant & 1)))) ++mant;
  const double v = std::ldexp(double(mant), extra - s - scale);
  if (!(v >= 0x1p-1022) || !std::isfinite(v)) throw TooLarge{};
  return num.negative() ? -v : v;
}

}  // namespace

namespace {

// ---------------------------------------------------------------- points

// Homogeneous point (X, Y, Z) / W with W > 0, in units of 2^-E.
struct Pt {
  Int c[4];  // x, y, z, w
  const Int &w() const { return c[3]; }
};

Pt make_pt(Int x, Int y, Int z, Int w) {
  if (w.sign() < 0) {
    x.negate();
    y.negate();
    z.negate();
    w.negate();
  }
  Pt p;
  p.c[0] = std::move(x);
  p.c[1] = std::move(y);
  p.c[2] = std::move(z);
  p.c[3] = std::move(w);
  return p;
}

bool same_point(const Pt &a, const Pt &b) {
  for (int k = 0; k < 3; ++k)
    if (a.c[k] * b.c[3] != b.c[k] * a.c[3]) return false;
  return true;
}

// Sign of a_k / a_w - b_k / b_w.
int cmp_coord(const Pt &a, const Pt &b, int k) { return cmp(a.c[k] * b.c[3], b.c[k] * a.c[3]); }

// Lexicographic order of the rational coordinates (x, then y, then z).
int cmp_lex(const Pt &a, const Pt &b) {
  for (int k = 0; k < 3; ++k) {
    const int c = cmp_coord(a, b, k);
    if (c) return c;
  }
  return 0;
}

// Orientation determinant of three homogeneous points projected on axes
// (i, j): its sign is the sign of the 2D orientation (every W > 0).
Int orient_h(const Pt &a, const Pt &b, const Pt &c, int i, int j) {
  const Int &ax = a.c[i], &ay = a.c[j], &aw = a.c[3];
  const Int &bx = b.c[i], &by = b.c[j], &bw = b.c[3];
  const Int &cx = c.c[i], &cy = c.c[j], &cw = c.c[3];
  return ax * (by * cw - bw * cy) - ay * (bx * cw - bw * cx) + aw * (bx * cy - by * cx);
}

// Three points on one line (all three axis-plane projections degenerate).
bool collinear(const Pt &u, const Pt &w, const Pt &x) {
  return orient_h(u, w, x, 0, 1).sign() == 0 && orient_h(u, w, x, 1, 2).sign() == 0 &&
         orient_h(u, w, x, 0, 2).sign() == 0;
}

// x strictly between u and w on the segment u-w (u != w): collinear, and
// strictly between them along an axis where they differ.
bool on_open_segment(const Pt &x, const Pt &u, const Pt &w, int &axis) {
  if (!collinear(u, w, x)) return false;
  for (int k = 0; k < 3; ++k) {
    const int d = cmp_coord(w, u, k);
    if (d == 0) continue;
    axis = k;
    const int a = cmp_coord(x, u, k), b = cmp_coord(w, x, k);
    return a == d && b == d;
  }
  return false;
}

// Correctly rounded binary64 coordinates of a point.
void round_pt(const Pt &p, int scale, double out[3]) {
  for (int k = 0; k < 3; ++k) out[k] = to_double(p.c[k], p.c[3], scale);
}

// ---------------------------------------------------------------- faces

// Exact form of one input triangle: vertices (W = 1), normal
// (v1 - v0) x (v2 - v0), offset normal . v0, and the dominant axis of the
// normal (the first of the largest magnitude).
struct FaceX {
  Pt v[3];
  Int n[3];
  Int off;
  bool degenerate = false;
  int dom = 2;
};

Int scaled(double x, int scale) {
  // x * 2^scale is an integer for every input coordinate.
  if (x == 0.0) return Int();
  int e;
  const double m = std::frexp(std::fabs(x), &e);  // |x| = m 2^e, m in [0.5, 1)
  u64 mant = u64(std::ldexp(m, 53));  // |x| = mant 2^(e - 53)
  const int tz = __builtin_ctzll(mant);
  mant >>= tz;
  const int shift = e - 53 + tz + scale;  // >= 0 by the choice of scale
  if (shift < 0) throw BadInput{};
  Int r = shl(Int{int64_t(mant)}, shift);
  if (x < 0) r.negate();
  return r;
}

FaceX face_exact(const double *t, int scale) {
  FaceX f;
  for (int k = 0; k < 3; ++k)
    f.v[k] = make_pt(scaled(t[3 * k], scale), scaled(t[3 * k + 1], scale),
                     scaled(t[3 * k + 2], scale), Int(1));
  Int d1[3], d2[3];
  for (int k = 0; k < 3; ++k) {
    d1[k] = f.v[1].c[k] - f.v[0].c[k];
    d2[k] = f.v[2].c[k] - f.v[0].c[k];
  }
  f.n[0] = d1[1] * d2[2] - d1[2] * d2[1];
  f.n[1] = d1[2] * d2[0] - d1[0] * d2[2];
  f.n[2] = d1[0] * d2[1] - d1[1] * d2[0];
  f.off = f.n[0] * f.v[0].c[0] + f.n[1] * f.v[0].c[1] + f.n[2] * f.v[0].c[2];
  f.degenerate = f.n[0].sign() == 0 && f.n[1].sign() == 0 && f.n[2].sign() == 0;
  int best = 0;
  for (int k = 1; k < 3; ++k)
    if (cmp_mag(f.n[k], f.n[best]) > 0) best = k;
  f.dom = best;
  return f;
}

bool is_vertex(const FaceX &f, const Pt &p) {
  for (int k = 0; k < 3; ++k)
    if (same_point(f.v[k], p)) return true;
  return false;
}

// The plane of `f` at p, times p's W (same sign as the plane value).
Int plane_value(const FaceX &f, const Pt &p) {
  return f.n[0] * p.c[0] + f.n[1] * p.c[1] + f.n[2] * p.c[2] - f.off * p.c[3];
}

// Axes of the projection that drops the dominant normal axis.
void plane_axes(int dom, int &i, int &j) {
  i = dom == 0 ? 1 : 0;
  j = dom == 2 ? 1 : 2;
}

// The segment p-r lies on the line of one of f's edges.
bool on_boundary(const FaceX &f, const Pt &p, const Pt &r) {
  for (int k = 0; k < 3; ++k) {
    const Pt &a = f.v[k], &b = f.v[(k + 1) % 3];
    if (collinear(a, b, p) && collinear(a, b, r)) return true;
  }
  return false;
}

// Points of `face` on `other`'s plane.  Returns 0 (strictly one side), 1
// (coplanar) or 2 (the distinct points, input vertices first, then edge
// crossings, in edge order).
int plane_section(const FaceX &face, const FaceX &other, std::vector<Pt> &out) {
  Int val[3];
  int pos = 0, neg = 0, zero = 0;
  for (int k = 0; k < 3; ++k) {
    val[k] = plane_value(other, face.v[k]);
    const int s = val[k].sign();
    pos += s > 0;
    neg += s < 0;
    zero += s == 0;
  }
  if (pos == 3 || neg == 3) return 0;
  if (zero == 3) return 1;
  out.clear();
  std::vector<Pt> points;
  for (int k = 0; k < 3; ++k)
    if (val[k].sign() == 0) points.push_back(face.v[k]);
  for (int k = 0; k < 3; ++k) {
    const Int &a = val[k], &b = val[(k + 1) % 3];
    if ((a.sign() < 0 && b.sign() > 0) || (b.sign() < 0 && a.sign() > 0)) {
      // (w a - u b) / (a - b) for the edge u -> w with plane values a, b.
      const Pt &u = face.v[k], &w = face.v[(k + 1) % 3];
      points.push_back(make_pt(w.c[0] * a - u.c[0] * b, w.c[1] * a - u.c[1] * b,
                               w.c[2] * a - u.c[2] * b, a - b));
    }
  }
  for (auto &p : points) {
    bool seen = false;
    for (auto &q : out) seen = seen || same_point(p, q);
    if (!seen) out.push_back(std::move(p));
  }
  return 2;
}

}  // namespace

namespace {

// ---------------------------------------------------------------- contacts

// The point on line a-b where the 2D orientation (axes i, j) against the
// line p-r vanishes (the lines are not parallel).
Pt intersect(const Pt &a, const Pt &b, const Pt &p, const Pt &r, int i, int j) {
  const Int da = orient_h(p, r, a, i, j), db = orient_h(p, r, b, i, j);
  return make_pt(b.c[0] * da - a.c[0] * db, b.c[1] * da - a.c[1] * db,
                 b.c[2] * da - a.c[2] * db, b.c[3] * da - a.c[3] * db);
}

// A polygon vertex and the line of its outgoing edge (two base points).
struct Vtx {
  Pt p;
  int la, lb;
};

// Touching points of two coplanar triangles; throws CoplanarOverlap when they
// overlap with positive area.  fb is clipped by fa's three edge half-planes
// in the projection that drops fa's dominant normal axis.
void coplanar_contact(const FaceX &fa, const FaceX &fb, int64_t ia, int64_t ib,
                      std::vector<Pt> &found) {
  int i, j;
  plane_axes(fa.dom, i, j);
  const Pt *base[6] = {&fa.v[0], &fa.v[1], &fa.v[2], &fb.v[0], &fb.v[1], &fb.v[2]};
  const int sa = orient_h(fa.v[0], fa.v[1], fa.v[2], i, j).sign() > 0 ? 1 : -1;
  std::vector<Vtx> poly;
  for (int k = 0; k < 3; ++k) poly.push_back({fb.v[k], 3 + k, 3 + (k + 1) % 3});
  for (int k = 0; k < 3; ++k) {
    const int ca = k, cb = (k + 1) % 3;
    const Pt &A = fa.v[ca], &B = fa.v[cb];
    std::vector<int> side(poly.size());
    for (size_t m = 0; m < poly.size(); ++m) side[m] = sa * orient_h(A, B, poly[m].p, i, j).sign();
    std::vector<Vtx> out;
    const size_t n = poly.size();
    for (size_t m = 0; m < n; ++m) {
      const Vtx &P = poly[m];
      const int sp = side[m], sq = side[(m + 1) % n];
      const bool cross = (sp > 0 && sq < 0) || (sq > 0 && sp < 0);
      if (sp >= 0) {
        if (sq >= 0 || cross) out.push_back({P.p, P.la, P.lb});
        else out.push_back({P.p, ca, cb});
      }
      if (cross) {
        Pt x = intersect(*base[P.la], *base[P.lb], A, B, i, j);
        if (sq > 0) out.push_back({std::move(x), P.la, P.lb});
        else out.push_back({std::move(x), ca, cb});
      }
    }
    poly = std::move(out);
    if (poly.empty()) return;
  }
  for (size_t m = 1; m + 1 < poly.size(); ++m)
    if (orient_h(poly[0].p, poly[m].p, poly[m + 1].p, i, j).sign() != 0)
      throw CoplanarOverlap{ia, ib};
  for (auto &v : poly) found.push_back(std::move(v.p));
}

// Exact contact of two non-degenerate triangles: the points (in `found`) and,
// when the contact is a segment, has_segment with its ends p (lower along
// fa.n x fb.n) and r.
struct Contact {
  std::vector<Pt> found;
  bool has_segment = false;
  Pt p, r;
};

void contact(const FaceX &fa, const FaceX &fb, int64_t ia, int64_t ib, Contact &out) {
  std::vector<Pt> sa, sb;
  const int ka = plane_section(fb, fa, sa);
  if (ka == 0) return;
  if (ka == 1) {
    coplanar_contact(fa, fb, ia, ib, out.found);
    return;
  }
  if (plane_section(fa, fb, sb) == 0) return;
  const Int line[3] = {fa.n[1] * fb.n[2] - fa.n[2] * fb.n[1], fa.n[2] * fb.n[0] - fa.n[0] * fb.n[2],
                       fa.n[0] * fb.n[1] - fa.n[1] * fb.n[0]};
  auto key = [&](const Pt &p) { return line[0] * p.c[0] + line[1] * p.c[1] + line[2] * p.c[2]; };
  // Order along the line (then lexicographic, as tuples compare).
  auto order = [&](const Pt &a, const Pt &b) {
    const int c = cmp(key(a) * b.c[3], key(b) * a.c[3]);
    return c ? c : cmp_lex(a, b);
  };
  auto lowest = [&](const std::vector<Pt> &v) {
    size_t best = 0;
    for (size_t m = 1; m < v.size(); ++m)
      if (order(v[m], v[best]) < 0) best = m;
    return best;
  };
  auto highest = [&](const std::vector<Pt> &v) {
    size_t best = 0;
    for (size_t m = 1; m < v.size(); ++m)
      if (order(v[m], v[best]) > 0) best = m;
    return best;
  };
  const Pt &a0 = sa[lowest(sa)], &b0 = sb[lowest(sb)];
  const Pt &a1 = sa[highest(sa)], &b1 = sb[highest(sb)];
  const Pt &lo = order(a0, b0) >= 0 ? a0 : b0;  // max, the first on ties
  const Pt &hi = order(a1, b1) <= 0 ? a1 : b1;  // min, the first on ties
  const int c = cmp(key(lo) * hi.c[3], key(hi) * lo.c[3]);
  if (c > 0) return;
  out.found.push_back(lo);
  if (c == 0) return;
  out.found.push_back(hi);
  out.has_segment = true;
  out.p = lo;
  out.r = hi;
}

// ---------------------------------------------------------------- pieces

// Sign of the side of v against the directed line p -> r in f's plane, as
// (r - p) x (v - p) . normal would give it: the projected orientation times
// the sign that the projection gives the normal's dominant component.
int plane_side(const FaceX &f, const Pt &p, const Pt &r, const Pt &v) {
  int i, j;
  plane_axes(f.dom, i, j);
  const int s = orient_h(p, r, v, i, j).sign();
  return s * f.n[f.dom].sign() * (f.dom == 1 ? -1 : 1);
}

bool has_area(const FaceX &f, const std::vector<Vtx> &poly) {
  int i, j;
  plane_axes(f.dom, i, j);
  for (size_t m = 1; m + 1 < poly.size(); ++m)
    if (orient_h(poly[0].p, poly[m].p, poly[m + 1].p, i, j).sign() != 0) return true;
  return false;
}

// Both sides of the convex polygon `poly` about the line through base[cp],
// base[cr] (parts without area dropped); new vertices are intersections of
// that line with the line of the edge they split.
void split(const FaceX &f, const std::vector<const Pt *> &base, int cp, int cr,
           std::vector<Vtx> &&poly, std::vector<std::vector<Vtx>> &parts) {
  const Pt &P = *base[cp], &R = *base[cr];
  const size_t n = poly.size();
  std::vector<int> side(n);
  bool any_pos = false, any_neg = false;
  for (size_t m = 0; m < n; ++m) {
    side[m] = plane_side(f, P, R, poly[m].p);
    any_pos = any_pos || side[m] > 0;
    any_neg = any_neg || side[m] < 0;
  }
  if (!any_pos || !any_neg) {
    parts.push_back(std::move(poly));
    return;
  }
  int i, j;
  plane_axes(f.dom, i, j);
  std::vector<Vtx> left, right;
  for (size_t m = 0; m < n; ++m) {
    const Vtx &u = poly[m];
    const int su = side[m], sw = side[(m + 1) % n];
    const bool cross = (su > 0 && sw < 0) || (sw > 0 && su < 0);
    if (su >= 0) left.push_back({u.p, (sw >= 0 || cross) ? u.la : cp, (sw >= 0 || cross) ? u.lb : cr});
    if (su <= 0) right.push_back({u.p, (sw <= 0 || cross) ? u.la : cp, (sw <= 0 || cross) ? u.lb : cr});
    if (cross) {
      Pt x = intersect(*base[u.la], *base[u.lb], P, R, i, j);
      left.push_back({x, sw > 0 ? u.la : cp, sw > 0 ? u.lb : cr});
      right.push_back({std::move(x), sw < 0 ? u.la : cp, sw < 0 ? u.lb : cr});
    }
  }
  for (auto *part : {&left, &right})
    if (part->size() >= 3 && has_area(f, *part)) parts.push_back(std::move(*part));
}

}  // namespace

namespace {

// ---------------------------------------------------------------- threads

// Calls f(begin, end) over [0, n) in chunks on `threads` threads; the first
// exception thrown by any chunk is rethrown after all threads finished.
template <class F>
void parallel_chunks(int64_t n, int threads, int64_t chunk, F f) {
  if (n <= 0) return;
  std::atomic<int64_t> next{0};
  std::vector<std::exception_ptr> errors(threads);
  auto work = [&](int t) {
    try {
      for (;;) {
        const int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        f(b, std::min(n, b + chunk));
      }
    } catch (...) {
      errors[t] = std::current_exception();
      next.store(n);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  for (auto &e : errors)
    if (e) std::rethrow_exception(e);
}

// ---------------------------------------------------------------- driver

struct PairResult {
  int64_t pair, fa, fb;  // pair index, input triangles
  std::vector<Pt> points;  // contact points that are not vertices of both triangles
  bool segment = false, cut_a = false, cut_b = false;
  Pt p, r;
};

// Python-compatible binary64 pre-test (shared vertices only): for each pair,
// true when the two triangles can meet only in vertices they share exactly
// (some vertex of one clearly off the other's plane, every such vertex on one
// side, the others vertices of the first); the margin 1e-12 M^3 is far above
// the rounding error of the side values.  A skipped pair would only have
// given points that are vertices of both triangles and, for a shared edge,
// a segment on both triangles' boundaries: it changes nothing.
bool shared_contact_only(const double *a, const double *b) {
  for (int dir = 0; dir < 2; ++dir) {
    const double *A = dir == 0 ? a : b, *B = dir == 0 ? b : a;
    double m = 0.0;
    for (int k = 0; k < 9; ++k) m = std::max(m, std::max(std::fabs(A[k]), std::fabs(B[k])));
    if (!(m >= 1e-50 && m <= 1e50)) continue;
    const double tol = 1e-12 * m * m * m;
    double e1[3], e2[3], nrm[3];
    for (int k = 0; k < 3; ++k) {
      e1[k] = A[3 + k] - A[k];
      e2[k] = A[6 + k] - A[k];
    }
    nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
    nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
    nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
    int pos = 0, neg = 0, clear = 0;
    bool ok = true;
    for (int v = 0; v < 3 && ok; ++v) {
      const double s = (B[3 * v] - A[0]) * nrm[0] + (B[3 * v + 1] - A[1]) * nrm[1] +
                       (B[3 * v + 2] - A[2]) * nrm[2];
      if (s > tol || s < -tol) {
        ++clear;
        pos += s > 0;
        neg += s < 0;
      } else {
        bool shared = false;
        for (int u = 0; u < 3; ++u)
          shared = shared || (B[3 * v] == A[3 * u] && B[3 * v + 1] == A[3 * u + 1] &&
                              B[3 * v + 2] == A[3 * u + 2]);
        ok = shared;
      }
    }
    if (ok && clear > 0 && (pos == 0 || neg == 0)) return true;
  }
  return false;
}


}  // namespace

struct edp_resolution {
  int status = EDP_RESOLVE_OK;
  int64_t overlap_a = -1, overlap_b = -1;
  int64_t summary[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> vertices;  // [T][3][3]
  std::vector<int64_t> parents;  // [T]
  std::string exact;             // "X Y Z W\n" per corner when asked
};

namespace {

// The scale exponent E: every coordinate times 2^E is an integer.
int choose_scale(const double *t, int64_t n) {
  int scale = 0;
  for (int64_t k = 0; k < 9 * n; ++k) {
    const double x = t[k];
    if (!std::isfinite(x)) throw BadInput{};
    if (x == 0.0) continue;
    if (std::fabs(x) < 0x1p-1022) throw BadInput{};
    int e;
    const double m = std::frexp(std::fabs(x), &e);
    const u64 mant = u64(std::ldexp(m, 53));
    scale = std::max(scale, 53 - e - __builtin_ctzll(mant));
  }
  return scale;
}

// Uniform grid over the created points' rounded coordinates.
struct PointGrid {
  double origin[3] = {0, 0, 0}, cell = 1.0;
  std::unordered_map<u64, std::vector<int>> cells;
  static u64 key(int64_t x, int64_t y, int64_t z) {
    return (u64(x & 0x1fffff) << 42) | (u64(y & 0x1fffff) << 21) | u64(z & 0x1fffff);
  }
  int64_t index(double v, int k) const { return int64_t(std::floor((v - origin[k]) / cell)); }
  void build(const std::vector<std::array<double, 3>> &pts, double size) {
    cell = size > 0 ? size : 1.0;
    if (!pts.empty())
      for (int k = 0; k < 3; ++k) {
        origin[k] = pts[0][k];
        for (auto &p : pts) origin[k] = std::min(origin[k], p[k]);
      }
    for (size_t i = 0; i < pts.size(); ++i)
      cells[key(index(pts[i][0], 0), index(pts[i][1], 1), index(pts[i][2], 2))].push_back(int(i));
  }
  // Points whose rounded coordinates lie in [lo, hi].
  void query(const double lo[3], const double hi[3], const std::vector<std::array<double, 3>> &pts,
             std::vector<int> &out) const {
    out.clear();
    if (pts.empty()) return;
    int64_t a[3], b[3];
    int64_t volume = 1;
    for (int k = 0; k < 3; ++k) {
      a[k] = index(lo[k], k);
      b[k] = index(hi[k], k);
      volume *= std::max<int64_t>(1, b[k] - a[k] + 1);
    }
    auto inside = [&](int i) {
      for (int k = 0; k < 3; ++k)
        if (!(pts[i][k] >= lo[k] && pts[i][k] <= hi[k])) return false;
      return true;
    };
    if (volume > int64_t(cells.size())) {
      for (const auto &c : cells)
        for (int i : c.second)
          if (inside(i)) out.push_back(i);
    } else {
      for (int64_t x = a[0]; x <= b[0]; ++x)
        for (int64_t y = a[1]; y <= b[1]; ++y)
          for (int64_t z = a[2]; z <= b[2]; ++z) {
            auto it = cells.find(key(x, y, z));
            if (it == cells.end()) continue;
            for (int i : it->second)
              if (inside(i)) out.push_back(i);
          }
    }
    std::sort(out.begin(), out.end());
  }
};

struct Output {
  std::vector<double> tris;  // 9 per triangle
  std::string text;
  bool trivial = true;       // the input triangle, unchanged
};

void write_text(const Pt &p, std::string &out) {
  for (int k = 0; k < 4; ++k) {
    out += hex(p.c[k]);
    out += k < 3 ? ' ' : '\n';
  }
}

struct Resolver {
  const double *tri;
  int64_t n;
  int threads;
  bool want_text;
  int scale = 0;
  std::vector<char> degenerate;
  std::vector<Pt> points;                       // distinct created points
  std::vector<std::array<double, 3>> rounded;   // their binary64 values
  PointGrid grid;
  std::vector<std::vector<std::vector<Pt>>> pieces;  // per face (cut faces only)
  std::vector<char> cut;
  std::vector<Output> out;
  int64_t summary[6] = {0, 0, 0, 0, 0, 0};

  // `poly` with every created point lying strictly inside one of its edges
  // inserted there, in order along the edge.
  std::vector<Pt> insert_points(const std::vector<Pt> &poly) const {
    const size_t n = poly.size();
    std::vector<std::array<double, 3>> corners(n);
    double m = 0.0, lo[3], hi[3];
    for (size_t v = 0; v < n; ++v) {
      double r[3];
      round_pt(poly[v], scale, r);
      for (int k = 0; k < 3; ++k) {
        corners[v][k] = r[k];
        m = std::max(m, std::fabs(r[k]));
        lo[k] = v ? std::min(lo[k], r[k]) : r[k];
        hi[k] = v ? std::max(hi[k], r[k]) : r[k];
      }
    }
    const double pad = 1e-9 * (m + 1.0);
    for (int k = 0; k < 3; ++k) {
      lo[k] -= pad;
      hi[k] += pad;
    }
    std::vector<int> near;
    grid.query(lo, hi, rounded, near);
    if (near.empty()) return poly;
    for (int i : near)
      for (int k = 0; k < 3; ++k) m = std::max(m, std::fabs(rounded[i][k]));
    const double tol = (m >= 1e-50 && m <= 1e50) ? 1e-12 * m * m : INFINITY;
    std::vector<Pt> result;
    for (size_t v = 0; v < n; ++v) {
      const Pt &u = poly[v], &w = poly[(v + 1) % n];
      result.push_back(u);
      const auto &fu = corners[v], &fw = corners[(v + 1) % n];
      const double d[3] = {fw[0] - fu[0], fw[1] - fu[1], fw[2] - fu[2]};
      std::vector<std::pair<int, int>> inside;  // point, axis
      for (int i : near) {
        const auto &c = rounded[i];
        const double e[3] = {c[0] - fu[0], c[1] - fu[1], c[2] - fu[2]};
        const double off = std::max({std::fabs(d[1] * e[2] - d[2] * e[1]),
                                     std::fabs(d[2] * e[0] - d[0] * e[2]),
                                     std::fabs(d[0] * e[1] - d[1] * e[0])});
        if (!(off <= tol)) continue;
        int axis;
        if (on_open_segment(points[i], u, w, axis)) inside.push_back({i, axis});
      }
      if (inside.empty()) continue;
      const int axis = inside[0].second;
      const int dir = cmp_coord(w, u, axis);
      std::sort(inside.begin(), inside.end(), [&](const std::pair<int, int> &a,
                                                  const std::pair<int, int> &b) {
        return cmp_coord(points[a.first], points[b.first], axis) * dir < 0;
      });
      for (auto &q : inside) result.push_back(points[q.first]);
    }
    return result;
  }
};

}  // namespace

namespace {

// Triangles of a convex piece of face f: the piece itself when it is a
// triangle; else a fan from its first corner whose two neighbours are corners
// too (no point inserted on the edges at that corner, so no fan triangle is
// degenerate), or, when every corner has an inserted neighbour, a fan around
// the centroid of its first three corners.  Corners are vertices not collinear
// with their neighbours.  Every boundary edge is kept, so no T-junctions.
void fan(const FaceX &f, const std::vector<Pt> &poly, std::vector<std::array<const Pt *, 3>> &tris,
         std::deque<Pt> &centers) {
  const size_t n = poly.size();
  if (n == 3) {
    tris.push_back({&poly[0], &poly[1], &poly[2]});
    return;
  }
  int i, j;
  plane_axes(f.dom, i, j);
  std::vector<char> corner(n);
  for (size_t v = 0; v < n; ++v)
    corner[v] = orient_h(poly[(v + n - 1) % n], poly[v], poly[(v + 1) % n], i, j).sign() != 0;
  for (size_t v = 0; v < n; ++v)
    if (corner[v] && corner[(v + n - 1) % n] && corner[(v + 1) % n]) {
      for (size_t t = 1; t + 1 < n; ++t)
        tris.push_back({&poly[v], &poly[(v + t) % n], &poly[(v + t + 1) % n]});
      return;
    }
  const Pt *c[3];
  int found = 0;
  for (size_t v = 0; v < n && found < 3; ++v)
    if (corner[v]) c[found++] = &poly[v];
  if (found < 3) throw TooLarge{};  // not reached: pieces have area
  const Int &w0 = c[0]->c[3], &w1 = c[1]->c[3], &w2 = c[2]->c[3];
  const Int w12 = w1 * w2, w02 = w0 * w2, w01 = w0 * w1;
  Int coord[3];
  for (int k = 0; k < 3; ++k) coord[k] = c[0]->c[k] * w12 + c[1]->c[k] * w02 + c[2]->c[k] * w01;
  centers.push_back(make_pt(coord[0], coord[1], coord[2], Int(3) * w0 * w12));
  const Pt *center = &centers.back();
  for (size_t v = 0; v < n; ++v) tris.push_back({center, &poly[v], &poly[(v + 1) % n]});
}

void resolve_all(Resolver &R) {
  const int64_t n = R.n;
  const double *tri = R.tri;
  const int threads = R.threads;
  R.scale = choose_scale(tri, n);
  const int scale = R.scale;
  R.summary[5] = scale;

  // Degenerate (zero-area) triangles pass through unchanged.
  R.degenerate.assign(n, 0);
  parallel_chunks(n, threads, 4096, [&](int64_t b, int64_t e) {
    for (int64_t f = b; f < e; ++f) R.degenerate[f] = face_exact(tri + 9 * f, scale).degenerate;
  });
  std::vector<int64_t> live;
  for (int64_t f = 0; f < n; ++f)
    if (!R.degenerate[f]) live.push_back(f);
  const int64_t L = int64_t(live.size());

  // Candidate pairs: padded boxes that overlap, swept along x.
  std::vector<std::array<double, 6>> box(L);  // lo xyz, hi xyz
  for (int64_t a = 0; a < L; ++a) {
    const double *t = tri + 9 * live[a];
    double m = 0.0;
    for (int k = 0; k < 9; ++k) m = std::max(m, std::fabs(t[k]));
    const double pad = 1e-9 * (m + 1.0);
    for (int k = 0; k < 3; ++k) {
      const double lo = std::min({t[k], t[3 + k], t[6 + k]});
      const double hi = std::max({t[k], t[3 + k], t[6 + k]});
      box[a][k] = lo - pad;
      box[a][3 + k] = hi + pad;
    }
  }
  std::vector<int64_t> order(L);
  for (int64_t a = 0; a < L; ++a) order[a] = a;
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t x, int64_t y) { return box[x][0] < box[y][0]; });
  // Every pair of overlapping boxes, as (earlier, later) in that order, in
  // increasing (earlier, later) position: the sweep's order.  A uniform grid
  // of cells twice the mean box extent finds them; boxes over more than 512
  // cells are checked against every later box.
  std::vector<int64_t> pos(L);
  for (int64_t k = 0; k < L; ++k) pos[order[k]] = k;
  double extent = 0.0, origin[3] = {0.0, 0.0, 0.0};
  for (int64_t a = 0; a < L; ++a) {
    extent += std::max({box[a][3] - box[a][0], box[a][4] - box[a][1], box[a][5] - box[a][2]});
    for (int k = 0; k < 3; ++k) origin[k] = a ? std::min(origin[k], box[a][k]) : box[a][k];
  }
  const double cell = L && extent > 0 ? 2.0 * extent / double(L) : 1.0;
  auto cell_of = [&](double v, int k) { return int64_t(std::floor((v - origin[k]) / cell)); };
  std::vector<std::pair<u64, int64_t>> entries;  // (cell key, position)
  std::vector<int64_t> big;                      // positions of boxes over many cells
  std::vector<char> is_big(L, 0);
  for (int64_t k = 0; k < L; ++k) {
    const auto &b = box[order[k]];
    int64_t lo[3], hi[3], volume = 1;
    for (int a = 0; a < 3; ++a) {
      lo[a] = cell_of(b[a], a);
      hi[a] = cell_of(b[3 + a], a);
      volume *= hi[a] - lo[a] + 1;
    }
    if (volume > 512) {
      big.push_back(k);
      is_big[k] = 1;
      continue;
    }
    for (int64_t x = lo[0]; x <= hi[0]; ++x)
      for (int64_t y = lo[1]; y <= hi[1]; ++y)
        for (int64_t z = lo[2]; z <= hi[2]; ++z) entries.push_back({PointGrid::key(x, y, z), k});
  }
  std::sort(entries.begin(), entries.end());
  const int64_t sweep_chunk = 2048;
  std::vector<std::vector<std::pair<int64_t, int64_t>>> swept((L + sweep_chunk - 1) / sweep_chunk);
  auto boxes_meet = [&](int64_t k, int64_t j) {
    const auto &bk = box[order[k]], &bj = box[order[j]];
    return bj[0] <= bk[3] && bj[1] <= bk[4] && bj[2] <= bk[5] && bj[4] >= bk[1] &&
           bj[5] >= bk[2];
  };
  parallel_chunks(L, threads, sweep_chunk, [&](int64_t b, int64_t e) {
    auto &mine = swept[b / sweep_chunk];
    std::vector<int64_t> cand;
    for (int64_t k = b; k < e; ++k) {
      cand.clear();
      if (is_big[k]) {
        for (int64_t j = k + 1; j < L; ++j) cand.push_back(j);
      } else {
        const auto &bk = box[order[k]];
        int64_t lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
          lo[a] = cell_of(bk[a], a);
          hi[a] = cell_of(bk[3 + a], a);
        }
        for (int64_t x = lo[0]; x <= hi[0]; ++x)
          for (int64_t y = lo[1]; y <= hi[1]; ++y)
            for (int64_t z = lo[2]; z <= hi[2]; ++z) {
              const u64 key = PointGrid::key(x, y, z);
              auto it = std::lower_bound(entries.begin(), entries.end(),
                                         std::make_pair(key, k + 1));
              for (; it != entries.end() && it->first == key; ++it) cand.push_back(it->second);
            }
        for (int64_t j : big)
          if (j > k) cand.push_back(j);
      }
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      for (int64_t j : cand) {
        // Positions j > k have lo_x >= k's, so the x intervals meet iff lo_j <= hi_k.
        const bool x_ok = box[order[j]][0] <= box[order[k]][3];
        if (x_ok && boxes_meet(k, j)) mine.push_back({order[k], order[j]});
      }
    }
  });
  std::vector<std::pair<int64_t, int64_t>> pairs;
  for (auto &s : swept) pairs.insert(pairs.end(), s.begin(), s.end());
  swept.clear();
  swept.shrink_to_fit();
  const int64_t P = int64_t(pairs.size());
  R.summary[2] = P;

  // Exact contacts of the pairs the binary64 pre-test keeps.
  const int64_t pair_chunk = 4096;
  std::vector<std::vector<PairResult>> found((P + pair_chunk - 1) / pair_chunk);
  std::atomic<int64_t> exact_pairs{0};
  std::atomic<int64_t> first_overlap{P};
  parallel_chunks(P, threads, pair_chunk, [&](int64_t b, int64_t e) {
    auto &mine = found[b / pair_chunk];
    int64_t tested = 0;
    for (int64_t q = b; q < e; ++q) {
      const int64_t fa_i = live[pairs[q].first], fb_i = live[pairs[q].second];
      if (shared_contact_only(tri + 9 * fa_i, tri + 9 * fb_i)) continue;
      ++tested;
      const FaceX fa = face_exact(tri + 9 * fa_i, scale), fb = face_exact(tri + 9 * fb_i, scale);
      Contact c;
      try {
        contact(fa, fb, fa_i, fb_i, c);
      } catch (const CoplanarOverlap &) {
        int64_t cur = first_overlap.load();
        while (q < cur && !first_overlap.compare_exchange_weak(cur, q)) {
        }
        break;
      }
      PairResult r;
      r.pair = q;
      r.fa = fa_i;
      r.fb = fb_i;
      for (auto &x : c.found)
        if (!(is_vertex(fa, x) && is_vertex(fb, x))) r.points.push_back(std::move(x));
      if (c.has_segment) {
        r.cut_a = !on_boundary(fa, c.p, c.r);
        r.cut_b = !on_boundary(fb, c.p, c.r);
        r.segment = r.cut_a || r.cut_b;
        r.p = std::move(c.p);
        r.r = std::move(c.r);
      }
      if (!r.points.empty() || r.segment) mine.push_back(std::move(r));
    }
    exact_pairs += tested;
  });
  R.summary[3] = exact_pairs.load();
  if (first_overlap.load() < P) {
    const int64_t q = first_overlap.load();
    throw CoplanarOverlap{live[pairs[q].first], live[pairs[q].second]};
  }
  pairs.clear();
  pairs.shrink_to_fit();

  // Cuts per face, in pair order; the contact points.
  std::vector<const PairResult *> results;
  for (auto &chunk : found)
    for (auto &r : chunk) results.push_back(&r);
  std::vector<const Pt *> made;  // every point made by a contact or a cut
  struct CutRef {
    int64_t face;
    const Pt *p, *r;
  };
  std::vector<CutRef> cuts;
  for (const PairResult *r : results) {
    for (auto &x : r->points) made.push_back(&x);
    if (!r->segment) continue;
    ++R.summary[0];
    if (r->cut_a) cuts.push_back({r->fa, &r->p, &r->r});
    if (r->cut_b) cuts.push_back({r->fb, &r->p, &r->r});
  }
  std::stable_sort(cuts.begin(), cuts.end(),
                   [](const CutRef &a, const CutRef &b) { return a.face < b.face; });
  std::vector<std::pair<int64_t, int64_t>> groups;  // [begin, end) per cut face
  for (int64_t k = 0; k < int64_t(cuts.size());) {
    int64_t e = k;
    while (e < int64_t(cuts.size()) && cuts[e].face == cuts[k].face) ++e;
    groups.push_back({k, e});
    k = e;
  }
  R.summary[1] = int64_t(groups.size());

  // Split every cut face by its distinct cut lines.
  R.cut.assign(n, 0);
  R.pieces.assign(n, {});
  std::vector<std::vector<Pt>> corners_made(groups.size());
  parallel_chunks(int64_t(groups.size()), threads, 64, [&](int64_t b, int64_t e) {
    for (int64_t g = b; g < e; ++g) {
      const int64_t face = cuts[groups[g].first].face;
      const FaceX F = face_exact(tri + 9 * face, scale);
      std::vector<const Pt *> base = {&F.v[0], &F.v[1], &F.v[2]};
      for (int64_t k = groups[g].first; k < groups[g].second; ++k) {
        const Pt &p = *cuts[k].p, &r = *cuts[k].r;
        bool seen = false;
        for (size_t c = 3; c < base.size() && !seen; c += 2)
          seen = collinear(*base[c], *base[c + 1], p) && collinear(*base[c], *base[c + 1], r);
        if (!seen) {
          base.push_back(&p);
          base.push_back(&r);
        }
      }
      std::vector<std::vector<Vtx>> parts(1);
      for (int k = 0; k < 3; ++k) parts[0].push_back({F.v[k], k, (k + 1) % 3});
      for (size_t c = 3; c < base.size(); c += 2) {
        std::vector<std::vector<Vtx>> next;
        for (auto &part : parts) split(F, base, int(c), int(c + 1), std::move(part), next);
        parts = std::move(next);
      }
      auto &mine = R.pieces[face];
      for (auto &part : parts) {
        std::vector<Pt> poly;
        for (auto &v : part) {
          if (!is_vertex(F, v.p)) corners_made[g].push_back(v.p);
          poly.push_back(std::move(v.p));
        }
        mine.push_back(std::move(poly));
      }
      R.cut[face] = 1;
    }
  });
  for (auto &v : corners_made)
    for (auto &x : v) made.push_back(&x);

  // Distinct points (by exact value), their binary64 values and a grid.
  std::vector<std::array<double, 3>> approx(made.size());
  parallel_chunks(int64_t(made.size()), threads, 1024, [&](int64_t b, int64_t e) {
    for (int64_t k = b; k < e; ++k) {
      double r[3];
      round_pt(*made[k], scale, r);
      approx[k] = {r[0], r[1], r[2]};
    }
  });
  // Equal points round alike: sort by the rounded values, then compare the
  // exact values within each run of equal roundings.
  std::vector<int64_t> by_value(made.size());
  for (size_t k = 0; k < made.size(); ++k) by_value[k] = int64_t(k);
  std::sort(by_value.begin(), by_value.end(), [&](int64_t x, int64_t y) {
    return approx[x] != approx[y] ? approx[x] < approx[y] : x < y;
  });
  for (size_t k = 0; k < by_value.size();) {
    size_t e = k;
    while (e < by_value.size() && approx[by_value[e]] == approx[by_value[k]]) ++e;
    const size_t first = R.points.size();
    for (size_t m = k; m < e; ++m) {
      const Pt &x = *made[by_value[m]];
      bool dup = false;
      for (size_t u = first; u < R.points.size() && !dup; ++u) dup = same_point(R.points[u], x);
      if (dup) continue;
      R.points.push_back(x);
      R.rounded.push_back(approx[by_value[m]]);
    }
    k = e;
  }
  R.summary[4] = int64_t(R.points.size());
  double size = 0.0;
  for (int64_t a = 0; a < L; ++a)
    size = std::max(size, std::max({box[a][3] - box[a][0], box[a][4] - box[a][1],
                                    box[a][5] - box[a][2]}));
  double mean = 0.0;
  for (int64_t a = 0; a < L; ++a)
    mean += std::max({box[a][3] - box[a][0], box[a][4] - box[a][1], box[a][5] - box[a][2]});
  mean = L ? mean / double(L) : 1.0;
  R.grid.build(R.rounded, mean > 0 ? 2.0 * mean : (size > 0 ? size : 1.0));

  // Every face's output triangles.
  R.out.assign(n, Output());
  parallel_chunks(n, threads, 256, [&](int64_t b, int64_t e) {
    std::vector<int> near;
    for (int64_t face = b; face < e; ++face) {
      if (R.degenerate[face]) continue;
      const double *t = tri + 9 * face;
      if (!R.cut[face]) {
        // Unchanged unless a made point lies on one of its edges.
        double m = 0.0, lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::min({t[k], t[3 + k], t[6 + k]});
          hi[k] = std::max({t[k], t[3 + k], t[6 + k]});
        }
        for (int k = 0; k < 9; ++k) m = std::max(m, std::fabs(t[k]));
        const double pad = 1e-9 * (m + 1.0);
        for (int k = 0; k < 3; ++k) {
          lo[k] -= pad;
          hi[k] += pad;
        }
        R.grid.query(lo, hi, R.rounded, near);
        if (near.empty()) continue;
      }
      const FaceX F = face_exact(t, scale);
      std::vector<std::vector<Pt>> polys;
      if (R.cut[face]) {
        for (auto &piece : R.pieces[face]) polys.push_back(R.insert_points(piece));
      } else {
        polys.push_back(R.insert_points({F.v[0], F.v[1], F.v[2]}));
        if (polys[0].size() == 3) continue;
      }
      Output &o = R.out[face];
      o.trivial = false;
      std::deque<Pt> centers;
      std::vector<std::array<const Pt *, 3>> tris;
      for (auto &poly : polys) fan(F, poly, tris, centers);
      for (auto &tr : tris)
        for (const Pt *p : tr) {
          double r[3];
          round_pt(*p, scale, r);
          o.tris.insert(o.tris.end(), r, r + 3);
          if (R.want_text) write_text(*p, o.text);
        }
    }
  });
  R.pieces.clear();
}

}  // namespace

extern "C" {

int edp_resolve_abi_version(void) { return EDP_RESOLVE_ABI_VERSION; }

int edp_resolve(const double *triangles, int64_t count, int threads, int exact_text,
                edp_resolution **out) {
  if (!out) return EDP_RESOLVE_BAD_INPUT;
  edp_resolution *res = new (std::nothrow) edp_resolution();
  *out = res;
  if (!res) return EDP_RESOLVE_NO_MEMORY;
  if (count < 0 || (count > 0 && !triangles)) return res->status = EDP_RESOLVE_BAD_INPUT;
  if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
  Resolver R;
  R.tri = triangles;
  R.n = count;
  R.threads = threads;
  R.want_text = exact_text != 0;
  try {
    resolve_all(R);
    std::vector<int64_t> start(count + 1, 0);
    for (int64_t f = 0; f < count; ++f)
      start[f + 1] = start[f] + (R.out[f].trivial ? 1 : int64_t(R.out[f].tris.size() / 9));
    const int64_t T = start[count];
    res->vertices.resize(size_t(9 * T));
    res->parents.resize(size_t(T));
    for (int64_t f = 0; f < count; ++f) {
      const Output &o = R.out[f];
      double *dst = res->vertices.data() + 9 * start[f];
      if (o.trivial) std::memcpy(dst, triangles + 9 * f, 9 * sizeof(double));
      else std::memcpy(dst, o.tris.data(), o.tris.size() * sizeof(double));
      for (int64_t t = start[f]; t < start[f + 1]; ++t) res->parents[t] = f;
      if (R.want_text) {
        if (o.trivial) {
          for (int k = 0; k < 3; ++k) {
            const double *v = triangles + 9 * f + 3 * k;
            write_text(make_pt(scaled(v[0], R.scale), scaled(v[1], R.scale),
                               scaled(v[2], R.scale), Int(1)),
                       res->exact);
          }
        } else {
          res->exact += o.text;
        }
      }
    }
    std::memcpy(res->summary, R.summary, sizeof(res->summary));
  } catch (const CoplanarOverlap &e) {
    res->overlap_a = e.a;
    res->overlap_b = e.b;
    res->status = EDP_RESOLVE_COPLANAR_OVERLAP;
  } catch (const TooLarge &) {
    res->status = EDP_RESOLVE_TOO_LARGE;
  } catch (const BadInput &) {
    res->status = EDP_RESOLVE_BAD_INPUT;
  } catch (const std::bad_alloc &) {
    res->status = EDP_RESOLVE_NO_MEMORY;
  }
  if (res->status != EDP_RESOLVE_OK) {
    res->vertices.clear();
    res->parents.clear();
    res->exact.clear();
  }
  return res->status;
}

int64_t edp_resolution_triangles(const edp_resolution *r) {
  return r ? int64_t(r->parents.size()) : 0;
}

void edp_resolution_summary(const edp_resolution *r, int64_t summary[6]) {
  for (int k = 0; k < 6; ++k) summary[k] = r ? r->summary[k] : 0;
}

int edp_resolution_binary64(const edp_resolution *r, double *vertices, int64_t *parents) {
  if (!r || r->status != EDP_RESOLVE_OK) return r ? r->status : EDP_RESOLVE_BAD_INPUT;
  if (vertices) std::memcpy(vertices, r->vertices.data(), r->vertices.size() * sizeof(double));
  if (parents) std::memcpy(parents, r->parents.data(), r->parents.size() * sizeof(int64_t));
  return EDP_RESOLVE_OK;
}

int64_t edp_resolution_exact(const edp_resolution *r, char *text, int64_t size) {
  if (!r || r->exact.empty()) return 0;
  const int64_t need = int64_t(r->exact.size()) + 1;
  if (text && size >= need) std::memcpy(text, r->exact.c_str(), size_t(need));
  return need;
}

void edp_resolution_overlap(const edp_resolution *r, int64_t *a, int64_t *b) {
  if (a) *a = r ? r->overlap_a : -1;
  if (b) *b = r ? r->overlap_b : -1;
}

void edp_resolution_free(edp_resolution *r) { delete r; }

}  // extern "C"
