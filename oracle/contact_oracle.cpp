// Test infrastructure, not product code: the oracle.
//
// A CPU restatement of MicroSimulator's capsule contact-mechanics step,
// templated on the scalar type.  With float it follows the reference's FP32
// operation order (no FMA, IEEE sqrt and division, the reference's fixed
// reduction grains) so that its results are bit-identical to the reference
// CPU backend; tests pin it against oracle/_ref (the reference itself) and
// against the reference tests' known answers.  With double it is the FP64
// oracle that every result's error is stated against.  Only tests/, the smoke
// check and bench.py's CPU-baseline leg load it (as _build/liboracle.so).
//
// Reference files followed (paths within the MicroSimulator tree):
//   broad phase      cpp/core/contact_graph.cpp:17-41,254-300
//   narrow phase     cpp/cpu/cpu_contacts.cpp:54-212
//   wall contacts    cpp/cpu/cpu_constraints.cpp:24-612
//   BB solve         cpp/core/contact_solver.hpp:44-120,
//                    cpp/cpu/cpu_contact_dynamics.cpp:40-338
//   stepper          cpp/core/contact_dynamics.cpp:55-782
//   axis rotation    cpp/core/mechanics_integration.cpp:9-20
//   world state      cpp/core/world_state.cpp:238-276,405-430

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <optional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../include/msb200.h"

namespace oracle {

constexpr std::uint32_t invalid_slot = 0xFFFFFFFFu;

template <typename T>
struct V3 {
  T x{0}, y{0}, z{0};
  V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator*(T s) const { return {x * s, y * s, z * s}; }
};

template <typename T>
T dot(const V3<T>& a, const V3<T>& b) {
  return (a.x * b.x) + (a.y * b.y) + (a.z * b.z);
}
template <typename T>
V3<T> cross(const V3<T>& a, const V3<T>& b) {
  return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
template <typename T>
T norm(const V3<T>& v) {
  return std::sqrt(dot(v, v));
}
template <typename T>
V3<T> normalized(const V3<T>& v) {
  const T m = norm(v);
  if (!std::isfinite(m) || m <= T(0)) {
    throw std::invalid_argument("cell direction must be finite and non-zero");
  }
  return v * (T(1) / m);
}
template <typename T>
bool finite3(const V3<T>& v) {
  return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}
template <typename T>
T clampv(T v, T lo, T hi) {
  return std::clamp(v, lo, hi);
}

template <typename T>
constexpr T inverse_sqrt_two() {
  if constexpr (std::is_same_v<T, float>) {
    return 0.7071067811865475F;
  } else {
    return 0.70710678118654752440;
  }
}

// ------------------------------------------------------------ world state

template <typename T>
struct World {
  std::vector<std::uint64_t> ids;
  std::vector<V3<T>> pos;
  std::vector<V3<T>> dir;
  std::vector<T> len;
  std::vector<T> rad;
  std::vector<T> growth;
  std::vector<std::uint8_t> fixed;
  std::size_t size() const { return ids.size(); }

  // WorldState::set_cell_geometry stores the normalized direction
  // (world_state.cpp:405-430).
  void set_geometry(std::size_t slot, V3<T> p, V3<T> d, T l) {
    if (!finite3(p) || !finite3(d) || !std::isfinite(l) || l < T(0)) {
      throw std::invalid_argument("cell fields must be finite");
    }
    pos[slot] = p;
    dir[slot] = normalized(d);
    len[slot] = l;
  }
};

template <typename T>
World<T> world_from(const msb_cell_arrays& c) {
  World<T> w;
  const auto n = c.count;
  w.ids.assign(c.ids, c.ids + n);
  w.pos.resize(n);
  w.dir.resize(n);
  w.len.resize(n);
  w.rad.resize(n);
  w.growth.resize(n);
  w.fixed.resize(n);
  for (std::size_t i = 0; i < n; ++i) {
    w.pos[i] = {T(c.position_x[i]), T(c.position_y[i]), T(c.position_z[i])};
    w.dir[i] = {T(c.direction_x[i]), T(c.direction_y[i]), T(c.direction_z[i])};
    w.len[i] = T(c.lengths[i]);
    w.rad[i] = T(c.radii[i]);
    w.growth[i] = c.growth_rates ? T(c.growth_rates[i]) : T(0);
    w.fixed[i] = c.fixed ? c.fixed[i] : 0;
  }
  return w;
}

template <typename T>
void world_to(const World<T>& w, msb_cell_arrays& c) {
  for (std::size_t i = 0; i < w.size(); ++i) {
    c.position_x[i] = float(w.pos[i].x);
    c.position_y[i] = float(w.pos[i].y);
    c.position_z[i] = float(w.pos[i].z);
    c.direction_x[i] = float(w.dir[i].x);
    c.direction_y[i] = float(w.dir[i].y);
    c.direction_z[i] = float(w.dir[i].z);
    c.lengths[i] = float(w.len[i]);
  }
}

// ------------------------------------------------------------ broad phase

struct Bounds {
  double lo[3];
  double hi[3];
};

// Padded box of one capsule, in FP64 whatever T is (contact_graph.cpp:258-283).
template <typename T>
Bounds bounds_of(const World<T>& w, std::size_t i, float margin) {
  const double half = double(w.len[i]) * 0.5;
  const double pad = double(w.rad[i]) + double(margin) * 0.5;
  const double c[3] = {double(w.pos[i].x), double(w.pos[i].y), double(w.pos[i].z)};
  const double d[3] = {double(w.dir[i].x), double(w.dir[i].y), double(w.dir[i].z)};
  Bounds b;
  for (int a = 0; a < 3; ++a) {
    const double e = std::abs(d[a]) * half + pad;
    b.lo[a] = c[a] - e;
    b.hi[a] = c[a] + e;
  }
  return b;
}

inline bool boxes_touch(const Bounds& l, const Bounds& r) {
  for (int a = 0; a < 3; ++a) {
    if (!(l.hi[a] >= r.lo[a] && r.hi[a] >= l.lo[a])) return false;
  }
  return true;
}

// All (first, second) slot pairs with first id < second id whose padded
// boxes overlap (touching counts), sorted by (first id, second id).  The
// search is a hashed uniform grid; the set it returns is the one the
// reference's grid or sweep returns.
template <typename T>
std::vector<std::pair<std::uint32_t, std::uint32_t>> candidates(const World<T>& w, float margin) {
  const auto n = w.size();
  std::vector<std::pair<std::uint32_t, std::uint32_t>> out;
  if (n < 2) return out;
  std::vector<Bounds> b(n);
  double width[3] = {0, 0, 0};
  double low[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                   std::numeric_limits<double>::infinity()};
  bool all_finite = true;
  for (std::size_t i = 0; i < n; ++i) {
    b[i] = bounds_of(w, i, margin);
    for (int a = 0; a < 3; ++a) {
      all_finite = all_finite && std::isfinite(b[i].lo[a]) && std::isfinite(b[i].hi[a]);
      width[a] = std::max(width[a], b[i].hi[a] - b[i].lo[a]);
      low[a] = std::min(low[a], b[i].lo[a]);
    }
  }
  if (!all_finite) throw std::invalid_argument("cell geometry is not finite");
  for (auto& v : width) v = std::max(v * 1.001, std::numeric_limits<double>::min());
  auto key_of = [&](std::int64_t x, std::int64_t y, std::int64_t z) {
    return (std::uint64_t(x) * 0x9E3779B97F4A7C15ull) ^ (std::uint64_t(y) * 0xC2B2AE3D27D4EB4Full) ^
           (std::uint64_t(z) * 0x165667B19E3779F9ull);
  };
  std::vector<std::array<std::int64_t, 3>> at(n);
  std::unordered_map<std::uint64_t, std::vector<std::uint32_t>> grid;
  grid.reserve(n * 2);
  for (std::size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      const double c = 0.5 * (b[i].lo[a] + b[i].hi[a]);
      at[i][a] = std::int64_t(std::floor((c - low[a]) / width[a]));
    }
    grid[key_of(at[i][0], at[i][1], at[i][2])].push_back(std::uint32_t(i));
  }
  std::vector<std::uint32_t> order(n);
  for (std::size_t i = 0; i < n; ++i) order[i] = std::uint32_t(i);
  std::sort(order.begin(), order.end(), [&](auto l, auto r) { return w.ids[l] < w.ids[r]; });
  std::vector<std::pair<std::uint64_t, std::uint32_t>> partners;
  for (const auto i : order) {
    partners.clear();
    for (std::int64_t dx = -1; dx <= 1; ++dx)
      for (std::int64_t dy = -1; dy <= 1; ++dy)
        for (std::int64_t dz = -1; dz <= 1; ++dz) {
          const std::array<std::int64_t, 3> q{at[i][0] + dx, at[i][1] + dy, at[i][2] + dz};
          const auto found = grid.find(key_of(q[0], q[1], q[2]));
          if (found == grid.end()) continue;
          for (const auto j : found->second) {
            if (at[j] != q) continue;
            if (w.ids[j] > w.ids[i] && boxes_touch(b[i], b[j])) partners.emplace_back(w.ids[j], j);
          }
        }
    std::sort(partners.begin(), partners.end());
    for (const auto& p : partners) out.emplace_back(i, p.second);
  }
  return out;
}

// ----------------------------------------------------------- narrow phase

template <typename T>
struct Capsule {
  std::uint64_t id;
  std::uint32_t slot;
  V3<T> c;
  V3<T> a;
  T len;
  T r;
};

template <typename T>
struct PointPair {
  V3<T> first, second;
};

// Closest points of two segments, clamped parameters (cpu_contacts.cpp:54-108).
template <typename T>
PointPair<T> closest_points(const Capsule<T>& p, const Capsule<T>& q, T eps) {
  const T ph = p.len * T(0.5);
  const T qh = q.len * T(0.5);
  const V3<T> p0 = p.c - (p.a * ph);
  const V3<T> p1 = p.c + (p.a * ph);
  const V3<T> q0 = q.c - (q.a * qh);
  const V3<T> q1 = q.c + (q.a * qh);
  const V3<T> d1 = p1 - p0;
  const V3<T> d2 = q1 - q0;
  const V3<T> r = p0 - q0;
  const T a = dot(d1, d1);
  const T e = dot(d2, d2);
  const T f = dot(d2, r);
  T s = 0, t = 0;
  if (a <= eps * eps && e <= eps * eps) return {p0, q0};
  if (a <= eps * eps) {
    t = clampv(f / e, T(0), T(1));
  } else {
    const T c = dot(d1, r);
    if (e <= eps * eps) {
      s = clampv(-c / a, T(0), T(1));
    } else {
      const T b = dot(d1, d2);
      const T denom = (a * e) - (b * b);
      const T tol = std::numeric_limits<T>::epsilon() * a * e;
      if (denom > tol) s = clampv(((b * f) - (c * e)) / denom, T(0), T(1));
      t = (b * s + f) / e;
      if (t < T(0)) {
        t = 0;
        s = clampv(-c / a, T(0), T(1));
      } else if (t > T(1)) {
        t = 1;
        s = clampv((b - c) / a, T(0), T(1));
      }
    }
  }
  return {p0 + (d1 * s), q0 + (d2 * t)};
}

template <typename T>
struct PointPairs {
  PointPair<T> pairs[2];
  int count{0};
};

// One contact point, or two at the ends of the axial overlap of a
// near-parallel pair (cpu_contacts.cpp:110-140).
template <typename T>
PointPairs<T> contact_points(const Capsule<T>& p, const Capsule<T>& q, T sine_threshold, T eps) {
  PointPairs<T> out;
  const T ad = clampv(dot(p.a, q.a), T(-1), T(1));
  const T sine = std::sqrt(std::max(T(0), T(1) - (ad * ad)));
  if (sine > sine_threshold || p.len <= eps || q.len <= eps) {
    out.pairs[0] = closest_points(p, q, eps);
    out.count = 1;
    return out;
  }
  const T ph = p.len * T(0.5);
  const T qh = q.len * T(0.5);
  const T cc = dot(q.c - p.c, p.a);
  const T proj = qh * std::abs(ad);
  const T begin = std::max(-ph, cc - proj);
  const T end = std::min(ph, cc + proj);
  if (end - begin <= eps) {
    out.pairs[0] = closest_points(p, q, eps);
    out.count = 1;
    return out;
  }
  for (const T s : {begin, end}) {
    const V3<T> on_p = p.c + (p.a * s);
    const T t = clampv(dot(on_p - q.c, q.a), -qh, qh);
    out.pairs[out.count++] = {on_p, q.c + (q.a * t)};
  }
  return out;
}

// Normal from the first capsule to the second, with fallbacks for
// coincident points (cpu_contacts.cpp:142-166).
template <typename T>
V3<T> deterministic_normal(const Capsule<T>& p, const Capsule<T>& q, const PointPair<T>& pts,
                           T eps) {
  const V3<T> delta = pts.second - pts.first;
  if (norm(delta) > eps) return normalized(delta);
  const V3<T> ax = cross(p.a, q.a);
  if (norm(ax) > eps) return normalized(ax);
  const V3<T> cd = q.c - p.c;
  const V3<T> tr = cd - (p.a * dot(cd, p.a));
  if (norm(tr) > eps) return normalized(tr);
  const V3<T> basis[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  int best = 0;
  for (int k = 1; k < 3; ++k) {
    if (std::abs(dot(p.a, basis[k])) < std::abs(dot(p.a, basis[best]))) best = k;
  }
  return normalized(cross(p.a, basis[best]));
}

template <typename T>
Capsule<T> capsule(const World<T>& w, std::uint32_t i) {
  return {w.ids[i], i, w.pos[i], w.dir[i], w.len[i], w.rad[i]};
}

template <typename T>
struct Contact {
  std::uint64_t first_id, second_id;
  std::uint32_t first_slot, second_slot;
  std::uint32_t ordinal;
  V3<T> point;
  V3<T> normal;
  T separation;
  T weight;
};

// find_cell_contacts_cpu (cpu_contacts.cpp:168-219).
template <typename T>
std::vector<Contact<T>> cell_contacts(const World<T>& w, const msb_contact_parameters& prm) {
  if (!std::isfinite(prm.activation_margin) || prm.activation_margin < 0.0F ||
      !std::isfinite(prm.parallel_sine_threshold) || prm.parallel_sine_threshold < 0.0F ||
      prm.parallel_sine_threshold > 1.0F || !std::isfinite(prm.degeneracy_epsilon) ||
      prm.degeneracy_epsilon <= 0.0F) {
    throw std::invalid_argument("contact parameters are invalid");
  }
  std::vector<Contact<T>> out;
  const T margin = T(prm.activation_margin);
  const T eps = T(prm.degeneracy_epsilon);
  for (const auto& [i, j] : candidates(w, prm.activation_margin)) {
    const auto p = capsule(w, i);
    const auto q = capsule(w, j);
    const auto pts = contact_points(p, q, T(prm.parallel_sine_threshold), eps);
    const T weight = pts.count == 2 ? inverse_sqrt_two<T>() : T(1);
    for (int k = 0; k < pts.count; ++k) {
      const auto& pair = pts.pairs[k];
      const T sep = norm(pair.second - pair.first) - (p.r + q.r);
      if (sep >= margin) continue;
      const V3<T> n = deterministic_normal(p, q, pair, eps);
      out.push_back({p.id, q.id, p.slot, q.slot, std::uint32_t(k), pair.first + (n * p.r), n, sep,
                     weight});
    }
  }
  return out;
}

// ---------------------------------------------------------- wall contacts

template <typename T>
struct Wall {
  std::uint64_t id;
  std::uint32_t kind;
  std::uint32_t region;
  V3<T> a, b;
  T radius, half_height, coefficient;
};

template <typename T>
struct External {
  std::uint64_t cell_id;
  std::uint64_t constraint_id;
  std::uint32_t slot;
  std::uint32_t kind;
  std::uint32_t location;
  V3<T> point;
  V3<T> normal;
  T separation;
  T weight;
};

template <typename T>
struct Surface {
  T distance;
  V3<T> outward;
};

template <typename T>
struct Endpoint {
  std::uint32_t location;
  V3<T> p;
};

template <typename T>
std::array<Endpoint<T>, 2> endpoints(const World<T>& w, std::size_t s) {
  const T h = w.len[s] * T(0.5);
  return {Endpoint<T>{MSB_ROD_NEGATIVE, w.pos[s] - w.dir[s] * h},
          Endpoint<T>{MSB_ROD_POSITIVE, w.pos[s] + w.dir[s] * h}};
}

// Slab test of a segment against an axis-aligned box (cpu_constraints.cpp:46-73).
template <typename T>
bool segment_hits_box(V3<T> s, V3<T> e, V3<T> lo, V3<T> hi) {
  const V3<T> d = e - s;
  const T ss[3] = {s.x, s.y, s.z}, dd[3] = {d.x, d.y, d.z}, ll[3] = {lo.x, lo.y, lo.z},
          uu[3] = {hi.x, hi.y, hi.z};
  T entry = 0, exit = 1;
  for (int a = 0; a < 3; ++a) {
    if (dd[a] == T(0)) {
      if (ss[a] < ll[a] || ss[a] > uu[a]) return false;
      continue;
    }
    T f = (ll[a] - ss[a]) / dd[a];
    T g = (uu[a] - ss[a]) / dd[a];
    if (f > g) std::swap(f, g);
    entry = std::max(entry, f);
    exit = std::min(exit, g);
    if (entry > exit) return false;
  }
  return true;
}

template <typename T>
struct Minimum {
  V3<T> point;
  Surface<T> surface;
};

// Ternary search of a surface distance along the centreline, then the best
// of five probes (cpu_constraints.cpp:75-105).  40 iterations
// (cpp/shared/constants.def: segment_minimization_iterations).
template <typename T, typename F>
Minimum<T> minimize_on_segment(V3<T> s, V3<T> e, const F& at) {
  const V3<T> d = e - s;
  T lo = 0, hi = 1;
  for (int it = 0; it < 40; ++it) {
    const T u = lo + (hi - lo) / T(3);
    const T v = hi - (hi - lo) / T(3);
    const auto fu = at(s + d * u);
    const auto fv = at(s + d * v);
    if (fu.distance < fv.distance) {
      hi = v;
    } else if (fv.distance < fu.distance) {
      lo = u;
    } else {
      lo = u;
      hi = v;
    }
  }
  Minimum<T> best{s, at(s)};
  const T probes[5] = {T(1), T(0.5), lo, (lo + hi) * T(0.5), hi};
  for (const T t : probes) {
    const V3<T> p = s + d * t;
    const auto f = at(p);
    if (f.distance < best.surface.distance) best = {p, f};
  }
  return best;
}

// Rows for a finite obstacle the cell must stay outside of
// (cpu_constraints.cpp:107-165).
template <typename T>
void outside_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                  const Wall<T>& c, const std::array<Endpoint<T>, 2>& ends,
                  const std::array<Surface<T>, 2>& surf, const Minimum<T>& m, T margin, T eps) {
  const T r = w.rad[s];
  if (m.surface.distance - r >= margin) return;
  const T nearest = std::min(surf[0].distance, surf[1].distance);
  const bool at_end = nearest - m.surface.distance <= eps;
  struct Cand {
    std::uint32_t loc;
    V3<T> p;
    Surface<T> f;
  };
  Cand cands[2];
  int count = 0;
  for (int k = 0; at_end && k < 2; ++k) {
    if (surf[k].distance - r < margin) cands[count++] = {ends[k].location, ends[k].p, surf[k]};
  }
  if (count == 0) cands[count++] = {MSB_ROD_INTERIOR, m.point, m.surface};
  const T weight = c.coefficient * (count == 2 ? inverse_sqrt_two<T>() : T(1));
  for (int k = 0; k < count; ++k) {
    const V3<T> n = cands[k].f.outward * T(-1);
    out.push_back({w.ids[s], c.id, std::uint32_t(s), c.kind, cands[k].loc, cands[k].p + n * r, n,
                   cands[k].f.distance - r, weight});
  }
}

// Endpoint rows of a container the cell must stay inside of, nearest face
// only (cpu_constraints.cpp:233-259, 410-436, 529-555).
template <typename T>
void inside_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                 const Wall<T>& c, const std::array<Endpoint<T>, 2>& ends,
                 const std::array<Surface<T>, 2>& surf, T margin) {
  T sep[2];
  bool active[2];
  for (int k = 0; k < 2; ++k) {
    sep[k] = -surf[k].distance - w.rad[s];
    active[k] = sep[k] < margin;
  }
  const unsigned n_active = unsigned(active[0]) + unsigned(active[1]);
  const T weight = c.coefficient * (n_active == 2 ? inverse_sqrt_two<T>() : T(1));
  for (int k = 0; k < 2; ++k) {
    if (!active[k]) continue;
    out.push_back({w.ids[s], c.id, std::uint32_t(s), c.kind, ends[k].location,
                   ends[k].p + surf[k].outward * w.rad[s], surf[k].outward, sep[k], weight});
  }
}

template <typename T>
Surface<T> box_surface(V3<T> p, const Wall<T>& box, T eps) {
  const V3<T> d = p - box.a;
  const V3<T> cl{clampv(d.x, -box.b.x, box.b.x), clampv(d.y, -box.b.y, box.b.y),
                 clampv(d.z, -box.b.z, box.b.z)};
  const V3<T> o = d - cl;
  const T od = norm(o);
  if (od > eps) return {od, o * (T(1) / od)};
  const T clear[3] = {box.b.x - std::abs(d.x), box.b.y - std::abs(d.y), box.b.z - std::abs(d.z)};
  int ax = 0;
  for (int k = 1; k < 3; ++k) {
    if (clear[k] < clear[ax]) ax = k;
  }
  const T off[3] = {d.x, d.y, d.z};
  const T sign = std::abs(off[ax]) <= eps || off[ax] >= T(0) ? T(1) : T(-1);
  V3<T> out{};
  (ax == 0 ? out.x : ax == 1 ? out.y : out.z) = sign;
  return {-clear[ax], out};
}

template <typename T>
Surface<T> cylinder_surface(V3<T> p, const Wall<T>& cy, T eps) {
  const V3<T> d{p.x - cy.a.x, p.y - cy.a.y, T(0)};
  const T rd = norm(d);
  const V3<T> radial = rd > eps ? d * (T(1) / rd) : V3<T>{1, 0, 0};
  const T zo = p.z - cy.a.z;
  const T zs = zo >= T(0) ? T(1) : T(-1);
  const V3<T> axial{0, 0, zs};
  const T re = rd - cy.radius;
  const T ae = std::abs(zo) - cy.half_height;
  if (re > T(0) && ae > T(0)) {
    const T dist = std::sqrt((re * re) + (ae * ae));
    return {dist, (radial * re + axial * ae) * (T(1) / dist)};
  }
  if (re > T(0)) return {re, radial};
  if (ae > T(0)) return {ae, axial};
  if (-re <= -ae) return {re, radial};
  return {ae, axial};
}

template <typename T>
void plane_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s, const Wall<T>& c,
                T margin) {
  const auto ends = endpoints(w, s);
  T sep[2];
  bool active[2];
  for (int k = 0; k < 2; ++k) {
    sep[k] = dot(ends[k].p - c.a, c.b) - w.rad[s];
    active[k] = sep[k] < margin;
  }
  const unsigned n_active = unsigned(active[0]) + unsigned(active[1]);
  const T weight = c.coefficient * (n_active == 2 ? inverse_sqrt_two<T>() : T(1));
  const V3<T> n = c.b * T(-1);
  for (int k = 0; k < 2; ++k) {
    if (!active[k]) continue;
    out.push_back({w.ids[s], c.id, std::uint32_t(s), c.kind, ends[k].location,
                   ends[k].p + n * w.rad[s], n, sep[k], weight});
  }
}

template <typename T>
void sphere_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                 const Wall<T>& c, T margin, T eps) {
  const auto ends = endpoints(w, s);
  std::array<Surface<T>, 2> surf;
  for (int k = 0; k < 2; ++k) {
    const V3<T> cd = ends[k].p - c.a;
    const T dist = norm(cd);
    const V3<T> radial = dist > eps ? cd * (T(1) / dist) : V3<T>{1, 0, 0};
    surf[k] = {dist - c.radius, radial};
  }
  if (c.region == MSB_REGION_OUTSIDE) {
    const V3<T> st = ends[0].p;
    const V3<T> d = ends[1].p - st;
    const T lsq = dot(d, d);
    const T t = lsq > eps * eps ? clampv(-dot(st - c.a, d) / lsq, T(0), T(1)) : T(0);
    const V3<T> p = st + d * t;
    const V3<T> cd = p - c.a;
    const T dist = norm(cd);
    const V3<T> radial = dist > eps ? cd * (T(1) / dist) : V3<T>{1, 0, 0};
    outside_rows(out, w, s, c, ends, surf, Minimum<T>{p, {dist - c.radius, radial}}, margin, eps);
    return;
  }
  inside_rows(out, w, s, c, ends, surf, margin);
}

template <typename T>
void box_face_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                   const Wall<T>& c, T margin) {
  const T r = w.rad[s];
  const T half[3] = {c.b.x, c.b.y, c.b.z};
  for (const auto& e : endpoints(w, s)) {
    const V3<T> d = e.p - c.a;
    const T off[3] = {d.x, d.y, d.z};
    for (int ax = 0; ax < 3; ++ax) {
      for (const T sign : {T(-1), T(1)}) {
        const T sep = half[ax] - sign * off[ax] - r;
        if (sep >= margin) continue;
        V3<T> n{};
        (ax == 0 ? n.x : ax == 1 ? n.y : n.z) = sign;
        out.push_back({w.ids[s], c.id, std::uint32_t(s), c.kind, e.location, e.p + n * r, n, sep,
                       c.coefficient});
      }
    }
  }
}

template <typename T>
void cylinder_face_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                        const Wall<T>& c, T margin, T eps) {
  const T r = w.rad[s];
  for (const auto& e : endpoints(w, s)) {
    auto push = [&](V3<T> n, T sep) {
      if (sep >= margin) return;
      out.push_back({w.ids[s], c.id, std::uint32_t(s), c.kind, e.location, e.p + n * r, n, sep,
                     c.coefficient});
    };
    const V3<T> rdel{e.p.x - c.a.x, e.p.y - c.a.y, T(0)};
    const T rd = norm(rdel);
    const V3<T> radial = rd > eps ? rdel * (T(1) / rd) : V3<T>{1, 0, 0};
    push(radial, c.radius - rd - r);
    const T zo = e.p.z - c.a.z;
    for (const T sign : {T(-1), T(1)}) push({0, 0, sign}, c.half_height - sign * zo - r);
  }
}

template <typename T>
void box_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s, const Wall<T>& c,
              T margin, T eps) {
  const auto ends = endpoints(w, s);
  std::array<Surface<T>, 2> surf;
  for (int k = 0; k < 2; ++k) surf[k] = box_surface(ends[k].p, c, eps);
  if (c.region == MSB_REGION_OUTSIDE) {
    const T reach = w.rad[s] + margin;
    const V3<T> lo{c.a.x - c.b.x - reach, c.a.y - c.b.y - reach, c.a.z - c.b.z - reach};
    const V3<T> hi{c.a.x + c.b.x + reach, c.a.y + c.b.y + reach, c.a.z + c.b.z + reach};
    if (!segment_hits_box(ends[0].p, ends[1].p, lo, hi)) return;
    const auto m = minimize_on_segment(ends[0].p, ends[1].p,
                                       [&](V3<T> p) { return box_surface(p, c, eps); });
    outside_rows(out, w, s, c, ends, surf, m, margin, eps);
    return;
  }
  inside_rows(out, w, s, c, ends, surf, margin);
}

template <typename T>
void cylinder_rows(std::vector<External<T>>& out, const World<T>& w, std::size_t s,
                   const Wall<T>& c, T margin, T eps) {
  const auto ends = endpoints(w, s);
  std::array<Surface<T>, 2> surf;
  for (int k = 0; k < 2; ++k) surf[k] = cylinder_surface(ends[k].p, c, eps);
  if (c.region == MSB_REGION_OUTSIDE) {
    const T reach = w.rad[s] + margin;
    const V3<T> lo{c.a.x - c.radius - reach, c.a.y - c.radius - reach,
                   c.a.z - c.half_height - reach};
    const V3<T> hi{c.a.x + c.radius + reach, c.a.y + c.radius + reach,
                   c.a.z + c.half_height + reach};
    if (!segment_hits_box(ends[0].p, ends[1].p, lo, hi)) return;
    const V3<T> st = ends[0].p, en = ends[1].p;
    auto at = [&](V3<T> p) { return cylinder_surface(p, c, eps); };
    auto m = minimize_on_segment(st, en, at);
    const V3<T> d = en - st;
    auto consider = [&](T t) {
      const V3<T> p = st + d * clampv(t, T(0), T(1));
      const auto f = at(p);
      if (f.distance <= m.surface.distance) m = {p, f};
    };
    if (std::abs(d.z) > eps) consider((c.a.z - st.z) / d.z);
    const T rl = d.x * d.x + d.y * d.y;
    if (rl > eps * eps) consider(-((st.x - c.a.x) * d.x + (st.y - c.a.y) * d.y) / rl);
    outside_rows(out, w, s, c, ends, surf, m, margin, eps);
    return;
  }
  inside_rows(out, w, s, c, ends, surf, margin);
}

template <typename T>
std::vector<Wall<T>> walls_from(const msb_constraint* cs, std::uint64_t n) {
  std::vector<Wall<T>> out;
  for (std::uint64_t i = 0; i < n; ++i) {
    const auto& c = cs[i];
    if (c.kind > MSB_CONSTRAINT_CYLINDER) throw std::invalid_argument("constraint kind is invalid");
    out.push_back({c.id, c.kind, c.allowed_region, {T(c.a.x), T(c.a.y), T(c.a.z)},
                   {T(c.b.x), T(c.b.y), T(c.b.z)}, T(c.radius), T(c.half_height),
                   T(c.coefficient)});
  }
  return out;
}

// external_contacts (cpu_constraints.cpp:563-598): per cell, planes, spheres,
// boxes then cylinders in insertion order, then a stable sort by
// (cell id, constraint id, location).
template <typename T>
std::vector<External<T>> external_contacts(const World<T>& w, const std::vector<Wall<T>>& walls,
                                           const msb_constraint_contact_parameters& prm,
                                           bool every_face) {
  if (!std::isfinite(prm.activation_margin) || prm.activation_margin < 0.0F ||
      !std::isfinite(prm.degeneracy_epsilon) || prm.degeneracy_epsilon <= 0.0F) {
    throw std::invalid_argument("constraint contact parameters are invalid");
  }
  const T margin = T(prm.activation_margin);
  const T eps = T(prm.degeneracy_epsilon);
  std::vector<External<T>> out;
  for (std::size_t s = 0; s < w.size(); ++s) {
    for (std::uint32_t kind = 0; kind < 4; ++kind) {
      for (const auto& c : walls) {
        if (c.kind != kind) continue;
        switch (kind) {
          case MSB_CONSTRAINT_PLANE:
            plane_rows(out, w, s, c, margin);
            break;
          case MSB_CONSTRAINT_SPHERE:
            sphere_rows(out, w, s, c, margin, eps);
            break;
          case MSB_CONSTRAINT_BOX:
            if (every_face && c.region == MSB_REGION_INSIDE) {
              box_face_rows(out, w, s, c, margin);
            } else {
              box_rows(out, w, s, c, margin, eps);
            }
            break;
          case MSB_CONSTRAINT_CYLINDER:
            if (every_face && c.region == MSB_REGION_INSIDE) {
              cylinder_face_rows(out, w, s, c, margin, eps);
            } else {
              cylinder_rows(out, w, s, c, margin, eps);
            }
            break;
        }
      }
    }
  }
  std::stable_sort(out.begin(), out.end(), [](const External<T>& l, const External<T>& r) {
    return std::tuple{l.cell_id, l.constraint_id, l.location} <
           std::tuple{r.cell_id, r.constraint_id, r.location};
  });
  return out;
}

// ---------------------------------------------------------------- solver

using W6 = std::array<double, 6>;

template <typename T>
using Wrench = std::array<T, 6>;

template <typename T>
struct Row {
  std::uint32_t s1, s2;
  Wrench<T> j1, j2;
  T l1, l2, offset, compliance;
};

template <typename T>
struct Body {
  V3<T> axis;
  T mt, mtr, ma, rate;
  Wrench<T> drift;
};

struct Growth {
  std::uint32_t law;
  float sensitivity, free_load, stall_load;
};

template <typename T>
struct System {
  std::vector<Row<T>> rows;
  std::vector<Body<T>> bodies;
  T dt;
  Growth growth;
};

template <typename T>
T wrench_dot(const Wrench<T>& a, const Wrench<T>& b) {
  T r = 0;
  for (int k = 0; k < 6; ++k) r += a[k] * b[k];
  return r;
}

// apply_mobility (cpu_contact_dynamics.cpp:40-53).
template <typename T>
Wrench<T> apply_mobility(const Body<T>& b, const Wrench<T>& w) {
  const V3<T> tq{w[3], w[4], w[5]};
  const V3<T> ang = tq * b.mtr + b.axis * ((b.ma - b.mtr) * dot(b.axis, tq));
  return {w[0] * b.mt, w[1] * b.mt, w[2] * b.mt, ang.x, ang.y, ang.z};
}

// growth_load_factor (contact_dynamics.cpp:600-612).
template <typename T>
T growth_factor(const Growth& g, T load) {
  switch (g.law) {
    case MSB_GROWTH_LAW_NONE:
      return T(1);
    case MSB_GROWTH_LAW_EXPONENTIAL:
      return std::exp(-T(g.sensitivity) * std::max(T(0), load));
    case MSB_GROWTH_LAW_LINEAR:
      return clampv(T(1) - (load - T(g.free_load)) / (T(g.stall_load) - T(g.free_load)), T(0),
                    T(1));
  }
  throw std::invalid_argument("growth load law is invalid");
}

template <typename T>
T loaded_rate(const Body<T>& b, const Growth& g, T load) {
  return b.rate > T(0) ? b.rate * growth_factor(g, load) : b.rate;
}

struct IncEntry {
  std::uint32_t row;
  bool second;
};

template <typename T>
struct Incidence {
  std::vector<std::uint32_t> offsets;
  std::vector<IncEntry> entries;
};

// make_incidence (cpu_contact_dynamics.cpp:78-106): per body, its rows in row order.
template <typename T>
Incidence<T> make_incidence(const System<T>& s) {
  Incidence<T> inc;
  inc.offsets.assign(s.bodies.size() + 1, 0);
  for (const auto& r : s.rows) {
    ++inc.offsets[r.s1 + 1];
    if (r.s2 != invalid_slot) ++inc.offsets[r.s2 + 1];
  }
  for (std::size_t i = 1; i < inc.offsets.size(); ++i) inc.offsets[i] += inc.offsets[i - 1];
  inc.entries.resize(inc.offsets.back());
  std::vector<std::uint32_t> cur(inc.offsets.begin(), inc.offsets.end() - 1);
  for (std::uint32_t i = 0; i < s.rows.size(); ++i) {
    inc.entries[cur[s.rows[i].s1]++] = {i, false};
    if (s.rows[i].s2 != invalid_slot) inc.entries[cur[s.rows[i].s2]++] = {i, true};
  }
  return inc;
}

template <typename T>
struct Eval {
  std::vector<Wrench<T>> vel;
  std::vector<T> load;
  std::vector<T> rate;
};

// evaluate (cpu_contact_dynamics.cpp:116-146): each body sums its rows in
// row order, skipping zero multipliers.
template <typename T, typename M>
void evaluate(const System<T>& s, const Incidence<T>& inc, const M& mult, Eval<T>& ev) {
  const auto n = s.bodies.size();
  ev.vel.resize(n);
  ev.load.resize(n);
  ev.rate.resize(n);
  for (std::size_t b = 0; b < n; ++b) {
    const auto& body = s.bodies[b];
    Wrench<T> w{};
    T load = 0;
    for (auto k = inc.offsets[b]; k < inc.offsets[b + 1]; ++k) {
      const auto& e = inc.entries[k];
      const T m = mult(e.row);
      if (m == T(0)) continue;
      const auto& row = s.rows[e.row];
      const auto& j = e.second ? row.j2 : row.j1;
      for (int c = 0; c < 6; ++c) w[c] += m * j[c];
      load += (e.second ? row.l2 : row.l1) * m;
    }
    auto v = apply_mobility(body, w);
    for (int c = 0; c < 6; ++c) v[c] += body.drift[c];
    ev.vel[b] = v;
    ev.load[b] = load;
    ev.rate[b] = loaded_rate(body, s.growth, load);
  }
}

// row_gap (cpu_contact_dynamics.cpp:149-159).
template <typename T>
T row_gap(const System<T>& s, const Eval<T>& ev, std::size_t i, T m) {
  const auto& r = s.rows[i];
  T rate = wrench_dot(r.j1, ev.vel[r.s1]) - r.l1 * ev.rate[r.s1];
  if (r.s2 != invalid_slot) rate += wrench_dot(r.j2, ev.vel[r.s2]) - r.l2 * ev.rate[r.s2];
  return r.offset + s.dt * rate + r.compliance * m;
}

template <typename T>
T row_residual(T m, T gap) {
  return m > T(0) ? std::abs(gap) : std::max(T(0), -gap);
}

struct Sums {
  double ss{0}, sy{0}, yy{0};
  double residual{0};
  bool finite{true};
};

constexpr std::size_t row_grain = 256;

// Residual of the gaps of `mult`, with the reference's grains
// (cpu_contact_dynamics.cpp:163-207).
template <typename T>
T evaluate_gaps(const System<T>& s, const Incidence<T>& inc, const std::vector<T>& mult,
                Eval<T>& ev, std::vector<T>& gaps) {
  evaluate(s, inc, [&](std::size_t i) { return mult[i]; }, ev);
  gaps.resize(s.rows.size());
  T residual = 0;
  bool finite = true;
  for (std::size_t i = 0; i < s.rows.size(); ++i) {
    gaps[i] = row_gap(s, ev, i, mult[i]);
    residual = std::max(residual, row_residual(mult[i], gaps[i]));
    finite = finite && std::isfinite(gaps[i]);
  }
  return finite ? residual : std::numeric_limits<T>::quiet_NaN();
}

template <typename T>
T diagonal_bound(const System<T>& s) {
  auto diag = [](const Body<T>& b, const Wrench<T>& j) { return wrench_dot(j, apply_mobility(b, j)); };
  T bound = 0;
  for (const auto& r : s.rows) {
    T e = diag(s.bodies[r.s1], r.j1);
    if (r.s2 != invalid_slot) e += diag(s.bodies[r.s2], r.j2);
    bound = std::max(bound, s.dt * e + r.compliance);
  }
  return bound;
}

template <typename T>
void validate_system(const System<T>& s) {
  if (!std::isfinite(s.dt) || s.dt <= T(0)) {
    throw std::invalid_argument("contact system time step must be finite and positive");
  }
  if (s.growth.law > MSB_GROWTH_LAW_LINEAR || !std::isfinite(s.growth.sensitivity) ||
      s.growth.sensitivity < 0.0F || !std::isfinite(s.growth.free_load) ||
      !std::isfinite(s.growth.stall_load) || s.growth.free_load < 0.0F ||
      s.growth.stall_load <= s.growth.free_load) {
    throw std::invalid_argument("growth load response is invalid");
  }
  for (const auto& b : s.bodies) {
    bool ok = finite3(b.axis) && std::isfinite(b.mt) && std::isfinite(b.mtr) &&
              std::isfinite(b.ma) && std::isfinite(b.rate) && b.mt >= T(0) && b.mtr >= T(0) &&
              b.ma >= T(0);
    for (auto v : b.drift) ok = ok && std::isfinite(v);
    if (!ok) throw std::invalid_argument("contact body is invalid");
  }
  for (const auto& r : s.rows) {
    if (r.s1 >= s.bodies.size() || (r.s2 != invalid_slot && r.s2 >= s.bodies.size())) {
      throw std::invalid_argument("contact row slot is out of range");
    }
    bool ok = std::isfinite(r.offset) && std::isfinite(r.compliance) && r.compliance >= T(0) &&
              std::isfinite(r.l1) && std::isfinite(r.l2) && r.l1 >= T(0) && r.l2 >= T(0);
    for (int k = 0; k < 6; ++k) ok = ok && std::isfinite(r.j1[k]) && std::isfinite(r.j2[k]);
    if (!ok) throw std::invalid_argument("contact row is invalid");
  }
}

template <typename T>
void require_multipliers(const System<T>& s, const std::vector<T>& m) {
  if (m.size() != s.rows.size()) {
    throw std::invalid_argument("contact multiplier count does not match the contact rows");
  }
  for (auto v : m) {
    if (!std::isfinite(v) || v < T(0)) {
      throw std::invalid_argument("contact multipliers must be finite and non-negative");
    }
  }
}

struct SolveReport {
  std::uint32_t status{MSB_SOLVE_CONVERGED};
  std::uint32_t iterations{0};
  double residual{0};
};

// next_contact_step_length (contact_solver.hpp:54-62).
template <typename T>
T next_step(T current, const Sums& s, std::uint32_t iteration) {
  if (!(s.sy > 0.0) || !(s.yy > 0.0)) return current;
  const double next = (iteration % 2U) == 1U ? s.ss / s.sy : s.sy / s.yy;
  return std::isfinite(next) && next > 0.0 ? T(next) : current;
}

// solve_contact_system_cpu (cpu_contact_dynamics.cpp:262-338) driven by
// solve_contact_system / iterate_contact_steps (contact_solver.hpp:66-120).
template <typename T>
SolveReport solve(const System<T>& s, std::vector<T>& mult, T tolerance,
                  std::uint32_t max_iterations) {
  validate_system(s);
  require_multipliers(s, mult);
  if (!std::isfinite(tolerance) || tolerance <= T(0)) {
    throw std::invalid_argument("contact solve tolerance must be finite and positive");
  }
  SolveReport report;
  if (s.rows.empty()) return report;
  const T bound = diagonal_bound(s);
  if (!std::isfinite(bound) || bound <= T(0)) {
    throw std::invalid_argument("contact system has no positive diagonal");
  }
  const auto inc = make_incidence(s);
  const auto n = s.rows.size();
  Eval<T> ev;
  std::vector<T> gaps, next_m(n), next_g(n);
  T step = T(1) / bound;
  report.residual = double(evaluate_gaps(s, inc, mult, ev, gaps));
  if (!std::isfinite(report.residual)) {
    report.status = MSB_SOLVE_BREAKDOWN;
    return report;
  }
  if (report.residual <= double(tolerance)) return report;
  report.status = MSB_SOLVE_ITERATION_LIMIT;
  std::uint32_t iteration = 0;
  while (report.iterations < max_iterations) {
    const T alpha = step;
    auto projected = [&](std::size_t i) { return std::max(T(0), mult[i] - alpha * gaps[i]); };
    evaluate(s, inc, projected, ev);
    Sums total;
    T residual = 0;
    bool finite = true;
    for (std::size_t begin = 0; begin < n; begin += row_grain) {
      Sums piece;
      T piece_res = 0;
      bool piece_fin = true;
      const auto end = std::min(n, begin + row_grain);
      for (std::size_t i = begin; i < end; ++i) {
        const T m = projected(i);
        const T g = row_gap(s, ev, i, m);
        const double moved = double(m) - double(mult[i]);
        const double change = double(g) - double(gaps[i]);
        piece.ss += moved * moved;
        piece.sy += moved * change;
        piece.yy += change * change;
        piece_res = std::max(piece_res, row_residual(m, g));
        piece_fin = piece_fin && std::isfinite(g);
        next_m[i] = m;
        next_g[i] = g;
      }
      total.ss += piece.ss;
      total.sy += piece.sy;
      total.yy += piece.yy;
      residual = std::max(residual, piece_res);
      finite = finite && piece_fin;
    }
    mult.swap(next_m);
    gaps.swap(next_g);
    const T reported = finite ? residual : std::numeric_limits<T>::quiet_NaN();
    ++iteration;
    ++report.iterations;
    report.residual = double(reported);
    if (!std::isfinite(reported)) {
      report.status = MSB_SOLVE_BREAKDOWN;
      return report;
    }
    if (!(reported > tolerance)) {
      report.status = MSB_SOLVE_CONVERGED;
      return report;
    }
    step = next_step(step, total, iteration);
  }
  return report;
}

// -------------------------------------------------------------- stepper

constexpr float minimum_lever_length = 1.0e-6F;
constexpr float solve_tolerance_fraction = 0.25F;
constexpr float load_resolution_fraction = 0.1F;
constexpr std::uint32_t easy_refinements = 2;
constexpr float maximum_substep_rotation = 0.5F;
constexpr float planned_substep_rotation = 0.8F * maximum_substep_rotation;
constexpr std::uint32_t rotation_probe_iterations = 128;

template <typename T>
struct Geometry {
  std::vector<V3<T>> pos, dir;
  std::vector<T> len;
  std::size_t size() const { return len.size(); }
};

template <typename T>
Geometry<T> capture(const World<T>& w) {
  return {w.pos, w.dir, w.len};
}

template <typename T>
void restore(World<T>& w, const Geometry<T>& g) {
  for (std::size_t i = 0; i < g.size(); ++i) w.set_geometry(i, g.pos[i], g.dir[i], g.len[i]);
}

struct Key {
  std::uint32_t first;
  bool wall;
  std::uint64_t partner;
  bool operator==(const Key& o) const {
    return first == o.first && wall == o.wall && partner == o.partner;
  }
};

template <typename T>
struct Touch {
  std::uint32_t s1, s2;
  std::uint64_t partner;
  V3<T> point, normal;
  T sep;
  Key key() const { return {s1, s2 == invalid_slot, partner}; }
};

struct Keyed {
  std::vector<std::uint32_t> offsets, rows;
  Keyed() = default;
  Keyed(std::size_t n, const std::vector<Key>& keys) : offsets(n + 1, 0), rows(keys.size()) {
    for (const auto& k : keys) ++offsets[k.first + 1];
    for (std::size_t i = 0; i < n; ++i) offsets[i + 1] += offsets[i];
    std::vector<std::uint32_t> cur(offsets.begin(), offsets.end() - 1);
    for (std::uint32_t r = 0; r < keys.size(); ++r) rows[cur[keys[r].first]++] = r;
  }
  template <typename F>
  void each(std::uint32_t slot, F&& f) const {
    if (offsets.empty()) return;
    for (auto k = offsets[slot]; k < offsets[slot + 1]; ++k) {
      if (!f(rows[k])) return;
    }
  }
};

template <typename T>
struct Memory {
  Keyed keyed;
  std::vector<Key> keys;
  std::vector<T> mult;
  T force(const Key& key, std::size_t occurrence) const {
    T found = 0;
    bool done = false;
    keyed.each(key.first, [&](std::uint32_t r) {
      if (keys[r] == key && occurrence-- == 0) {
        found = mult[r];
        done = true;
        return false;
      }
      return true;
    });
    return done ? found : T(0);
  }
};

template <typename T>
std::vector<Touch<T>> find_touches(const World<T>& w, const std::vector<Wall<T>>& walls,
                                   msb_contact_parameters cp,
                                   msb_constraint_contact_parameters wp, float margin) {
  cp.activation_margin = margin;
  wp.activation_margin = margin;
  std::vector<Touch<T>> out;
  for (const auto& c : cell_contacts(w, cp)) {
    out.push_back({c.first_slot, c.second_slot, c.second_slot, c.point, c.normal, c.separation});
  }
  if (!walls.empty()) {
    for (const auto& e : external_contacts(w, walls, wp, true)) {
      out.push_back({e.slot, invalid_slot, e.constraint_id, e.point, e.normal, e.separation});
    }
  }
  return out;
}

// length_lever (contact_dynamics.cpp:215-224).
template <typename T>
T length_lever(const Geometry<T>& g, std::uint32_t s, V3<T> centre, V3<T> outward) {
  const T l = g.len[s];
  if (l <= T(minimum_lever_length)) return T(0);
  const V3<T>& ax = g.dir[s];
  const T coord = dot(ax, centre - g.pos[s]) / l;
  return std::max(T(0), clampv(coord, T(-0.5), T(0.5)) * dot(ax, outward));
}

// make_row (contact_dynamics.cpp:230-252).
template <typename T>
Row<T> make_row(const Geometry<T>& g, const std::vector<T>& radii, const Touch<T>& t,
                T compliance, T recovery) {
  Row<T> r{};
  r.s1 = t.s1;
  r.s2 = t.s2;
  r.offset = std::max(t.sep, -recovery);
  r.compliance = t.sep < -recovery ? compliance * recovery / -t.sep : compliance;
  const V3<T>& n = t.normal;
  const V3<T> a1 = cross(t.point - g.pos[t.s1], n);
  r.j1 = {-n.x, -n.y, -n.z, -a1.x, -a1.y, -a1.z};
  r.l1 = length_lever(g, t.s1, t.point - n * radii[t.s1], n);
  if (t.s2 != invalid_slot) {
    const V3<T> a2 = cross(t.point - g.pos[t.s2], n);
    r.j2 = {n.x, n.y, n.z, a2.x, a2.y, a2.z};
    r.l2 = length_lever(g, t.s2, t.point + n * (t.sep + radii[t.s2]), n * T(-1));
  }
  return r;
}

// make_bodies (contact_dynamics.cpp:257-284).
template <typename T>
std::vector<Body<T>> make_bodies(const World<T>& w, const std::vector<T>& rate_lengths, T drag) {
  std::vector<Body<T>> out(w.size());
  for (std::size_t s = 0; s < w.size(); ++s) {
    auto& b = out[s];
    b.axis = w.dir[s];
    b.rate = w.growth[s] * rate_lengths[s];
    b.mt = b.mtr = b.ma = T(0);
    b.drift = {};
    if (w.fixed[s] != 0) continue;
    const T r = w.rad[s];
    const T total = w.len[s] + T(2) * r;
    const T tr = drag * total;
    const T ax = T(0.5) * tr * r * r;
    const T tv = tr * ((total * total) + T(3) * r * r) / T(12);
    b.mt = T(1) / tr;
    b.ma = T(1) / ax;
    b.mtr = T(1) / tv;
  }
  return out;
}

// rotate_axis_angle (cpp/core/mechanics_integration.cpp:9-20).
template <typename T>
V3<T> rotate_axis_angle(V3<T> d, V3<T> rot, T max_rot) {
  const T mag = norm(rot);
  if (mag <= T(1.0e-12F) || max_rot == T(0)) return d;
  const T angle = std::min(mag, max_rot);
  const V3<T> ax = rot * (T(1) / mag);
  const T c = std::cos(angle);
  const T s = std::sin(angle);
  return normalized(d * c + cross(ax, d) * s + ax * (dot(ax, d) * (T(1) - c)));
}

template <typename T>
struct Move {
  std::optional<Geometry<T>> geometry;
  T rotation{0};
};

// moved (contact_dynamics.cpp:311-356).
template <typename T>
Move<T> moved(const Geometry<T>& base, const Eval<T>& resp, T dt) {
  Geometry<T> g;
  const auto n = base.size();
  g.pos.resize(n);
  g.dir.resize(n);
  g.len.resize(n);
  T rotation = 0;
  bool valid = true;
  for (std::size_t s = 0; s < n; ++s) {
    const auto& v = resp.vel[s];
    const V3<T> rot{v[3] * dt, v[4] * dt, v[5] * dt};
    if (!finite3(rot)) {
      valid = false;
      continue;
    }
    const T angle = norm(rot);
    rotation = std::max(rotation, angle);
    if (angle > T(maximum_substep_rotation)) {
      valid = false;
      continue;
    }
    g.pos[s] = base.pos[s] + V3<T>{v[0], v[1], v[2]} * dt;
    g.dir[s] = rotate_axis_angle(base.dir[s], rot, T(maximum_substep_rotation));
    g.len[s] = base.len[s] + resp.rate[s] * dt;
    if (!finite3(g.pos[s]) || !finite3(g.dir[s]) || !std::isfinite(g.len[s]) || g.len[s] < T(0)) {
      valid = false;
    }
  }
  if (!valid) return {std::nullopt, rotation};
  return {std::move(g), rotation};
}

template <typename T>
T largest_rotation(const Eval<T>& resp, T dt) {
  T largest = 0;
  for (const auto& v : resp.vel) {
    const T a = norm(V3<T>{v[3] * dt, v[4] * dt, v[5] * dt});
    largest = std::isfinite(a) ? std::max(largest, a) : std::numeric_limits<T>::infinity();
  }
  return largest;
}

template <typename T>
T effective_tolerance(const msb_contact_dynamics_parameters& p) {
  T scale = 0;
  if (p.growth.law == MSB_GROWTH_LAW_LINEAR) {
    scale = T(p.growth.stall_load) - T(p.growth.free_load);
  } else if (p.growth.law == MSB_GROWTH_LAW_EXPONENTIAL && p.growth.sensitivity > 0.0F) {
    scale = T(1) / T(p.growth.sensitivity);
  }
  if (scale <= T(0)) return T(p.overlap_tolerance);
  return std::min(T(p.overlap_tolerance),
                  T(load_resolution_fraction) * scale / T(p.contact_stiffness));
}

template <typename T>
struct Substep {
  Geometry<T> geometry;
  std::vector<Wrench<T>> vel;
  std::vector<T> loads;
  Memory<T> forces;
  std::uint32_t refinements{0};
  std::size_t rows{0};
  T max_overlap{0};
};

template <typename T>
struct Attempt {
  std::optional<Substep<T>> substep;
  T rotation{0};
};

template <typename T>
void validate_dynamics(const msb_contact_dynamics_parameters& p) {
  auto positive = [](float v) { return std::isfinite(v) && v > 0.0F; };
  if (!positive(p.drag) || !positive(p.contact_stiffness) || !positive(p.wall_stiffness) ||
      !positive(p.overlap_tolerance) || !std::isfinite(p.candidate_margin) ||
      p.candidate_margin < 0.0F || !positive(p.max_overlap_recovery) ||
      !positive(p.max_growth_fraction) || p.max_iterations == 0 || p.flow_drift != 0) {
    throw std::invalid_argument("contact dynamics parameters are invalid");
  }
  if (p.growth.law > MSB_GROWTH_LAW_LINEAR || !std::isfinite(p.growth.sensitivity) ||
      p.growth.sensitivity < 0.0F || !std::isfinite(p.growth.free_load) ||
      !std::isfinite(p.growth.stall_load) || p.growth.free_load < 0.0F ||
      p.growth.stall_load <= p.growth.free_load) {
    throw std::invalid_argument("growth load response is invalid");
  }
}

// advance_substep (contact_dynamics.cpp:418-582).
template <typename T>
Attempt<T> advance_substep(World<T>& w, const Geometry<T>& base, const std::vector<T>& rate_lengths,
                           const std::vector<Wall<T>>& walls, T dt,
                           const msb_contact_dynamics_parameters& p,
                           const msb_contact_parameters& cp,
                           const msb_constraint_contact_parameters& wp, const Memory<T>& remembered,
                           bool probe, std::uint64_t& iterations) {
  const auto& radii = w.rad;
  auto bodies = make_bodies(w, rate_lengths, T(p.drag));
  const auto cands = find_touches(w, walls, cp, wp, p.candidate_margin);
  auto compliance_of = [&](const Touch<T>& t) {
    return T(1) / (t.s2 == invalid_slot ? T(p.wall_stiffness) : T(p.contact_stiffness));
  };
  std::vector<Row<T>> rows(cands.size());
  std::vector<Key> keys(cands.size());
  T starting = 0;
  for (std::size_t i = 0; i < cands.size(); ++i) {
    starting = std::max(starting, -cands[i].sep);
    rows[i] = make_row(base, radii, cands[i], compliance_of(cands[i]), T(p.max_overlap_recovery));
    keys[i] = cands[i].key();
  }
  const T tolerance = effective_tolerance<T>(p);
  const T slack = tolerance + std::max(T(0), starting - T(p.max_overlap_recovery));
  const T solve_tol = T(solve_tolerance_fraction) * tolerance;
  Keyed keyed(bodies.size(), keys);
  T rotation = 0;
  std::vector<T> mult(rows.size(), T(0));
  for (std::size_t i = 0; i < rows.size(); ++i) {
    std::size_t occurrence = 0;
    keyed.each(keys[i].first, [&](std::uint32_t r) {
      if (r >= i) return false;
      occurrence += keys[r] == keys[i] ? 1 : 0;
      return true;
    });
    mult[i] = remembered.force(keys[i], occurrence);
  }
  for (std::uint32_t refinement = 0; refinement <= p.max_refinements; ++refinement) {
    System<T> sys{rows, bodies, dt, {p.growth.law, p.growth.sensitivity, p.growth.free_load,
                                     p.growth.stall_load}};
    auto remaining = p.max_iterations;
    if (probe && refinement == 0 && remaining > rotation_probe_iterations) {
      auto early = mult;
      const auto rep = solve(sys, early, solve_tol, rotation_probe_iterations);
      iterations += rep.iterations;
      remaining -= rep.iterations;
      if (rep.status == MSB_SOLVE_BREAKDOWN) break;
      mult = std::move(early);
      if (rep.status != MSB_SOLVE_CONVERGED) {
        Eval<T> ev;
        evaluate(sys, make_incidence(sys), [&](std::size_t i) { return mult[i]; }, ev);
        rotation = largest_rotation(ev, dt);
        if (rotation > T(maximum_substep_rotation)) break;
      }
    }
    auto solved = mult;
    const auto rep = solve(sys, solved, solve_tol, remaining);
    iterations += rep.iterations;
    if (rep.status != MSB_SOLVE_CONVERGED) break;
    mult = std::move(solved);
    Eval<T> resp;
    evaluate(sys, make_incidence(sys), [&](std::size_t i) { return mult[i]; }, resp);
    auto mv = moved(base, resp, dt);
    rotation = mv.rotation;
    if (!mv.geometry) break;
    const auto& trial = *mv.geometry;
    restore(w, trial);
    const auto found = find_touches(w, walls, cp, wp, 0.0F);
    auto force_on = [&](const Key& key) {
      T f = 0;
      keyed.each(key.first, [&](std::uint32_t r) {
        if (keys[r] == key) f += mult[r];
        return true;
      });
      return f;
    };
    T max_overlap = 0;
    std::vector<Touch<T>> overlapping;
    for (const auto& t : found) {
      max_overlap = std::max(max_overlap, -t.sep);
      const T allowed = slack + force_on(t.key()) * compliance_of(t);
      if (t.sep < -allowed) overlapping.push_back(t);
    }
    if (overlapping.empty()) {
      Substep<T> sub{*mv.geometry, resp.vel, resp.load, {keyed, keys, mult}, refinement,
                     rows.size(), max_overlap};
      return {std::move(sub), rotation};
    }
    for (const auto& t : overlapping) {
      auto row = make_row(trial, radii, t, compliance_of(t), T(p.max_overlap_recovery));
      T rate = wrench_dot(row.j1, resp.vel[row.s1]) - row.l1 * resp.rate[row.s1];
      if (row.s2 != invalid_slot) {
        rate += wrench_dot(row.j2, resp.vel[row.s2]) - row.l2 * resp.rate[row.s2];
      }
      row.offset -= dt * rate;
      rows.push_back(row);
      keys.push_back(t.key());
      mult.push_back(T(0));
    }
    keyed = Keyed(bodies.size(), keys);
  }
  restore(w, base);
  return {std::nullopt, rotation};
}

template <typename T>
struct StepResult {
  msb_contact_dynamics_report report{};
  std::vector<V3<T>> velocities;
  std::vector<T> loads;
  std::vector<T> increments;
};

// advance_contact_dynamics (contact_dynamics.cpp:676-782).
template <typename T>
StepResult<T> advance(World<T>& w, const std::vector<Wall<T>>& walls, float dt_in,
                      const msb_contact_dynamics_parameters& p, const msb_contact_parameters& cp,
                      const msb_constraint_contact_parameters& wp) {
  if (!std::isfinite(dt_in) || dt_in < 0.0F) {
    throw std::invalid_argument("time step must be finite and non-negative");
  }
  validate_dynamics<T>(p);
  StepResult<T> result;
  result.velocities.assign(w.size(), V3<T>{});
  result.loads.assign(w.size(), T(0));
  result.increments.assign(w.size(), T(0));
  if (w.size() == 0 || dt_in == 0.0F) return result;
  const T dt = T(dt_in);
  const auto initial = capture(w);
  auto base = initial;
  try {
    T growth = 0;
    for (std::size_t s = 0; s < w.size(); ++s) {
      growth = std::max(growth, std::abs(w.growth[s]) * w.len[s] * T(0.5) * dt / w.rad[s]);
    }
    const T pieces = std::max(T(1), std::ceil(growth / T(p.max_growth_fraction)));
    if (!std::isfinite(pieces)) throw std::runtime_error("contact dynamics growth per step is not finite");
    const T longest = dt / pieces;
    const T shortest = std::ldexp(longest, -int(p.max_step_halvings));
    double remaining = double(dt);
    T length = longest;
    T proven = 0;
    Memory<T> forces;
    while (remaining > 0.0) {
      if (double(length) >= remaining * (1.0 - 1.0e-6)) length = T(remaining);
      auto attempt = advance_substep(w, base, initial.len, walls, length, p, cp, wp, forces,
                                     length > proven, result.report.iterations);
      if (!attempt.substep) {
        const T excess = attempt.rotation / T(planned_substep_rotation);
        const std::uint32_t halvings =
            excess > T(2) ? std::uint32_t(std::ceil(std::log2(excess))) : 1u;
        const T failed = length;
        length = std::ldexp(length, -int(std::min<std::uint32_t>(halvings, 64)));
        result.report.halvings += halvings;
        if (length < shortest) {
          throw std::runtime_error(
              "contact dynamics did not resolve the contacts of a substep of " +
              std::to_string(double(failed)));
        }
        continue;
      }
      auto& sub = *attempt.substep;
      remaining -= double(length);
      proven = std::max(proven, length);
      base = std::move(sub.geometry);
      if (remaining <= 0.0) {
        for (std::size_t s = 0; s < w.size(); ++s) {
          result.velocities[s] = {sub.vel[s][0], sub.vel[s][1], sub.vel[s][2]};
        }
      }
      result.loads = sub.loads;
      ++result.report.substeps;
      result.report.refinements += sub.refinements;
      result.report.max_rows = std::max<std::uint64_t>(result.report.max_rows, sub.rows);
      result.report.max_overlap = float(sub.max_overlap);
      forces = std::move(sub.forces);
      if (sub.refinements <= easy_refinements &&
          T(2) * attempt.rotation <= T(planned_substep_rotation)) {
        length = std::min(longest, length * T(2));
      }
    }
  } catch (...) {
    restore(w, initial);
    throw;
  }
  for (std::size_t s = 0; s < initial.size(); ++s) result.increments[s] = base.len[s] - initial.len[s];
  return result;
}

// ------------------------------------------------------------ conversion

template <typename T>
System<T> system_from(const msb_contact_system& s) {
  System<T> out;
  out.rows.resize(s.row_count);
  for (std::uint64_t i = 0; i < s.row_count; ++i) {
    const auto& r = s.rows[i];
    auto& o = out.rows[i];
    o.s1 = r.first_slot;
    o.s2 = r.second_slot;
    for (int k = 0; k < 6; ++k) {
      o.j1[k] = T(r.first_jacobian[k]);
      o.j2[k] = T(r.second_jacobian[k]);
    }
    o.l1 = T(r.first_length_lever);
    o.l2 = T(r.second_length_lever);
    o.offset = T(r.offset);
    o.compliance = T(r.compliance);
  }
  out.bodies.resize(s.body_count);
  for (std::uint64_t i = 0; i < s.body_count; ++i) {
    const auto& b = s.bodies[i];
    auto& o = out.bodies[i];
    o.axis = {T(b.axis.x), T(b.axis.y), T(b.axis.z)};
    o.mt = T(b.translational_mobility);
    o.mtr = T(b.transverse_mobility);
    o.ma = T(b.axial_mobility);
    o.rate = T(b.length_rate);
    for (int k = 0; k < 6; ++k) o.drift[k] = T(b.drift[k]);
  }
  out.dt = T(s.dt);
  out.growth = {s.growth.law, s.growth.sensitivity, s.growth.free_load, s.growth.stall_load};
  return out;
}

thread_local std::string last_error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    last_error.clear();
    return MSB_OK;
  } catch (const std::invalid_argument& e) {
    last_error = e.what();
    return MSB_ERR_INVALID_ARGUMENT;
  } catch (const std::overflow_error& e) {
    last_error = e.what();
    return MSB_ERR_OVERFLOW;
  } catch (const std::length_error& e) {
    last_error = e.what();
    return MSB_ERR_CAPACITY;
  } catch (const std::exception& e) {
    last_error = e.what();
    return MSB_ERR_RUNTIME;
  }
}

template <typename T>
void cell_contacts_out(const msb_cell_arrays* cells, const msb_contact_parameters* prm,
                       msb_cell_contact* out, std::uint64_t cap, std::uint64_t* count) {
  const auto w = world_from<T>(*cells);
  const auto contacts = cell_contacts(w, *prm);
  *count = contacts.size();
  if (contacts.size() > cap) throw std::length_error("capacity");
  for (std::size_t i = 0; i < contacts.size(); ++i) {
    const auto& c = contacts[i];
    out[i] = {c.first_id,
              c.second_id,
              c.first_slot,
              c.second_slot,
              c.ordinal,
              {float(c.point.x), float(c.point.y), float(c.point.z)},
              {float(c.normal.x), float(c.normal.y), float(c.normal.z)},
              float(c.separation),
              float(c.weight),
              0};
  }
}

template <typename T>
void external_out(const msb_cell_arrays* cells, const msb_constraint* cs, std::uint64_t n,
                  const msb_constraint_contact_parameters* prm, std::uint32_t every_face,
                  msb_external_contact* out, std::uint64_t cap, std::uint64_t* count) {
  const auto w = world_from<T>(*cells);
  const auto contacts = external_contacts(w, walls_from<T>(cs, n), *prm, every_face != 0);
  *count = contacts.size();
  if (contacts.size() > cap) throw std::length_error("capacity");
  for (std::size_t i = 0; i < contacts.size(); ++i) {
    const auto& c = contacts[i];
    out[i] = {c.cell_id,
              c.constraint_id,
              c.slot,
              c.kind,
              c.location,
              {float(c.point.x), float(c.point.y), float(c.point.z)},
              {float(c.normal.x), float(c.normal.y), float(c.normal.z)},
              float(c.separation),
              float(c.weight),
              0};
  }
}

}  // namespace oracle

using namespace oracle;

extern "C" {

const char* oracle_last_error(void) {
  return oracle::last_error.c_str();
}

// precision: 0 = FP32 (the reference's arithmetic), 1 = FP64.
int oracle_find_cell_contacts(uint32_t precision, const msb_cell_arrays* cells,
                              const msb_contact_parameters* prm, msb_cell_contact* out,
                              uint64_t cap, uint64_t* count) {
  return guarded([&] {
    if (precision == 0) {
      cell_contacts_out<float>(cells, prm, out, cap, count);
    } else {
      cell_contacts_out<double>(cells, prm, out, cap, count);
    }
  });
}

int oracle_find_cell_contact_candidates(const msb_cell_arrays* cells, float margin, uint32_t* pairs,
                                        uint64_t cap, uint64_t* count) {
  return guarded([&] {
    const auto w = world_from<float>(*cells);
    const auto c = candidates(w, margin);
    *count = c.size();
    if (c.size() > cap) throw std::length_error("capacity");
    for (std::size_t i = 0; i < c.size(); ++i) {
      pairs[2 * i] = c[i].first;
      pairs[2 * i + 1] = c[i].second;
    }
  });
}

int oracle_find_external_contacts(uint32_t precision, const msb_cell_arrays* cells,
                                  const msb_constraint* cs, uint64_t n,
                                  const msb_constraint_contact_parameters* prm,
                                  uint32_t every_face, msb_external_contact* out, uint64_t cap,
                                  uint64_t* count) {
  return guarded([&] {
    if (precision == 0) {
      external_out<float>(cells, cs, n, prm, every_face, out, cap, count);
    } else {
      external_out<double>(cells, cs, n, prm, every_face, out, cap, count);
    }
  });
}

int oracle_solve_contact_forces(uint32_t precision, const msb_contact_system* system,
                                const float* initial, const msb_contact_solve_parameters* prm,
                                float* mult_out, msb_contact_solve_report* report) {
  return guarded([&] {
    auto run = [&](auto zero) {
      using T = decltype(zero);
      const auto sys = system_from<T>(*system);
      std::vector<T> mult(initial, initial + system->row_count);
      const auto rep = solve(sys, mult, T(prm->tolerance), prm->max_iterations);
      for (std::size_t i = 0; i < mult.size(); ++i) mult_out[i] = float(mult[i]);
      report->status = rep.status;
      report->iterations = rep.iterations;
      report->residual = float(rep.residual);
    };
    if (precision == 0) {
      run(0.0F);
    } else {
      run(0.0);
    }
  });
}

int oracle_evaluate_contact_response(uint32_t precision, const msb_contact_system* system,
                                     const float* mult_in, float* velocities, float* loads,
                                     float* rates) {
  return guarded([&] {
    auto run = [&](auto zero) {
      using T = decltype(zero);
      const auto sys = system_from<T>(*system);
      validate_system(sys);
      std::vector<T> mult(mult_in, mult_in + system->row_count);
      require_multipliers(sys, mult);
      Eval<T> ev;
      evaluate(sys, make_incidence(sys), [&](std::size_t i) { return mult[i]; }, ev);
      for (std::size_t b = 0; b < sys.bodies.size(); ++b) {
        if (velocities) {
          for (int k = 0; k < 6; ++k) velocities[6 * b + k] = float(ev.vel[b][k]);
        }
        if (loads) loads[b] = float(ev.load[b]);
        if (rates) rates[b] = float(ev.rate[b]);
      }
    };
    if (precision == 0) {
      run(0.0F);
    } else {
      run(0.0);
    }
  });
}

int oracle_evaluate_contact_gaps(uint32_t precision, const msb_contact_system* system,
                                 const float* mult_in, float* gaps_out) {
  return guarded([&] {
    auto run = [&](auto zero) {
      using T = decltype(zero);
      const auto sys = system_from<T>(*system);
      validate_system(sys);
      std::vector<T> mult(mult_in, mult_in + system->row_count);
      require_multipliers(sys, mult);
      Eval<T> ev;
      std::vector<T> gaps;
      evaluate_gaps(sys, make_incidence(sys), mult, ev, gaps);
      for (std::size_t i = 0; i < gaps.size(); ++i) gaps_out[i] = float(gaps[i]);
    };
    if (precision == 0) {
      run(0.0F);
    } else {
      run(0.0);
    }
  });
}

int oracle_contact_system_diagonal_bound(uint32_t precision, const msb_contact_system* system,
                                         float* bound) {
  return guarded([&] {
    if (precision == 0) {
      *bound = diagonal_bound(system_from<float>(*system));
    } else {
      *bound = float(diagonal_bound(system_from<double>(*system)));
    }
  });
}

int oracle_advance_contact_dynamics(uint32_t precision, msb_cell_arrays* cells,
                                    const msb_constraint* cs, uint64_t n, float dt,
                                    const msb_contact_dynamics_parameters* dyn,
                                    const msb_contact_parameters* cp,
                                    const msb_constraint_contact_parameters* wp,
                                    msb_contact_dynamics_report* report,
                                    msb_contact_dynamics_outputs* outputs) {
  return guarded([&] {
    auto run = [&](auto zero) {
      using T = decltype(zero);
      auto w = world_from<T>(*cells);
      const auto walls = walls_from<T>(cs, n);
      const auto r = advance(w, walls, dt, *dyn, *cp, *wp);
      world_to(w, *cells);
      *report = r.report;
      if (outputs) {
        for (std::size_t s = 0; s < w.size(); ++s) {
          if (outputs->center_velocities) {
            outputs->center_velocities[3 * s] = float(r.velocities[s].x);
            outputs->center_velocities[3 * s + 1] = float(r.velocities[s].y);
            outputs->center_velocities[3 * s + 2] = float(r.velocities[s].z);
          }
          if (outputs->axial_loads) outputs->axial_loads[s] = float(r.loads[s]);
          if (outputs->length_increments) outputs->length_increments[s] = float(r.increments[s]);
        }
      }
    };
    if (precision == 0) {
      run(0.0F);
    } else {
      run(0.0);
    }
  });
}

}  // extern "C"
