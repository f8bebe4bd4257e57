// =====================================================================================
// cc_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU restatement of CutCellMethods.jl's `update_cache!` hot path (MarchingSquaresCutCell,
// MarchingCubesCutCell, PLICCutCell, calc_volume), used only by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU baseline leg as the checker. Nothing in the
// product links or calls it.
//
// Every construction follows the reference's expression order (StaticArrays left folds,
// elementwise division, no FMA contraction: build with -ffp-contract=off -fno-fast-math), so
// that a device kernel compiled with --fmad=false can be compared bit for bit.
//
// What this file cannot restate bit-exactly, because the code is absent from the reference
// checkout (third-party packages pinned in Manifest.toml but not vendored):
//   * SDFLibrary 0.10.5 `sdf_value` / `get_sdf`: replaced by the op-tape primitives defined in
//     include/cutcell_b200.h, written from each body's mathematics. The PLIC normal is the
//     forward-mode gradient of the same expression.
//   * CartesianMeshes 0.2.3 `get_node` / `get_elem_centroid` / `get_volume_fraction`: node
//     coordinates are taken as x0 + T(i)*d (0-based i), centroids as x0 + T(i + 0.5)*d, and the
//     plane-cube clip is the analytic formula of Scardovelli & Zaleski (2000).
//   * MarchingCubes.jl 0.1.11 Lewiner tables: the per-cube dispatch of
//     src/marching_cubes/marching_cubes.jl:538-651 is restated here over a table blob passed in by
//     the caller (the format of include/cutcell_b200.h); the tests pass a project-designed tiling.
// Parity of these pieces against the reference is therefore "unpinned" here; everything else is
// pinned against the reference tests' golden values (tests/test_oracle_*.py).
// =====================================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <map>
#include <utility>
#include <algorithm>
#include <thread>
#include <atomic>
#include <type_traits>
#include "../include/cutcell_b200.h"

namespace oc {

// ----------------------------------------------------------------------------------
// Host threading: a static split of [0, n) over std::threads (the toolchain here has no OpenMP
// runtime). Each index is processed by exactly one thread and every output slot is written by
// the index that owns it, so results do not depend on the thread count.
static int g_threads = 1;
template <class F>
void parallel_for(int64_t n, F f) {
  int nt = g_threads;
  if (nt <= 1 || n < 2) { for (int64_t i = 0; i < n; ++i) f(i); return; }
  if (nt > n) nt = int(n);
  std::atomic<int64_t> next(0);
  const int64_t chunk = std::max<int64_t>(1, n / (int64_t(nt) * 16));
  auto work = [&]() {
    for (;;) {
      const int64_t b = next.fetch_add(chunk);
      if (b >= n) break;
      const int64_t e = std::min(n, b + chunk);
      for (int64_t i = b; i < e; ++i) f(i);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
}

// ----------------------------------------------------------------------------------
// Forward-mode dual numbers: the value and its gradient in D coordinates.
template <class T, int D>
struct Dual {
  T v;
  T g[D];
};
template <class T> inline T val(T x) { return x; }
template <class T, int D> inline T val(const Dual<T, D>& x) { return x.v; }

template <class T, int D> inline Dual<T, D> dconst(T c) {
  Dual<T, D> r; r.v = c; for (int i = 0; i < D; ++i) r.g[i] = T(0); return r;
}
template <class T, int D> inline Dual<T, D> operator+(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v + b.v; for (int i = 0; i < D; ++i) r.g[i] = a.g[i] + b.g[i]; return r;
}
template <class T, int D> inline Dual<T, D> operator-(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v - b.v; for (int i = 0; i < D; ++i) r.g[i] = a.g[i] - b.g[i]; return r;
}
template <class T, int D> inline Dual<T, D> operator-(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = -a.v; for (int i = 0; i < D; ++i) r.g[i] = -a.g[i]; return r;
}
template <class T, int D> inline Dual<T, D> operator*(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v * b.v;
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
template <class T, int D> inline Dual<T, D> operator/(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v / b.v;
  const T bb = b.v * b.v;
  for (int i = 0; i < D; ++i) r.g[i] = (a.g[i] * b.v - a.v * b.g[i]) / bb;
  return r;
}
template <class T, int D> inline Dual<T, D> operator+(const Dual<T, D>& a, T c) { Dual<T, D> r = a; r.v = a.v + c; return r; }
template <class T, int D> inline Dual<T, D> operator-(const Dual<T, D>& a, T c) { Dual<T, D> r = a; r.v = a.v - c; return r; }
template <class T, int D> inline Dual<T, D> operator-(T c, const Dual<T, D>& a) { Dual<T, D> r = -a; r.v = c - a.v; return r; }
template <class T, int D> inline Dual<T, D> operator*(T c, const Dual<T, D>& a) {
  Dual<T, D> r; r.v = c * a.v; for (int i = 0; i < D; ++i) r.g[i] = c * a.g[i]; return r;
}
template <class T, int D> inline Dual<T, D> operator*(const Dual<T, D>& a, T c) {
  Dual<T, D> r; r.v = a.v * c; for (int i = 0; i < D; ++i) r.g[i] = a.g[i] * c; return r;
}
template <class T, int D> inline Dual<T, D> operator/(const Dual<T, D>& a, T c) {
  Dual<T, D> r; r.v = a.v / c; for (int i = 0; i < D; ++i) r.g[i] = a.g[i] / c; return r;
}
template <class T, int D> inline Dual<T, D> dsqrt(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = std::sqrt(a.v);
  const T two_s = T(2) * r.v;
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] / two_s;
  return r;
}
template <class T, int D> inline Dual<T, D> dabs(const Dual<T, D>& a) {
  // sign(0) == 0, so the gradient of |x| at x == 0 is zero.
  const T sg = a.v > T(0) ? T(1) : (a.v < T(0) ? T(-1) : T(0));
  Dual<T, D> r; r.v = std::fabs(a.v); for (int i = 0; i < D; ++i) r.g[i] = sg * a.g[i]; return r;
}
template <class T, int D> inline Dual<T, D> dsin(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = std::sin(a.v); const T c = std::cos(a.v);
  for (int i = 0; i < D; ++i) r.g[i] = c * a.g[i];
  return r;
}
template <class T, int D> inline Dual<T, D> dcos(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = std::cos(a.v); const T s = -std::sin(a.v);
  for (int i = 0; i < D; ++i) r.g[i] = s * a.g[i];
  return r;
}
template <class T, int D> inline Dual<T, D> datan2(const Dual<T, D>& y, const Dual<T, D>& x) {
  Dual<T, D> r; r.v = std::atan2(y.v, x.v);
  const T den = x.v * x.v + y.v * y.v;
  for (int i = 0; i < D; ++i) r.g[i] = (x.v * y.g[i] - y.v * x.g[i]) / den;
  return r;
}
// scalar overloads so one template serves T and Dual<T,D>
template <class T> inline T dsqrt(T a) { return std::sqrt(a); }
template <class T> inline T dabs(T a) { return std::fabs(a); }
template <class T> inline T dsin(T a) { return std::sin(a); }
template <class T> inline T dcos(T a) { return std::cos(a); }
template <class T> inline T datan2(T y, T x) { return std::atan2(y, x); }

template <class S> struct Lift;  // constant of the evaluation type
template <> struct Lift<float> { static float c(float x) { return x; } };
template <> struct Lift<double> { static double c(double x) { return x; } };
template <class T, int D> struct Lift<Dual<T, D>> { static Dual<T, D> c(T x) { return dconst<T, D>(x); } };

// ----------------------------------------------------------------------------------
// The op-tape: SDF primitives and CSG combinators (include/cutcell_b200.h). Stands in for
// SDFLibrary.jl's `sdf_value` (src/marching_squares/cache.jl:69) and `get_sdf`
// (src/plic/plic.jl:74).
template <class T>
struct Tape {
  std::vector<cc_op> ops;
  std::vector<T> p;
};

template <class T, int D, class S>
inline S prim(const cc_op& op, const T* p, const S* x) {
  switch (op.opcode) {
    case CC_OP_SPHERE: {
      const T* c = p + op.poff;
      S u = (x[0] - c[0]) * (x[0] - c[0]);
      for (int a = 1; a < D; ++a) u = u + (x[a] - c[a]) * (x[a] - c[a]);
      return dsqrt(u) - c[D];
    }
    case CC_OP_BOX: {
      const T* c = p + op.poff;
      const T* h = c + D;
      S q[D];
      for (int a = 0; a < D; ++a) q[a] = dabs(x[a] - c[a]) - h[a];
      // outside part: |max(q, 0)|
      S zero = Lift<S>::c(T(0));
      S qp0 = val(q[0]) > T(0) ? q[0] : zero;
      S u = qp0 * qp0;
      for (int a = 1; a < D; ++a) { S qa = val(q[a]) > T(0) ? q[a] : zero; u = u + qa * qa; }
      S outside = dsqrt(u);
      // inside part: min(max_a q_a, 0)
      S m = q[0];
      for (int a = 1; a < D; ++a) m = val(q[a]) > val(m) ? q[a] : m;
      S inside = val(m) < T(0) ? m : zero;
      return outside + inside;
    }
    case CC_OP_TORUS: if constexpr (D == 3) {
      const T* c = p + op.poff;
      const T* R = c + 3;
      S d0 = x[0] - c[0], d1 = x[1] - c[1], d2 = x[2] - c[2];
      S l0 = R[0] * d0 + R[1] * d1 + R[2] * d2;
      S l1 = R[3] * d0 + R[4] * d1 + R[5] * d2;
      S l2 = R[6] * d0 + R[7] * d1 + R[8] * d2;
      S qx = dsqrt(l0 * l0 + l1 * l1) - c[12];
      return dsqrt(qx * qx + l2 * l2) - c[13];
    } else { return Lift<S>::c(std::numeric_limits<T>::quiet_NaN()); }
    case CC_OP_PLANE: {
      const T* pt = p + op.poff;
      const T* n = pt + D;
      S s = n[0] * (x[0] - pt[0]);
      for (int a = 1; a < D; ++a) s = s + n[a] * (x[a] - pt[a]);
      return s;
    }
    case CC_OP_TRIG: {
      const T* q = p + op.poff;
      S s = q[0] * dsin(q[1] * x[0]);
      for (int a = 1; a < D; ++a) s = s * dsin(q[1 + a] * x[a]);
      return s + q[1 + D];
    }
    case CC_OP_CONST:
      return Lift<S>::c(p[op.poff]);
    case CC_OP_STAR: if constexpr (D == 2) {
      const T* q = p + op.poff;
      S dx = x[0] - q[0], dy = x[1] - q[1];
      S rad = dsqrt(dx * dx + dy * dy);
      S th = datan2(dy, dx);
      S r = Lift<S>::c(q[2]);
      for (int k = 2; k <= 6; ++k) r = r + q[3 + (k - 2)] * dcos(T(k) * th + q[8 + (k - 2)]);
      return rad - r;
    } else { return Lift<S>::c(std::numeric_limits<T>::quiet_NaN()); }
    default:
      return Lift<S>::c(std::numeric_limits<T>::quiet_NaN());
  }
}

template <class T, class S>
inline S combine(int mode, const S& top, const S& v, T k) {
  switch (mode) {
    case CC_COMB_MIN: return val(v) < val(top) ? v : top;
    case CC_COMB_MAX: return val(v) > val(top) ? v : top;
    case CC_COMB_SUB: { S w = -v; return val(w) > val(top) ? w : top; }
    case CC_COMB_SMIN: {
      // polynomial smooth minimum: min(a,b) - h^2 k / 4, h = max(k - |a-b|, 0) / k
      S ad = dabs(top - v);
      S hk = k - ad;
      S zero = Lift<S>::c(T(0));
      S h = (val(hk) > T(0) ? hk : zero) / k;
      S m = val(v) < val(top) ? v : top;
      return m - ((h * h) * k) * T(0.25);
    }
    default: return v;
  }
}

template <class T, int D, class S>
inline S eval_tape(const Tape<T>& t, const S* x) {
  S st[CC_TAPE_MAX_STACK];
  int sp = 0;
  for (size_t i = 0; i < t.ops.size(); ++i) {
    const cc_op& op = t.ops[i];
    S v;
    if (op.opcode == CC_OP_NONE) {
      if (op.combine == CC_COMB_NEG) { st[sp - 1] = -st[sp - 1]; continue; }
      v = st[--sp];
    } else {
      v = prim<T, D, S>(op, t.p.data(), x);
    }
    if (op.combine == CC_COMB_PUSH) st[sp++] = v;
    else st[sp - 1] = combine<T, S>(op.combine, st[sp - 1], v, op.combine == CC_COMB_SMIN ? t.p[op.kparam] : T(0));
  }
  return st[0];
}

// ----------------------------------------------------------------------------------
// CartesianMeshes stand-ins.
template <class T> inline T node_coord(T x0, T d, int64_t i) { return x0 + T(i) * d; }
template <class T> inline T centroid_coord(T x0, T d, int64_t i) { return x0 + T(double(i) + 0.5) * d; }

// Solid fraction of the unit square {n . xi <= a}, Scardovelli & Zaleski (2000), 2D form.
template <class T>
inline T gvf2(T n1, T n2, T a) {
  T m1 = std::fabs(n1), m2 = std::fabs(n2);
  T alpha = a;
  if (n1 < T(0)) alpha = alpha + m1;
  if (n2 < T(0)) alpha = alpha + m2;
  const T s = m1 + m2;
  if (!(s > T(0))) return alpha >= T(0) ? T(1) : T(0);
  m1 = m1 / s; m2 = m2 / s; alpha = alpha / s;
  if (alpha <= T(0)) return T(0);
  if (alpha >= T(1)) return T(1);
  const bool flip = alpha > T(0.5);
  if (flip) alpha = T(1) - alpha;
  if (m1 > m2) std::swap(m1, m2);
  T v;
  if (alpha < m1) v = (alpha * alpha) / (T(2) * m1 * m2);
  else v = (alpha - T(0.5) * m1) / m2;
  return flip ? T(1) - v : v;
}

// Solid fraction of the unit cube {n . xi <= a}, Scardovelli & Zaleski (2000).
template <class T>
inline T gvf3(T n1, T n2, T n3, T a) {
  T m[3] = {std::fabs(n1), std::fabs(n2), std::fabs(n3)};
  T alpha = a;
  if (n1 < T(0)) alpha = alpha + m[0];
  if (n2 < T(0)) alpha = alpha + m[1];
  if (n3 < T(0)) alpha = alpha + m[2];
  const T s = (m[0] + m[1]) + m[2];
  if (!(s > T(0))) return alpha >= T(0) ? T(1) : T(0);
  m[0] = m[0] / s; m[1] = m[1] / s; m[2] = m[2] / s; alpha = alpha / s;
  if (alpha <= T(0)) return T(0);
  if (alpha >= T(1)) return T(1);
  const bool flip = alpha > T(0.5);
  if (flip) alpha = T(1) - alpha;
  if (m[0] > m[1]) std::swap(m[0], m[1]);
  if (m[1] > m[2]) std::swap(m[1], m[2]);
  if (m[0] > m[1]) std::swap(m[0], m[1]);
  const T m1 = m[0], m2 = m[1], m3 = m[2];
  const T m12 = m1 + m2;
  T v;
  // alpha^3 - (alpha - m1)^3 is expanded as m1 * (3 alpha^2 - 3 alpha m1 + m1^2) so that no branch
  // divides a cancelling difference by a small m1; the remaining cubes (alpha - m2)^3 and
  // (alpha - m3)^3 are below m1^3 wherever they appear.
  if (alpha < m1) {
    v = (alpha * alpha * alpha) / (T(6) * m1 * m2 * m3);
  } else {
    const T core = (T(3) * alpha * alpha - T(3) * alpha * m1 + m1 * m1) / (T(6) * m2 * m3);
    if (alpha < m2) {
      v = core;
    } else if (alpha < std::min(m12, m3)) {
      const T u = alpha - m2;
      v = core - (u * u * u) / (T(6) * m1 * m2 * m3);
    } else if (m3 < m12) {
      const T u = alpha - m2, w = alpha - m3;
      v = core - (u * u * u + w * w * w) / (T(6) * m1 * m2 * m3);
    } else {
      v = (T(2) * alpha - m12) / (T(2) * m3);
    }
  }
  return flip ? T(1) - v : v;
}

// ----------------------------------------------------------------------------------
// Marching squares (src/marching_squares/marching_squares.jl, src/marching_squares/moments.jl).
// Edges 0..3 of the counter-clockwise walk; 0-based forms of MS_EDGE_DIRECTION /
// MS_DIRECTION_EDGE (marching_squares.jl:81-82).
static const int MS_DIRECTION_EDGE0[4] = {3, 1, 0, 2};
inline int ms_next(int k) { return (k + 1) & 3; }
inline int ms_prev(int k) { return (k + 3) & 3; }

// Mixed precision (prec 2 at the C entry points): Float32 data and arithmetic with Float64
// islands -- the edge root when the Float32 denominator is below 2^-100, the asymptotic deciders,
// the PLIC plane-cube clips. A process-wide flag, set for the duration of one entry-point call.
inline bool& mixed_flag() {
  static bool m = false;
  return m;
}
struct MixedScope {
  bool old;
  explicit MixedScope(bool m) : old(mixed_flag()) { mixed_flag() = m; }
  ~MixedScope() { mixed_flag() = old; }
};
template <class T> inline bool mixed_on() { return std::is_same<T, float>::value && mixed_flag(); }
constexpr float MIXED_TINY = 7.8886090522101181e-31f;  // 2^-100

// _open_fraction, marching_squares.jl:192-198
template <class T>
inline T open_fraction(T pa, T pb) {
  const bool fa = pa >= T(0), fb = pb >= T(0);
  if (fa && fb) return T(1);
  if (!fa && !fb) return T(0);
  if (mixed_on<T>()) {
    const T den = fa ? pa - pb : pb - pa;
    if (std::fabs(den) < T(MIXED_TINY))
      return T(fa ? double(pa) / (double(pa) - double(pb)) : double(pb) / (double(pb) - double(pa)));
  }
  return fa ? pa / (pa - pb) : pb / (pb - pa);
}

// The plane-cube clips; under mixed precision evaluated in Float64 and rounded once.
template <class T> inline T gvf2p(T n1, T n2, T a) {
  return mixed_on<T>() ? T(gvf2<double>(n1, n2, a)) : gvf2<T>(n1, n2, a);
}
template <class T> inline T gvf3p(T n1, T n2, T n3, T a) {
  return mixed_on<T>() ? T(gvf3<double>(n1, n2, n3, a)) : gvf3<T>(n1, n2, n3, a);
}

// _open_segment, marching_squares.jl:208-217
template <class T>
inline void open_segment(const T* pa, const T* pb, T fa, T fb, T frac, T* a, T* b) {
  if (fa >= T(0) && fb >= T(0)) {
    a[0] = pa[0]; a[1] = pa[1]; b[0] = pb[0]; b[1] = pb[1];
  } else if (fa >= T(0)) {
    a[0] = pa[0]; a[1] = pa[1];
    b[0] = pa[0] + frac * (pb[0] - pa[0]);
    b[1] = pa[1] + frac * (pb[1] - pa[1]);
  } else {
    a[0] = pb[0] + frac * (pa[0] - pb[0]);
    a[1] = pb[1] + frac * (pa[1] - pb[1]);
    b[0] = pb[0]; b[1] = pb[1];
  }
}

// cell_boundary_walk, marching_squares.jl:240-251
template <class T>
struct Walk {
  T fracs[4];
  bool present[4];
  T sa[4][2];
  T sb[4][2];
};
template <class T>
inline void boundary_walk(const T nodes[4][2], const T phi[4], Walk<T>& w) {
  for (int k = 0; k < 4; ++k) w.fracs[k] = open_fraction(phi[k], phi[ms_next(k)]);
  for (int k = 0; k < 4; ++k) w.present[k] = phi[k] >= T(0) || phi[ms_next(k)] >= T(0);
  for (int k = 0; k < 4; ++k)
    open_segment(nodes[k], nodes[ms_next(k)], phi[k], phi[ms_next(k)], w.fracs[k], w.sa[k], w.sb[k]);
}

// _next_present, marching_squares.jl:255-264
inline int next_present(const bool present[4], int k) {
  int j = ms_next(k);
  if (present[j]) return j;
  j = ms_next(j);
  if (present[j]) return j;
  j = ms_next(j);
  if (present[j]) return j;
  return k;
}

// cell_gap_segments, marching_squares.jl:291-317
template <class T>
inline int gap_segments(const Walk<T>& w, T ia[2][2], T ib[2][2]) {
  int n = 0;
  ia[0][0] = ia[0][1] = ia[1][0] = ia[1][1] = T(0);
  ib[0][0] = ib[0][1] = ib[1][0] = ib[1][1] = T(0);
  for (int k = 0; k < 4; ++k) {
    if (!w.present[k]) continue;
    const int j = next_present(w.present, k);
    const T* a = w.sb[k];
    const T* b = w.sa[j];
    if (a[0] != b[0] || a[1] != b[1]) {
      ++n;
      if (n == 1) { ia[0][0] = a[0]; ia[0][1] = a[1]; ib[0][0] = b[0]; ib[0][1] = b[1]; }
      else if (n == 2) { ia[1][0] = a[0]; ia[1][1] = a[1]; ib[1][0] = b[0]; ib[1][1] = b[1]; }
    }
  }
  return std::min(n, 2);
}

template <class T, int D>
struct CellOut {
  int8_t kind;
  uint8_t amb;
  T vf;
  T c[D];
  T ff[2 * D];
  T fcl[2 * D * (D - 1)];
  T ic[D];
};

// cut_cell_moments (2D), src/marching_squares/moments.jl:66-164
template <class T>
inline void ms_moments(const T nodes[4][2], const T phi[4], const T cs[2], CellOut<T, 2>& o) {
  const T* origin = nodes[0];
  const T centre[2] = {origin[0] + T(0.5) * cs[0], origin[1] + T(0.5) * cs[1]};
  const T vol_cell = cs[0] * cs[1];
  int noutside = 0;
  for (int k = 0; k < 4; ++k) noutside += phi[k] >= T(0) ? 1 : 0;

  auto full_face_centre = [&](int dir, T* x) {  // moments.jl:39-42
    const int k = MS_DIRECTION_EDGE0[dir];
    x[0] = T(0.5) * (nodes[k][0] + nodes[ms_next(k)][0]);
    x[1] = T(0.5) * (nodes[k][1] + nodes[ms_next(k)][1]);
  };
  auto face_offset = [&](const T* x, int dir) -> T {  // moments.jl:48-51
    const int p = dir < 2 ? 1 : 0;  // 3 - direction_axis(dir), 0-based
    return x[p] - origin[p];
  };

  if (noutside == 4 || noutside == 0) {  // moments.jl:84-93
    const bool outside = noutside == 4;
    o.kind = outside ? 1 : 0;
    o.amb = 0;
    o.vf = outside ? T(1) : T(0);
    o.c[0] = centre[0]; o.c[1] = centre[1];
    for (int dir = 0; dir < 4; ++dir) {
      o.ff[dir] = outside ? T(1) : T(0);
      T x[2]; full_face_centre(dir, x);
      o.fcl[dir] = face_offset(x, dir);
    }
    o.ic[0] = centre[0]; o.ic[1] = centre[1];
    return;
  }
  Walk<T> w;
  boundary_walk(nodes, phi, w);
  for (int dir = 0; dir < 4; ++dir) {
    const int k = MS_DIRECTION_EDGE0[dir];
    o.ff[dir] = w.fracs[k];
    T x[2];
    if (w.present[k]) { x[0] = T(0.5) * (w.sa[k][0] + w.sb[k][0]); x[1] = T(0.5) * (w.sa[k][1] + w.sb[k][1]); }
    else full_face_centre(dir, x);
    o.fcl[dir] = face_offset(x, dir);
  }
  T area2 = T(0), cm0 = T(0), cm1 = T(0);
  for (int k = 0; k < 4; ++k) {
    if (!w.present[k]) continue;
    const T la0 = w.sa[k][0] - origin[0], la1 = w.sa[k][1] - origin[1];
    const T lb0 = w.sb[k][0] - origin[0], lb1 = w.sb[k][1] - origin[1];
    const T cr = la0 * lb1 - la1 * lb0;
    area2 = area2 + cr;
    cm0 = cm0 + (la0 + lb0) * cr;
    cm1 = cm1 + (la1 + lb1) * cr;
  }
  T ia[2][2], ib[2][2];
  const int nint = gap_segments(w, ia, ib);
  T ilen = T(0), icm0 = T(0), icm1 = T(0);
  for (int s = 0; s < nint; ++s) {
    const T* a = ia[s];
    const T* b = ib[s];
    const T la0 = a[0] - origin[0], la1 = a[1] - origin[1];
    const T lb0 = b[0] - origin[0], lb1 = b[1] - origin[1];
    const T cr = la0 * lb1 - la1 * lb0;
    area2 = area2 + cr;
    cm0 = cm0 + (la0 + lb0) * cr;
    cm1 = cm1 + (la1 + lb1) * cr;
    const T v0 = b[0] - a[0], v1 = b[1] - a[1];
    const T len = std::sqrt(v0 * v0 + v1 * v1);
    ilen = ilen + len;
    const T hl = T(0.5) * len;
    icm0 = icm0 + hl * (a[0] + b[0]);
    icm1 = icm1 + hl * (a[1] + b[1]);
  }
  const T area = T(0.5) * area2;
  o.kind = 2;
  o.amb = nint > 1 ? 1 : 0;
  o.vf = area / vol_cell;
  if (area2 != T(0)) {
    const T den = T(3) * area2;
    o.c[0] = origin[0] + cm0 / den;
    o.c[1] = origin[1] + cm1 / den;
  } else { o.c[0] = centre[0]; o.c[1] = centre[1]; }
  if (ilen > T(0)) { o.ic[0] = icm0 / ilen; o.ic[1] = icm1 / ilen; }
  else { o.ic[0] = centre[0]; o.ic[1] = centre[1]; }
}

// ----------------------------------------------------------------------------------
// Marching cubes (src/marching_cubes/marching_cubes.jl, src/marching_cubes/moments.jl).
// MC_NODE_BITS :106-107, MC_EDGE_NODES :135-137 (1-based node pairs),
// MC_TEST_FACE_QUADS :372-373.
static const int MC_BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int MC_EDGE_NODES1[12][2] = {{1, 2}, {2, 3}, {4, 3}, {1, 4}, {5, 6}, {6, 7},
                                          {8, 7}, {5, 8}, {1, 5}, {2, 6}, {3, 7}, {4, 8}};
static const int MC_TEST_FACE_QUADS1[6][4] = {{1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 8, 4},
                                              {4, 8, 5, 1}, {1, 4, 3, 2}, {5, 8, 7, 6}};
// Derived once, as the reference derives them (:146-180, :385-388).
struct McConst {
  int face_axes[6][2];  // 0-based in-plane axes (p, q)
  int face_nodes[6][4]; // 0-based corner indices
  int face_test_code[6];
  McConst() {
    for (int dir = 0; dir < 6; ++dir) {
      const int ax = dir >> 1;
      int pq[2], np = 0;
      for (int a = 0; a < 3; ++a) if (a != ax) pq[np++] = a;
      face_axes[dir][0] = pq[0]; face_axes[dir][1] = pq[1];
      const int bax = (dir & 1) ? 1 : 0;
      static const int MSB[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
      for (int k = 0; k < 4; ++k) {
        int bits[3];
        for (int a = 0; a < 3; ++a) bits[a] = a == ax ? bax : (a == pq[0] ? MSB[k][0] : MSB[k][1]);
        for (int c = 0; c < 8; ++c)
          if (MC_BITS[c][0] == bits[0] && MC_BITS[c][1] == bits[1] && MC_BITS[c][2] == bits[2]) face_nodes[dir][k] = c;
      }
      for (int f = 0; f < 6; ++f) {
        int hit = 0;
        for (int k = 0; k < 4; ++k)
          for (int l = 0; l < 4; ++l) hit += (MC_TEST_FACE_QUADS1[f][l] - 1) == face_nodes[dir][k];
        if (hit == 4) face_test_code[dir] = f + 1;
      }
    }
  }
};
static const McConst MCC;

// nudge_zeros, marching_cubes.jl:240-243
template <class T> inline T nudge(T v) {
  const T e = std::numeric_limits<T>::epsilon();
  return std::fabs(v) < e ? e : v;
}

// _test_face, marching_cubes.jl:401-406, evaluated in R (T, or Float64 under mixed precision)
// with the threshold eps(T).
template <class T, class R>
inline bool test_face_r(const T* cb, int face) {
  const int* q = MC_TEST_FACE_QUADS1[std::abs(face) - 1];
  const R A = cb[q[0] - 1], B = cb[q[1] - 1], C = cb[q[2] - 1], D = cb[q[3] - 1];
  const R det = A * C - B * D;
  if (std::fabs(det) < R(std::numeric_limits<T>::epsilon())) return face >= 0;
  return (R(face) * A) * det >= R(0);
}
template <class T>
inline bool test_face(const T* cb, int face) {
  return mixed_on<T>() ? test_face_r<T, double>(cb, face) : test_face_r<T, T>(cb, face);
}

// _test_interior, marching_cubes.jl:427-504. Reference edges 0..11 as
// (t numerator corner, t other corner, B pair, C pair, D pair), 1-based corners, restating the
// twelve branches of :450-486.
static const int MC_INTERIOR_EDGE1[12][8] = {
    {1, 2, 4, 3, 8, 7, 5, 6}, {2, 3, 1, 4, 5, 8, 6, 7}, {3, 4, 2, 1, 6, 5, 7, 8},
    {4, 1, 3, 2, 7, 6, 8, 5}, {5, 6, 8, 7, 4, 3, 1, 2}, {6, 7, 5, 8, 1, 4, 2, 3},
    {7, 8, 6, 5, 2, 1, 3, 4}, {8, 5, 7, 6, 3, 2, 4, 1}, {1, 5, 4, 8, 3, 7, 2, 6},
    {2, 6, 1, 5, 4, 8, 3, 7}, {3, 7, 2, 6, 1, 5, 4, 8}, {4, 8, 3, 7, 2, 6, 1, 5}};
template <class T, class R>
inline bool test_interior_r(int itype, int edge, const T* cb, int s) {
  R At = R(0), Bt = R(0), Ct = R(0), Dt = R(0);
  auto c = [&](int i) { return R(cb[i - 1]); };
  if (itype == CC_MC_INTERIOR_CASE4_10) {
    const R a = (c(5) - c(1)) * (c(7) - c(3)) - (c(8) - c(4)) * (c(6) - c(2));
    const R b = ((c(3) * (c(5) - c(1)) + c(1) * (c(7) - c(3))) - c(2) * (c(8) - c(4))) - c(4) * (c(6) - c(2));
    const R t = -b / (R(2) * a);
    if (t < R(0) || t > R(1)) return s > 0;
    At = c(1) + (c(5) - c(1)) * t;
    Bt = c(4) + (c(8) - c(4)) * t;
    Ct = c(3) + (c(7) - c(3)) * t;
    Dt = c(2) + (c(6) - c(2)) * t;
  } else {
    const int* e = MC_INTERIOR_EDGE1[edge];
    const R t = c(e[0]) / (c(e[0]) - c(e[1]));
    Bt = c(e[2]) + (c(e[3]) - c(e[2])) * t;
    Ct = c(e[4]) + (c(e[5]) - c(e[4])) * t;
    Dt = c(e[6]) + (c(e[7]) - c(e[6])) * t;
  }
  int test = 0;
  if (At >= R(0)) test += 1;
  if (Bt >= R(0)) test += 2;
  if (Ct >= R(0)) test += 4;
  if (Dt >= R(0)) test += 8;
  const R eps = R(std::numeric_limits<T>::epsilon());
  if (test == 6 || test == 8 || test == 9 || test == 12 || (test >= 0 && test <= 4)) return s > 0;
  if (test == 5) return (At * Ct - Bt * Dt < eps) ? s > 0 : s < 0;
  if (test == 10) return (At * Ct - Bt * Dt >= eps) ? s > 0 : s < 0;
  return s < 0;
}
template <class T>
inline bool test_interior(int itype, int edge, const T* cb, int s) {
  return mixed_on<T>() ? test_interior_r<T, double>(itype, edge, cb, s) : test_interior_r<T, T>(itype, edge, cb, s);
}

struct McTable {
  const cc_mc_table_header* h = nullptr;
  const cc_mc_lut* luts = nullptr;
  const cc_mc_outcome* outs = nullptr;
  const cc_mc_tile* tiles = nullptr;
  const uint8_t* codes = nullptr;
  bool parse(const uint8_t* blob) {
    h = reinterpret_cast<const cc_mc_table_header*>(blob);
    if (h->magic != CC_MC_TABLE_MAGIC) return false;
    luts = reinterpret_cast<const cc_mc_lut*>(blob + sizeof(cc_mc_table_header));
    outs = reinterpret_cast<const cc_mc_outcome*>(luts + 256);
    tiles = reinterpret_cast<const cc_mc_tile*>(outs + h->n_outcomes);
    codes = reinterpret_cast<const uint8_t*>(tiles + h->n_tiles);
    return true;
  }
};

// cell_case, marching_cubes.jl:343-349 (returned 0-based: lut - 1)
template <class T> inline int cell_case0(const T* phi) {
  int lut = 0;
  for (int p = 0; p < 8; ++p) if (phi[p] >= T(0)) lut |= 1 << p;
  return lut;
}

// cell_triangles, marching_cubes.jl:538-651, over the table blob: the face tests, then the
// optional interior test, pick one tiling. Returns the triangle count and the tile's codes.
template <class T>
inline int cell_triangles(const McTable& tb, const T* phi, const uint8_t** codes, int* lcase) {
  const int lut = cell_case0(phi);
  const cc_mc_lut& e = tb.luts[lut];
  *lcase = e.lcase;
  int o = 0;
  for (int i = 0; i < e.ntests; ++i) if (test_face(phi, e.face[i])) o |= 1 << i;
  const cc_mc_outcome& oc = tb.outs[e.outcome_base + o];
  int tile = oc.tile_true;
  if (oc.itype != CC_MC_INTERIOR_NONE && !test_interior(oc.itype, oc.edge, phi, oc.s)) tile = oc.tile_false;
  *codes = tb.codes + tb.tiles[tile].code_off;
  return tb.tiles[tile].ntris;
}

// _chord_target, moments.jl:91-98 (returns -1 for none)
template <class T>
inline int chord_target(const T* fphi, int k, bool forward) {
  int j = k;
  for (int it = 0; it < 4; ++it) {
    j = forward ? ms_next(j) : ms_prev(j);
    if (fphi[j] < T(0) && fphi[ms_next(j)] >= T(0)) return j;
  }
  return -1;
}

// _face_polygon, moments.jl:111-139
template <class T>
inline void face_polygon(const T fn[4][2], const T* fphi, bool connect, T& area2, T& c0, T& c1) {
  Walk<T> w;
  boundary_walk(fn, fphi, w);
  area2 = T(0); c0 = T(0); c1 = T(0);
  for (int k = 0; k < 4; ++k) {
    if (!w.present[k]) continue;
    const T* la = w.sa[k]; const T* lb = w.sb[k];
    const T cr = la[0] * lb[1] - la[1] * lb[0];
    area2 = area2 + cr;
    c0 = c0 + (la[0] + lb[0]) * cr;
    c1 = c1 + (la[1] + lb[1]) * cr;
  }
  for (int k = 0; k < 4; ++k) {
    if (!(fphi[k] >= T(0) && fphi[ms_next(k)] < T(0))) continue;
    const int j = chord_target(fphi, k, connect);
    if (j < 0) continue;
    const T* la = w.sb[k]; const T* lb = w.sa[j];
    const T cr = la[0] * lb[1] - la[1] * lb[0];
    area2 = area2 + cr;
    c0 = c0 + (la[0] + lb[0]) * cr;
    c1 = c1 + (la[1] + lb[1]) * cr;
  }
}

// full_face_area (3D), src/cut_cell.jl:190-197
template <class T> inline T full_face_area3(const T* cs, int dir) {
  const int ax = dir >> 1;
  T p = T(1);
  for (int a = 0; a < 3; ++a) if (a != ax) p = p * cs[a];
  return p;
}

// _edge_crossing, marching_cubes.jl:284-287
template <class T>
inline void edge_crossing(const T* pa, const T* pb, T fa, T fb, T* out) {
  const T s = open_fraction(fa, fb);
  if (fa >= T(0)) for (int i = 0; i < 3; ++i) out[i] = pa[i] + s * (pb[i] - pa[i]);
  else for (int i = 0; i < 3; ++i) out[i] = pb[i] + s * (pa[i] - pb[i]);
}

// cut_cell_moments (3D), moments.jl:275-346, with cut_cell_faces (:224-257) and
// _cut_cell_face (:150-196) inlined.
template <class T>
inline void mc_moments(const McTable& tb, const T nodes[8][3], const T phi_raw[8], const T cs[3],
                       CellOut<T, 3>& o) {
  T phi[8];
  for (int k = 0; k < 8; ++k) phi[k] = nudge(phi_raw[k]);
  const T* origin = nodes[0];
  T centre[3];
  for (int a = 0; a < 3; ++a) centre[a] = origin[a] + T(0.5) * cs[a];
  const T vol_cell = (cs[0] * cs[1]) * cs[2];
  const uint8_t* codes = nullptr;
  int lcase = 1;
  const int ntri = cell_triangles(tb, phi, &codes, &lcase);

  T ln[8][3];
  for (int k = 0; k < 8; ++k) for (int a = 0; a < 3; ++a) ln[k][a] = nodes[k][a] - origin[a];
  int noutside = 0;
  for (int k = 0; k < 8; ++k) noutside += phi[k] >= T(0) ? 1 : 0;
  const int kind = noutside == 8 ? 1 : (noutside == 0 ? 0 : 2);
  bool amb_face = false;
  for (int dir = 0; dir < 6; ++dir) {
    const int p = MCC.face_axes[dir][0], q = MCC.face_axes[dir][1];
    const int* idx = MCC.face_nodes[dir];
    T fn[4][2], fphi[4];
    for (int k = 0; k < 4; ++k) { fn[k][0] = ln[idx[k]][p]; fn[k][1] = ln[idx[k]][q]; fphi[k] = phi[idx[k]]; }
    int nout = 0;
    for (int k = 0; k < 4; ++k) nout += fphi[k] >= T(0) ? 1 : 0;
    const bool amb_dir = (nout == 2) && ((fphi[0] >= T(0)) == (fphi[2] >= T(0)));
    T frac, c0, c1;
    const T avg0 = T(0.25) * (((fn[0][0] + fn[1][0]) + fn[2][0]) + fn[3][0]);
    const T avg1 = T(0.25) * (((fn[0][1] + fn[1][1]) + fn[2][1]) + fn[3][1]);
    if (nout == 4 || nout == 0) {
      frac = nout == 4 ? T(1) : T(0);
      c0 = avg0; c1 = avg1;
    } else {
      T area2, m0, m1;
      face_polygon(fn, fphi, test_face(phi, MCC.face_test_code[dir]), area2, m0, m1);
      frac = (T(0.5) * area2) / full_face_area3(cs, dir);
      if (area2 != T(0)) { const T den = T(3) * area2; c0 = m0 / den; c1 = m1 / den; }
      else { c0 = avg0; c1 = avg1; }
    }
    o.ff[dir] = frac;
    o.fcl[2 * dir] = c0;
    o.fcl[2 * dir + 1] = c1;
    amb_face = amb_face || amb_dir;
  }
  o.kind = int8_t(kind);
  if (kind != 2) {
    o.amb = 0;
    o.vf = kind == 1 ? T(1) : T(0);
    for (int a = 0; a < 3; ++a) { o.c[a] = centre[a]; o.ic[a] = centre[a]; }
    return;
  }
  // edge_crossings, marching_cubes.jl:306-330
  T pts[13][3];
  T acc[3] = {T(0), T(0), T(0)};
  int ncr = 0;
  for (int e = 0; e < 12; ++e) {
    const int a = MC_EDGE_NODES1[e][0] - 1, b = MC_EDGE_NODES1[e][1] - 1;
    const bool crossed = (phi[a] >= T(0)) != (phi[b] >= T(0));
    if (crossed) {
      edge_crossing(ln[a], ln[b], phi[a], phi[b], pts[e]);
      for (int i = 0; i < 3; ++i) acc[i] = acc[i] + pts[e][i];
      ++ncr;
    } else {
      pts[e][0] = pts[e][1] = pts[e][2] = T(0);
    }
  }
  for (int i = 0; i < 3; ++i) pts[12][i] = ncr > 0 ? acc[i] / T(ncr) : T(0);

  T vol3 = T(0);
  T cm2[3] = {T(0), T(0), T(0)};
  for (int dir = 0; dir < 6; ++dir) {
    const int ax = dir >> 1;
    const T s = (dir & 1) ? T(1) : T(-1);
    const T x_ax = ln[MCC.face_nodes[dir][0]][ax];
    const T a_open = o.ff[dir] * full_face_area3(cs, dir);
    vol3 = vol3 + (s * x_ax) * a_open;
    for (int a = 0; a < 3; ++a) cm2[a] = cm2[a] + (a == ax ? ((s * x_ax) * x_ax) * a_open : T(0));
  }
  T iarea = T(0);
  T icm[3] = {T(0), T(0), T(0)};
  for (int t = 0; t < ntri; ++t) {
    const T* A = pts[codes[3 * t] - 1];
    const T* B = pts[codes[3 * t + 1] - 1];
    const T* Dd = pts[codes[3 * t + 2] - 1];
    T u[3], v[3];
    for (int i = 0; i < 3; ++i) { u[i] = B[i] - A[i]; v[i] = Dd[i] - A[i]; }
    T w[3] = {T(0.5) * (u[1] * v[2] - u[2] * v[1]), T(0.5) * (u[2] * v[0] - u[0] * v[2]),
              T(0.5) * (u[0] * v[1] - u[1] * v[0])};
    T xc[3];
    for (int i = 0; i < 3; ++i) xc[i] = ((A[i] + B[i]) + Dd[i]) / T(3);
    vol3 = vol3 - ((w[0] * xc[0] + w[1] * xc[1]) + w[2] * xc[2]);
    for (int i = 0; i < 3; ++i) {
      const T m2 = (((((A[i] * A[i] + B[i] * B[i]) + Dd[i] * Dd[i]) + A[i] * B[i]) + B[i] * Dd[i]) + Dd[i] * A[i]) / T(6);
      cm2[i] = cm2[i] - w[i] * m2;
    }
    const T len = std::sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
    iarea = iarea + len;
    for (int i = 0; i < 3; ++i) icm[i] = icm[i] + len * xc[i];
  }
  const T volume = vol3 / T(3);
  if (volume > T(0)) { const T den = T(2) * volume; for (int a = 0; a < 3; ++a) o.c[a] = origin[a] + cm2[a] / den; }
  else for (int a = 0; a < 3; ++a) o.c[a] = centre[a];
  if (iarea > T(0)) for (int a = 0; a < 3; ++a) o.ic[a] = origin[a] + icm[a] / iarea;
  else for (int a = 0; a < 3; ++a) o.ic[a] = centre[a];
  const bool amb_case = lcase == 5 || lcase == 7 || lcase == 8 || lcase == 11 || lcase == 13 || lcase == 14;
  o.amb = (amb_face || amb_case) ? 1 : 0;
  o.vf = volume / vol_cell;
}

// ----------------------------------------------------------------------------------
// Column writers (the StructArray layout of include/cutcell_b200.h).
template <class T, int D>
inline void store(const cc_cells& c, int64_t ci, const CellOut<T, D>& o) {
  c.kind[ci] = o.kind;
  c.ambiguous[ci] = o.amb;
  static_cast<T*>(c.volume_fraction)[ci] = o.vf;
  for (int a = 0; a < D; ++a) static_cast<T*>(c.centroid)[D * ci + a] = o.c[a];
  for (int a = 0; a < 2 * D; ++a) static_cast<T*>(c.face_fraction)[2 * D * ci + a] = o.ff[a];
  for (int a = 0; a < 2 * D * (D - 1); ++a) static_cast<T*>(c.face_centroid_local)[2 * D * (D - 1) * ci + a] = o.fcl[a];
  for (int a = 0; a < D; ++a) static_cast<T*>(c.interface_centroid)[D * ci + a] = o.ic[a];
}

template <class T>
Tape<T> make_tape(const cc_optape* t) {
  Tape<T> r;
  r.ops.assign(t->ops, t->ops + t->n_ops);
  r.p.resize(t->n_params);
  for (int i = 0; i < t->n_params; ++i) r.p[i] = T(t->params[i]);
  return r;
}

// _sample_nodes_kernel!, src/marching_squares/cache.jl:67-70, over the node layers kn0..kn1
// (inclusive; 3D) of the full grid: every node's coordinates are get_node's expression with its
// global index, and phi holds the layers from kn0 on.
template <class T, int D>
void sample_nodes_range(const cc_grid& g, const Tape<T>& tp, T* phi, int64_t kn0, int64_t kn1) {
  const int64_t nx = g.n[0] + 1, ny = g.n[1] + 1, nz = D == 3 ? kn1 - kn0 + 1 : 1;
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])};
  const T d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  parallel_for(ny * nz, [&](int64_t row) {
    const int64_t j = row % ny, kl = row / ny;
    for (int64_t i = 0; i < nx; ++i) {
      T x[3];
      x[0] = node_coord(x0[0], d[0], i);
      x[1] = node_coord(x0[1], d[1], j);
      x[2] = node_coord(x0[2], d[2], D == 3 ? kn0 + kl : kl);
      phi[i + nx * (j + ny * kl)] = eval_tape<T, D, T>(tp, x);
    }
  });
}

template <class T, int D>
void sample_nodes(const cc_grid& g, const Tape<T>& tp, T* phi) {
  sample_nodes_range<T, D>(g, tp, phi, 0, D == 3 ? g.n[2] : 0);
}

// _nodal_cells_kernel!, src/marching_squares/cache.jl:75-78, 3D, over the cell layers k0..k1-1
// of the full grid: phi holds the node layers k0..k1 and the columns the cell layers from k0 on;
// node coordinates use the global indices.
template <class T>
void mc_cells_range(const cc_grid& g, const McTable& tb, const T* phi, const cc_cells& c, int64_t k0, int64_t k1) {
  const int64_t n0 = g.n[0], n1 = g.n[1];
  const int64_t nx = n0 + 1, ny = n1 + 1;
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])};
  const T d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  parallel_for(n1 * (k1 - k0), [&](int64_t row) {
    const int64_t j = row % n1, kl = row / n1, k = k0 + kl;
    for (int64_t i = 0; i < n0; ++i) {
        T nodes[8][3], ph[8];
        for (int q = 0; q < 8; ++q) {
          const int64_t ii = i + MC_BITS[q][0], jj = j + MC_BITS[q][1], kk = k + MC_BITS[q][2];
          nodes[q][0] = node_coord(x0[0], d[0], ii);
          nodes[q][1] = node_coord(x0[1], d[1], jj);
          nodes[q][2] = node_coord(x0[2], d[2], kk);
          ph[q] = phi[ii + nx * (jj + ny * (kk - k0))];
        }
        CellOut<T, 3> o;
        mc_moments(tb, nodes, ph, d, o);
        store<T, 3>(c, i + n0 * (j + n1 * kl), o);
    }
  });
}

template <class T>
void mc_cells(const cc_grid& g, const McTable& tb, const T* phi, const cc_cells& c) {
  mc_cells_range<T>(g, tb, phi, c, 0, g.n[2]);
}

// generate_mesh (src/marching_cubes/surface.jl:82-112) restated for the project's device mesh:
// every cut cell's triangles are its tile's, each edge vertex the crossing anchored on the
// outside node in world coordinates, shared; code 13 the mean of the cell's crossings. Numbered
// serially: edge vertices by lower node (linear order) then axis, interior vertices by cell,
// triangles by cell.
template <class T>
struct Mesh {
  std::vector<T> verts;
  std::vector<int32_t> tris;
  std::vector<int64_t> cells;
};

template <class T>
inline T nudged_at(const T* phi, int64_t v) { return nudge(phi[v]); }

template <class T>
void edge_vertex(const T x0[3], const T d[3], const T* phi, const int64_t n[3], int64_t i, int64_t j, int64_t k,
                 int a, T out[3]) {
  const int64_t nx = n[0] + 1, ny = n[1] + 1;
  const int64_t v = i + nx * (j + ny * k);
  const int64_t w = v + (a == 0 ? 1 : a == 1 ? nx : nx * ny);
  const T fa = nudge(phi[v]), fb = nudge(phi[w]);
  const int64_t idx[3] = {i, j, k};
  T xa[3], xb[3];
  for (int q = 0; q < 3; ++q) {
    xa[q] = node_coord(x0[q], d[q], idx[q]);
    xb[q] = node_coord(x0[q], d[q], idx[q] + (q == a ? 1 : 0));
  }
  const T s = open_fraction(fa, fb);
  for (int q = 0; q < 3; ++q) out[q] = fa >= T(0) ? xa[q] + s * (xb[q] - xa[q]) : xb[q] + s * (xa[q] - xb[q]);
}

template <class T>
Mesh<T> mc_mesh(const cc_grid& g, const McTable& tb, const T* phi) {
  const int64_t n[3] = {g.n[0], g.n[1], g.n[2]};
  const int64_t nx = n[0] + 1, ny = n[1] + 1, nz = n[2] + 1;
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])};
  const T d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  Mesh<T> m;
  std::vector<uint32_t> vbase(size_t(nx * ny * nz));
  auto out = [&](int64_t v) { return nudge(phi[v]) >= T(0); };
  auto edges = [&](int64_t i, int64_t j, int64_t k) {
    const int64_t v = i + nx * (j + ny * k);
    unsigned msk = 0;
    if (i < n[0] && out(v + 1) != out(v)) msk |= 1u;
    if (j < n[1] && out(v + nx) != out(v)) msk |= 2u;
    if (k < n[2] && out(v + nx * ny) != out(v)) msk |= 4u;
    return msk;
  };
  uint32_t id = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        const unsigned msk = edges(i, j, k);
        vbase[size_t(i + nx * (j + ny * k))] = id;
        for (int a = 0; a < 3; ++a) {
          if (!(msk >> a & 1u)) continue;
          T p[3];
          edge_vertex(x0, d, phi, n, i, j, k, a, p);
          m.verts.insert(m.verts.end(), p, p + 3);
          ++id;
        }
      }
  std::vector<T> interior;
  for (int64_t k = 0; k < n[2]; ++k)
    for (int64_t j = 0; j < n[1]; ++j)
      for (int64_t i = 0; i < n[0]; ++i) {
        T ph[8];
        int nout = 0;
        for (int q = 0; q < 8; ++q) {
          ph[q] = nudge(phi[(i + MC_BITS[q][0]) + nx * ((j + MC_BITS[q][1]) + ny * (k + MC_BITS[q][2]))]);
          nout += ph[q] >= T(0) ? 1 : 0;
        }
        if (nout == 0 || nout == 8) continue;
        const uint8_t* codes;
        int lcase;
        const int nt = cell_triangles(tb, ph, &codes, &lcase);
        uint32_t vid[12];
        T acc[3] = {T(0), T(0), T(0)};
        int ncr = 0;
        for (int e = 0; e < 12; ++e) {
          const int ca = MC_EDGE_NODES1[e][0] - 1, cb = MC_EDGE_NODES1[e][1] - 1;
          const int a = MC_BITS[ca][0] != MC_BITS[cb][0] ? 0 : (MC_BITS[ca][1] != MC_BITS[cb][1] ? 1 : 2);
          const int lo = MC_BITS[ca][a] < MC_BITS[cb][a] ? ca : cb;
          const int64_t li = i + MC_BITS[lo][0], lj = j + MC_BITS[lo][1], lk = k + MC_BITS[lo][2];
          const unsigned msk = edges(li, lj, lk);
          vid[e] = vbase[size_t(li + nx * (lj + ny * lk))] + uint32_t(__builtin_popcount(msk & ((1u << a) - 1u)));
          if ((ph[ca] >= T(0)) != (ph[cb] >= T(0))) {
            T p[3];
            edge_vertex(x0, d, phi, n, li, lj, lk, a, p);
            acc[0] = acc[0] + p[0]; acc[1] = acc[1] + p[1]; acc[2] = acc[2] + p[2];
            ++ncr;
          }
        }
        bool uses13 = false;
        for (int q = 0; q < 3 * nt; ++q) uses13 = uses13 || codes[q] == 13;
        uint32_t centre = 0;
        if (uses13) {
          centre = uint32_t(interior.size() / 3);
          interior.push_back(acc[0] / T(ncr));
          interior.push_back(acc[1] / T(ncr));
          interior.push_back(acc[2] / T(ncr));
        }
        for (int r = 0; r < nt; ++r) {
          for (int q = 0; q < 3; ++q) {
            const int code = codes[3 * r + q];
            // an interior vertex is numbered after all edge vertices: a placeholder until then
            m.tris.push_back(code == 13 ? -1 - int32_t(centre) : int32_t(vid[code - 1]));
          }
          m.cells.push_back(i + n[0] * (j + n[1] * k));
        }
      }
  const int32_t ne = int32_t(m.verts.size() / 3);
  for (auto& t : m.tris)
    if (t < 0) t = ne + (-1 - t);
  m.verts.insert(m.verts.end(), interior.begin(), interior.end());
  return m;
}

static const int MS_BITS[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};

template <class T>
void ms_cells(const cc_grid& g, const T* phi, const cc_cells& c) {
  const int64_t n0 = g.n[0], n1 = g.n[1], nx = n0 + 1;
  const T x0[2] = {T(g.x0[0]), T(g.x0[1])};
  const T d[2] = {T(g.d[0]), T(g.d[1])};
  parallel_for(n1, [&](int64_t j) {
    for (int64_t i = 0; i < n0; ++i) {
      T nodes[4][2], ph[4];
      for (int q = 0; q < 4; ++q) {
        const int64_t ii = i + MS_BITS[q][0], jj = j + MS_BITS[q][1];
        nodes[q][0] = node_coord(x0[0], d[0], ii);
        nodes[q][1] = node_coord(x0[1], d[1], jj);
        ph[q] = phi[ii + nx * jj];
      }
      CellOut<T, 2> o;
      ms_moments(nodes, ph, d, o);
      store<T, 2>(c, i + n0 * j, o);
    }
  });
}

// generate_mesh for marching squares (src/marching_squares/surface.jl:70-111, 153-176): cut cells in
// order, each cell_interface segment (the gaps, endpoints swapped: out of the body) appended with
// its vertices welded by exact coordinate equality in a map, numbered by first occurrence.
template <class T>
struct Contour {
  std::vector<T> verts;
  std::vector<int32_t> segs;
  std::vector<int64_t> cells;
  std::map<std::pair<T, T>, int32_t> ids;
  int32_t vertex(const T* x) {
    const std::pair<T, T> key(x[0] + T(0), x[1] + T(0));
    auto it = ids.find(key);
    if (it != ids.end()) return it->second;
    const int32_t id = int32_t(verts.size() / 2);
    ids.emplace(key, id);
    verts.push_back(key.first);
    verts.push_back(key.second);
    return id;
  }
  void add_cell(const T nodes[4][2], const T ph[4], int64_t cell) {
    Walk<T> w;
    boundary_walk(nodes, ph, w);
    T ia[2][2], ib[2][2];
    const int n = gap_segments(w, ia, ib);
    for (int s = 0; s < n; ++s) {  // cell_interface: (n, b, a)
      const int32_t i1 = vertex(ib[s]);
      const int32_t i2 = vertex(ia[s]);
      segs.push_back(i1);
      segs.push_back(i2);
      cells.push_back(cell);
    }
  }
};

template <class T>
Contour<T> ms_mesh_grid(const cc_grid& g, const T* phi) {
  const int64_t n0 = g.n[0], n1 = g.n[1], nx = n0 + 1;
  const T x0[2] = {T(g.x0[0]), T(g.x0[1])};
  const T d[2] = {T(g.d[0]), T(g.d[1])};
  Contour<T> c;
  for (int64_t j = 0; j < n1; ++j)
    for (int64_t i = 0; i < n0; ++i) {
      T nodes[4][2], ph[4];
      for (int q = 0; q < 4; ++q) {
        const int64_t ii = i + MS_BITS[q][0], jj = j + MS_BITS[q][1];
        nodes[q][0] = node_coord(x0[0], d[0], ii);
        nodes[q][1] = node_coord(x0[1], d[1], jj);
        ph[q] = phi[ii + nx * jj];
      }
      c.add_cell(nodes, ph, i + n0 * j);
    }
  return c;
}

template <class T>
Contour<T> ms_mesh_tree(const double* x0d, const double* based, int64_t nl, const int32_t* level,
                        const int32_t* coord, const T* phi4) {
  const T x0[2] = {T(x0d[0]), T(x0d[1])};
  Contour<T> c;
  for (int64_t i = 0; i < nl; ++i) {
    const T scale = T(std::ldexp(1.0, -level[i]));
    const T h[2] = {T(based[0]) * scale, T(based[1]) * scale};
    T nodes[4][2], ph[4];
    for (int q = 0; q < 4; ++q) {
      nodes[q][0] = x0[0] + T(int64_t(coord[2 * i]) + MS_BITS[q][0]) * h[0];
      nodes[q][1] = x0[1] + T(int64_t(coord[2 * i + 1]) + MS_BITS[q][1]) * h[1];
      ph[q] = phi4[4 * i + q];
    }
    c.add_cell(nodes, ph, i);
  }
  return c;
}

// _leaf_cells_kernel!, src/marching_squares/cache.jl:129-137
template <class T>
void ms_tree(const double* x0d, const double* based, int64_t nl, const int32_t* level,
             const int32_t* coord, const Tape<T>& tp, T* phi4, const cc_cells& c) {
  const T x0[2] = {T(x0d[0]), T(x0d[1])};
  parallel_for(nl, [&](int64_t i) {
    const T scale = T(std::ldexp(1.0, -level[i]));
    const T h[2] = {T(based[0]) * scale, T(based[1]) * scale};
    T nodes[4][2], ph[4];
    for (int q = 0; q < 4; ++q) {
      nodes[q][0] = x0[0] + T(int64_t(coord[2 * i]) + MS_BITS[q][0]) * h[0];
      nodes[q][1] = x0[1] + T(int64_t(coord[2 * i + 1]) + MS_BITS[q][1]) * h[1];
      ph[q] = eval_tape<T, 2, T>(tp, nodes[q]);
      phi4[4 * i + q] = ph[q];
    }
    CellOut<T, 2> o;
    ms_moments(nodes, ph, h, o);
    store<T, 2>(c, i, o);
  });
}

// ----------------------------------------------------------------------------------
// PLIC (src/plic/plic.jl:72-88, src/plic/apertures.jl:73-125, src/plic/cache.jl:96-162)
template <class T, int D>
struct Plane {
  T n[D];
  T a;
  T fraction;  // solid
  bool valid;
};

template <class T, int D>
inline Plane<T, D> cell_plane(const Tape<T>& tp, const T* x0, const T* d, const int64_t* idx) {
  Dual<T, D> x[D];
  for (int a = 0; a < D; ++a) {
    x[a] = dconst<T, D>(centroid_coord(x0[a], d[a], idx[a]));
    x[a].g[a] = T(1);
  }
  const Dual<T, D> r = eval_tape<T, D, Dual<T, D>>(tp, x);
  const T dist = r.v;
  T s = r.g[0];
  for (int a = 1; a < D; ++a) s = s + r.g[a];
  const T a = T(0.5) * s - dist / d[0];
  bool allzero = true;
  for (int q = 0; q < D; ++q) allzero = allzero && (r.g[q] == T(0));
  Plane<T, D> pl;
  if (std::isnan(a) || allzero) {
    for (int q = 0; q < D; ++q) pl.n[q] = T(0);
    pl.a = T(0);
    pl.fraction = dist <= T(0) ? T(1) : T(0);
    pl.valid = false;
    return pl;
  }
  for (int q = 0; q < D; ++q) pl.n[q] = r.g[q];
  pl.a = a;
  pl.fraction = D == 2 ? gvf2p(r.g[0], r.g[1], a) : gvf3p(r.g[0], r.g[1], r.g[D - 1], a);
  pl.valid = true;
  return pl;
}

// _cell_wet + _face_area (2D and 3D), apertures.jl:73-125
template <class T, int D>
inline T face_area(const T* n, T a, T frac, bool valid, const T* cs, int k /*0-based*/) {
  const T s = (k & 1) ? T(1) : T(0);
  if (D == 2) {
    const int c = k < 2 ? 0 : 1, p = k < 2 ? 1 : 0;
    const T len = cs[p];
    if (!valid) return frac < T(0.5) ? T(0) : len;
    const T base = n[c] * s - a;
    return open_fraction(base, base + n[p]) * len;
  } else {
    int c, p, q;
    if (k < 2) { c = 0; p = 1; q = 2; }
    else if (k < 4) { c = 1; p = 0; q = 2; }
    else { c = 2; p = 0; q = 1; }
    const T U = cs[p], V = cs[q];
    if (!valid) return frac < T(0.5) ? T(0) : U * V;
    const T base = n[c] * s - a;
    if (n[p] == T(0) && n[q] == T(0)) return base >= T(0) ? U * V : T(0);
    const T solid = gvf2p(n[p], n[q], -base);
    return (U * V) * (T(1) - solid);
  }
}

// _plic_fit_kernel! + _plic_face_fraction_kernel! (src/plic/cache.jl:96-162) over the cell layers
// k0..k1-1 of the full grid (3D; 2D takes the whole grid): the planes of the layers k0-1..k1 (those
// inside the grid) are fitted, so the slab's faces resolve against the same neighbours as in the
// whole-grid update. The columns, normals, intercepts and flags hold the slab's cells from k0 on.
template <class T, int D>
void plic_update_range(const cc_grid& g, const Tape<T>& tp, const cc_cells& c, T* normals, T* intercepts,
                       uint8_t* is_valid, int64_t k0, int64_t k1) {
  const int64_t n[3] = {g.n[0], g.n[1], D == 3 ? g.n[2] : 1};
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])};
  const T d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  if (D == 2) { k0 = 0; k1 = 1; }
  const int64_t h0 = k0 > 0 ? k0 - 1 : 0, h1 = k1 < n[2] ? k1 + 1 : n[2];  // fitted layers [h0, h1)
  const int64_t nlay = n[0] * n[1];
  const int64_t nfit = nlay * (h1 - h0);
  std::vector<T> hn(size_t(nfit) * D), ha(nfit), hvf(nfit);
  std::vector<uint8_t> hv(nfit);
  parallel_for(nfit, [&](int64_t li) {
    const int64_t ci = li + nlay * h0;
    const int64_t idx[3] = {ci % n[0], (ci / n[0]) % n[1], ci / (n[0] * n[1])};
    Plane<T, D> pl = cell_plane<T, D>(tp, x0, d, idx);
    for (int a = 0; a < D; ++a) hn[D * li + a] = pl.n[a];
    ha[li] = pl.a;
    hv[li] = pl.valid ? 1 : 0;
    hvf[li] = T(1) - pl.fraction;
  });
  T* vf = static_cast<T*>(c.volume_fraction);
  T* ff = static_cast<T*>(c.face_fraction);
  const int64_t nout = nlay * (k1 - k0);
  parallel_for(nout, [&](int64_t oi) {
    const int64_t ci = oi + nlay * k0;  // global cell index
    const int64_t li = ci - nlay * h0;  // index among the fitted layers
    const int64_t idx[3] = {ci % n[0], (ci / n[0]) % n[1], ci / (n[0] * n[1])};
    const T frac = hvf[li];
    for (int a = 0; a < D; ++a) normals[D * oi + a] = hn[D * li + a];
    intercepts[oi] = ha[li];
    is_valid[oi] = hv[li];
    vf[oi] = frac;
    c.kind[oi] = frac == T(0) ? 0 : (frac == T(1) ? 1 : 2);
    for (int k = 0; k < 2 * D; ++k) {
      const int cax = k >> 1;
      int64_t stride = 1;
      for (int a = 0; a < cax; ++a) stride *= n[a];
      T full;
      if (D == 2) full = d[1 - cax];
      else full = full_face_area3(d, k);
      auto area_of = [&](int64_t lj, int kk) {
        return face_area<T, D>(hn.data() + D * lj, ha[lj], hvf[lj], hv[lj] != 0, d, kk);
      };
      const T own = area_of(li, k);
      T r;
      if ((k & 1) == 0) {
        const bool has = idx[cax] >= 1;
        const T below = area_of(has ? li - stride : li, k + 1);
        r = has ? (below / full + own / full) / T(2) : own / full;
      } else {
        const bool has = idx[cax] <= n[cax] - 2;
        const T above = area_of(has ? li + stride : li, k - 1);
        r = has ? (own / full + above / full) / T(2) : own / full;
      }
      ff[2 * D * oi + k] = r;
    }
  });
}

template <class T, int D>
void plic_update(const cc_grid& g, const Tape<T>& tp, const cc_cells& c, T* normals, T* intercepts,
                 uint8_t* is_valid) {
  plic_update_range<T, D>(g, tp, c, normals, intercepts, is_valid, 0, D == 3 ? g.n[2] : 1);
}

template <class T, int D>
T calc_volume(const cc_grid& g, const Tape<T>& tp) {
  const int64_t n[3] = {g.n[0], g.n[1], D == 3 ? g.n[2] : 1};
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])};
  const T d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  T vol = T(0);
  for (int64_t k = 0; k < n[2]; ++k)
    for (int64_t j = 0; j < n[1]; ++j)
      for (int64_t i = 0; i < n[0]; ++i) {
        const int64_t idx[3] = {i, j, k};
        vol = vol + cell_plane<T, D>(tp, x0, d, idx).fraction;
      }
  T pd = d[0];
  for (int a = 1; a < D; ++a) pd = pd * d[a];
  return vol * pd;
}

// ---- generate_mesh for a PLIC cache (src/plic/surface.jl:28-267), serially ----
// CartesianMeshes 0.2.3 `cell_plane_clip` / `local_to_global` are absent from the checkout; the
// clip is written from the geometry: the plane n . xi = a in the unit cell meets the square's /
// cube's edges where the corner values n . xi - a change sign strictly, and a corner with value 0
// is a point of its own. The world point is x_node + xi * d.

// Monotone stand-in for atan2(y, x) over (-pi, pi], in (-2, 2]: the order of the reference's
// angle sort (surface.jl:254-265) without a transcendental, so it is reproducible bit for bit.
template <class T> inline T pseudo_angle(T y, T x) {
  if (x == T(0) && y == T(0)) return T(0);
  if (y >= T(0)) return x >= T(0) ? y / (x + y) : T(1) + (-x) / (y - x);
  return x >= T(0) ? -((-y) / (x - y)) : -(T(1) + (-x) / (-x - y));
}

template <class T> struct PlicMesh {
  std::vector<T> nodes;
  std::vector<int32_t> elems;
  std::vector<int64_t> cells;
};

// 2D: one segment per cell -- the two crossings, walking the square's edges (0,0)->(1,0)->(1,1)->
// (0,1); a line that does not cross draws a zero-length segment (at the one corner it touches,
// else at the lower corner; a degenerate fit at the lower corner). Kept when its length is at
// least min_frac * min(d) (surface.jl:91-94).
template <class T>
PlicMesh<T> plic_mesh2(const cc_grid& g, const T* normals, const T* intercepts, const uint8_t* valid, T min_frac) {
  PlicMesh<T> out;
  const T x0[2] = {T(g.x0[0]), T(g.x0[1])}, d[2] = {T(g.d[0]), T(g.d[1])};
  const T min_d = d[1] < d[0] ? d[1] : d[0];
  const T corner[4][2] = {{T(0), T(0)}, {T(1), T(0)}, {T(1), T(1)}, {T(0), T(1)}};
  for (int64_t j = 0; j < g.n[1]; ++j)
    for (int64_t i = 0; i < g.n[0]; ++i) {
      const int64_t ci = i + g.n[0] * j;
      const T org[2] = {node_coord(x0[0], d[0], i), node_coord(x0[1], d[1], j)};
      T xi[2][2] = {{T(0), T(0)}, {T(0), T(0)}};
      if (valid[ci]) {
        const T n0 = normals[2 * ci], n1 = normals[2 * ci + 1], a = intercepts[ci];
        T s[4];
        for (int k = 0; k < 4; ++k) s[k] = (n0 * corner[k][0] + n1 * corner[k][1]) - a;
        int m = 0;
        for (int k = 0; k < 4 && m < 2; ++k) {
          if (s[k] == T(0)) { xi[m][0] = corner[k][0]; xi[m][1] = corner[k][1]; ++m; continue; }
          const int k1 = (k + 1) & 3;
          if ((s[k] < T(0) && s[k1] > T(0)) || (s[k] > T(0) && s[k1] < T(0))) {
            const T t = s[k] / (s[k] - s[k1]);
            xi[m][0] = corner[k][0] + t * (corner[k1][0] - corner[k][0]);
            xi[m][1] = corner[k][1] + t * (corner[k1][1] - corner[k][1]);
            ++m;
          }
        }
        if (m == 0) xi[0][0] = xi[0][1] = T(0);
        if (m < 2) { xi[1][0] = xi[0][0]; xi[1][1] = xi[0][1]; }
      }
      T p[2][2];
      for (int q = 0; q < 2; ++q) {
        p[q][0] = org[0] + xi[q][0] * d[0];
        p[q][1] = org[1] + xi[q][1] * d[1];
      }
      const T dx = p[1][0] - p[0][0], dy = p[1][1] - p[0][1];
      if (!(std::sqrt(dx * dx + dy * dy) >= min_frac * min_d)) continue;
      const int32_t base = int32_t(out.nodes.size() / 2);
      for (int q = 0; q < 2; ++q) { out.nodes.push_back(p[q][0]); out.nodes.push_back(p[q][1]); }
      out.elems.push_back(base);
      out.elems.push_back(base + 1);
      out.cells.push_back(ci);
    }
  return out;
}

// 3D: the polygon (corners on the plane, then strict edge crossings in the order x-edges, y-edges,
// z-edges), ordered about its centroid in the basis of surface.jl:247-249, fanned from its first
// vertex with the area floor of surface.jl:162-181. Cells with fewer than 3 points draw nothing.
template <class T>
PlicMesh<T> plic_mesh3(const cc_grid& g, const T* normals, const T* intercepts, const uint8_t* valid, T min_frac) {
  PlicMesh<T> out;
  const T x0[3] = {T(g.x0[0]), T(g.x0[1]), T(g.x0[2])}, d[3] = {T(g.d[0]), T(g.d[1]), T(g.d[2])};
  T min_d = d[0];
  for (int a = 1; a < 3; ++a) min_d = d[a] < min_d ? d[a] : min_d;
  const T min_area = min_frac * (min_d * min_d);
  const T min_cross_sq = (T(2) * min_area) * (T(2) * min_area);
  static const int edge[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                  {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int64_t k3 = 0; k3 < g.n[2]; ++k3)
    for (int64_t j = 0; j < g.n[1]; ++j)
      for (int64_t i = 0; i < g.n[0]; ++i) {
        const int64_t ci = i + g.n[0] * (j + g.n[1] * k3);
        if (!valid[ci]) continue;
        const T nr[3] = {normals[3 * ci], normals[3 * ci + 1], normals[3 * ci + 2]};
        const T a = intercepts[ci];
        const T org[3] = {node_coord(x0[0], d[0], i), node_coord(x0[1], d[1], j), node_coord(x0[2], d[2], k3)};
        T s[8];
        for (int c = 0; c < 8; ++c)
          s[c] = ((nr[0] * T(c & 1) + nr[1] * T((c >> 1) & 1)) + nr[2] * T((c >> 2) & 1)) - a;
        T xi[6][3];
        int m = 0;
        for (int c = 0; c < 8 && m < 6; ++c)
          if (s[c] == T(0)) { xi[m][0] = T(c & 1); xi[m][1] = T((c >> 1) & 1); xi[m][2] = T((c >> 2) & 1); ++m; }
        for (int e = 0; e < 12 && m < 6; ++e) {
          const int p = edge[e][0], q = edge[e][1];
          if ((s[p] < T(0) && s[q] > T(0)) || (s[p] > T(0) && s[q] < T(0))) {
            const T t = s[p] / (s[p] - s[q]);
            for (int ax = 0; ax < 3; ++ax) {
              const T cp = T((p >> ax) & 1), cq = T((q >> ax) & 1);
              xi[m][ax] = cp + t * (cq - cp);
            }
            ++m;
          }
        }
        if (m < 3) continue;
        T pt[6][3];
        for (int v = 0; v < m; ++v)
          for (int ax = 0; ax < 3; ++ax) pt[v][ax] = org[ax] + xi[v][ax] * d[ax];
        T cen[3] = {T(0), T(0), T(0)};
        for (int v = 0; v < m; ++v)
          for (int ax = 0; ax < 3; ++ax) cen[ax] = cen[ax] + pt[v][ax];
        for (int ax = 0; ax < 3; ++ax) cen[ax] = cen[ax] / T(m);
        const bool zr = std::fabs(nr[2]) < T(0.9);
        const T r[3] = {zr ? T(0) : T(1), T(0), zr ? T(1) : T(0)};
        T u[3] = {r[1] * nr[2] - r[2] * nr[1], r[2] * nr[0] - r[0] * nr[2], r[0] * nr[1] - r[1] * nr[0]};
        const T ul = std::sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
        for (int ax = 0; ax < 3; ++ax) u[ax] = u[ax] / ul;
        const T v[3] = {nr[1] * u[2] - nr[2] * u[1], nr[2] * u[0] - nr[0] * u[2], nr[0] * u[1] - nr[1] * u[0]};
        T ang[6];
        for (int q = 0; q < m; ++q) {
          const T dx = pt[q][0] - cen[0], dy = pt[q][1] - cen[1], dz = pt[q][2] - cen[2];
          ang[q] = pseudo_angle((dx * v[0] + dy * v[1]) + dz * v[2], (dx * u[0] + dy * u[1]) + dz * u[2]);
        }
        for (int q = 1; q < m; ++q) {  // insertion sort, as surface.jl:256-265
          const T ka = ang[q];
          T kp[3] = {pt[q][0], pt[q][1], pt[q][2]};
          int w = q - 1;
          while (w >= 0 && ang[w] > ka) {
            ang[w + 1] = ang[w];
            for (int ax = 0; ax < 3; ++ax) pt[w + 1][ax] = pt[w][ax];
            --w;
          }
          ang[w + 1] = ka;
          for (int ax = 0; ax < 3; ++ax) pt[w + 1][ax] = kp[ax];
        }
        const int32_t base = int32_t(out.nodes.size() / 3);
        for (int q = 0; q < m; ++q)
          for (int ax = 0; ax < 3; ++ax) out.nodes.push_back(pt[q][ax]);
        for (int q = 1; q < m - 1; ++q) {
          const T a0 = pt[q][0] - pt[0][0], a1 = pt[q][1] - pt[0][1], a2 = pt[q][2] - pt[0][2];
          const T b0 = pt[q + 1][0] - pt[0][0], b1 = pt[q + 1][1] - pt[0][1], b2 = pt[q + 1][2] - pt[0][2];
          const T c0 = a1 * b2 - a2 * b1, c1 = a2 * b0 - a0 * b2, c2 = a0 * b1 - a1 * b0;
          if ((c0 * c0 + c1 * c1) + c2 * c2 >= min_cross_sq) {
            out.elems.push_back(base);
            out.elems.push_back(base + q);
            out.elems.push_back(base + q + 1);
            out.cells.push_back(ci);
          }
        }
      }
  return out;
}

}  // namespace oc

// ======================================================================================
// C entry points for the test harness (ctypes). prec: 0 = Float32, 1 = Float64, 2 = mixed
// (Float32 data with the Float64 islands).
extern "C" {

int oc_set_threads(int n) {
  if (n > 0) oc::g_threads = n;
  return oc::g_threads;
}

int oc_sample_nodes(int prec, const cc_grid* g, const cc_optape* t, void* phi) {
  oc::MixedScope mixed(prec == 2);
  if (g->dim == 3) {
    if (prec == 1) oc::sample_nodes<double, 3>(*g, oc::make_tape<double>(t), (double*)phi);
    else oc::sample_nodes<float, 3>(*g, oc::make_tape<float>(t), (float*)phi);
  } else {
    if (prec == 1) oc::sample_nodes<double, 2>(*g, oc::make_tape<double>(t), (double*)phi);
    else oc::sample_nodes<float, 2>(*g, oc::make_tape<float>(t), (float*)phi);
  }
  return 0;
}

int oc_mc_cells_from_phi(int prec, const cc_grid* g, const uint8_t* table, const void* phi,
                         const cc_cells* c) {
  oc::MixedScope mixed(prec == 2);
  oc::McTable tb;
  if (!tb.parse(table)) return CC_BAD_TABLE;
  if (prec == 1) oc::mc_cells<double>(*g, tb, (const double*)phi, *c);
  else oc::mc_cells<float>(*g, tb, (const float*)phi, *c);
  return 0;
}

// The learned correction's label of cut cell `ci` of the 3D grid g: the fluid volume fraction of
// update_cache! on the one-cell grid CartesianGrid(get_node(g, ci), (8,8,8), g.d/8) in Float64 (the
// idiom of test/test_mc_moments.jl:67-69,91-98), its 512 fractions summed in the order the device
// sums them: four sub-cells per thread (t, t+128, t+256, t+384), a butterfly over each warp's 32
// threads, then (w0 + w1) + (w2 + w3); divided by 512.
int oc_mc_labels(const cc_grid* g, const cc_optape* t, const uint8_t* table, const int64_t* cells, int64_t n,
                 double* out) {
  if (g->dim != 3) return CC_BAD_ARG;
  oc::McTable tb;
  if (!tb.parse(table)) return CC_BAD_TABLE;
  const oc::Tape<double> tp = oc::make_tape<double>(t);
  for (int64_t q = 0; q < n; ++q) {
    const int64_t ci = cells[q];
    const int64_t idx[3] = {ci % g->n[0], (ci / g->n[0]) % g->n[1], ci / (g->n[0] * g->n[1])};
    cc_grid sub{};
    sub.dim = 3;
    for (int a = 0; a < 3; ++a) {
      sub.x0[a] = oc::node_coord(g->x0[a], g->d[a], idx[a]);
      sub.d[a] = g->d[a] / 8.0;
      sub.n[a] = 8;
    }
    std::vector<double> phi(729);
    oc::sample_nodes_range<double, 3>(sub, tp, phi.data(), 0, 8);
    std::vector<int8_t> kind(512);
    std::vector<uint8_t> amb(512);
    std::vector<double> vf(512), c(512 * 3), ff(512 * 6), fcl(512 * 12), ic(512 * 3);
    const cc_cells cols{kind.data(), amb.data(), vf.data(), c.data(), ff.data(), fcl.data(), ic.data()};
    oc::mc_cells_range<double>(sub, tb, phi.data(), cols, 0, 8);
    double lane[128];
    for (int th = 0; th < 128; ++th) {
      double acc = 0.0;
      for (int r = 0; r < 4; ++r) acc = acc + vf[th + 128 * r];
      lane[th] = acc;
    }
    double red[4];
    for (int w = 0; w < 4; ++w) {
      double b[32];
      for (int l = 0; l < 32; ++l) b[l] = lane[32 * w + l];
      for (int o = 16; o > 0; o >>= 1) {
        double nb[32];
        for (int l = 0; l < 32; ++l) nb[l] = b[l] + b[l ^ o];
        for (int l = 0; l < 32; ++l) b[l] = nb[l];
      }
      red[w] = b[0];
    }
    out[q] = ((red[0] + red[1]) + (red[2] + red[3])) / 512.0;
  }
  return 0;
}

// Marching cubes over the cell layers k0..k1-1 of the full grid g: phi receives the node layers
// k0..k1 and the columns the slab's cells, each computed with its global indices.
int oc_mc_update_slab(int prec, const cc_grid* g, const cc_optape* t, const uint8_t* table, int64_t k0,
                      int64_t k1, void* phi, const cc_cells* c) {
  if (g->dim != 3 || k0 < 0 || k1 > g->n[2] || k0 >= k1) return CC_BAD_ARG;
  oc::MixedScope mixed(prec == 2);
  oc::McTable tb;
  if (!tb.parse(table)) return CC_BAD_TABLE;
  if (prec == 1) {
    oc::sample_nodes_range<double, 3>(*g, oc::make_tape<double>(t), (double*)phi, k0, k1);
    oc::mc_cells_range<double>(*g, tb, (const double*)phi, *c, k0, k1);
  } else {
    oc::sample_nodes_range<float, 3>(*g, oc::make_tape<float>(t), (float*)phi, k0, k1);
    oc::mc_cells_range<float>(*g, tb, (const float*)phi, *c, k0, k1);
  }
  return 0;
}

// PLIC over the cell layers k0..k1-1 of the full 3D grid g (the layers either side fitted too, so
// the faces resolve as in the whole-grid update); outputs hold the slab's cells.
int oc_plic_update_slab(int prec, const cc_grid* g, const cc_optape* t, int64_t k0, int64_t k1, const cc_cells* c,
                        void* normals, void* intercepts, uint8_t* is_valid) {
  if (g->dim != 3 || k0 < 0 || k1 > g->n[2] || k0 >= k1) return CC_BAD_ARG;
  oc::MixedScope mixed(prec == 2);
  if (prec == 1)
    oc::plic_update_range<double, 3>(*g, oc::make_tape<double>(t), *c, (double*)normals, (double*)intercepts,
                                     is_valid, k0, k1);
  else
    oc::plic_update_range<float, 3>(*g, oc::make_tape<float>(t), *c, (float*)normals, (float*)intercepts,
                                    is_valid, k0, k1);
  return 0;
}

int oc_mc_update(int prec, const cc_grid* g, const cc_optape* t, const uint8_t* table, void* phi,
                 const cc_cells* c) {
  oc::MixedScope mixed(prec == 2);
  oc_sample_nodes(prec, g, t, phi);
  return oc_mc_cells_from_phi(prec, g, table, phi, c);
}

// generate_mesh: counts into *nv / *nt; arrays written when non-null (capacities checked).
int oc_mc_mesh(int prec, const cc_grid* g, const uint8_t* table, const void* phi, void* verts, int64_t vcap,
               int32_t* tris, int64_t tcap, int64_t* cells, int64_t* nv, int64_t* nt) {
  oc::MixedScope mixed(prec == 2);
  oc::McTable tb;
  if (!tb.parse(table)) return CC_BAD_TABLE;
  auto run = [&](auto m) {
    using TT = typename std::decay<decltype(m.verts[0])>::type;
    *nv = int64_t(m.verts.size() / 3);
    *nt = int64_t(m.tris.size() / 3);
    if (verts && *nv <= vcap) std::memcpy(verts, m.verts.data(), m.verts.size() * sizeof(TT));
    if (tris && *nt <= tcap) std::memcpy(tris, m.tris.data(), m.tris.size() * sizeof(int32_t));
    if (cells && *nt <= tcap) std::memcpy(cells, m.cells.data(), m.cells.size() * sizeof(int64_t));
    return 0;
  };
  if (prec == 1) return run(oc::mc_mesh<double>(*g, tb, (const double*)phi));
  return run(oc::mc_mesh<float>(*g, tb, (const float*)phi));
}

// generate_mesh for marching squares: a grid (tree == 0) or leaves (tree != 0, then x0, base_d,
// nl, level, coord describe them). Counts into *nv / *ns; arrays written when non-null.
int oc_ms_mesh(int prec, int tree, const cc_grid* g, const double* x0, const double* based, int64_t nl,
               const int32_t* level, const int32_t* coord, const void* phi, void* verts, int32_t* segs,
               int64_t* cells, int64_t* nv, int64_t* ns) {
  oc::MixedScope mixed(prec == 2);
  auto out = [&](auto c) {
    using TT = typename std::decay<decltype(c.verts[0])>::type;
    *nv = int64_t(c.verts.size() / 2);
    *ns = int64_t(c.cells.size());
    if (verts) std::memcpy(verts, c.verts.data(), c.verts.size() * sizeof(TT));
    if (segs) std::memcpy(segs, c.segs.data(), c.segs.size() * sizeof(int32_t));
    if (cells) std::memcpy(cells, c.cells.data(), c.cells.size() * sizeof(int64_t));
    return 0;
  };
  if (prec == 1)
    return tree ? out(oc::ms_mesh_tree<double>(x0, based, nl, level, coord, (const double*)phi))
                : out(oc::ms_mesh_grid<double>(*g, (const double*)phi));
  return tree ? out(oc::ms_mesh_tree<float>(x0, based, nl, level, coord, (const float*)phi))
              : out(oc::ms_mesh_grid<float>(*g, (const float*)phi));
}

// generate_mesh for a PLIC cache: counts into *nn / *ne; arrays written when non-null.
int oc_plic_mesh(int prec, const cc_grid* g, const void* normals, const void* intercepts, const uint8_t* valid,
                 double min_frac, void* nodes, int32_t* elems, int64_t* cells, int64_t* nn, int64_t* ne) {
  auto out = [&](auto c, int D) {
    using TT = typename std::decay<decltype(c.nodes[0])>::type;
    *nn = int64_t(c.nodes.size() / D);
    *ne = int64_t(c.cells.size());
    if (nodes) std::memcpy(nodes, c.nodes.data(), c.nodes.size() * sizeof(TT));
    if (elems) std::memcpy(elems, c.elems.data(), c.elems.size() * sizeof(int32_t));
    if (cells) std::memcpy(cells, c.cells.data(), c.cells.size() * sizeof(int64_t));
    return 0;
  };
  if (g->dim == 3) {
    if (prec == 1)
      return out(oc::plic_mesh3<double>(*g, (const double*)normals, (const double*)intercepts, valid, min_frac), 3);
    return out(oc::plic_mesh3<float>(*g, (const float*)normals, (const float*)intercepts, valid, float(min_frac)), 3);
  }
  if (prec == 1)
    return out(oc::plic_mesh2<double>(*g, (const double*)normals, (const double*)intercepts, valid, min_frac), 2);
  return out(oc::plic_mesh2<float>(*g, (const float*)normals, (const float*)intercepts, valid, float(min_frac)), 2);
}

int oc_ms_cells_from_phi(int prec, const cc_grid* g, const void* phi, const cc_cells* c) {
  oc::MixedScope mixed(prec == 2);
  if (prec == 1) oc::ms_cells<double>(*g, (const double*)phi, *c);
  else oc::ms_cells<float>(*g, (const float*)phi, *c);
  return 0;
}

int oc_ms_update(int prec, const cc_grid* g, const cc_optape* t, void* phi, const cc_cells* c) {
  oc::MixedScope mixed(prec == 2);
  oc_sample_nodes(prec, g, t, phi);
  return oc_ms_cells_from_phi(prec, g, phi, c);
}

int oc_ms_tree_update(int prec, const double* x0, const double* base_d, int64_t nleaves,
                      const int32_t* level, const int32_t* coord, const cc_optape* t, void* phi4,
                      const cc_cells* c) {
  oc::MixedScope mixed(prec == 2);
  if (prec == 1) oc::ms_tree<double>(x0, base_d, nleaves, level, coord, oc::make_tape<double>(t), (double*)phi4, *c);
  else oc::ms_tree<float>(x0, base_d, nleaves, level, coord, oc::make_tape<float>(t), (float*)phi4, *c);
  return 0;
}

int oc_plic_update(int prec, const cc_grid* g, const cc_optape* t, const cc_cells* c, void* normals,
                   void* intercepts, uint8_t* is_valid) {
  oc::MixedScope mixed(prec == 2);
  if (g->dim == 3) {
    if (prec == 1) oc::plic_update<double, 3>(*g, oc::make_tape<double>(t), *c, (double*)normals, (double*)intercepts, is_valid);
    else oc::plic_update<float, 3>(*g, oc::make_tape<float>(t), *c, (float*)normals, (float*)intercepts, is_valid);
  } else {
    if (prec == 1) oc::plic_update<double, 2>(*g, oc::make_tape<double>(t), *c, (double*)normals, (double*)intercepts, is_valid);
    else oc::plic_update<float, 2>(*g, oc::make_tape<float>(t), *c, (float*)normals, (float*)intercepts, is_valid);
  }
  return 0;
}

double oc_calc_volume(int prec, const cc_grid* g, const cc_optape* t) {
  oc::MixedScope mixed(prec == 2);
  if (g->dim == 3) {
    if (prec == 1) return oc::calc_volume<double, 3>(*g, oc::make_tape<double>(t));
    return double(oc::calc_volume<float, 3>(*g, oc::make_tape<float>(t)));
  }
  if (prec == 1) return oc::calc_volume<double, 2>(*g, oc::make_tape<double>(t));
  return double(oc::calc_volume<float, 2>(*g, oc::make_tape<float>(t)));
}

// Every cell's cell_plane solid fraction, widened to double (the calc_volume integrand).
int oc_plic_fractions(int prec, const cc_grid* g, const cc_optape* t, double* out) {
  oc::MixedScope mixed(prec == 2);
  const int64_t n[3] = {g->n[0], g->n[1], g->dim == 3 ? g->n[2] : 1};
  const int64_t ncell = n[0] * n[1] * n[2];
  auto run = [&](auto zero, auto dimc) {
    using T = decltype(zero);
    constexpr int D = decltype(dimc)::value;
    const oc::Tape<T> tp = oc::make_tape<T>(t);
    const T x0[3] = {T(g->x0[0]), T(g->x0[1]), T(g->x0[2])};
    const T d[3] = {T(g->d[0]), T(g->d[1]), T(g->d[2])};
    oc::parallel_for(ncell, [&](int64_t ci) {
      const int64_t idx[3] = {ci % n[0], (ci / n[0]) % n[1], ci / (n[0] * n[1])};
      out[ci] = double(oc::cell_plane<T, D>(tp, x0, d, idx).fraction);
    });
  };
  if (g->dim == 3) { if (prec == 1) run(0.0, std::integral_constant<int, 3>()); else run(0.0f, std::integral_constant<int, 3>()); }
  else { if (prec == 1) run(0.0, std::integral_constant<int, 2>()); else run(0.0f, std::integral_constant<int, 2>()); }
  return 0;
}

double oc_gvf3(double n1, double n2, double n3, double a) { return oc::gvf3(n1, n2, n3, a); }
double oc_gvf2(double n1, double n2, double a) { return oc::gvf2(n1, n2, a); }
float oc_gvf3f(float n1, float n2, float n3, float a) { return oc::gvf3(n1, n2, n3, a); }

// Per-cube dispatch pieces, exposed for the table tests.
int oc_mc_triangles(const uint8_t* table, const double* phi8, uint8_t* codes_out, int* lcase) {
  oc::McTable tb;
  if (!tb.parse(table)) return -1;
  double ph[8];
  for (int k = 0; k < 8; ++k) ph[k] = oc::nudge(phi8[k]);
  const uint8_t* codes = nullptr;
  const int n = oc::cell_triangles(tb, ph, &codes, lcase);
  std::memcpy(codes_out, codes, 3 * n);
  return n;
}
int oc_test_face(const double* phi8, int face) { return oc::test_face(phi8, face) ? 1 : 0; }
int oc_test_interior(int itype, int edge, const double* phi8, int s) {
  return oc::test_interior(itype, edge, phi8, s) ? 1 : 0;
}
int oc_face_test_code(int dir) { return oc::MCC.face_test_code[dir]; }
int oc_face_node(int dir, int k) { return oc::MCC.face_nodes[dir][k]; }

double oc_eval_tape(int dim, int prec, const cc_optape* t, const double* x, double* grad) {
  if (dim == 3) {
    if (prec == 1) {
      oc::Tape<double> tp = oc::make_tape<double>(t);
      oc::Dual<double, 3> xs[3];
      for (int a = 0; a < 3; ++a) { xs[a] = oc::dconst<double, 3>(x[a]); xs[a].g[a] = 1.0; }
      auto r = oc::eval_tape<double, 3, oc::Dual<double, 3>>(tp, xs);
      if (grad) for (int a = 0; a < 3; ++a) grad[a] = r.g[a];
      return r.v;
    }
    oc::Tape<float> tp = oc::make_tape<float>(t);
    float xs[3] = {float(x[0]), float(x[1]), float(x[2])};
    return oc::eval_tape<float, 3, float>(tp, xs);
  }
  if (prec == 1) {
    oc::Tape<double> tp = oc::make_tape<double>(t);
    oc::Dual<double, 2> xs[2];
    for (int a = 0; a < 2; ++a) { xs[a] = oc::dconst<double, 2>(x[a]); xs[a].g[a] = 1.0; }
    auto r = oc::eval_tape<double, 2, oc::Dual<double, 2>>(tp, xs);
    if (grad) for (int a = 0; a < 2; ++a) grad[a] = r.g[a];
    return r.v;
  }
  oc::Tape<float> tp = oc::make_tape<float>(t);
  float xs[2] = {float(x[0]), float(x[1])};
  return oc::eval_tape<float, 2, float>(tp, xs);
}

}  // extern "C"
