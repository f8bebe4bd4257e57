// mc_cell.cuh -- the per-cell marching-cubes construction (cut cells), shared by the update
// kernels and the learned-correction kernels.
//
// cut_cell_moments for a cut cell (src/marching_cubes/moments.jl:275-346): the six face clips
// (cut_cell_faces / _cut_cell_face, :150-257, with the walk of
// src/marching_squares/marching_squares.jl:240-251), the Lewiner dispatch over a tiling table
// (src/marching_cubes/marching_cubes.jl:538-651, deciders :401-504), the edge crossings
// (:306-330) and the divergence-theorem sums.
#pragma once
#include <cstdint>
#include <type_traits>
#include "cc_device.cuh"
#include "cc_internal.h"

namespace ccmc {

using namespace ccd;
using cci::DevTable;

// MC_NODE_BITS (src/marching_cubes/marching_cubes.jl:106-107), bit of corner c along axis a.
__host__ __device__ constexpr int cbit(int c, int a) {
  return a == 0 ? ((c ^ (c >> 1)) & 1) : (a == 1 ? ((c >> 1) & 1) : ((c >> 2) & 1));
}
// MC_FACE_NODES (:169-180), 0-based directions and corners.
__host__ __device__ constexpr int face_node(int dir, int k) {
  constexpr int t[6][4] = {{0, 3, 7, 4}, {1, 2, 6, 5}, {0, 1, 5, 4}, {3, 2, 6, 7}, {0, 1, 2, 3}, {4, 5, 6, 7}};
  return t[dir][k];
}
// MC_FACE_TEST_CODE (:385-388)
__host__ __device__ constexpr int face_test_code(int dir) {
  constexpr int t[6] = {4, 2, 1, 3, 5, 6};
  return t[dir];
}
// MC_EDGE_NODES (:135-137), 0-based corners.
__host__ __device__ constexpr int edge_node(int e, int s) {
  constexpr int t[12][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}, {4, 5}, {5, 6}, {7, 6}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  return t[e][s];
}

// MC_TEST_FACE_QUADS (:372-373) and the twelve reference-edge branches of _test_interior
// (:450-486), 0-based corners, for indices only known at run time.
static __constant__ uint8_t c_quads[6][4] = {{0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 4, 0}, {0, 3, 2, 1}, {4, 7, 6, 5}};
static __constant__ uint8_t c_iedge[12][8] = {
    {0, 1, 3, 2, 7, 6, 4, 5}, {1, 2, 0, 3, 4, 7, 5, 6}, {2, 3, 1, 0, 5, 4, 6, 7}, {3, 0, 2, 1, 6, 5, 7, 4},
    {4, 5, 7, 6, 3, 2, 0, 1}, {5, 6, 4, 7, 0, 3, 1, 2}, {6, 7, 5, 4, 1, 0, 2, 3}, {7, 4, 6, 5, 2, 1, 3, 0},
    {0, 4, 3, 7, 2, 6, 1, 5}, {1, 5, 0, 4, 3, 7, 2, 6}, {2, 6, 1, 5, 0, 4, 3, 7}, {3, 7, 2, 6, 1, 5, 0, 4}};

template <class T>
__device__ __forceinline__ T nudge(T v) {
  const T e = Eps<T>::v();
  return fabs(v) < e ? e : v;
}

// _test_face, src/marching_cubes/marching_cubes.jl:401-406. With MX the determinant and the
// final product are evaluated in FP64 (R) from the FP32 corner values; the threshold stays eps(T).
template <class T, bool MX = false>
__device__ __forceinline__ bool test_face(const T* cb, int face) {
  using R = typename std::conditional<MX, double, T>::type;
  const int f = (face < 0 ? -face : face) - 1;
  const R A = cb[c_quads[f][0]], B = cb[c_quads[f][1]], C = cb[c_quads[f][2]], D = cb[c_quads[f][3]];
  const R det = A * C - B * D;
  if (fabs(det) < R(Eps<T>::v())) return face >= 0;
  return (R(face) * A) * det >= R(0);
}
// The same decider for a face code known at compile time (face_outside_connected, :421-422).
template <class T, int FACE, bool MX = false>
__device__ __forceinline__ bool test_face_c(const T* cb) {
  using R = typename std::conditional<MX, double, T>::type;
  constexpr int q[6][4] = {{0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 4, 0}, {0, 3, 2, 1}, {4, 7, 6, 5}};
  const R A = cb[q[FACE - 1][0]], B = cb[q[FACE - 1][1]], C = cb[q[FACE - 1][2]], D = cb[q[FACE - 1][3]];
  const R det = A * C - B * D;
  if (fabs(det) < R(Eps<T>::v())) return true;
  return (R(FACE) * A) * det >= R(0);
}

// _test_interior, :427-504. With MX every step runs in FP64 (R) from the FP32 corner values; the
// thresholds stay eps(T).
template <class T, bool MX = false>
__device__ bool test_interior(int itype, int edge, const T* cbt, int s) {
  using R = typename std::conditional<MX, double, T>::type;
  R cb[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) cb[k] = cbt[k];
  R At = R(0), Bt = R(0), Ct = R(0), Dt = R(0);
  if (itype == CC_MC_INTERIOR_CASE4_10) {
    const R a = (cb[4] - cb[0]) * (cb[6] - cb[2]) - (cb[7] - cb[3]) * (cb[5] - cb[1]);
    const R b = ((cb[2] * (cb[4] - cb[0]) + cb[0] * (cb[6] - cb[2])) - cb[1] * (cb[7] - cb[3])) - cb[3] * (cb[5] - cb[1]);
    const R t = -b / (R(2) * a);
    if (t < R(0) || t > R(1)) return s > 0;
    At = cb[0] + (cb[4] - cb[0]) * t;
    Bt = cb[3] + (cb[7] - cb[3]) * t;
    Ct = cb[2] + (cb[6] - cb[2]) * t;
    Dt = cb[1] + (cb[5] - cb[1]) * t;
  } else {
    const uint8_t* e = c_iedge[edge];
    const R t = cb[e[0]] / (cb[e[0]] - cb[e[1]]);
    Bt = cb[e[2]] + (cb[e[3]] - cb[e[2]]) * t;
    Ct = cb[e[4]] + (cb[e[5]] - cb[e[4]]) * t;
    Dt = cb[e[6]] + (cb[e[7]] - cb[e[6]]) * t;
  }
  int test = 0;
  if (At >= R(0)) test += 1;
  if (Bt >= R(0)) test += 2;
  if (Ct >= R(0)) test += 4;
  if (Dt >= R(0)) test += 8;
  const R eps = R(Eps<T>::v());
  if (test == 6 || test == 8 || test == 9 || test == 12 || (test >= 0 && test <= 4)) return s > 0;
  if (test == 5) return (At * Ct - Bt * Dt < eps) ? s > 0 : s < 0;
  if (test == 10) return (At * Ct - Bt * Dt >= eps) ? s > 0 : s < 0;
  return s < 0;
}

// The open polygon of one cube face in its own (p, q) frame: cell_boundary_walk
// (src/marching_squares/marching_squares.jl:240-251) then _face_polygon
// (src/marching_cubes/moments.jl:111-139) with _chord_target (:91-98).
template <class T, bool MX = false>
__device__ __forceinline__ void face_polygon(const T fn[4][2], const T fphi[4], bool connect, T& area2,
                                             T& m0, T& m1) {
  T sa[4][2], sb[4][2];
  bool present[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int k1 = (k + 1) & 3;
    const T fa = fphi[k], fb = fphi[k1];
    const T frac = open_fraction<T, MX>(fa, fb);
    present[k] = fa >= T(0) || fb >= T(0);
    if (fa >= T(0) && fb >= T(0)) {
      sa[k][0] = fn[k][0]; sa[k][1] = fn[k][1]; sb[k][0] = fn[k1][0]; sb[k][1] = fn[k1][1];
    } else if (fa >= T(0)) {
      sa[k][0] = fn[k][0]; sa[k][1] = fn[k][1];
      sb[k][0] = fn[k][0] + frac * (fn[k1][0] - fn[k][0]);
      sb[k][1] = fn[k][1] + frac * (fn[k1][1] - fn[k][1]);
    } else {
      sa[k][0] = fn[k1][0] + frac * (fn[k][0] - fn[k1][0]);
      sa[k][1] = fn[k1][1] + frac * (fn[k][1] - fn[k1][1]);
      sb[k][0] = fn[k1][0]; sb[k][1] = fn[k1][1];
    }
  }
  area2 = T(0); m0 = T(0); m1 = T(0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (present[k]) {
      const T cr = sa[k][0] * sb[k][1] - sa[k][1] * sb[k][0];
      area2 = area2 + cr;
      m0 = m0 + (sa[k][0] + sb[k][0]) * cr;
      m1 = m1 + (sa[k][1] + sb[k][1]) * cr;
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!(fphi[k] >= T(0) && fphi[(k + 1) & 3] < T(0))) continue;
    int j = k, hit = -1;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      j = connect ? ((j + 1) & 3) : ((j + 3) & 3);
      if (hit < 0 && fphi[j] < T(0) && fphi[(j + 1) & 3] >= T(0)) hit = j;
    }
    if (hit < 0) continue;
    const T lb0 = hit == 0 ? sa[0][0] : hit == 1 ? sa[1][0] : hit == 2 ? sa[2][0] : sa[3][0];
    const T lb1 = hit == 0 ? sa[0][1] : hit == 1 ? sa[1][1] : hit == 2 ? sa[2][1] : sa[3][1];
    const T la0 = sb[k][0], la1 = sb[k][1];
    const T cr = la0 * lb1 - la1 * lb0;
    area2 = area2 + cr;
    m0 = m0 + (la0 + lb0) * cr;
    m1 = m1 + (la1 + lb1) * cr;
  }
}

// Shared-memory staging of one tile's output columns.
template <class T>
struct Stage {
  int8_t* kind;
  uint8_t* amb;
  T* vf;
  T* c;
  T* ff;
  T* fcl;
  T* ic;
};

template <class T>
__device__ __forceinline__ void put_vec(T* dst, const T* v, int n);

template <>
__device__ __forceinline__ void put_vec<float>(float* dst, const float* v, int n) {
  // n is 6 or 12 with dst 8- or 16-byte aligned respectively
  if (n == 12) {
    float4* d4 = reinterpret_cast<float4*>(dst);
    d4[0] = make_float4(v[0], v[1], v[2], v[3]);
    d4[1] = make_float4(v[4], v[5], v[6], v[7]);
    d4[2] = make_float4(v[8], v[9], v[10], v[11]);
  } else {
    float2* d2 = reinterpret_cast<float2*>(dst);
    d2[0] = make_float2(v[0], v[1]);
    d2[1] = make_float2(v[2], v[3]);
    d2[2] = make_float2(v[4], v[5]);
  }
}
template <>
__device__ __forceinline__ void put_vec<double>(double* dst, const double* v, int n) {
  double2* d2 = reinterpret_cast<double2*>(dst);
  for (int i = 0; i < n / 2; ++i) d2[i] = make_double2(v[2 * i], v[2 * i + 1]);
}

template <class T>
__device__ __forceinline__ void put_cell(const Stage<T>& st, long long lc, int kind, int amb, T vf, const T c[3],
                                         const T ff[6], const T fcl[12], const T ic[3]) {
  st.kind[lc] = int8_t(kind);
  st.amb[lc] = uint8_t(amb);
  st.vf[lc] = vf;
  st.c[3 * lc] = c[0]; st.c[3 * lc + 1] = c[1]; st.c[3 * lc + 2] = c[2];
  put_vec<T>(st.ff + 6 * lc, ff, 6);
  put_vec<T>(st.fcl + 12 * lc, fcl, 12);
  st.ic[3 * lc] = ic[0]; st.ic[3 * lc + 1] = ic[1]; st.ic[3 * lc + 2] = ic[2];
}

// cell_triangles over the table (src/marching_cubes/marching_cubes.jl:538-651): the tile of a cube
// with nudged corner values `phi` (MC_NODE_BITS order).
template <class T, bool MX = false>
__device__ __forceinline__ int mc_tile(const T phi[8], const DevTable& tb) {
  int lut = 0;
#pragma unroll
  for (int p = 0; p < 8; ++p) lut |= (phi[p] >= T(0) ? 1 : 0) << p;
  const cc_mc_lut ent = tb.luts[lut];
  int o = 0;
  for (int i = 0; i < ent.ntests; ++i) o |= (test_face<T, MX>(phi, ent.face[i]) ? 1 : 0) << i;
  const cc_mc_outcome oc = tb.outs[ent.outcome_base + o];
  int tile = oc.tile_true;
  if (oc.itype != CC_MC_INTERIOR_NONE && !test_interior<T, MX>(oc.itype, oc.edge, phi, oc.s)) tile = oc.tile_false;
  return tile;
}

// cut_cell_moments (3D) for a cut cell, src/marching_cubes/moments.jl:275-346. `phr` are the
// raw corner values in MC_NODE_BITS order, `l` the cell's lattice edge lengths
// (x_{i+1} - x_i per axis: every corner's cell-local coordinate is 0 or l exactly), `org` the
// lower corner and `cs` the grid's cell size.
template <class T, bool MX = false>
__device__ __noinline__ void mc_cut_cell(const T phr[8], const T l[3], const T org[3], const T cs[3],
                                         const DevTable tb, const Stage<T> st, long long lc) {
  T phi[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) phi[k] = nudge(phr[k]);
  T centre[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) centre[a] = org[a] + T(0.5) * cs[a];
  const T vol_cell = (cs[0] * cs[1]) * cs[2];

  const cc_mc_tile tl = tb.tiles[mc_tile<T, MX>(phi, tb)];

  // the six face clips (cut_cell_faces / _cut_cell_face, moments.jl:150-257)
  T ff[6], fcl[12];
  bool amb_face = false;
#pragma unroll
  for (int dir = 0; dir < 6; ++dir) {
    const int ax = dir >> 1;
    const int p = ax == 0 ? 1 : 0;
    const int q = ax == 2 ? 1 : 2;
    T fn[4][2], fphi[4];
    int nout = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int c = face_node(dir, k);
      fn[k][0] = cbit(c, p) ? l[p] : T(0);
      fn[k][1] = cbit(c, q) ? l[q] : T(0);
      fphi[k] = phi[c];
      nout += fphi[k] >= T(0) ? 1 : 0;
    }
    amb_face = amb_face || ((nout == 2) && ((fphi[0] >= T(0)) == (fphi[2] >= T(0))));
    const T avg0 = T(0.25) * (((fn[0][0] + fn[1][0]) + fn[2][0]) + fn[3][0]);
    const T avg1 = T(0.25) * (((fn[0][1] + fn[1][1]) + fn[2][1]) + fn[3][1]);
    T frac, c0, c1;
    if (nout == 4 || nout == 0) {
      frac = nout == 4 ? T(1) : T(0);
      c0 = avg0; c1 = avg1;
    } else {
      bool connect;
      switch (dir) {
        case 0: connect = test_face_c<T, face_test_code(0), MX>(phi); break;
        case 1: connect = test_face_c<T, face_test_code(1), MX>(phi); break;
        case 2: connect = test_face_c<T, face_test_code(2), MX>(phi); break;
        case 3: connect = test_face_c<T, face_test_code(3), MX>(phi); break;
        case 4: connect = test_face_c<T, face_test_code(4), MX>(phi); break;
        default: connect = test_face_c<T, face_test_code(5), MX>(phi); break;
      }
      T area2, m0, m1;
      face_polygon<T, MX>(fn, fphi, connect, area2, m0, m1);
      const T full = (T(1) * cs[p]) * cs[q];
      frac = (T(0.5) * area2) / full;
      if (area2 != T(0)) { const T den = T(3) * area2; c0 = m0 / den; c1 = m1 / den; }
      else { c0 = avg0; c1 = avg1; }
    }
    ff[dir] = frac;
    fcl[2 * dir] = c0;
    fcl[2 * dir + 1] = c1;
  }

  // edge_crossings (marching_cubes.jl:306-330)
  T pts[13][3];
  T acc0 = T(0), acc1 = T(0), acc2 = T(0);
  int ncr = 0;
#pragma unroll
  for (int e = 0; e < 12; ++e) {
    const int a = edge_node(e, 0), b = edge_node(e, 1);
    const T fa = phi[a], fb = phi[b];
    if ((fa >= T(0)) != (fb >= T(0))) {
      const T s = open_fraction<T, MX>(fa, fb);
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const T pa = cbit(a, x) ? l[x] : T(0);
        const T pb = cbit(b, x) ? l[x] : T(0);
        pts[e][x] = fa >= T(0) ? pa + s * (pb - pa) : pb + s * (pa - pb);
      }
      acc0 = acc0 + pts[e][0]; acc1 = acc1 + pts[e][1]; acc2 = acc2 + pts[e][2];
      ++ncr;
    } else {
      pts[e][0] = T(0); pts[e][1] = T(0); pts[e][2] = T(0);
    }
  }
  pts[12][0] = ncr > 0 ? acc0 / T(ncr) : T(0);
  pts[12][1] = ncr > 0 ? acc1 / T(ncr) : T(0);
  pts[12][2] = ncr > 0 ? acc2 / T(ncr) : T(0);

  // divergence theorem over the closed polyhedron (moments.jl:304-336)
  T vol3 = T(0);
  T cm0 = T(0), cm1 = T(0), cm2 = T(0);
#pragma unroll
  for (int dir = 0; dir < 6; ++dir) {
    const int ax = dir >> 1;
    const int p = ax == 0 ? 1 : 0;
    const int q = ax == 2 ? 1 : 2;
    const T s = (dir & 1) ? T(1) : T(-1);
    const T x_ax = (dir & 1) ? l[ax] : T(0);
    const T a_open = ff[dir] * ((T(1) * cs[p]) * cs[q]);
    vol3 = vol3 + (s * x_ax) * a_open;
    const T m = ((s * x_ax) * x_ax) * a_open;
    cm0 = cm0 + (ax == 0 ? m : T(0));
    cm1 = cm1 + (ax == 1 ? m : T(0));
    cm2 = cm2 + (ax == 2 ? m : T(0));
  }
  T iarea = T(0), ic0 = T(0), ic1 = T(0), ic2 = T(0);
  const uint8_t* codes = tb.codes + tl.code_off;
  for (int t = 0; t < tl.ntris; ++t) {
    const int ca = codes[3 * t] - 1, cb = codes[3 * t + 1] - 1, cd = codes[3 * t + 2] - 1;
    const T A0 = pts[ca][0], A1 = pts[ca][1], A2 = pts[ca][2];
    const T B0 = pts[cb][0], B1 = pts[cb][1], B2 = pts[cb][2];
    const T D0 = pts[cd][0], D1 = pts[cd][1], D2 = pts[cd][2];
    const T u0 = B0 - A0, u1 = B1 - A1, u2 = B2 - A2;
    const T v0 = D0 - A0, v1 = D1 - A1, v2 = D2 - A2;
    const T w0 = T(0.5) * (u1 * v2 - u2 * v1);
    const T w1 = T(0.5) * (u2 * v0 - u0 * v2);
    const T w2 = T(0.5) * (u0 * v1 - u1 * v0);
    const T x0 = ((A0 + B0) + D0) / T(3);
    const T x1 = ((A1 + B1) + D1) / T(3);
    const T x2 = ((A2 + B2) + D2) / T(3);
    vol3 = vol3 - ((w0 * x0 + w1 * x1) + w2 * x2);
    const T q0 = (((((A0 * A0 + B0 * B0) + D0 * D0) + A0 * B0) + B0 * D0) + D0 * A0) / T(6);
    const T q1 = (((((A1 * A1 + B1 * B1) + D1 * D1) + A1 * B1) + B1 * D1) + D1 * A1) / T(6);
    const T q2 = (((((A2 * A2 + B2 * B2) + D2 * D2) + A2 * B2) + B2 * D2) + D2 * A2) / T(6);
    cm0 = cm0 - w0 * q0;
    cm1 = cm1 - w1 * q1;
    cm2 = cm2 - w2 * q2;
    const T len = sqrt((w0 * w0 + w1 * w1) + w2 * w2);
    iarea = iarea + len;
    ic0 = ic0 + len * x0;
    ic1 = ic1 + len * x1;
    ic2 = ic2 + len * x2;
  }
  const T volume = vol3 / T(3);
  T c[3], ic[3];
  if (volume > T(0)) {
    const T den = T(2) * volume;
    c[0] = org[0] + cm0 / den; c[1] = org[1] + cm1 / den; c[2] = org[2] + cm2 / den;
  } else {
    c[0] = centre[0]; c[1] = centre[1]; c[2] = centre[2];
  }
  if (iarea > T(0)) {
    ic[0] = org[0] + ic0 / iarea; ic[1] = org[1] + ic1 / iarea; ic[2] = org[2] + ic2 / iarea;
  } else {
    ic[0] = centre[0]; ic[1] = centre[1]; ic[2] = centre[2];
  }
  int lut = 0;
#pragma unroll
  for (int p = 0; p < 8; ++p) lut |= (phi[p] >= T(0) ? 1 : 0) << p;
  const int lc_case = tb.luts[lut].lcase;
  const bool amb_case = lc_case == 5 || lc_case == 7 || lc_case == 8 || lc_case == 11 || lc_case == 13 || lc_case == 14;
  put_cell<T>(st, lc, 2, (amb_face || amb_case) ? 1 : 0, volume / vol_cell, c, ff, fcl, ic);
}

}  // namespace ccmc
