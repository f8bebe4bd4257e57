// mc.cu -- MarchingCubesCutCell update_cache! on sm_100a.
//
// Two kernels replace the reference's two KernelAbstractions launches
// (_sample_nodes_kernel! and _nodal_cells_kernel!, src/marching_squares/cache.jl:55-78):
//
//   * mc_fill_kernel: a CTA owns a pencil of TX x 4 cells in (x, y) and marches KZ slices along
//     z. Each slice it samples one new slab of (TX+1) x 5 node values from the op-tape into shared
//     memory (the slab below is kept from the previous slice), so a node is evaluated once per
//     CTA and written to phi once, by the CTA that owns it. Every thread classifies one cell from
//     its eight corners. Uncut cells (all corners of one sign) get their fields directly -- their
//     face centroids are half the lattice edge lengths, a cheap affine fill -- into a
//     double-buffered shared-memory staging tile that leaves as contiguous row spans of each
//     StructArray column through the TMA bulk-copy engine (cp.async.bulk, shared -> global), so
//     the SM's threads never issue the column stores. Cut cells are compacted with a warp ballot
//     into a global work list.
//   * mc_cut_kernel: one lane per listed cut cell runs the full construction of
//     src/marching_cubes/moments.jl:275-346 densely and writes that cell's fields.
#include <cstdint>
#include <cstring>
#include <cuda.h>
#include "cc_device.cuh"
#include "cc_internal.h"

namespace {

using namespace ccd;
using cci::Cols;
using cci::DevGrid;
using cci::DevTable;
using cci::DevTape;

// Fill-kernel tile: TX cells along x (32 at Float32, 16 at Float64, so a staging buffer is about
// 26 KB either way) by TY = 8 rows, one thread per cell, marching KZ slices along z. A slab of
// (TX+1) x (TY+1) nodes serves TX x TY cells: 1.16 node evaluations per cell at Float32.
template <class T> struct Tile {
  static constexpr int TX = sizeof(T) == 4 ? 32 : 16;
  static constexpr int TY = 8;
  static constexpr int NT = TX * TY;
  static constexpr int NSX = TX + 1;
  static constexpr int NSLAB = (TX + 1) * (TY + 1);
  static constexpr int MINB = sizeof(T) == 4 ? 3 : 4;
};
constexpr int KZ = 32;  // z slices marched per CTA
constexpr int NS = 4;   // node slabs sampled per round (one op-major tape pass per thread)
constexpr int CUT_NT = 128;

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
__constant__ uint8_t c_quads[6][4] = {{0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 4, 0}, {0, 3, 2, 1}, {4, 7, 6, 5}};
__constant__ uint8_t c_iedge[12][8] = {
    {0, 1, 3, 2, 7, 6, 4, 5}, {1, 2, 0, 3, 4, 7, 5, 6}, {2, 3, 1, 0, 5, 4, 6, 7}, {3, 0, 2, 1, 6, 5, 7, 4},
    {4, 5, 7, 6, 3, 2, 0, 1}, {5, 6, 4, 7, 0, 3, 1, 2}, {6, 7, 5, 4, 1, 0, 2, 3}, {7, 4, 6, 5, 2, 1, 3, 0},
    {0, 4, 3, 7, 2, 6, 1, 5}, {1, 5, 0, 4, 3, 7, 2, 6}, {2, 6, 1, 5, 0, 4, 3, 7}, {3, 7, 2, 6, 1, 5, 0, 4}};

template <class T>
__device__ __forceinline__ T nudge(T v) {
  const T e = Eps<T>::v();
  return fabs(v) < e ? e : v;
}

// _test_face, src/marching_cubes/marching_cubes.jl:401-406
template <class T>
__device__ __forceinline__ bool test_face(const T* cb, int face) {
  const int f = (face < 0 ? -face : face) - 1;
  const T A = cb[c_quads[f][0]], B = cb[c_quads[f][1]], C = cb[c_quads[f][2]], D = cb[c_quads[f][3]];
  const T det = A * C - B * D;
  if (fabs(det) < Eps<T>::v()) return face >= 0;
  return (T(face) * A) * det >= T(0);
}
// The same decider for a face code known at compile time (face_outside_connected, :421-422).
template <class T, int FACE>
__device__ __forceinline__ bool test_face_c(const T* cb) {
  constexpr int q[6][4] = {{0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 4, 0}, {0, 3, 2, 1}, {4, 7, 6, 5}};
  const T A = cb[q[FACE - 1][0]], B = cb[q[FACE - 1][1]], C = cb[q[FACE - 1][2]], D = cb[q[FACE - 1][3]];
  const T det = A * C - B * D;
  if (fabs(det) < Eps<T>::v()) return true;
  return (T(FACE) * A) * det >= T(0);
}

// _test_interior, :427-504
template <class T>
__device__ bool test_interior(int itype, int edge, const T* cb, int s) {
  T At = T(0), Bt = T(0), Ct = T(0), Dt = T(0);
  if (itype == CC_MC_INTERIOR_CASE4_10) {
    const T a = (cb[4] - cb[0]) * (cb[6] - cb[2]) - (cb[7] - cb[3]) * (cb[5] - cb[1]);
    const T b = ((cb[2] * (cb[4] - cb[0]) + cb[0] * (cb[6] - cb[2])) - cb[1] * (cb[7] - cb[3])) - cb[3] * (cb[5] - cb[1]);
    const T t = -b / (T(2) * a);
    if (t < T(0) || t > T(1)) return s > 0;
    At = cb[0] + (cb[4] - cb[0]) * t;
    Bt = cb[3] + (cb[7] - cb[3]) * t;
    Ct = cb[2] + (cb[6] - cb[2]) * t;
    Dt = cb[1] + (cb[5] - cb[1]) * t;
  } else {
    const uint8_t* e = c_iedge[edge];
    const T t = cb[e[0]] / (cb[e[0]] - cb[e[1]]);
    Bt = cb[e[2]] + (cb[e[3]] - cb[e[2]]) * t;
    Ct = cb[e[4]] + (cb[e[5]] - cb[e[4]]) * t;
    Dt = cb[e[6]] + (cb[e[7]] - cb[e[6]]) * t;
  }
  int test = 0;
  if (At >= T(0)) test += 1;
  if (Bt >= T(0)) test += 2;
  if (Ct >= T(0)) test += 4;
  if (Dt >= T(0)) test += 8;
  const T eps = Eps<T>::v();
  if (test == 6 || test == 8 || test == 9 || test == 12 || (test >= 0 && test <= 4)) return s > 0;
  if (test == 5) return (At * Ct - Bt * Dt < eps) ? s > 0 : s < 0;
  if (test == 10) return (At * Ct - Bt * Dt >= eps) ? s > 0 : s < 0;
  return s < 0;
}

// The open polygon of one cube face in its own (p, q) frame: cell_boundary_walk
// (src/marching_squares/marching_squares.jl:240-251) then _face_polygon
// (src/marching_cubes/moments.jl:111-139) with _chord_target (:91-98).
template <class T>
__device__ __forceinline__ void face_polygon(const T fn[4][2], const T fphi[4], bool connect, T& area2,
                                             T& m0, T& m1) {
  T sa[4][2], sb[4][2];
  bool present[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int k1 = (k + 1) & 3;
    const T fa = fphi[k], fb = fphi[k1];
    const T frac = open_fraction(fa, fb);
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

// cut_cell_moments (3D) for a cut cell, src/marching_cubes/moments.jl:275-346. `phr` are the
// raw corner values in MC_NODE_BITS order, `l` the cell's lattice edge lengths
// (x_{i+1} - x_i per axis: every corner's cell-local coordinate is 0 or l exactly), `org` the
// lower corner and `cs` the grid's cell size.
template <class T>
__device__ __noinline__ void mc_cut_cell(const T phr[8], const T l[3], const T org[3], const T cs[3],
                                         const DevTable tb, const Stage<T> st, long long lc) {
  T phi[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) phi[k] = nudge(phr[k]);
  T centre[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) centre[a] = org[a] + T(0.5) * cs[a];
  const T vol_cell = (cs[0] * cs[1]) * cs[2];

  // cell_triangles over the table (src/marching_cubes/marching_cubes.jl:538-651)
  int lut = 0;
#pragma unroll
  for (int p = 0; p < 8; ++p) lut |= (phi[p] >= T(0) ? 1 : 0) << p;
  const cc_mc_lut ent = tb.luts[lut];
  int o = 0;
  for (int i = 0; i < ent.ntests; ++i) o |= (test_face(phi, ent.face[i]) ? 1 : 0) << i;
  const cc_mc_outcome oc = tb.outs[ent.outcome_base + o];
  int tile = oc.tile_true;
  if (oc.itype != CC_MC_INTERIOR_NONE && !test_interior(oc.itype, oc.edge, phi, oc.s)) tile = oc.tile_false;
  const cc_mc_tile tl = tb.tiles[tile];

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
        case 0: connect = test_face_c<T, face_test_code(0)>(phi); break;
        case 1: connect = test_face_c<T, face_test_code(1)>(phi); break;
        case 2: connect = test_face_c<T, face_test_code(2)>(phi); break;
        case 3: connect = test_face_c<T, face_test_code(3)>(phi); break;
        case 4: connect = test_face_c<T, face_test_code(4)>(phi); break;
        default: connect = test_face_c<T, face_test_code(5)>(phi); break;
      }
      T area2, m0, m1;
      face_polygon(fn, fphi, connect, area2, m0, m1);
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
      const T s = open_fraction(fa, fb);
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
  const int lc_case = ent.lcase;
  const bool amb_case = lc_case == 5 || lc_case == 7 || lc_case == 8 || lc_case == 11 || lc_case == 13 || lc_case == 14;
  put_cell<T>(st, lc, 2, (amb_face || amb_case) ? 1 : 0, volume / vol_cell, c, ff, fcl, ic);
}

template <class T>
struct McArgs {
  DevGrid<T> g;
  DevTape tape;
  const T* phi_in;
  T* phi_out;
  Cols cols;
  DevTable tb;
  unsigned* cut_list;
  unsigned* cut_count;
  int n_itiles, n_jtiles;
  int use_tma;  // output columns leave through TMA tensor stores (maps below are valid)
};

// One TMA tensor map per output column: kind, ambiguous, volume_fraction (n0 x n1 x n2), centroid
// and interface_centroid (3 n0 x n1 x n2), face_fraction (6 n0 x n1 x n2), face_centroid_local
// (12 x n0 x n1 x n2). A staged tile is exactly one box of each.
struct ColumnMaps {
  CUtensorMap m[7];
};

// TMA bulk copy engine, shared -> global (cp.async.bulk, sm_90+), and its group bookkeeping.
__device__ __forceinline__ void bulk_s2g(void* gdst, const void* ssrc, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gdst),
               "r"((unsigned)__cvta_generic_to_shared(ssrc)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait() { asm volatile("cp.async.bulk.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_store3(const CUtensorMap* m, const void* ssrc, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(m),
               "r"((unsigned)__cvta_generic_to_shared(ssrc)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void tma_store4(const CUtensorMap* m, const void* ssrc, int c0, int c1, int c2, int c3) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];\n" ::"l"(m),
               "r"((unsigned)__cvta_generic_to_shared(ssrc)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}

// Shared-memory byte layout of one fill CTA: two staging buffers, two node slabs, the tape.
template <class T>
struct Layout {
  using TL = Tile<T>;
  static constexpr int NC = TL::NT;  // cells per staging buffer
  static constexpr int kind = 0;
  static constexpr int amb = kind + NC;
  static constexpr int vf = amb + NC;
  static constexpr int c = vf + NC * int(sizeof(T));
  static constexpr int ff = c + 3 * NC * int(sizeof(T));
  static constexpr int fcl = ff + 6 * NC * int(sizeof(T));
  static constexpr int ic = fcl + 12 * NC * int(sizeof(T));
  static constexpr int stage_bytes = ((ic + 3 * NC * int(sizeof(T)) + 127) / 128) * 128;
  static constexpr int slab_bytes = ((TL::NSLAB * int(sizeof(T)) + 15) / 16) * 16;
  static constexpr int slab0 = 2 * stage_bytes;
  static constexpr int tape = slab0 + (NS + 1) * slab_bytes;
  // TMA tensor stores read each staged column from a 128-byte aligned base
  static_assert(amb % 128 == 0 && vf % 128 == 0 && c % 128 == 0 && ff % 128 == 0 && fcl % 128 == 0 &&
                    ic % 128 == 0 && stage_bytes % 128 == 0,
                "staged columns must start on 128-byte boundaries");
};

// bytes per staged row of output column `col` (kind, amb, vf, c, ff, fcl, ic) and its offset
template <class T>
__device__ __forceinline__ constexpr int col_bytes(int col) {
  return col < 2 ? Tile<T>::TX
                 : (col == 2 ? 1 : col == 3 ? 3 : col == 4 ? 6 : col == 5 ? 12 : 3) * Tile<T>::TX * int(sizeof(T));
}
template <class T>
__device__ __forceinline__ constexpr int col_offset(int col) {
  return col == 0 ? Layout<T>::kind : col == 1 ? Layout<T>::amb : col == 2 ? Layout<T>::vf : col == 3 ? Layout<T>::c
       : col == 4 ? Layout<T>::ff : col == 5 ? Layout<T>::fcl : Layout<T>::ic;
}
__device__ __forceinline__ constexpr int col_elem(int col, int tsize) {
  return col < 2 ? 1 : (col == 2 ? 1 : col == 3 ? 3 : col == 4 ? 6 : col == 5 ? 12 : 3) * tsize;
}

template <class T>
__device__ __forceinline__ Stage<T> stage_at(unsigned char* base) {
  using L = Layout<T>;
  Stage<T> st;
  st.kind = reinterpret_cast<int8_t*>(base + L::kind);
  st.amb = base + L::amb;
  st.vf = reinterpret_cast<T*>(base + L::vf);
  st.c = reinterpret_cast<T*>(base + L::c);
  st.ff = reinterpret_cast<T*>(base + L::ff);
  st.fcl = reinterpret_cast<T*>(base + L::fcl);
  st.ic = reinterpret_cast<T*>(base + L::ic);
  return st;
}

template <class T, bool SAMPLE>
__global__ void __launch_bounds__(Tile<T>::NT, Tile<T>::MINB) mc_fill_kernel(const McArgs<T> A,
                                                                            const __grid_constant__ ColumnMaps maps) {
  using TL = Tile<T>;
  using L = Layout<T>;
  constexpr int TX = TL::TX, TY = TL::TY, NT = TL::NT, NSX = TL::NSX, NSLAB = TL::NSLAB;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x;
  const long long n0 = A.g.n[0], n1 = A.g.n[1], n2 = A.g.n[2];
  const long long nx = n0 + 1, ny = n1 + 1;

  int b = blockIdx.x;
  const int it = b % A.n_itiles; b /= A.n_itiles;
  const int jt = b % A.n_jtiles; b /= A.n_jtiles;
  const long long i0 = (long long)it * TX, j0 = (long long)jt * TY;
  const long long k0 = (long long)b * KZ;
  const long long k1 = (k0 + KZ < n2) ? k0 + KZ : n2;

  STape<T> tape;
  if (SAMPLE) tape = load_tape<T>(A.tape.bytes, A.tape.n_ops, A.tape.n_params, smem + L::tape);
  T* const ring = reinterpret_cast<T*>(smem + L::slab0);
  constexpr int RS = L::slab_bytes / int(sizeof(T));  // ring slot stride, elements
  if (SAMPLE) __syncthreads();

  const T x0 = A.g.x0[0], y0 = A.g.x0[1], z0 = A.g.x0[2];
  const T dx = A.g.d[0], dy = A.g.d[1], dz = A.g.d[2];
  const long long nxy = nx * ny;

  // This thread's node slots for one sampling round of NS slabs, fixed for the whole march:
  // which of the round's slabs, the slab index, coordinates, the node index in the z = 0 plane,
  // and whether this CTA owns (writes) the node.
  constexpr int NSL = (NS * NSLAB + NT - 1) / NT;
  int sl_s[NSL], sl_v[NSL];
  T sl_x[NSL], sl_y[NSL];
  long long sl_g[NSL];
  bool sl_ok[NSL], sl_own[NSL];
#pragma unroll
  for (int q = 0; q < NSL; ++q) {
    const int flat = tid + q * NT;
    const int s = flat / NSLAB, v = flat - s * NSLAB;
    const int tx = v % NSX, ty = v / NSX;
    const long long i = i0 + tx, j = j0 + ty;
    sl_s[q] = s;
    sl_v[q] = v;
    sl_ok[q] = s < NS && i <= n0 && j <= n1;
    sl_own[q] = (tx < TX || i == n0) && (ty < TY || j == n1);
    sl_x[q] = node_coord(x0, dx, i);
    sl_y[q] = node_coord(y0, dy, j);
    sl_g[q] = i + nx * j;
  }

  // One round: slabs zbase, zbase+1, ... (slot s samples slab zbase + s, for slabs <= zlast),
  // into ring slot z % (NS + 1); phi written for owned nodes of owned slabs. `first` samples
  // only slab zbase (the first slab of the march).
  auto sample_round = [&](long long zbase, long long zlast, bool first) {
    T pts[NSL][3];
    T val[NSL];
    bool use[NSL];
#pragma unroll
    for (int q = 0; q < NSL; ++q) {
      const long long z = zbase + sl_s[q];
      use[q] = sl_ok[q] && z <= zlast && (!first || sl_s[q] == 0);
      pts[q][0] = sl_x[q];
      pts[q][1] = sl_y[q];
      pts[q][2] = node_coord(z0, dz, (long long)(int)z);
    }
    if (SAMPLE) {
      tape_eval_multi<T, 3, NSL>(tape, pts, val);
    }
#pragma unroll
    for (int q = 0; q < NSL; ++q) {
      if (!use[q]) continue;
      const long long z = zbase + sl_s[q];
      const long long gi = sl_g[q] + nxy * z;
      T v;
      if (SAMPLE) {
        v = val[q];
        const bool own_slab = z < k1 || z == n2;
        if (own_slab && sl_own[q]) A.phi_out[gi] = v;
      } else {
        v = A.phi_in[gi];
      }
      ring[(int)(z - k0) % (NS + 1) * RS + sl_v[q]] = v;
    }
  };

  sample_round(k0, k0, true);

  const int tx = tid % TX, ty = tid / TX;
  const long long ci = i0 + tx, cj = j0 + ty;
  const bool valid = ci < n0 && cj < n1;
  const T xa = node_coord(x0, dx, ci), xb = node_coord(x0, dx, ci + 1);
  const T ya = node_coord(y0, dy, cj), yb = node_coord(y0, dy, cj + 1);
  const T hx = T(0.5) * (xb - xa), hy = T(0.5) * (yb - ya);
  const T cx = xa + T(0.5) * dx, cy = ya + T(0.5) * dy;
  const int lc = ty * TX + tx;
  const int s00 = ty * NSX + tx;
  const bool fast = A.use_tma != 0;
  const int rows = (int)((n1 - j0) < TY ? (n1 - j0) : TY);
  const int cnt = (int)((n0 - i0) < TX ? (n0 - i0) : TX);
  unsigned char* gcol[7] = {reinterpret_cast<unsigned char*>(A.cols.kind), A.cols.amb,
                            reinterpret_cast<unsigned char*>(A.cols.vf), reinterpret_cast<unsigned char*>(A.cols.c),
                            reinterpret_cast<unsigned char*>(A.cols.ff), reinterpret_cast<unsigned char*>(A.cols.fcl),
                            reinterpret_cast<unsigned char*>(A.cols.ic)};

  for (long long k = k0; k < k1; ++k) {
    const int sb = (int)((k - k0) & 1);
    unsigned char* sbase = smem + sb * L::stage_bytes;
    if (((k - k0) % NS) == 0) sample_round(k + 1, k1, false);
    if (fast && tid == 0) bulk_wait_read<1>();  // staging buffer sb: its copy two slices ago has been read
    __syncthreads();  // slabs k and k+1 ready; staging sb free

    const T za = node_coord(z0, dz, (long long)(int)k), zb = node_coord(z0, dz, (long long)(int)(k + 1));
    bool is_cut = false;
    if (valid) {
      const int rk = (int)(k - k0) % (NS + 1);
      const T* sa = ring + rk * RS;
      const T* sbb = ring + (rk == NS ? 0 : rk + 1) * RS;
      const T ph[8] = {sa[s00], sa[s00 + 1], sa[s00 + NSX + 1], sa[s00 + NSX],
                       sbb[s00], sbb[s00 + 1], sbb[s00 + NSX + 1], sbb[s00 + NSX]};
      // nudge_zeros(v) >= 0  <=>  v > -eps  (and false for NaN, as there)
      const T neps = -Eps<T>::v();
      int nout = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) nout += ph[q] > neps ? 1 : 0;
      if (nout == 0 || nout == 8) {
        const T hz = T(0.5) * (zb - za);
        const T one = nout == 8 ? T(1) : T(0);
        const T cen[3] = {cx, cy, za + T(0.5) * dz};
        const T ff[6] = {one, one, one, one, one, one};
        const T fcl[12] = {hy, hz, hy, hz, hx, hz, hx, hz, hx, hy, hx, hy};
        put_cell<T>(stage_at<T>(sbase), lc, nout == 8 ? 1 : 0, 0, one, cen, ff, fcl, cen);
      } else {
        is_cut = true;
      }
    }
    // Warp-ballot compaction of the cut band into the global work list. A cut cell's staged slot
    // is left as it is: the span is copied out whole and the cut kernel, which runs after this
    // one in stream order, overwrites the cell.
    const unsigned m = __ballot_sync(0xffffffffu, is_cut);
    if (m) {
      const int lane = tid & 31;
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(A.cut_count, (unsigned)__popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (is_cut) A.cut_list[base + __popc(m & ((1u << lane) - 1))] = (unsigned)(ci + n0 * (cj + n1 * k));
    }
    if (fast) fence_proxy_async_smem();  // staged writes visible to the bulk-copy engine
    __syncthreads();  // staging sb complete

    const long long row0 = i0 + n0 * (j0 + n1 * k);
    if (fast) {
      // one thread stores the staged tile: one TMA box per column (the hardware clips the box
      // at the grid's edge)
      if (tid == 0) {
        const int ci0 = (int)i0, cj0 = (int)j0, ck = (int)k;
        tma_store3(&maps.m[0], sbase + col_offset<T>(0), ci0, cj0, ck);
        tma_store3(&maps.m[1], sbase + col_offset<T>(1), ci0, cj0, ck);
        tma_store3(&maps.m[2], sbase + col_offset<T>(2), ci0, cj0, ck);
        tma_store3(&maps.m[3], sbase + col_offset<T>(3), 3 * ci0, cj0, ck);
        tma_store3(&maps.m[4], sbase + col_offset<T>(4), 6 * ci0, cj0, ck);
        tma_store4(&maps.m[5], sbase + col_offset<T>(5), 0, ci0, cj0, ck);
        tma_store3(&maps.m[6], sbase + col_offset<T>(6), 3 * ci0, cj0, ck);
        bulk_commit();
      }
    } else {
      for (int r = 0; r < rows; ++r) {
        const long long rowc = row0 + (long long)r * n0;
#pragma unroll
        for (int col = 0; col < 7; ++col) {
          const int es = col_elem(col, int(sizeof(T)));
          const unsigned char* src = sbase + col_offset<T>(col) + r * col_bytes<T>(col);
          unsigned char* dst = gcol[col] + rowc * es;
          if (col >= 2) {
            const T* s2 = reinterpret_cast<const T*>(src);
            T* d2 = reinterpret_cast<T*>(dst);
            const int ne = cnt * es / int(sizeof(T));
            for (int v = tid; v < ne; v += NT) d2[v] = s2[v];
          } else {
            for (int v = tid; v < cnt; v += NT) dst[v] = src[v];
          }
        }
      }
    }
  }
  if (fast && tid == 0) bulk_wait<0>();  // all tensor stores complete before the CTA retires
}

template <class T, bool SAMPLE>
__global__ void __launch_bounds__(CUT_NT) mc_cut_kernel(const McArgs<T> A) {
  const long long n0 = A.g.n[0], n1 = A.g.n[1];
  const long long nx = n0 + 1, ny = n1 + 1;
  const T* phi = SAMPLE ? A.phi_out : A.phi_in;
  Stage<T> st;
  st.kind = A.cols.kind;
  st.amb = A.cols.amb;
  st.vf = static_cast<T*>(A.cols.vf);
  st.c = static_cast<T*>(A.cols.c);
  st.ff = static_cast<T*>(A.cols.ff);
  st.fcl = static_cast<T*>(A.cols.fcl);
  st.ic = static_cast<T*>(A.cols.ic);
  const T cs[3] = {A.g.d[0], A.g.d[1], A.g.d[2]};
  const unsigned total = *A.cut_count;
  for (unsigned q = blockIdx.x * CUT_NT + threadIdx.x; q < total; q += gridDim.x * CUT_NT) {
    const long long ci = A.cut_list[q];
    const long long i = ci % n0, j = (ci / n0) % n1, k = ci / (n0 * n1);
    const long long b0 = i + nx * (j + ny * k);
    const long long bz = nx * ny;
    const T ph[8] = {phi[b0], phi[b0 + 1], phi[b0 + nx + 1], phi[b0 + nx],
                     phi[b0 + bz], phi[b0 + bz + 1], phi[b0 + bz + nx + 1], phi[b0 + bz + nx]};
    const T org[3] = {node_coord(A.g.x0[0], A.g.d[0], i), node_coord(A.g.x0[1], A.g.d[1], j),
                      node_coord(A.g.x0[2], A.g.d[2], k)};
    const T l[3] = {node_coord(A.g.x0[0], A.g.d[0], i + 1) - org[0], node_coord(A.g.x0[1], A.g.d[1], j + 1) - org[1],
                    node_coord(A.g.x0[2], A.g.d[2], k + 1) - org[2]};
    mc_cut_cell<T>(ph, l, org, cs, A.tb, st, ci);
  }
}

template <class T>
constexpr int smem_bytes(int tape_bytes) {
  return Layout<T>::tape + ((tape_bytes + 15) / 16) * 16;
}

}  // namespace

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// The seven column maps of a marching-cubes cache, or false where TMA cannot address the columns
// (a row of the kind column is not a multiple of 16 bytes, a base not 16-byte aligned, or a
// dimension past 2^31); the fill kernel then stores with its threads.
template <class T>
bool make_column_maps(const DevGrid<T>& g, const Cols& cols, ColumnMaps* maps) {
  using TL = Tile<T>;
  const long long n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  if (n0 % 16 != 0 || 12 * n0 >= 0x7fffffffLL || n1 >= 0x7fffffffLL || n2 >= 0x7fffffffLL) return false;
  void* base[7] = {cols.kind, cols.amb, cols.vf, cols.c, cols.ff, cols.fcl, cols.ic};
  for (void* b : base)
    if (reinterpret_cast<uintptr_t>(b) & 15u) return false;
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  const CUtensorMapDataType tt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint64_t es = sizeof(T);
  const int width[7] = {1, 1, 1, 3, 6, 12, 3};
  for (int c = 0; c < 7; ++c) {
    const CUtensorMapDataType dt = c < 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : tt;
    const cuuint64_t e = c < 2 ? 1 : es;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r;
    if (c == 5) {
      const cuuint64_t dims[4] = {12, (cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
      const cuuint64_t strides[3] = {12 * e, 12 * e * n0, 12 * e * n0 * n1};
      const cuuint32_t box[4] = {12, (cuuint32_t)TL::TX, (cuuint32_t)TL::TY, 1};
      r = enc(&maps->m[c], dt, 4, base[c], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
      const cuuint64_t w = width[c];
      const cuuint64_t dims[3] = {w * n0, (cuuint64_t)n1, (cuuint64_t)n2};
      const cuuint64_t strides[2] = {w * e * n0, w * e * n0 * n1};
      const cuuint32_t box[3] = {(cuuint32_t)(w * TL::TX), (cuuint32_t)TL::TY, 1};
      r = enc(&maps->m[c], dt, 3, base[c], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

}  // namespace

namespace cci {

template <class T>
cudaError_t launch_mc(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, const DevTable& tb, unsigned* cut_list, unsigned* cut_count,
                      cudaStream_t s) {
  using TL = Tile<T>;
  McArgs<T> a;
  a.g = g;
  a.tape = tape;
  a.phi_in = phi_in;
  a.phi_out = phi_out;
  a.cols = cols;
  a.tb = tb;
  a.cut_list = cut_list;
  a.cut_count = cut_count;
  ColumnMaps maps;
  std::memset(&maps, 0, sizeof maps);
  a.use_tma = make_column_maps<T>(g, cols, &maps) ? 1 : 0;
  a.n_itiles = int((g.n[0] + TL::TX - 1) / TL::TX);
  a.n_jtiles = int((g.n[1] + TL::TY - 1) / TL::TY);
  const long long nk = (g.n[2] + KZ - 1) / KZ;
  const long long blocks = (long long)a.n_itiles * a.n_jtiles * nk;
  if (blocks <= 0 || blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaMemsetAsync(cut_count, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  const bool sample = phi_in == nullptr;
  const int sm = smem_bytes<T>(sample ? tape.bytes_len : 0);
  const int cut_blocks = 148 * 8;
  if (sample) {
    e = cudaFuncSetAttribute(mc_fill_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    mc_fill_kernel<T, true><<<unsigned(blocks), TL::NT, sm, s>>>(a, maps);
    mc_cut_kernel<T, true><<<cut_blocks, CUT_NT, 0, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(mc_fill_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    mc_fill_kernel<T, false><<<unsigned(blocks), TL::NT, sm, s>>>(a, maps);
    mc_cut_kernel<T, false><<<cut_blocks, CUT_NT, 0, s>>>(a);
  }
  return cudaGetLastError();
}

template cudaError_t launch_mc<float>(const DevGrid<float>&, const DevTape&, const float*, float*,
                                      const Cols&, const DevTable&, unsigned*, unsigned*, cudaStream_t);
template cudaError_t launch_mc<double>(const DevGrid<double>&, const DevTape&, const double*, double*,
                                       const Cols&, const DevTable&, unsigned*, unsigned*, cudaStream_t);

}  // namespace cci
