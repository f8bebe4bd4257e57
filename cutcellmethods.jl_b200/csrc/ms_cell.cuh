// ms_cell.cuh -- the per-cell marching-squares construction, shared by the grid, tree and
// batched kernels: cut_cell_moments (2D), src/marching_squares/moments.jl:66-164, with
// cell_boundary_walk (src/marching_squares/marching_squares.jl:240-251) and cell_gap_segments
// (:291-317).
#pragma once
#include <cstdint>
#include "cc_device.cuh"
#include "cc_internal.h"

namespace ccms {

using namespace ccd;
using cci::Cols;

// MS_DIRECTION_EDGE (0-based), src/marching_squares/marching_squares.jl:81-82
__host__ __device__ constexpr int dir_edge(int dir) { return dir == 0 ? 3 : dir == 1 ? 1 : dir == 2 ? 0 : 2; }

// cut_cell_moments (2D), src/marching_squares/moments.jl:66-164, from global corner
// coordinates `nd` (MS_NODE_BITS order) and corner values `ph`; writes cell `ci`'s columns.
// One cell's fields into the columns. Where the four wide columns are 16-byte aligned (every
// caller's allocation here), a cell's centroid and interface centroid leave as one 2-vector each
// and its face fractions and face centroids as 16-byte vectors, so a warp's store covers whole
// sectors; otherwise element by element.
template <class T>
__device__ __forceinline__ void store_cell2(const Cols& cols, long long ci, int kind, int amb, T vf, T c0, T c1,
                                            const T ff[4], const T fcl[4], T i0, T i1) {
  cols.kind[ci] = int8_t(kind);
  cols.amb[ci] = uint8_t(amb);
  static_cast<T*>(cols.vf)[ci] = vf;
  T* c = static_cast<T*>(cols.c);
  T* f = static_cast<T*>(cols.ff);
  T* l = static_cast<T*>(cols.fcl);
  T* ic = static_cast<T*>(cols.ic);
  const bool vec = ((reinterpret_cast<uintptr_t>(c) | reinterpret_cast<uintptr_t>(f) | reinterpret_cast<uintptr_t>(l) |
                     reinterpret_cast<uintptr_t>(ic)) & 15u) == 0;
  if (vec) {
    if (sizeof(T) == 4) {
      reinterpret_cast<float2*>(c)[ci] = make_float2(float(c0), float(c1));
      reinterpret_cast<float2*>(ic)[ci] = make_float2(float(i0), float(i1));
      reinterpret_cast<float4*>(f)[ci] = make_float4(float(ff[0]), float(ff[1]), float(ff[2]), float(ff[3]));
      reinterpret_cast<float4*>(l)[ci] = make_float4(float(fcl[0]), float(fcl[1]), float(fcl[2]), float(fcl[3]));
    } else {
      reinterpret_cast<double2*>(c)[ci] = make_double2(double(c0), double(c1));
      reinterpret_cast<double2*>(ic)[ci] = make_double2(double(i0), double(i1));
      reinterpret_cast<double2*>(f)[2 * ci] = make_double2(double(ff[0]), double(ff[1]));
      reinterpret_cast<double2*>(f)[2 * ci + 1] = make_double2(double(ff[2]), double(ff[3]));
      reinterpret_cast<double2*>(l)[2 * ci] = make_double2(double(fcl[0]), double(fcl[1]));
      reinterpret_cast<double2*>(l)[2 * ci + 1] = make_double2(double(fcl[2]), double(fcl[3]));
    }
    return;
  }
  c[2 * ci] = c0; c[2 * ci + 1] = c1;
#pragma unroll
  for (int dir = 0; dir < 4; ++dir) { f[4 * ci + dir] = ff[dir]; l[4 * ci + dir] = fcl[dir]; }
  ic[2 * ci] = i0; ic[2 * ci + 1] = i1;
}

template <class T, bool MX>
__device__ void ms_cell(const T nd[4][2], const T ph[4], const T cs[2], const Cols& cols, long long ci) {
  const T o0 = nd[0][0], o1 = nd[0][1];
  const T ce0 = o0 + T(0.5) * cs[0], ce1 = o1 + T(0.5) * cs[1];
  const T vol_cell = cs[0] * cs[1];
  int nout = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) nout += ph[k] >= T(0) ? 1 : 0;
  T fc[4], ffv[4];
  if (nout == 4 || nout == 0) {
    const bool out = nout == 4;
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      const int k = dir_edge(dir), k1 = (k + 1) & 3;
      const int p = dir < 2 ? 1 : 0;
      fc[dir] = T(0.5) * (nd[k][p] + nd[k1][p]) - nd[0][p];
      ffv[dir] = out ? T(1) : T(0);
    }
    store_cell2<T>(cols, ci, out ? 1 : 0, 0, out ? T(1) : T(0), ce0, ce1, ffv, fc, ce0, ce1);
    return;
  }
  // cell_boundary_walk, marching_squares.jl:240-251
  T fr[4], sa[4][2], sb[4][2];
  bool pr[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int k1 = (k + 1) & 3;
    const T fa = ph[k], fb = ph[k1];
    fr[k] = open_fraction<T, MX>(fa, fb);
    pr[k] = fa >= T(0) || fb >= T(0);
    if (fa >= T(0) && fb >= T(0)) {
      sa[k][0] = nd[k][0]; sa[k][1] = nd[k][1]; sb[k][0] = nd[k1][0]; sb[k][1] = nd[k1][1];
    } else if (fa >= T(0)) {
      sa[k][0] = nd[k][0]; sa[k][1] = nd[k][1];
      sb[k][0] = nd[k][0] + fr[k] * (nd[k1][0] - nd[k][0]);
      sb[k][1] = nd[k][1] + fr[k] * (nd[k1][1] - nd[k][1]);
    } else {
      sa[k][0] = nd[k1][0] + fr[k] * (nd[k][0] - nd[k1][0]);
      sa[k][1] = nd[k1][1] + fr[k] * (nd[k][1] - nd[k1][1]);
      sb[k][0] = nd[k1][0]; sb[k][1] = nd[k1][1];
    }
  }
#pragma unroll
  for (int dir = 0; dir < 4; ++dir) {
    const int k = dir_edge(dir), k1 = (k + 1) & 3;
    const int p = dir < 2 ? 1 : 0;
    const T x = pr[k] ? T(0.5) * (sa[k][p] + sb[k][p]) : T(0.5) * (nd[k][p] + nd[k1][p]);
    fc[dir] = x - nd[0][p];
    ffv[dir] = fr[k];
  }
  T area2 = T(0), m0 = T(0), m1 = T(0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!pr[k]) continue;
    const T la0 = sa[k][0] - o0, la1 = sa[k][1] - o1, lb0 = sb[k][0] - o0, lb1 = sb[k][1] - o1;
    const T cr = la0 * lb1 - la1 * lb0;
    area2 = area2 + cr;
    m0 = m0 + (la0 + lb0) * cr;
    m1 = m1 + (la1 + lb1) * cr;
  }
  // cell_gap_segments, marching_squares.jl:291-317 (with _next_present, :255-264)
  int nint = 0;
  T ilen = T(0), im0 = T(0), im1 = T(0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!pr[k]) continue;
    int j = (k + 1) & 3;
    if (!pr[j]) { j = (j + 1) & 3; if (!pr[j]) { j = (j + 1) & 3; if (!pr[j]) j = k; } }
    const T a0 = sb[k][0], a1 = sb[k][1];
    const T b0 = j == 0 ? sa[0][0] : j == 1 ? sa[1][0] : j == 2 ? sa[2][0] : sa[3][0];
    const T b1 = j == 0 ? sa[0][1] : j == 1 ? sa[1][1] : j == 2 ? sa[2][1] : sa[3][1];
    if (a0 != b0 || a1 != b1) {
      ++nint;
      if (nint <= 2) {
        const T la0 = a0 - o0, la1 = a1 - o1, lb0 = b0 - o0, lb1 = b1 - o1;
        const T cr = la0 * lb1 - la1 * lb0;
        area2 = area2 + cr;
        m0 = m0 + (la0 + lb0) * cr;
        m1 = m1 + (la1 + lb1) * cr;
        const T v0 = b0 - a0, v1 = b1 - a1;
        const T len = sqrt(v0 * v0 + v1 * v1);
        ilen = ilen + len;
        const T hl = T(0.5) * len;
        im0 = im0 + hl * (a0 + b0);
        im1 = im1 + hl * (a1 + b1);
      }
    }
  }
  const T area = T(0.5) * area2;
  T c0 = ce0, c1 = ce1, i0 = ce0, i1 = ce1;
  if (area2 != T(0)) {
    const T den = T(3) * area2;
    c0 = o0 + m0 / den;
    c1 = o1 + m1 / den;
  }
  if (ilen > T(0)) {
    i0 = im0 / ilen;
    i1 = im1 / ilen;
  }
  store_cell2<T>(cols, ci, 2, nint > 1 ? 1 : 0, area / vol_cell, c0, c1, ffv, fc, i0, i1);
}

// cell_interface (src/marching_squares/marching_squares.jl:343-351): the cell's n <= 2 contour
// segments, the s-th from a[s] to b[s], oriented out of the body -- the walk of
// cell_boundary_walk and the gaps of cell_gap_segments exactly as ms_cell builds them, endpoints
// swapped.
template <class T, bool MX>
__device__ __forceinline__ int ms_interface(const T nd[4][2], const T ph[4], T a[2][2], T b[2][2]) {
  T sa[4][2], sb[4][2];
  bool pr[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int k1 = (k + 1) & 3;
    const T fa = ph[k], fb = ph[k1];
    const T fr = open_fraction<T, MX>(fa, fb);
    pr[k] = fa >= T(0) || fb >= T(0);
    if (fa >= T(0) && fb >= T(0)) {
      sa[k][0] = nd[k][0]; sa[k][1] = nd[k][1]; sb[k][0] = nd[k1][0]; sb[k][1] = nd[k1][1];
    } else if (fa >= T(0)) {
      sa[k][0] = nd[k][0]; sa[k][1] = nd[k][1];
      sb[k][0] = nd[k][0] + fr * (nd[k1][0] - nd[k][0]);
      sb[k][1] = nd[k][1] + fr * (nd[k1][1] - nd[k][1]);
    } else {
      sa[k][0] = nd[k1][0] + fr * (nd[k][0] - nd[k1][0]);
      sa[k][1] = nd[k1][1] + fr * (nd[k][1] - nd[k1][1]);
      sb[k][0] = nd[k1][0]; sb[k][1] = nd[k1][1];
    }
  }
  int n = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!pr[k]) continue;
    int j = (k + 1) & 3;
    if (!pr[j]) { j = (j + 1) & 3; if (!pr[j]) { j = (j + 1) & 3; if (!pr[j]) j = k; } }
    const T a0 = sb[k][0], a1 = sb[k][1];
    const T b0 = j == 0 ? sa[0][0] : j == 1 ? sa[1][0] : j == 2 ? sa[2][0] : sa[3][0];
    const T b1 = j == 0 ? sa[0][1] : j == 1 ? sa[1][1] : j == 2 ? sa[2][1] : sa[3][1];
    if (a0 != b0 || a1 != b1) {
      if (n < 2) {  // the public orientation: from the gap's end to its start
        a[n][0] = b0; a[n][1] = b1;
        b[n][0] = a0; b[n][1] = a1;
      }
      ++n;
    }
  }
  return n < 2 ? n : 2;
}

}  // namespace ccms
