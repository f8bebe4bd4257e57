// ms.cu -- MarchingSquaresCutCell update_cache! on sm_100a: a grid (nodal phi block) and the
// leaves of an AdaptiveMesh{2} quadtree.
//
// Grid: one pass samples every node from the op-tape (the reference's _sample_nodes_kernel!,
// src/marching_squares/cache.jl:67-70), a second builds every cell from its four corners
// (_nodal_cells_kernel!, :75-78). Tree: one thread per leaf samples its four lattice corners and
// builds its moments from exactly those (_leaf_cells_kernel!, :129-137).
#include <cstdint>
#include "cc_device.cuh"
#include "cc_internal.h"

namespace {

using namespace ccd;
using cci::Cols;
using cci::DevGrid;
using cci::DevTape;

constexpr int NT = 256;

// MS_DIRECTION_EDGE (0-based), src/marching_squares/marching_squares.jl:81-82
__host__ __device__ constexpr int dir_edge(int dir) { return dir == 0 ? 3 : dir == 1 ? 1 : dir == 2 ? 0 : 2; }

// cut_cell_moments (2D), src/marching_squares/moments.jl:66-164, from global corner
// coordinates `nd` (MS_NODE_BITS order) and corner values `ph`; writes cell `ci`'s columns.
template <class T, bool MX>
__device__ void ms_cell(const T nd[4][2], const T ph[4], const T cs[2], const Cols& cols, long long ci) {
  const T o0 = nd[0][0], o1 = nd[0][1];
  const T ce0 = o0 + T(0.5) * cs[0], ce1 = o1 + T(0.5) * cs[1];
  const T vol_cell = cs[0] * cs[1];
  int nout = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) nout += ph[k] >= T(0) ? 1 : 0;
  T* vf = static_cast<T*>(cols.vf);
  T* c = static_cast<T*>(cols.c);
  T* ff = static_cast<T*>(cols.ff);
  T* fcl = static_cast<T*>(cols.fcl);
  T* ic = static_cast<T*>(cols.ic);
  T fc[4];
  if (nout == 4 || nout == 0) {
    const bool out = nout == 4;
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
      const int k = dir_edge(dir), k1 = (k + 1) & 3;
      const int p = dir < 2 ? 1 : 0;
      fc[dir] = T(0.5) * (nd[k][p] + nd[k1][p]) - nd[0][p];
    }
    cols.kind[ci] = out ? 1 : 0;
    cols.amb[ci] = 0;
    vf[ci] = out ? T(1) : T(0);
    c[2 * ci] = ce0; c[2 * ci + 1] = ce1;
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) { ff[4 * ci + dir] = out ? T(1) : T(0); fcl[4 * ci + dir] = fc[dir]; }
    ic[2 * ci] = ce0; ic[2 * ci + 1] = ce1;
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
    ff[4 * ci + dir] = fr[k];
    fcl[4 * ci + dir] = fc[dir];
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
  cols.kind[ci] = 2;
  cols.amb[ci] = nint > 1 ? 1 : 0;
  vf[ci] = area / vol_cell;
  if (area2 != T(0)) {
    const T den = T(3) * area2;
    c[2 * ci] = o0 + m0 / den; c[2 * ci + 1] = o1 + m1 / den;
  } else {
    c[2 * ci] = ce0; c[2 * ci + 1] = ce1;
  }
  if (ilen > T(0)) { ic[2 * ci] = im0 / ilen; ic[2 * ci + 1] = im1 / ilen; }
  else { ic[2 * ci] = ce0; ic[2 * ci + 1] = ce1; }
}

template <class T>
__global__ void __launch_bounds__(NT) ms_sample_kernel(const DevGrid<T> g, const DevTape tape, T* phi) {
  extern __shared__ __align__(16) unsigned char smem[];
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1, total = nx * ny;
  for (long long v = blockIdx.x * (long long)NT + threadIdx.x; v < total; v += (long long)gridDim.x * NT) {
    const long long i = v % nx, j = v / nx;
    const T x[2] = {node_coord(g.x0[0], g.d[0], i), node_coord(g.x0[1], g.d[1], j)};
    phi[v] = tape_eval<T, 2, T>(t, x);
  }
}

template <class T, bool MX>
__global__ void __launch_bounds__(NT) ms_cells_kernel(const DevGrid<T> g, const T* __restrict__ phi, const Cols cols) {
  const long long n0 = g.n[0], n1 = g.n[1], nx = n0 + 1, total = n0 * n1;
  const T cs[2] = {g.d[0], g.d[1]};
  for (long long ci = blockIdx.x * (long long)NT + threadIdx.x; ci < total; ci += (long long)gridDim.x * NT) {
    const long long i = ci % n0, j = ci / n0;
    const T xa = node_coord(g.x0[0], g.d[0], i), xb = node_coord(g.x0[0], g.d[0], i + 1);
    const T ya = node_coord(g.x0[1], g.d[1], j), yb = node_coord(g.x0[1], g.d[1], j + 1);
    const T nd[4][2] = {{xa, ya}, {xb, ya}, {xb, yb}, {xa, yb}};
    const long long b = i + nx * j;
    const T ph[4] = {phi[b], phi[b + 1], phi[b + nx + 1], phi[b + nx]};
    ms_cell<T, MX>(nd, ph, cs, cols, ci);
  }
}

template <class T, bool MX>
__global__ void __launch_bounds__(NT) ms_tree_kernel(const T x00, const T x01, const double bd0, const double bd1,
                                                     long long nl, const int32_t* __restrict__ level,
                                                     const int32_t* __restrict__ coord, const DevTape tape, T* phi4,
                                                     const Cols cols) {
  extern __shared__ __align__(16) unsigned char smem[];
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < nl; i += (long long)gridDim.x * NT) {
    const int lv = level[i];
    const T scale = T(ldexp(1.0, -lv));
    const T h[2] = {T(bd0) * scale, T(bd1) * scale};
    const long long cx = coord[2 * i], cy = coord[2 * i + 1];
    const T xa = x00 + T(cx) * h[0], xb = x00 + T(cx + 1) * h[0];
    const T ya = x01 + T(cy) * h[1], yb = x01 + T(cy + 1) * h[1];
    const T nd[4][2] = {{xa, ya}, {xb, ya}, {xb, yb}, {xa, yb}};
    T ph[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ph[q] = tape_eval<T, 2, T>(t, nd[q]);
      phi4[4 * i + q] = ph[q];
    }
    ms_cell<T, MX>(nd, ph, h, cols, i);
  }
}

int grid_blocks(long long work) {
  long long b = (work + NT - 1) / NT;
  const long long cap = 148LL * 16;
  return int(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

namespace cci {

template <class T>
cudaError_t launch_ms(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, cudaStream_t s, bool mixed) {
  const T* phi = phi_in;
  if (!phi_in) {
    const int sm = ((tape.bytes_len + 15) / 16) * 16;
    ms_sample_kernel<T><<<grid_blocks((g.n[0] + 1) * (g.n[1] + 1)), NT, sm, s>>>(g, tape, phi_out);
    phi = phi_out;
  }
  if (mixed && sizeof(T) == 4) ms_cells_kernel<T, true><<<grid_blocks(g.n[0] * g.n[1]), NT, 0, s>>>(g, phi, cols);
  else ms_cells_kernel<T, false><<<grid_blocks(g.n[0] * g.n[1]), NT, 0, s>>>(g, phi, cols);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_ms_tree(const T x0[2], const double base_d[2], long long nleaves, const int32_t* level,
                           const int32_t* coord, const DevTape& tape, T* phi4, const Cols& cols, cudaStream_t s,
                           bool mixed) {
  if (nleaves <= 0) return cudaSuccess;
  const int sm = ((tape.bytes_len + 15) / 16) * 16;
  if (mixed && sizeof(T) == 4)
    ms_tree_kernel<T, true><<<grid_blocks(nleaves), NT, sm, s>>>(x0[0], x0[1], base_d[0], base_d[1], nleaves, level,
                                                                 coord, tape, phi4, cols);
  else
    ms_tree_kernel<T, false><<<grid_blocks(nleaves), NT, sm, s>>>(x0[0], x0[1], base_d[0], base_d[1], nleaves, level,
                                                                  coord, tape, phi4, cols);
  return cudaGetLastError();
}

template cudaError_t launch_ms<float>(const DevGrid<float>&, const DevTape&, const float*, float*, const Cols&, cudaStream_t,
                                      bool);
template cudaError_t launch_ms<double>(const DevGrid<double>&, const DevTape&, const double*, double*, const Cols&,
                                       cudaStream_t, bool);
template cudaError_t launch_ms_tree<float>(const float*, const double*, long long, const int32_t*, const int32_t*,
                                           const DevTape&, float*, const Cols&, cudaStream_t, bool);
template cudaError_t launch_ms_tree<double>(const double*, const double*, long long, const int32_t*, const int32_t*,
                                            const DevTape&, double*, const Cols&, cudaStream_t, bool);

}  // namespace cci
