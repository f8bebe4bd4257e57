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
#include "ms_cell.cuh"

namespace {

using namespace ccd;
using namespace ccms;
using cci::Cols;
using cci::DevGrid;
using cci::DevTape;

constexpr int NT = 256;

// (i, j) of item v of an n0-wide box: a 32-bit quotient where the box has fewer than 2^32 items
// (every grid that fits a device), else 64-bit.
__device__ __forceinline__ void split2(long long v, long long n0, bool small, long long& i, long long& j) {
  if (small) {
    const unsigned q = unsigned(v) / unsigned(n0);
    j = q;
    i = (long long)(unsigned(v) - q * unsigned(n0));
  } else {
    j = v / n0;
    i = v - j * n0;
  }
}


template <class T>
__global__ void __launch_bounds__(NT) ms_sample_kernel(const DevGrid<T> g, const DevTape tape, T* phi) {
  extern __shared__ __align__(16) unsigned char smem[];
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1, total = nx * ny;
  const bool small = total + (long long)gridDim.x * NT < (1LL << 32);
  for (long long v = blockIdx.x * (long long)NT + threadIdx.x; v < total; v += (long long)gridDim.x * NT) {
    long long i, j;
    split2(v, nx, small, i, j);
    const T x[2] = {node_coord(g.x0[0], g.d[0], i), node_coord(g.x0[1], g.d[1], j)};
    phi[v] = tape_eval<T, 2, T>(t, x);
  }
}

template <class T, bool MX>
__global__ void __launch_bounds__(NT) ms_cells_kernel(const DevGrid<T> g, const T* __restrict__ phi, const Cols cols) {
  const long long n0 = g.n[0], n1 = g.n[1], nx = n0 + 1, total = n0 * n1;
  const T cs[2] = {g.d[0], g.d[1]};
  const bool small = total + (long long)gridDim.x * NT < (1LL << 32);
  for (long long ci = blockIdx.x * (long long)NT + threadIdx.x; ci < total; ci += (long long)gridDim.x * NT) {
    long long i, j;
    split2(ci, n0, small, i, j);
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
