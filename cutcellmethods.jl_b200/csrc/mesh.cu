// mesh.cu -- generate_mesh for a marching-cubes cache on the device
// (src/marching_cubes/surface.jl:82-112, where the reference marches cache.phi serially on the host).
//
// The surface is the one the cache's cut cells integrate: every cut cell's triangles are the
// tile its moments used (the same table, the same face and interior deciders), and a vertex on
// a grid edge is that edge's crossing as the cells place it, anchored on the outside node:
// x_out + s (x_in - x_out), s = phi_out / (phi_out - phi_in), nudged corner values. Every cell
// around an edge computes the same vertex, so the vertex is stored once and shared: the mesh is
// watertight and wound so each triangle's normal points out of the body. A tile's code 13 is
// the cell's interior vertex, the mean of its crossings.
//
// The numbering is deterministic: first the edge vertices, each owned by its edge's lower node,
// nodes in linear order (x fastest) and each node's x, y, z edges in that order; then the
// interior vertices, cells in linear order; triangles by cell in linear order, each cell's in
// tile order.
//
// Two passes, edge vertices (nodes) and cells. Each counts per block of 8192 items, the block
// counts are scanned, and an emit writes through in-block scans; both compact the thin band that
// contributes (nodes with a cut edge, cut cells) per block before the long work, so it runs on
// dense warps (compact.cuh). The count call keeps each block's survivors and the scanned offsets
// on the handle, and an emit call that follows it for the same phi and grid, with no update in
// between, starts from them. The edge pass keeps each surviving node's first vertex, so a cell's
// triangles can name the vertices of edges other nodes own. Every write of an emit is checked
// against the output capacities.
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"
#include "mc_cell.cuh"
#include "compact.cuh"

namespace {

using namespace ccd;
using namespace ccmc;
using cci::DevGrid;
using cci::DevTable;

constexpr int MB = 256;          // threads per block
constexpr int IPT = 32;          // rounds per block
constexpr int BLK = MB * IPT;    // nodes or cells per block
constexpr int KEEP = 1024;       // survivors a block hands from the count to the emit pass

template <class T>
__device__ __forceinline__ bool outside(T v) { return nudge(v) >= T(0); }

// Bit a set: node (i,j,k)'s edge to the next node along axis a crosses the surface.
template <class T>
__device__ __forceinline__ unsigned node_edges(const T* __restrict__ phi, long long i, long long j, long long k,
                                               const long long n[3]) {
  const long long nx = n[0] + 1, ny = n[1] + 1;
  const long long v = i + nx * (j + ny * k);
  const bool o = outside(phi[v]);
  unsigned m = 0;
  if (i < n[0] && outside(phi[v + 1]) != o) m |= 1u;
  if (j < n[1] && outside(phi[v + nx]) != o) m |= 2u;
  if (k < n[2] && outside(phi[v + nx * ny]) != o) m |= 4u;
  return m;
}

// The crossing on node v's edge along axis a (world coordinates), as the cells place it.
template <class T>
__device__ __forceinline__ void edge_vertex(const T* __restrict__ phi, const DevGrid<T>& g, long long i, long long j,
                                            long long k, int a, T out[3]) {
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1;
  const long long v = i + nx * (j + ny * k);
  const long long w = v + (a == 0 ? 1 : a == 1 ? nx : nx * ny);
  const T fa = nudge(phi[v]), fb = nudge(phi[w]);
  const long long idx[3] = {i, j, k};
  T xa[3], xb[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    xa[q] = node_coord(g.x0[q], g.d[q], idx[q]);
    xb[q] = node_coord(g.x0[q], g.d[q], idx[q] + (q == a ? 1 : 0));
  }
  const T s = open_fraction(fa, fb);
#pragma unroll
  for (int q = 0; q < 3; ++q) out[q] = fa >= T(0) ? xa[q] + s * (xb[q] - xa[q]) : xb[q] + s * (xa[q] - xb[q]);
}

// Walks item coordinates (i, j, k) over an n0 x n1 x * box from item `start + threadIdx.x` in steps
// of MB (one 64-bit division at the start), carrying the item's node index b = i + sx j + sz k
// (for the node box, b is the item itself; for the cell box, the cell's lower corner). Indices
// are 32-bit: a mesh grid has fewer than 2^32 nodes. The steps are arithmetic only, so the loads
// they address do not wait on one another.
struct Walker {
  unsigned v, b;
  int i, j, k;
  const int n0, n1;
  const unsigned sx, sz;
  __device__ Walker(long long start, long long n0_, long long n1_, long long sx_, long long sz_)
      : n0(int(n0_)), n1(int(n1_)), sx(unsigned(sx_)), sz(unsigned(sz_)) {
    const long long v64 = start + threadIdx.x;
    v = unsigned(v64);
    i = int(v64 % n0_);
    j = int((v64 / n0_) % n1_);
    k = int(v64 / (n0_ * n1_));
    b = unsigned(i) + sx * unsigned(j) + sz * unsigned(k);
  }
  __device__ __forceinline__ void step() {
    v += MB;
    i += MB;
    b += MB;
    while (i >= n0) {
      i -= n0;
      b += sx - unsigned(n0);
      if (++j == n1) {
        j = 0;
        ++k;
        b += sz - sx * unsigned(n1);
      }
    }
  }
};

// outside(v) without the nudge: |v| < eps reads as +eps, so v is outside exactly when v > -eps
// (a NaN is neither).
template <class T>
__device__ __forceinline__ bool out_fast(T v) { return v > -Eps<T>::v(); }

// The cheap tests, in groups of G rounds: each round's item is clamped to the box's last item
// (past it the round answers false), and every load of the group is issued before any is tested.
// A node has a cut edge when a neighbour along +x, +y or +z (inside the box) lies on the other side;
// a cell is cut when its corners are not all on one side.
template <class T, int G>
__device__ __forceinline__ unsigned nodes_with_cut(const T* __restrict__ phi, Walker& w, unsigned nn, int m0, int m1,
                                                   int m2, unsigned nx, unsigned nz, bool full) {
  T p0[G], px[G], py[G], pz[G];
  bool in[G];
#pragma unroll
  for (int u = 0; u < G; ++u) {
    in[u] = full || w.v < nn;
    const T* p = phi + (in[u] ? w.b : nn - 1);
    p0[u] = p[0];
    px[u] = p[in[u] && w.i < m0 ? 1u : 0u];
    py[u] = p[in[u] && w.j < m1 ? nx : 0u];
    pz[u] = p[in[u] && w.k < m2 ? nz : 0u];
    w.step();
  }
  unsigned m = 0;
#pragma unroll
  for (int u = 0; u < G; ++u) {
    const bool o = out_fast(p0[u]);
    const bool cut = (out_fast(px[u]) != o) | (out_fast(py[u]) != o) | (out_fast(pz[u]) != o);
    if (in[u] & cut) m |= 1u << u;
  }
  return m;
}

template <class T, int G>
__device__ __forceinline__ unsigned cells_with_cut(const T* __restrict__ phi, Walker& w, unsigned nc, unsigned nx,
                                                   unsigned nz, bool full) {
  T c[G][8];
  bool in[G];
#pragma unroll
  for (int u = 0; u < G; ++u) {
    in[u] = full || w.v < nc;
    const T* p = phi + (in[u] ? w.b : 0u);
    c[u][0] = p[0]; c[u][1] = p[1]; c[u][2] = p[nx]; c[u][3] = p[nx + 1];
    c[u][4] = p[nz]; c[u][5] = p[nz + 1]; c[u][6] = p[nz + nx]; c[u][7] = p[nz + nx + 1];
    w.step();
  }
  unsigned m = 0;
#pragma unroll
  for (int u = 0; u < G; ++u) {
    const bool o = out_fast(c[u][0]);
    bool cut = false;
#pragma unroll
    for (int q = 1; q < 8; ++q) cut |= out_fast(c[u][q]) != o;
    if (in[u] & cut) m |= 1u << u;
  }
  return m;
}

template <class T> struct Groups { static constexpr int node = 8, cell = 4; };
template <> struct Groups<double> { static constexpr int node = 4, cell = 2; };

// This block's survivors: from the count pass (kept_n >= 0) or compacted again (kept_n < 0,
// more than KEEP). Returns their number (block-uniform).
template <int G, class Keep>
__device__ __forceinline__ int survivors(int* cand, const int* kept, const int* kept_n, Keep keep) {
  int n = kept_n[blockIdx.x];
  if (n == 0) return 0;
  if (n > 0) {
    for (int x = threadIdx.x; x < n; x += MB) cand[x] = kept[(size_t)blockIdx.x * KEEP + x];
    __syncthreads();
    return n;
  }
  return cccompact::compact<MB, IPT, G>(cand, keep);
}

__device__ __forceinline__ void keep_survivors(const int* cand, int n, int* kept, int* kept_n) {
  if (threadIdx.x == 0) kept_n[blockIdx.x] = n <= KEEP ? n : -1;
  if (n <= KEEP)
    for (int x = threadIdx.x; x < n; x += MB) kept[(size_t)blockIdx.x * KEEP + x] = cand[x];
}

// ---- the edge vertices ----------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(MB, 4) node_count_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                           unsigned long long* bsum, int* kept, int* kept_n) {
  __shared__ int cand[BLK];
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1, nn = nx * ny * (g.n[2] + 1);
  const long long start = (long long)blockIdx.x * BLK;
  Walker w(start, nx, ny, nx, nx * ny);
  const bool full = start + BLK <= nn;  // block-uniform: no item past the grid
  const int n = cccompact::compact<MB, IPT, Groups<T>::node>(cand, [&](int) {
    return nodes_with_cut<T, Groups<T>::node>(phi, w, unsigned(nn), int(g.n[0]), int(g.n[1]), int(g.n[2]),
                                              unsigned(nx), unsigned(nx * ny), full);
  });
  keep_survivors(cand, n, kept, kept_n);
  unsigned long long c = 0;
  for (int x = threadIdx.x; x < n; x += MB) {
    const long long v = start + cand[x];
    c += __popc(node_edges(phi, v % nx, (v / nx) % ny, v / (nx * ny), g.n));
  }
  unsigned long long total;
  cccompact::block_scan<MB>(c, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

template <class T>
__global__ void __launch_bounds__(MB, 4) node_emit_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                          const unsigned long long* __restrict__ boff,
                                                          const int* kept, const int* kept_n, unsigned* __restrict__ vbase,
                                                          T* __restrict__ verts, unsigned long long vcap,
                                                          unsigned long long* overflow) {
  __shared__ int cand[BLK];
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1, nn = nx * ny * (g.n[2] + 1);
  const long long start = (long long)blockIdx.x * BLK;
  Walker w(start, nx, ny, nx, nx * ny);
  const bool full = start + BLK <= nn;  // block-uniform: no item past the grid
  const int n = survivors<Groups<T>::node>(cand, kept, kept_n, [&](int) {
    return nodes_with_cut<T, Groups<T>::node>(phi, w, unsigned(nn), int(g.n[0]), int(g.n[1]), int(g.n[2]),
                                              unsigned(nx), unsigned(nx * ny), full);
  });
  unsigned long long run = boff[blockIdx.x];
  for (int c0 = 0; c0 < n; c0 += MB) {  // block-uniform
    const int x = c0 + threadIdx.x;
    const long long v = x < n ? start + cand[x] : 0;
    const long long i = v % nx, j = (v / nx) % ny, k = v / (nx * ny);
    const unsigned m = x < n ? node_edges(phi, i, j, k, g.n) : 0u;
    unsigned long long total;
    unsigned long long id = run + cccompact::block_scan<MB>((unsigned long long)__popc(m), &total);
    run += total;
    if (x >= n) continue;
    if (id + __popc(m) > vcap) {
      atomicOr(overflow, 1ull);
      continue;
    }
    vbase[v] = unsigned(id);
    for (int a = 0; a < 3; ++a) {
      if (!(m >> a & 1u)) continue;
      T p[3];
      edge_vertex(phi, g, i, j, k, a, p);
      verts[3 * id] = p[0]; verts[3 * id + 1] = p[1]; verts[3 * id + 2] = p[2];
      ++id;
    }
  }
}

// ---- the cells: triangles and interior vertices ----------------------------------------------
template <class T>
__device__ __forceinline__ void corners(const T* __restrict__ phi, const long long n[3], long long i, long long j,
                                        long long k, T ph[8]) {
  const long long nx = n[0] + 1, ny = n[1] + 1;
  const long long b0 = i + nx * (j + ny * k), bz = nx * ny;
  const T r[8] = {phi[b0], phi[b0 + 1], phi[b0 + nx + 1], phi[b0 + nx],
                  phi[b0 + bz], phi[b0 + bz + 1], phi[b0 + bz + nx + 1], phi[b0 + bz + nx]};
#pragma unroll
  for (int c = 0; c < 8; ++c) ph[c] = nudge(r[c]);
}

// A cell's triangle count and whether its tile uses the interior vertex (code 13); -1 tile if
// the cell is not cut.
template <class T, bool MX>
__device__ __forceinline__ int cell_tile(const T ph[8], const DevTable& tb, int& ntris, int& interior) {
  int nout = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) nout += ph[c] >= T(0) ? 1 : 0;
  ntris = 0;
  interior = 0;
  if (nout == 0 || nout == 8) return -1;
  const int tile = mc_tile<T, MX>(ph, tb);
  const cc_mc_tile tl = tb.tiles[tile];
  ntris = tl.ntris;
  const uint8_t* codes = tb.codes + tl.code_off;
  for (int q = 0; q < 3 * tl.ntris; ++q) interior |= codes[q] == 13 ? 1 : 0;
  return tile;
}

template <class T, bool MX>
__global__ void __launch_bounds__(MB, 4) cell_count_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                           const DevTable tb, unsigned long long* bsum, int* kept,
                                                           int* kept_n) {
  __shared__ int cand[BLK];
  const long long n0 = g.n[0], n1 = g.n[1], nc = n0 * n1 * g.n[2];
  const long long start = (long long)blockIdx.x * BLK;
  const long long nx = n0 + 1, nz = (n0 + 1) * (n1 + 1);
  Walker w(start, n0, n1, nx, nz);
  const bool full = start + BLK <= nc;  // block-uniform: no item past the grid
  const int n = cccompact::compact<MB, IPT, Groups<T>::cell>(cand, [&](int) {
    return cells_with_cut<T, Groups<T>::cell>(phi, w, unsigned(nc), unsigned(nx), unsigned(nz), full);
  });
  keep_survivors(cand, n, kept, kept_n);
  unsigned long long t = 0, in = 0;
  for (int x = threadIdx.x; x < n; x += MB) {
    const long long c = start + cand[x];
    T ph[8];
    corners(phi, g.n, c % n0, (c / n0) % n1, c / (n0 * n1), ph);
    int nt, it;
    cell_tile<T, MX>(ph, tb, nt, it);
    t += nt;
    in += it;
  }
  unsigned long long tt, ti;
  cccompact::block_scan<MB>(t, &tt);
  cccompact::block_scan<MB>(in, &ti);
  if (threadIdx.x == 0) {
    bsum[2 * blockIdx.x] = tt;
    bsum[2 * blockIdx.x + 1] = ti;
  }
}

template <class T, bool MX>
__global__ void __launch_bounds__(MB, 4) cell_emit_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                          const DevTable tb, const unsigned long long* __restrict__ boff,
                                                          const int* kept, const int* kept_n,
                                                          const unsigned* __restrict__ vbase,
                                                          unsigned long long n_edge_verts, T* __restrict__ verts,
                                                          unsigned long long vcap, int32_t* __restrict__ tris,
                                                          unsigned long long tcap, int64_t* __restrict__ tri_cells,
                                                          unsigned long long* overflow) {
  __shared__ int cand[BLK];
  const long long n0 = g.n[0], n1 = g.n[1], nc = n0 * n1 * g.n[2];
  const long long start = (long long)blockIdx.x * BLK;
  const long long nx = n0 + 1, nz = (n0 + 1) * (n1 + 1);
  Walker w(start, n0, n1, nx, nz);
  const bool full = start + BLK <= nc;  // block-uniform: no item past the grid
  const int n = survivors<Groups<T>::cell>(cand, kept, kept_n, [&](int) {
    return cells_with_cut<T, Groups<T>::cell>(phi, w, unsigned(nc), unsigned(nx), unsigned(nz), full);
  });
  unsigned long long run_t = boff[2 * blockIdx.x], run_i = n_edge_verts + boff[2 * blockIdx.x + 1];
  for (int c0 = 0; c0 < n; c0 += MB) {  // block-uniform
    const int x = c0 + threadIdx.x;
    const long long c = x < n ? start + cand[x] : 0;
    const long long i = c % n0, j = (c / n0) % n1, k = c / (n0 * n1);
    T ph[8];
    int nt = 0, it = 0, tile = -1;
    if (x < n) {
      corners(phi, g.n, i, j, k, ph);
      tile = cell_tile<T, MX>(ph, tb, nt, it);
    }
    unsigned long long tot;
    const unsigned long long pre =
        cccompact::block_scan<MB>(((unsigned long long)nt << 32) | (unsigned long long)it, &tot);
    unsigned long long tri_id = run_t + (pre >> 32), int_id = run_i + (pre & 0xffffffffull);
    run_t += tot >> 32;
    run_i += tot & 0xffffffffull;
    if (tile < 0) continue;
    if (tri_id + nt > tcap || (it && int_id >= vcap)) {
      atomicOr(overflow, 1ull);
      continue;
    }
    // the vertex of each of the cell's cut edges (code e + 1), from its lower node's numbering
    unsigned vid[12];
#pragma unroll
    for (int e = 0; e < 12; ++e) {
      const int ca = edge_node(e, 0), cb = edge_node(e, 1);
      vid[e] = 0;
      if ((ph[ca] >= T(0)) == (ph[cb] >= T(0))) continue;
      const int a = cbit(ca, 0) != cbit(cb, 0) ? 0 : (cbit(ca, 1) != cbit(cb, 1) ? 1 : 2);
      const int lo = cbit(ca, a) < cbit(cb, a) ? ca : cb;
      const long long li = i + cbit(lo, 0), lj = j + cbit(lo, 1), lk = k + cbit(lo, 2);
      const unsigned m = node_edges(phi, li, lj, lk, g.n);
      const long long v = li + (g.n[0] + 1) * (lj + (g.n[1] + 1) * lk);
      vid[e] = vbase[v] + __popc(m & ((1u << a) - 1u));
    }
    unsigned centre = 0;
    if (it) {
      centre = unsigned(int_id);
      T acc[3] = {T(0), T(0), T(0)};
      int ncr = 0;
      for (int e = 0; e < 12; ++e) {
        const int ca = edge_node(e, 0), cb = edge_node(e, 1);
        if ((ph[ca] >= T(0)) == (ph[cb] >= T(0))) continue;
        const int a = cbit(ca, 0) != cbit(cb, 0) ? 0 : (cbit(ca, 1) != cbit(cb, 1) ? 1 : 2);
        const int lo = cbit(ca, a) < cbit(cb, a) ? ca : cb;
        T p[3];
        edge_vertex(phi, g, i + cbit(lo, 0), j + cbit(lo, 1), k + cbit(lo, 2), a, p);
        acc[0] = acc[0] + p[0]; acc[1] = acc[1] + p[1]; acc[2] = acc[2] + p[2];
        ++ncr;
      }
      verts[3 * (long long)centre] = acc[0] / T(ncr);
      verts[3 * (long long)centre + 1] = acc[1] / T(ncr);
      verts[3 * (long long)centre + 2] = acc[2] / T(ncr);
    }
    const cc_mc_tile tl = tb.tiles[tile];
    const uint8_t* codes = tb.codes + tl.code_off;
    for (int r = 0; r < tl.ntris; ++r, ++tri_id) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int code = codes[3 * r + q];
        tris[3 * tri_id + q] = int32_t(code == 13 ? centre : vid[code - 1]);
      }
      if (tri_cells) tri_cells[tri_id] = c;
    }
  }
}

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);
  return s;
}
cc_status cuda_fail(cudaError_t e, const char* where) {
  cci::set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
  return CC_CUDA_ERR;
}

template <class T>
DevGrid<T> grid_of(const cc_grid* g) {
  DevGrid<T> d;
  for (int a = 0; a < 3; ++a) {
    d.x0[a] = T(g->x0[a]);
    d.d[a] = T(g->d[a]);
    d.n[a] = g->n[a];
  }
  return d;
}

template <class T, bool MX>
cc_status run_mesh(cc_handle* h, const cc_grid* gg, const T* phi, T* verts, int64_t vcap, int32_t* tris, int64_t tcap,
                   int64_t* tri_cells, int64_t* nv, int64_t* nt, cudaStream_t s) {
  const DevGrid<T> g = grid_of<T>(gg);
  const long long nn = (g.n[0] + 1) * (g.n[1] + 1) * (g.n[2] + 1);
  const long long nc = g.n[0] * g.n[1] * g.n[2];
  const long long nbn = (nn + BLK - 1) / BLK, nbc = (nc + BLK - 1) / BLK;
  // 32-bit item indices, with room for the last block's rounds past the end
  if (nn > 0xffffffffLL - BLK) return fail(CC_TOO_LARGE, "generate_mesh takes fewer than 2^32 - 8192 nodes");
  cci::MeshKey& key = h->mesh_key;
  cudaError_t e = cudaSuccess;
  if (size_t(nn) > h->mesh_vbase_n) {
    if (h->mesh_vbase) cudaFree(h->mesh_vbase);
    h->mesh_vbase = nullptr;
    h->mesh_vbase_n = 0;
    key.valid = false;
    if ((e = cudaMalloc(&h->mesh_vbase, size_t(nn) * sizeof(unsigned))) != cudaSuccess)
      return cuda_fail(e, "generate_mesh scratch");
    h->mesh_vbase_n = size_t(nn);
  }
  // 64-bit words: node block offsets, cell block offsets (tris, interior) interleaved, 3 totals,
  // the overflow flag; then 32-bit: node kept_n, node kept, cell kept_n, cell kept
  const size_t words = size_t(nbn + 2 * nbc + 4);
  const size_t ints = size_t(nbn) * (KEEP + 1) + size_t(nbc) * (KEEP + 1);
  const size_t scan_n = words + (ints + 1) / 2;
  if (scan_n > h->mesh_scan_n) {
    if (h->mesh_scan) cudaFree(h->mesh_scan);
    h->mesh_scan = nullptr;
    h->mesh_scan_n = 0;
    key.valid = false;
    if ((e = cudaMalloc(&h->mesh_scan, scan_n * sizeof(unsigned long long))) != cudaSuccess)
      return cuda_fail(e, "generate_mesh scratch");
    h->mesh_scan_n = scan_n;
  }
  unsigned long long* nb = h->mesh_scan;              // node blocks
  unsigned long long* cb = nb + nbn;                  // cell blocks (tris, interior) interleaved
  unsigned long long* tot = cb + 2 * nbc;             // edge vertices, tris, interior vertices
  unsigned long long* overflow = tot + 3;
  int* node_kept_n = reinterpret_cast<int*>(h->mesh_scan + words);
  int* node_kept = node_kept_n + nbn;
  int* cell_kept_n = node_kept + size_t(nbn) * KEEP;
  int* cell_kept = cell_kept_n + nbc;
  const bool emit = verts || tris;
  bool reuse = emit && key.valid && key.generation == h->generation && key.phi == phi && key.prec == h->prec;
  for (int a = 0; a < 3 && reuse; ++a)
    reuse = key.g.n[a] == gg->n[a] && key.g.x0[a] == gg->x0[a] && key.g.d[a] == gg->d[a];
  unsigned long long t[3] = {key.tot[0], key.tot[1], key.tot[2]};
  if (!reuse) {
    key.valid = false;
    node_count_kernel<T><<<unsigned(nbn), MB, 0, s>>>(phi, g, nb, node_kept, node_kept_n);
    cccompact::scan_series_kernel<MB><<<1, MB, 0, s>>>(nb, nbn, 1, tot);
    cell_count_kernel<T, MX><<<unsigned(nbc), MB, 0, s>>>(phi, g, h->tb, cb, cell_kept, cell_kept_n);
    cccompact::scan_series_kernel<MB><<<1, MB, 0, s>>>(cb, nbc, 2, tot + 1);
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaMemcpyAsync(t, tot, sizeof t, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "generate_mesh count");
    key.valid = true;
    key.generation = h->generation;
    key.phi = phi;
    key.prec = h->prec;
    key.g = *gg;
    for (int q = 0; q < 3; ++q) key.tot[q] = t[q];
  }
  const long long n_vert = (long long)(t[0] + t[2]), n_tri = (long long)t[1];
  if (nv) *nv = n_vert;
  if (nt) *nt = n_tri;
  if (!emit) return CC_OK;  // counting only
  if (!verts || !tris || vcap < n_vert || tcap < n_tri)
    return fail(CC_BAD_ARG, "generate_mesh output smaller than the counted surface");
  if (n_vert > 0xffffffffLL) return fail(CC_TOO_LARGE, "generate_mesh numbers at most 2^32 - 1 vertices");
  unsigned long long flag = 0;
  e = cudaMemsetAsync(overflow, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) {
    node_emit_kernel<T><<<unsigned(nbn), MB, 0, s>>>(phi, g, nb, node_kept, node_kept_n, h->mesh_vbase, verts,
                                                     (unsigned long long)vcap, overflow);
    cell_emit_kernel<T, MX><<<unsigned(nbc), MB, 0, s>>>(phi, g, h->tb, cb, cell_kept, cell_kept_n, h->mesh_vbase, t[0],
                                                         verts, (unsigned long long)vcap, tris,
                                                         (unsigned long long)tcap, tri_cells, overflow);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, overflow, sizeof flag, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  key.valid = false;  // one emit per count
  if (e != cudaSuccess) return cuda_fail(e, "generate_mesh emit");
  if (flag) return fail(CC_BAD_ARG, "generate_mesh: phi changed between the count and the emit call");
  return CC_OK;
}

// cell_indices (src/marching_cubes/surface.jl:128-143): the cell of each triangle, from its
// vertices' centroid (summed and divided in the mesh's precision) floored against the grid in
// Float64, clamped to the grid.
template <class T>
__global__ void cell_index_kernel(const cc_grid g, const T* __restrict__ verts, const int32_t* __restrict__ tris,
                                  long long nt, int64_t* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt; t += (long long)gridDim.x * blockDim.x) {
    const long long va = tris[3 * t], vb = tris[3 * t + 1], vc = tris[3 * t + 2];
    long long idx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T cT = ((verts[3 * va + a] + verts[3 * vb + a]) + verts[3 * vc + a]) / T(3);
      const double c = double(cT);
      long long q = (long long)floor((c - g.x0[a]) / g.d[a]);
      q = q < 0 ? 0 : (q > g.n[a] - 1 ? g.n[a] - 1 : q);
      idx[a] = q;
    }
    out[t] = idx[0] + g.n[0] * (idx[1] + g.n[1] * idx[2]);
  }
}

}  // namespace

extern "C" {

cc_status cc_mc_mesh(cc_handle* h, const cc_grid* g, const void* phi, void* vertices, int64_t vertex_capacity,
                     int32_t* triangles, int64_t triangle_capacity, int64_t* triangle_cells, int64_t* n_vertices,
                     int64_t* n_triangles, void* stream) {
  if (!h || !g || !phi) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_MARCHING_CUBES) return fail(CC_BAD_ARG, "handle was created for another method");
  if (g->dim != 3) return fail(CC_DIM_MISMATCH, "grid dimension differs from the cache's");
  for (int a = 0; a < 3; ++a)
    if (g->n[a] != h->n[a]) return fail(CC_DIM_MISMATCH, "grid size differs from the cache's");
  if (!h->table_dev) return fail(CC_NO_TABLE, "no marching-cubes tiling table set on the handle");
  int old = -1;
  cudaGetDevice(&old);
  if (old != h->device) cudaSetDevice(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cc_status st;
  if (h->prec == CC_F64)
    st = run_mesh<double, false>(h, g, static_cast<const double*>(phi), static_cast<double*>(vertices), vertex_capacity,
                                 triangles, triangle_capacity, triangle_cells, n_vertices, n_triangles, s);
  else if (h->prec == CC_MIXED)
    st = run_mesh<float, true>(h, g, static_cast<const float*>(phi), static_cast<float*>(vertices), vertex_capacity,
                               triangles, triangle_capacity, triangle_cells, n_vertices, n_triangles, s);
  else
    st = run_mesh<float, false>(h, g, static_cast<const float*>(phi), static_cast<float*>(vertices), vertex_capacity,
                                triangles, triangle_capacity, triangle_cells, n_vertices, n_triangles, s);
  if (old >= 0 && old != h->device) cudaSetDevice(old);
  return st;
}

cc_status cc_mc_mesh_cell_indices(cc_handle* h, const cc_grid* g, const void* vertices, const int32_t* triangles,
                                  int64_t n_triangles, int64_t* cells, void* stream) {
  if (!h || !g || (n_triangles > 0 && (!vertices || !triangles || !cells)) || n_triangles < 0)
    return fail(CC_BAD_ARG, "null argument");
  if (g->dim != 3) return fail(CC_DIM_MISMATCH, "a 3D grid");
  if (n_triangles == 0) return CC_OK;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = int(n_triangles / 256 + 1 < 148 * 16 ? n_triangles / 256 + 1 : 148 * 16);
  if (h->prec == CC_F64)
    cell_index_kernel<double><<<blocks, 256, 0, s>>>(*g, static_cast<const double*>(vertices), triangles, n_triangles, cells);
  else
    cell_index_kernel<float><<<blocks, 256, 0, s>>>(*g, static_cast<const float*>(vertices), triangles, n_triangles, cells);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? CC_OK : cuda_fail(e, "cell_indices");
}

}  // extern "C"
