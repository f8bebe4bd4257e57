// plic_mesh.cu -- extract_surface_plic / generate_mesh for a PLIC cache on the device
// (src/plic/surface.jl:28-267, where the clip runs as a kernel but the sort, fan and compaction on
// host arrays).
//
// Every entry's plane n . xi = a (its cell's unit frame, xi in [0,1]^D) is clipped to its cell:
// in 3D the points where the plane crosses the cube's edges (sign change of n . xi - a between the
// edge's corners; a corner exactly on the plane taken once), 0 to 6 of them; in 2D the square's two
// crossings. The points map to the world as x_node + xi * d. A 3D polygon's vertices are ordered by
// angle about their centroid in the plane basis u = normalize(r x n), v = n x u (r = e_z unless
// |n_z| >= 0.9, then e_x) -- a pseudo-angle, monotone in atan2, keeps that order reproducible bit
// for bit -- then fanned from the first vertex; a fan triangle with |cross|^2 < (2 min_area)^2,
// min_area = min_tri_area_fraction * min(d)^2, is dropped (its vertices stay). A 2D segment
// shorter than min_tri_area_fraction * min(d) is dropped with its nodes; an entry whose line does
// not cross its cell (or with a degenerate fit) has a zero-length segment, so at fraction 0 every
// 2D entry draws one, and a 3D entry draws only a polygon of 3 or more points. Entries contribute
// in order; elements do not share nodes (each plane is its own cell's).
//
// CartesianMeshes.cell_plane_clip itself is not available here: this clip is written from the
// geometry, so its vertex order may differ from that package's; the sort makes the polygon's
// winding the same.
//
// Two passes over the entries (count, then emit at scanned offsets), each thread owning IPT
// consecutive entries, so the output is in entry order with no atomics.
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"

namespace {

using namespace ccd;

constexpr int MB = 256;
constexpr int IPT = 8;
constexpr int BLK = MB * IPT;

template <class T, int D>
struct PlicIn {
  T x0[3], d[3];
  long long n[3];
  const int64_t* index;  // entry k draws cell index[k] (linear); null: entry k is cell k
  long long count;       // entries
  const T* normals;
  const T* intercepts;
  const uint8_t* valid;  // null: a zero normal marks a degenerate fit
  T min_frac;
};

// A pseudo-angle of (x, y): strictly increasing with atan2(y, x) over (-pi, pi], valued in (-2, 2],
// from one correctly rounded division, so the order it gives is the same on every IEEE machine.
template <class T>
__device__ __forceinline__ T pseudo_angle(T y, T x) {
  if (x == T(0) && y == T(0)) return T(0);
  if (y >= T(0)) return x >= T(0) ? y / (x + y) : T(1) + (-x) / (y - x);
  return x >= T(0) ? -((-y) / (x - y)) : -(T(1) + (-x) / (-x - y));
}

// The clipped polygon of one entry in world coordinates, ordered (3D); returns its vertex count
// (always 2 in 2D, where a miss is a zero-length segment).
template <class T, int D>
__device__ int clip_cell(const PlicIn<T, D>& P, long long entry, T out[6][3]) {
  const long long ci = P.index ? (long long)P.index[entry] : entry;
  const long long idx[3] = {ci % P.n[0], (ci / P.n[0]) % P.n[1], D == 3 ? ci / (P.n[0] * P.n[1]) : 0};
  T nrm[3] = {P.normals[D * entry], P.normals[D * entry + 1], D == 3 ? P.normals[D * entry + 2] : T(0)};
  const T a = P.intercepts[entry];
  const bool ok = P.valid ? P.valid[entry] != 0 : (nrm[0] != T(0) || nrm[1] != T(0) || nrm[2] != T(0));
  T org[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) org[q] = q < D ? node_coord(P.x0[q], P.d[q], idx[q]) : T(0);
  int m = 0;
  T xi[6][3];
  if (D == 2) {
    // the square's corners (0,0) (1,0) (1,1) (0,1) and edges k -> k+1
    const T c[4][2] = {{T(0), T(0)}, {T(1), T(0)}, {T(1), T(1)}, {T(0), T(1)}};
    T s[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] = (nrm[0] * c[k][0] + nrm[1] * c[k][1]) - a;
    for (int k = 0; k < 4 && m < 2 && ok; ++k) {
      if (s[k] == T(0)) { xi[m][0] = c[k][0]; xi[m][1] = c[k][1]; ++m; continue; }
      const int k1 = (k + 1) & 3;
      if ((s[k] < T(0) && s[k1] > T(0)) || (s[k] > T(0) && s[k1] < T(0))) {
        const T t = s[k] / (s[k] - s[k1]);
        xi[m][0] = c[k][0] + t * (c[k1][0] - c[k][0]);
        xi[m][1] = c[k][1] + t * (c[k1][1] - c[k][1]);
        ++m;
      }
    }
    if (m < 2) {
      // no crossing: a zero-length segment at the one corner the line touches, else (a miss, or
      // a degenerate fit's zero plane) at the cell's lower corner
      if (m == 0) xi[0][0] = xi[0][1] = T(0);
      xi[1][0] = xi[0][0];
      xi[1][1] = xi[0][1];
    }
    for (int q = 0; q < 2; ++q) {
      out[q][0] = org[0] + xi[q][0] * P.d[0];
      out[q][1] = org[1] + xi[q][1] * P.d[1];
      out[q][2] = T(0);
    }
    return 2;
  }
  if (!ok) return 0;
  // 3D: corners by bits (x = bit 0, y = bit 1, z = bit 2); the 12 edges as corner pairs
  T s[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) s[c] = ((nrm[0] * T(c & 1) + nrm[1] * T((c >> 1) & 1)) + nrm[2] * T((c >> 2) & 1)) - a;
  for (int c = 0; c < 8 && m < 6; ++c)
    if (s[c] == T(0)) { xi[m][0] = T(c & 1); xi[m][1] = T((c >> 1) & 1); xi[m][2] = T((c >> 2) & 1); ++m; }
  const int e[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int k = 0; k < 12 && m < 6; ++k) {
    const int p = e[k][0], q = e[k][1];
    if ((s[p] < T(0) && s[q] > T(0)) || (s[p] > T(0) && s[q] < T(0))) {
      const T t = s[p] / (s[p] - s[q]);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const T cp = T((p >> ax) & 1), cq = T((q >> ax) & 1);
        xi[m][ax] = cp + t * (cq - cp);
      }
      ++m;
    }
  }
  if (m < 3) return 0;
  for (int k = 0; k < m; ++k)
#pragma unroll
    for (int q = 0; q < 3; ++q) out[k][q] = org[q] + xi[k][q] * P.d[q];
  // order by angle about the centroid in the plane's basis
  T cen[3] = {T(0), T(0), T(0)};
  for (int k = 0; k < m; ++k) { cen[0] = cen[0] + out[k][0]; cen[1] = cen[1] + out[k][1]; cen[2] = cen[2] + out[k][2]; }
  cen[0] = cen[0] / T(m); cen[1] = cen[1] / T(m); cen[2] = cen[2] / T(m);
  const bool zr = fabs(nrm[2]) < T(0.9);
  const T r[3] = {zr ? T(0) : T(1), T(0), zr ? T(1) : T(0)};
  T u[3] = {r[1] * nrm[2] - r[2] * nrm[1], r[2] * nrm[0] - r[0] * nrm[2], r[0] * nrm[1] - r[1] * nrm[0]};
  const T ul = sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
  u[0] = u[0] / ul; u[1] = u[1] / ul; u[2] = u[2] / ul;
  const T v[3] = {nrm[1] * u[2] - nrm[2] * u[1], nrm[2] * u[0] - nrm[0] * u[2], nrm[0] * u[1] - nrm[1] * u[0]};
  T ang[6];
  for (int k = 0; k < m; ++k) {
    const T dx = out[k][0] - cen[0], dy = out[k][1] - cen[1], dz = out[k][2] - cen[2];
    ang[k] = pseudo_angle((dx * v[0] + dy * v[1]) + dz * v[2], (dx * u[0] + dy * u[1]) + dz * u[2]);
  }
  for (int i = 1; i < m; ++i) {  // insertion sort, as the reference's sort kernel
    const T ka = ang[i], k0 = out[i][0], k1 = out[i][1], k2 = out[i][2];
    int j = i - 1;
    while (j >= 0 && ang[j] > ka) {
      ang[j + 1] = ang[j];
      out[j + 1][0] = out[j][0]; out[j + 1][1] = out[j][1]; out[j + 1][2] = out[j][2];
      --j;
    }
    ang[j + 1] = ka;
    out[j + 1][0] = k0; out[j + 1][1] = k1; out[j + 1][2] = k2;
  }
  return m;
}

// Nodes and elements one clipped entry contributes; keep bit v marks fan triangle (0, v, v+1).
template <class T, int D>
__device__ __forceinline__ void cell_counts(const PlicIn<T, D>& P, int m, const T p[6][3], T min_d, int& nodes,
                                            int& elems, unsigned& keep) {
  nodes = elems = 0;
  keep = 0;
  if (D == 2) {
    if (m < 2) return;
    const T dx = p[1][0] - p[0][0], dy = p[1][1] - p[0][1];
    if (sqrt(dx * dx + dy * dy) >= P.min_frac * min_d) { nodes = 2; elems = 1; keep = 1; }
    return;
  }
  if (m < 3) return;
  nodes = m;
  const T min_area = P.min_frac * (min_d * min_d);
  const T min_cross_sq = (T(2) * min_area) * (T(2) * min_area);
  for (int v = 1; v < m - 1; ++v) {
    const T a0 = p[v][0] - p[0][0], a1 = p[v][1] - p[0][1], a2 = p[v][2] - p[0][2];
    const T b0 = p[v + 1][0] - p[0][0], b1 = p[v + 1][1] - p[0][1], b2 = p[v + 1][2] - p[0][2];
    const T c0 = a1 * b2 - a2 * b1, c1 = a2 * b0 - a0 * b2, c2 = a0 * b1 - a1 * b0;
    if ((c0 * c0 + c1 * c1) + c2 * c2 >= min_cross_sq) { ++elems; keep |= 1u << v; }
  }
}

// Exclusive scan of x over the block; *total gets the block's sum.
__device__ __forceinline__ unsigned long long block_scan(unsigned long long x, unsigned long long* total) {
  __shared__ unsigned long long warp_sum[MB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) warp_sum[w] = v;
  __syncthreads();
  unsigned long long base = 0, all = 0;
  for (int q = 0; q < MB / 32; ++q) {
    if (q < w) base += warp_sum[q];
    all += warp_sum[q];
  }
  __syncthreads();
  *total = all;
  return base + v - x;
}

// In-place exclusive scan of the per-block (nodes, elements) pairs; the totals go to total[0..1].
__global__ void scan2_kernel(unsigned long long* a, long long n, unsigned long long* total) {
  __shared__ unsigned long long carry[2];
  if (threadIdx.x < 2) carry[threadIdx.x] = 0;
  __syncthreads();
  for (int l = 0; l < 2; ++l)
    for (long long base = 0; base < n; base += MB) {
      const long long q = base + threadIdx.x;
      const unsigned long long x = q < n ? a[2 * q + l] : 0ull;
      unsigned long long t;
      const unsigned long long pre = block_scan(x, &t);
      if (q < n) a[2 * q + l] = carry[l] + pre;
      __syncthreads();
      if (threadIdx.x == 0) carry[l] += t;
      __syncthreads();
    }
  if (threadIdx.x < 2) total[threadIdx.x] = carry[threadIdx.x];
}

template <class T, int D>
__global__ void __launch_bounds__(MB) plic_count_kernel(const PlicIn<T, D> P, T min_d, unsigned long long* bsum) {
  const long long nc = P.count;
  const long long c0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long nn = 0, ne = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long k = c0 + q;
    if (k >= nc) break;
    T p[6][3];
    const int m = clip_cell<T, D>(P, k, p);
    int a, b;
    unsigned keep;
    cell_counts<T, D>(P, m, p, min_d, a, b, keep);
    nn += a;
    ne += b;
  }
  unsigned long long t0, t1;
  block_scan(nn, &t0);
  block_scan(ne, &t1);
  if (threadIdx.x == 0) { bsum[2 * blockIdx.x] = t0; bsum[2 * blockIdx.x + 1] = t1; }
}

template <class T, int D>
__global__ void __launch_bounds__(MB) plic_emit_kernel(const PlicIn<T, D> P, T min_d, const unsigned long long* boff,
                                                       T* nodes, int32_t* elems, int64_t* cells) {
  const long long nc = P.count;
  const long long c0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long nn = 0, ne = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long k = c0 + q;
    if (k >= nc) break;
    T p[6][3];
    const int m = clip_cell<T, D>(P, k, p);
    int a, b;
    unsigned keep;
    cell_counts<T, D>(P, m, p, min_d, a, b, keep);
    nn += a;
    ne += b;
  }
  unsigned long long t0, t1;
  unsigned long long vn = boff[2 * blockIdx.x] + block_scan(nn, &t0);
  unsigned long long ve = boff[2 * blockIdx.x + 1] + block_scan(ne, &t1);
  for (int q = 0; q < IPT; ++q) {
    const long long k = c0 + q;
    if (k >= nc) break;
    T p[6][3];
    const int m = clip_cell<T, D>(P, k, p);
    int a, b;
    unsigned keep;
    cell_counts<T, D>(P, m, p, min_d, a, b, keep);
    if (a == 0) continue;
    const long long ci = P.index ? (long long)P.index[k] : k;
    for (int v = 0; v < a; ++v)
#pragma unroll
      for (int x = 0; x < D; ++x) nodes[D * (vn + v) + x] = p[v][x];
    if (D == 2) {
      if (b) {
        elems[2 * ve] = int32_t(vn);
        elems[2 * ve + 1] = int32_t(vn + 1);
        cells[ve] = ci;
        ++ve;
      }
    } else {
      for (int v = 1; v < m - 1; ++v) {
        if (!(keep >> v & 1u)) continue;
        elems[3 * ve] = int32_t(vn);
        elems[3 * ve + 1] = int32_t(vn + v);
        elems[3 * ve + 2] = int32_t(vn + v + 1);
        cells[ve] = ci;
        ++ve;
      }
    }
    vn += a;
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

template <class T, int D>
cc_status run(const cc_grid* g, const void* normals, const void* intercepts, const uint8_t* valid,
              const int64_t* index, int64_t count, double min_frac, void* nodes, int64_t ncap, int32_t* elems,
              int64_t ecap, int64_t* cells, int64_t* n_nodes, int64_t* n_elems, cudaStream_t s) {
  PlicIn<T, D> P;
  for (int a = 0; a < 3; ++a) {
    P.x0[a] = a < D ? T(g->x0[a]) : T(0);
    P.d[a] = a < D ? T(g->d[a]) : T(1);
    P.n[a] = a < D ? g->n[a] : 1;
  }
  P.index = index;
  P.count = index ? count : P.n[0] * P.n[1] * P.n[2];
  P.normals = static_cast<const T*>(normals);
  P.intercepts = static_cast<const T*>(intercepts);
  P.valid = valid;
  P.min_frac = T(min_frac);
  T min_d = P.d[0];
  for (int a = 1; a < D; ++a) min_d = P.d[a] < min_d ? P.d[a] : min_d;
  const long long nc = P.count;
  if (nc == 0) {
    if (n_nodes) *n_nodes = 0;
    if (n_elems) *n_elems = 0;
    return CC_OK;
  }
  const long long nb = (nc + BLK - 1) / BLK;
  unsigned long long* bsum = nullptr;
  cudaError_t e = cudaMalloc(&bsum, (2 * size_t(nb) + 2) * sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "generate_mesh scratch");
  plic_count_kernel<T, D><<<unsigned(nb), MB, 0, s>>>(P, min_d, bsum);
  scan2_kernel<<<1, MB, 0, s>>>(bsum, nb, bsum + 2 * nb);
  unsigned long long tot[2] = {0, 0};
  if ((e = cudaGetLastError()) == cudaSuccess)
    e = cudaMemcpyAsync(tot, bsum + 2 * nb, sizeof tot, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    if (n_nodes) *n_nodes = (int64_t)tot[0];
    if (n_elems) *n_elems = (int64_t)tot[1];
    if (tot[0] > 0x7fffffffull) {
      cudaFree(bsum);
      return fail(CC_TOO_LARGE, "generate_mesh: more nodes than int32 element indices address");
    }
    if (nodes || elems) {
      if (!nodes || !elems || !cells || ncap < (int64_t)tot[0] || ecap < (int64_t)tot[1]) {
        cudaFree(bsum);
        return fail(CC_BAD_ARG, "generate_mesh output smaller than the counted surface");
      }
      if (tot[1] > 0)
        plic_emit_kernel<T, D><<<unsigned(nb), MB, 0, s>>>(P, min_d, bsum, static_cast<T*>(nodes), elems, cells);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
  }
  cudaFree(bsum);
  return e == cudaSuccess ? CC_OK : cuda_fail(e, "generate_mesh");
}

cc_status surface(int prec, const cc_grid* g, const void* normals, const void* intercepts, const uint8_t* valid,
                  const int64_t* index, int64_t count, double min_frac, void* nodes, int64_t ncap, int32_t* elems,
                  int64_t ecap, int64_t* cells, int64_t* n_nodes, int64_t* n_elems, cudaStream_t s) {
  if (prec == CC_F64)
    return g->dim == 3 ? run<double, 3>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                        cells, n_nodes, n_elems, s)
                       : run<double, 2>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                        cells, n_nodes, n_elems, s);
  return g->dim == 3 ? run<float, 3>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                     cells, n_nodes, n_elems, s)
                     : run<float, 2>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                     cells, n_nodes, n_elems, s);
}

}  // namespace

extern "C" {

cc_status cc_plic_surface(int prec, const cc_grid* g, const void* normals, const void* intercepts,
                          const uint8_t* is_valid, const int64_t* cell_index, int64_t n_entries,
                          double min_tri_area_fraction, void* nodes, int64_t node_capacity, int32_t* elements,
                          int64_t element_capacity, int64_t* element_cells, int64_t* n_nodes, int64_t* n_elements,
                          void* stream) {
  if (!g) return fail(CC_BAD_ARG, "null argument");
  if (g->dim != 2 && g->dim != 3) return fail(CC_BAD_ARG, "grid dimension must be 2 or 3");
  if (prec != CC_F32 && prec != CC_F64 && prec != CC_MIXED) return fail(CC_BAD_ARG, "unknown precision");
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] < 1) return fail(CC_BAD_ARG, "grid needs at least one cell per axis");
  if (cell_index && n_entries < 0) return fail(CC_BAD_ARG, "n_entries must be >= 0");
  if ((!cell_index || n_entries > 0) && (!normals || !intercepts)) return fail(CC_BAD_ARG, "null argument");
  if (!(min_tri_area_fraction >= 0.0)) return fail(CC_BAD_ARG, "min_tri_area_fraction must be >= 0");
  return surface(prec, g, normals, intercepts, is_valid, cell_index, n_entries, min_tri_area_fraction, nodes,
                 node_capacity, elements, element_capacity, element_cells, n_nodes, n_elements,
                 static_cast<cudaStream_t>(stream));
}

cc_status cc_plic_mesh(cc_handle* h, const cc_grid* g, const void* normals, const void* intercepts,
                       const uint8_t* is_valid, double min_tri_area_fraction, void* nodes, int64_t node_capacity,
                       int32_t* elements, int64_t element_capacity, int64_t* element_cells, int64_t* n_nodes,
                       int64_t* n_elements, void* stream) {
  if (!h || !g || !normals || !intercepts || !is_valid) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_PLIC) return fail(CC_BAD_ARG, "handle was created for another method");
  if (g->dim != h->dim) return fail(CC_DIM_MISMATCH, "grid dimension differs from the cache's");
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] != h->n[a]) return fail(CC_DIM_MISMATCH, "grid size differs from the cache's");
  if (!(min_tri_area_fraction >= 0.0)) return fail(CC_BAD_ARG, "min_tri_area_fraction must be >= 0");
  int old = -1;
  cudaGetDevice(&old);
  if (old != h->device) cudaSetDevice(h->device);
  const cc_status st = surface(h->prec, g, normals, intercepts, is_valid, nullptr, 0, min_tri_area_fraction, nodes,
                               node_capacity, elements, element_capacity, element_cells, n_nodes, n_elements,
                               static_cast<cudaStream_t>(stream));
  if (old >= 0 && old != h->device) cudaSetDevice(old);
  return st;
}

}  // extern "C"
