// ms_mesh.cu -- generate_mesh for a marching-squares cache on the device: the contour of a grid
// cache's nodal phi, or of a quadtree cache's per-leaf corners (src/marching_squares/surface.jl:
// 70-111, where the reference walks the cut cells serially and welds vertices in a host Dict).
//
// Elements are the cells' cell_interface segments (oriented out of the body), in cell (or leaf)
// order; vertices are welded by exact coordinate equality, -0.0 normalised to 0.0, and numbered by
// first occurrence -- segment order, each segment's start before its end -- which is the
// numbering the reference's serial Dict weld produces. On the device: count and scan the
// segments, emit their endpoint occurrences, hash the occurrences by coordinate (open addressing,
// each slot keeping the smallest occurrence of its coordinate), flag first occurrences, scan the
// flags into vertex numbers, and resolve every element endpoint. Every probe sequence is bounded
// by the table size; a full table (not reachable at the load factor used) is an error, not a wait.
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"
#include "ms_cell.cuh"

namespace {

using namespace ccd;
using namespace ccms;

constexpr int MB = 256;
constexpr int IPT = 8;
constexpr int BLK = MB * IPT;

// One item: a grid cell or a tree leaf.
template <class T>
struct MsDomain {
  int tree;
  T x0[2], d[2];        // grid origin / cell size (as T)
  long long n0, n1;     // grid cells per axis; tree: n0 = leaves
  double base_d[2];     // tree
  const int32_t* level;
  const int32_t* coord;
  const T* phi;         // grid: nodal block; tree: 4 corners per leaf
  __host__ __device__ long long items() const { return tree ? n0 : n0 * n1; }
};

template <class T>
__device__ __forceinline__ void item_corners(const MsDomain<T>& D, long long it, T nd[4][2], T ph[4]) {
  if (!D.tree) {
    const long long i = it % D.n0, j = it / D.n0, nx = D.n0 + 1;
    const T xa = node_coord(D.x0[0], D.d[0], i), xb = node_coord(D.x0[0], D.d[0], i + 1);
    const T ya = node_coord(D.x0[1], D.d[1], j), yb = node_coord(D.x0[1], D.d[1], j + 1);
    nd[0][0] = xa; nd[0][1] = ya; nd[1][0] = xb; nd[1][1] = ya;
    nd[2][0] = xb; nd[2][1] = yb; nd[3][0] = xa; nd[3][1] = yb;
    const long long b = i + nx * j;
    ph[0] = D.phi[b]; ph[1] = D.phi[b + 1]; ph[2] = D.phi[b + nx + 1]; ph[3] = D.phi[b + nx];
  } else {
    const T scale = T(ldexp(1.0, -D.level[it]));
    const T h0 = T(D.base_d[0]) * scale, h1 = T(D.base_d[1]) * scale;
    const long long cx = D.coord[2 * it], cy = D.coord[2 * it + 1];
    const T xa = D.x0[0] + T(cx) * h0, xb = D.x0[0] + T(cx + 1) * h0;
    const T ya = D.x0[1] + T(cy) * h1, yb = D.x0[1] + T(cy + 1) * h1;
    nd[0][0] = xa; nd[0][1] = ya; nd[1][0] = xb; nd[1][1] = ya;
    nd[2][0] = xb; nd[2][1] = yb; nd[3][0] = xa; nd[3][1] = yb;
#pragma unroll
    for (int q = 0; q < 4; ++q) ph[q] = D.phi[4 * it + q];
  }
}

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

// Exclusive scan of `n` block counts in one CTA, in place; *total their sum.
__global__ void scan_kernel(unsigned long long* a, long long n, unsigned long long* total) {
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < n; base += MB) {
    const long long q = base + threadIdx.x;
    const unsigned long long x = q < n ? a[q] : 0ull;
    unsigned long long t;
    const unsigned long long pre = block_scan(x, &t);
    if (q < n) a[q] = carry + pre;
    __syncthreads();
    if (threadIdx.x == 0) carry += t;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

template <class T, bool MX>
__global__ void __launch_bounds__(MB) seg_count_kernel(const MsDomain<T> D, unsigned long long* bsum) {
  const long long n = D.items(), i0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long c = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long it = i0 + q;
    if (it >= n) break;
    T nd[4][2], ph[4], a[2][2], b[2][2];
    item_corners(D, it, nd, ph);
    c += ms_interface<T, MX>(nd, ph, a, b);
  }
  unsigned long long t;
  block_scan(c, &t);
  if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

// Each segment s: occurrences 2s (its start) and 2s + 1 (its end), coordinates normalised.
template <class T, bool MX>
__global__ void __launch_bounds__(MB) seg_emit_kernel(const MsDomain<T> D, const unsigned long long* boff, T* occ,
                                                      int64_t* cells) {
  const long long n = D.items(), i0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long c = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long it = i0 + q;
    if (it >= n) break;
    T nd[4][2], ph[4], a[2][2], b[2][2];
    item_corners(D, it, nd, ph);
    c += ms_interface<T, MX>(nd, ph, a, b);
  }
  unsigned long long t;
  unsigned long long s = boff[blockIdx.x] + block_scan(c, &t);
  for (int q = 0; q < IPT; ++q) {
    const long long it = i0 + q;
    if (it >= n) break;
    T nd[4][2], ph[4], a[2][2], b[2][2];
    item_corners(D, it, nd, ph);
    const int m = ms_interface<T, MX>(nd, ph, a, b);
    for (int r = 0; r < m; ++r, ++s) {
      occ[4 * s] = a[r][0] + T(0);
      occ[4 * s + 1] = a[r][1] + T(0);
      occ[4 * s + 2] = b[r][0] + T(0);
      occ[4 * s + 3] = b[r][1] + T(0);
      cells[s] = it;
    }
  }
}

template <class T> struct Bits;
template <> struct Bits<float> {
  using U = unsigned;
  static __device__ __forceinline__ U of(float v) { return __float_as_uint(v); }
};
template <> struct Bits<double> {
  using U = unsigned long long;
  static __device__ __forceinline__ U of(double v) { return (unsigned long long)__double_as_longlong(v); }
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class T>
__device__ __forceinline__ unsigned long long occ_hash(const T* occ, long long o) {
  return mix64((unsigned long long)Bits<T>::of(occ[2 * o]) * 0x100000001B3ull ^ mix64(Bits<T>::of(occ[2 * o + 1])));
}

template <class T>
__device__ __forceinline__ bool same(const T* occ, long long o, long long p) {
  return Bits<T>::of(occ[2 * o]) == Bits<T>::of(occ[2 * p]) && Bits<T>::of(occ[2 * o + 1]) == Bits<T>::of(occ[2 * p + 1]);
}

// Insert every occurrence; each slot's owner is the first occurrence to claim it, and minocc the
// smallest occurrence with that coordinate.
template <class T>
__global__ void hash_insert_kernel(const T* occ, long long nocc, long long* owner, unsigned long long* minocc,
                                   unsigned long long mask, int* err) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < nocc; o += (long long)gridDim.x * blockDim.x) {
    unsigned long long h = occ_hash(occ, o) & mask;
    bool done = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      const long long cur = (long long)atomicCAS((unsigned long long*)&owner[h], ~0ull, (unsigned long long)o);
      if (cur == -1 || same(occ, o, cur)) {
        atomicMin(&minocc[h], (unsigned long long)o);
        done = true;
        break;
      }
      h = (h + 1) & mask;
    }
    if (!done) atomicExch(err, 1);
  }
}

// The first occurrence of each occurrence's coordinate, and whether it is its own.
template <class T>
__global__ void __launch_bounds__(MB) first_kernel(const T* occ, long long nocc, const long long* owner,
                                                   const unsigned long long* minocc, unsigned long long mask,
                                                   long long* first, unsigned long long* bsum) {
  const long long o0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long c = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long o = o0 + q;
    if (o >= nocc) break;
    unsigned long long h = occ_hash(occ, o) & mask;
    long long f = o;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      const long long cur = owner[h];
      if (cur == -1) break;  // (not reachable: o itself was inserted)
      if (same(occ, o, cur)) {
        f = (long long)minocc[h];
        break;
      }
      h = (h + 1) & mask;
    }
    first[o] = f;
    c += f == o ? 1 : 0;
  }
  unsigned long long t;
  block_scan(c, &t);
  if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

// Number the first occurrences in occurrence order and write their vertices.
template <class T>
__global__ void __launch_bounds__(MB) vertex_kernel(const T* occ, long long nocc, const long long* first,
                                                   const unsigned long long* boff, unsigned* vid, T* verts) {
  const long long o0 = (long long)blockIdx.x * BLK + (long long)threadIdx.x * IPT;
  unsigned long long c = 0;
  for (int q = 0; q < IPT; ++q) {
    const long long o = o0 + q;
    if (o >= nocc) break;
    c += first[o] == o ? 1 : 0;
  }
  unsigned long long t;
  unsigned long long v = boff[blockIdx.x] + block_scan(c, &t);
  for (int q = 0; q < IPT; ++q) {
    const long long o = o0 + q;
    if (o >= nocc) break;
    if (first[o] == o) {
      vid[o] = unsigned(v);
      verts[2 * v] = occ[2 * o];
      verts[2 * v + 1] = occ[2 * o + 1];
      ++v;
    }
  }
}

__global__ void element_kernel(long long nocc, const long long* first, const unsigned* vid, int32_t* elements) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < nocc; o += (long long)gridDim.x * blockDim.x)
    elements[o] = int32_t(vid[first[o]]);
}

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);
  return s;
}
cc_status cuda_fail(cudaError_t e, const char* where) {
  cci::set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
  return CC_CUDA_ERR;
}

}  // namespace

// The contour the handle last built, until the next build or the handle's end.
struct cc_ms_mesh_store {
  void* verts = nullptr;
  int32_t* elements = nullptr;
  int64_t* cells = nullptr;
  long long nv = 0, ns = 0;
};

namespace {

void free_store(cc_handle* h) {
  cc_ms_mesh_store* st = static_cast<cc_ms_mesh_store*>(h->ms_mesh);
  if (!st) return;
  cudaFree(st->verts);
  cudaFree(st->elements);
  cudaFree(st->cells);
  delete st;
  h->ms_mesh = nullptr;
}

template <class T, bool MX>
cc_status build(cc_handle* h, const MsDomain<T>& D, cudaStream_t s, int64_t* nv, int64_t* ns) {
  free_store(h);
  const long long items = D.items();
  const long long nb = items > 0 ? (items + BLK - 1) / BLK : 1;
  unsigned long long *bsum = nullptr, *tot = nullptr;
  cudaError_t e = cudaMalloc(&bsum, (size_t(nb) + 4) * sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "generate_mesh scratch");
  tot = bsum + nb;
  seg_count_kernel<T, MX><<<unsigned(nb), MB, 0, s>>>(D, bsum);
  scan_kernel<<<1, MB, 0, s>>>(bsum, nb, tot);
  unsigned long long nseg = 0;
  if ((e = cudaGetLastError()) == cudaSuccess) e = cudaMemcpyAsync(&nseg, tot, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cc_ms_mesh_store* st = new cc_ms_mesh_store();
  h->ms_mesh = st;
  st->ns = (long long)nseg;
  const long long nocc = 2 * (long long)nseg;
  T* occ = nullptr;
  long long *owner = nullptr, *first = nullptr;
  unsigned long long* minocc = nullptr;
  unsigned* vid = nullptr;
  int* err = nullptr;
  unsigned long long size = 1;
  while (size < 4ull * (unsigned long long)(nocc > 0 ? nocc : 1)) size <<= 1;
  const long long nbo = nocc > 0 ? (nocc + BLK - 1) / BLK : 1;
  unsigned long long* osum = nullptr;
  if (e == cudaSuccess && nseg > 0) {
    e = cudaMalloc(&st->cells, nseg * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&st->elements, nocc * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&occ, nocc * 2 * sizeof(T));
    if (e == cudaSuccess) e = cudaMalloc(&owner, size * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&minocc, size * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&first, nocc * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&vid, nocc * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&osum, (size_t(nbo) + 2) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(owner, 0xff, size * sizeof(long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(minocc, 0xff, size * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess) {
      seg_emit_kernel<T, MX><<<unsigned(nb), MB, 0, s>>>(D, bsum, occ, st->cells);
      const int g = int(nocc / 256 + 1 < 148 * 8 ? nocc / 256 + 1 : 148 * 8);
      hash_insert_kernel<T><<<g, 256, 0, s>>>(occ, nocc, owner, minocc, size - 1, err);
      first_kernel<T><<<unsigned(nbo), MB, 0, s>>>(occ, nocc, owner, minocc, size - 1, first, osum);
      scan_kernel<<<1, MB, 0, s>>>(osum, nbo, osum + nbo);
      unsigned long long nvert = 0;
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(&nvert, osum + nbo, 8, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e == cudaSuccess) {
        st->nv = (long long)nvert;
        e = cudaMalloc(&st->verts, (nvert > 0 ? nvert : 1) * 2 * sizeof(T));
      }
      if (e == cudaSuccess) {
        vertex_kernel<T><<<unsigned(nbo), MB, 0, s>>>(occ, nocc, first, osum, vid, static_cast<T*>(st->verts));
        element_kernel<<<g, 256, 0, s>>>(nocc, first, vid, st->elements);
        e = cudaGetLastError();
      }
      int bad = 0;
      if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, err, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e == cudaSuccess && bad) {
        cudaFree(occ); cudaFree(owner); cudaFree(minocc); cudaFree(first); cudaFree(vid); cudaFree(osum);
        cudaFree(err); cudaFree(bsum);
        free_store(h);
        return fail(CC_CUDA_ERR, "generate_mesh: vertex table full");
      }
    }
  }
  cudaFree(occ); cudaFree(owner); cudaFree(minocc); cudaFree(first); cudaFree(vid); cudaFree(osum); cudaFree(err);
  cudaFree(bsum);
  if (e != cudaSuccess) {
    free_store(h);
    return cuda_fail(e, "generate_mesh");
  }
  if (nv) *nv = st->nv;
  if (ns) *ns = st->ns;
  return CC_OK;
}

template <class T>
MsDomain<T> grid_domain(const cc_grid* g, const void* phi) {
  MsDomain<T> D{};
  D.tree = 0;
  D.x0[0] = T(g->x0[0]); D.x0[1] = T(g->x0[1]);
  D.d[0] = T(g->d[0]); D.d[1] = T(g->d[1]);
  D.n0 = g->n[0];
  D.n1 = g->n[1];
  D.phi = static_cast<const T*>(phi);
  return D;
}

template <class T>
MsDomain<T> tree_domain(const cc_tree* t, const void* phi4) {
  MsDomain<T> D{};
  D.tree = 1;
  D.x0[0] = T(t->x0[0]); D.x0[1] = T(t->x0[1]);
  D.n0 = t->nleaves;
  D.base_d[0] = t->base_d[0]; D.base_d[1] = t->base_d[1];
  D.level = t->level;
  D.coord = t->coord;
  D.phi = static_cast<const T*>(phi4);
  return D;
}

struct DevGuard {
  int old = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&old);
    if (old != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (old >= 0 && cur != old) cudaSetDevice(old);
  }
};

}  // namespace

namespace cci {
void free_ms_mesh(cc_handle* h) { free_store(h); }
}  // namespace cci

extern "C" {

cc_status cc_ms_mesh_grid(cc_handle* h, const cc_grid* g, const void* phi, int64_t* n_vertices, int64_t* n_segments,
                          void* stream) {
  if (!h || !g || !phi) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_MARCHING_SQUARES || h->tree) return fail(CC_BAD_ARG, "not a grid marching-squares handle");
  if (g->dim != 2 || g->n[0] != h->n[0] || g->n[1] != h->n[1])
    return fail(CC_DIM_MISMATCH, "grid size differs from the cache's");
  DevGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (h->prec == CC_F64) return build<double, false>(h, grid_domain<double>(g, phi), s, n_vertices, n_segments);
  if (h->prec == CC_MIXED) return build<float, true>(h, grid_domain<float>(g, phi), s, n_vertices, n_segments);
  return build<float, false>(h, grid_domain<float>(g, phi), s, n_vertices, n_segments);
}

cc_status cc_ms_mesh_tree(cc_handle* h, const cc_tree* t, const void* phi4, int64_t* n_vertices, int64_t* n_segments,
                          void* stream) {
  if (!h || !t || !phi4) return fail(CC_BAD_ARG, "null argument");
  if (h->method != CC_MARCHING_SQUARES || !h->tree) return fail(CC_BAD_ARG, "not a tree marching-squares handle");
  if (t->nleaves != h->n[0]) return fail(CC_DIM_MISMATCH, "leaf count differs from the cache's");
  if (t->nleaves > 0 && (!t->level || !t->coord)) return fail(CC_BAD_ARG, "null leaf arrays");
  DevGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (h->prec == CC_F64) return build<double, false>(h, tree_domain<double>(t, phi4), s, n_vertices, n_segments);
  if (h->prec == CC_MIXED) return build<float, true>(h, tree_domain<float>(t, phi4), s, n_vertices, n_segments);
  return build<float, false>(h, tree_domain<float>(t, phi4), s, n_vertices, n_segments);
}

cc_status cc_ms_mesh_fetch(cc_handle* h, void* vertices, int32_t* segments, int64_t* cells, void* stream) {
  if (!h) return fail(CC_BAD_ARG, "null handle");
  cc_ms_mesh_store* st = static_cast<cc_ms_mesh_store*>(h->ms_mesh);
  if (!st) return fail(CC_BAD_ARG, "no contour built on this handle");
  DevGuard dg(h->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t es = h->prec == CC_F64 ? 8 : 4;
  cudaError_t e = cudaSuccess;
  if (vertices && st->nv > 0) e = cudaMemcpyAsync(vertices, st->verts, st->nv * 2 * es, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && segments && st->ns > 0)
    e = cudaMemcpyAsync(segments, st->elements, st->ns * 2 * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && cells && st->ns > 0)
    e = cudaMemcpyAsync(cells, st->cells, st->ns * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? CC_OK : cuda_fail(e, "generate_mesh fetch");
}

}  // extern "C"
