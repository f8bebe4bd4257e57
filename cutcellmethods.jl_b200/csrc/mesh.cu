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
// The surface lives in a thin band (about one node in a hundred at 512^3), so the passes first
// find it cheaply. A sign pass reads phi once and writes one bit per node (outside or not); every
// later test is word arithmetic on that bitmap, 32 nodes at a time: an edge crosses where its two
// nodes' bits differ, a cell is cut where its corners' bits are not all equal. A band count pass
// sums, per block of words, the cut nodes, their edge vertices (popcounts) and the cut cells; the
// block counts are scanned; a band list pass writes the cut nodes (with their first vertex and
// edge bits) and the cut cells in order into two flat lists. The long work -- each cut cell's
// tile for the triangle counts, the edge crossings, the triangles -- then runs over the lists one
// survivor per thread, so a block that a grid-aligned face fills with cut cells is no tail. The
// count call keeps the bitmap, the lists (whose capacity carries over between calls) and the
// scanned offsets on the handle, and an emit call that follows it for the same phi and grid, with
// no update in between, starts from them. The node emit stores each cut node's first vertex, so
// a cell's triangles can name the vertices of edges other nodes own. Every write of an emit is
// checked against the output capacities.
#include <cstdint>
#include <string>
#include <tuple>
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
constexpr int IPT = 4;           // rounds per block, one bitmap word per thread and round
constexpr int BW = MB * IPT;     // bitmap words per block (32768 nodes)

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

// outside(v) without the nudge: |v| < eps reads as +eps, so v is outside exactly when v > -eps
// (a NaN is neither).
template <class T>
__device__ __forceinline__ bool out_fast(T v) { return v > -Eps<T>::v(); }

// The sign bitmap. Node row r = j + ny k keeps its nx nodes in W 32-bit words, bit b of word w set
// when node i = 32 w + b is outside (bits past nx stay clear); word u = r W + w. Rows are padded to
// whole words so that every word lies in one row: its +y and +z neighbours are the words W and
// W ny further on, and a 32-node test is a few word operations.
// Quotient and remainder of a 32-bit value by a fixed divisor d >= 1 through one multiply-high
// (division by invariant integers, Granlund and Montgomery 1994): with m = floor((2^32 - 1) / d),
// umulhi(u, m) is floor(u / d) or one less, and a single correction step makes it exact.
struct FastDiv {
  unsigned d, m;
  static FastDiv of(unsigned d) { return FastDiv{d, 0xffffffffu / d}; }
  __device__ __forceinline__ unsigned div(unsigned u, unsigned& rem) const {
    unsigned q = __umulhi(u, m), r = u - q * d;
    if (r >= d) {
      ++q;
      r -= d;
    }
    rem = r;
    return q;
  }
};

struct Signs {
  unsigned* s;
  unsigned W, ny, words;
  int n0, n1, n2;
  FastDiv byW, byny;
};

// One warp per node row: lane b tests node 32 w + b of each of the row's W words in turn and a
// ballot forms the word. One load per lane in flight per warp, many warps per SM: on a 513^3
// Float32 field this read 5.2 TB/s where batches of 4, 8 and 16 loads per lane read 4.8, 4.1 and
// 3.5. No index needs a division.
template <class T>
__global__ void __launch_bounds__(256) sign_kernel(const T* __restrict__ phi, const Signs sg, unsigned nx,
                                                   unsigned rows) {
  const unsigned lane = threadIdx.x & 31u, r = blockIdx.x * 8u + (threadIdx.x >> 5);
  if (r >= rows) return;  // warp-uniform
  const T* __restrict__ row = phi + (size_t)nx * r;
  unsigned* __restrict__ out = sg.s + (size_t)sg.W * r;
  for (unsigned w = 0; w < sg.W; ++w) {
    const unsigned i = 32u * w + lane;
    const unsigned m = __ballot_sync(0xffffffffu, i < nx && out_fast(row[i < nx ? i : 0u]));
    if (lane == 0) out[w] = m;
  }
}

// The cuts of bitmap word u, one bit per node: its x, y and z edges to the next node that cross
// the surface (ax, ay, az), and the cut cells it is the lower corner of (cell). All zero past the
// last word. An edge crosses where its two nodes' bits differ; a cell is cut unless its eight
// corners share node (i, j, k)'s bit, i.e. unless the (j, k) face corners agree at i and at i + 1
// and bit i equals bit i + 1.
struct Cuts {
  unsigned ax, ay, az, cell;
};
__device__ __forceinline__ Cuts word_cuts(const Signs& sg, unsigned u) {
  const bool in = u < sg.words;
  const unsigned uc = in ? u : 0u;
  unsigned w, j;
  const unsigned r = sg.byW.div(uc, w), k = sg.byny.div(r, j);
  const bool hx = w + 1u < sg.W, hy = int(j) < sg.n1, hz = int(k) < sg.n2;
  const unsigned ox = hx ? 1u : 0u, oy = hy ? sg.W : 0u, oz = hz ? sg.W * sg.ny : 0u;
  const unsigned* p = sg.s + uc;  // every address below stays inside the bitmap
  const unsigned A = p[0], B = p[oy], C = p[oz], D = p[oy + oz];
  unsigned An = p[ox], Bn = p[oy + ox], Cn = p[oz + ox], Dn = p[oy + oz + ox];
  if (!hx) An = Bn = Cn = Dn = 0u;  // the row's last word: bit 31 is past n0 and masked below
  const int lo = sg.n0 - int(32u * w);
  const unsigned xm = lo >= 32 ? 0xffffffffu : lo <= 0 ? 0u : (1u << lo) - 1u;  // nodes with i < n0
  Cuts c{0u, 0u, 0u, 0u};
  if (!in) return c;
  c.ax = (A ^ ((A >> 1) | (An << 31))) & xm;
  c.ay = A ^ B;  // B is A itself on the last row along y, C on the last layer along z
  c.az = A ^ C;
  const unsigned d = (A ^ B) | (A ^ C) | (A ^ D), dn = (An ^ Bn) | (An ^ Cn) | (An ^ Dn);
  c.cell = hy && hz ? (d | (d >> 1) | (dn << 31) | c.ax) & xm : 0u;
  return c;
}

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

// ---- the band: per block of words, its cut nodes, their edge vertices and its cut cells -------
__global__ void __launch_bounds__(MB) band_count_kernel(const Signs sg, unsigned long long* bsum) {
  const unsigned u0 = blockIdx.x * unsigned(BW);
  unsigned long long packed = 0;  // cut nodes | edge vertices << 21 | cut cells << 42, each < 2^21
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    const Cuts c = word_cuts(sg, u0 + q * MB + threadIdx.x);
    packed += (unsigned long long)__popc(c.ax | c.ay | c.az) +
              ((unsigned long long)(__popc(c.ax) + __popc(c.ay) + __popc(c.az)) << 21) +
              ((unsigned long long)__popc(c.cell) << 42);
  }
  unsigned long long t;
  cccompact::block_scan<MB>(packed, &t);
  if (threadIdx.x == 0) {
    bsum[3 * blockIdx.x] = t & 0x1fffffull;
    bsum[3 * blockIdx.x + 1] = (t >> 21) & 0x1fffffull;
    bsum[3 * blockIdx.x + 2] = t >> 42;
  }
}

// Writes the block's cut nodes (node, first vertex, edge bits) and cut cells (lower node) at
// their places in the two ordered lists, as far as the lists' capacities reach. Each word's owner
// writes its own bits: the writes are short, and the long work runs later on the flat lists, one
// survivor per thread.
__global__ void __launch_bounds__(MB) band_list_kernel(const Signs sg, unsigned nx,
                                                       const unsigned long long* __restrict__ boff,
                                                       const unsigned long long* __restrict__ tot,
                                                       uint4* __restrict__ nodes, unsigned long long node_cap,
                                                       unsigned* __restrict__ cells, unsigned long long cell_cap) {
  const unsigned u0 = blockIdx.x * unsigned(BW);
  const unsigned long long nb = boff[3 * blockIdx.x], vb = boff[3 * blockIdx.x + 1], cb = boff[3 * blockIdx.x + 2];
  // the block's own counts, from the next block's offsets (the totals after the last block)
  const unsigned long long* next = blockIdx.x + 1 < gridDim.x ? boff + 3 * (blockIdx.x + 1) : tot;
  if (next[0] == nb && next[2] == cb) return;  // block-uniform: no cut node, no cut cell
  unsigned ax[IPT], ay[IPT], az[IPT], cm[IPT];
  unsigned long long cnt[IPT], pre[IPT];  // cut nodes | edge vertices << 21 | cut cells << 42
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    const Cuts c = word_cuts(sg, u0 + q * MB + threadIdx.x);
    ax[q] = c.ax;
    ay[q] = c.ay;
    az[q] = c.az;
    cm[q] = c.cell;
    cnt[q] = (unsigned long long)__popc(c.ax | c.ay | c.az) +
             ((unsigned long long)(__popc(c.ax) + __popc(c.ay) + __popc(c.az)) << 21) +
             ((unsigned long long)__popc(c.cell) << 42);
  }
  cccompact::round_prefix<MB, IPT>(cnt, pre);
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    const unsigned u = u0 + q * MB + threadIdx.x;
    if (u >= sg.words) continue;
    unsigned w;
    const unsigned r = sg.byW.div(u, w), v0 = 32u * w + nx * r;  // the node of bit 0
    unsigned bits = ax[q] | ay[q] | az[q];
    unsigned long long x = nb + (pre[q] & 0x1fffffull), vid = vb + ((pre[q] >> 21) & 0x1fffffull);
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1u;
      const unsigned m = (ax[q] >> b & 1u) | (ay[q] >> b & 1u) << 1 | (az[q] >> b & 1u) << 2;
      if (x < node_cap) nodes[x] = make_uint4(v0 + unsigned(b), unsigned(vid), m, 0u);
      ++x;
      vid += __popc(m);
    }
    bits = cm[q];
    x = cb + (pre[q] >> 42);
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1u;
      if (x < cell_cap) cells[x] = v0 + unsigned(b);
      ++x;
    }
  }
}

struct NodeDiv {
  FastDiv bynx, byny;
};
__device__ __forceinline__ void split_node(unsigned v, const NodeDiv& nd, long long& i, long long& j, long long& k) {
  unsigned ri, rj;
  const unsigned r = nd.bynx.div(v, ri), rk = nd.byny.div(r, rj);
  i = ri;
  j = rj;
  k = rk;
}

// Per block of MB cut cells: its triangles and interior vertices. The list holds
// min(*n_cells, cap) cells (the count is read on the device; blocks past it write zeros).
template <class T, bool MX>
__global__ void __launch_bounds__(MB) tile_count_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                        const NodeDiv nd, const DevTable tb,
                                                        const unsigned* __restrict__ cells,
                                                        const unsigned long long* __restrict__ n_cells,
                                                        unsigned long long cap, unsigned long long* bsum) {
  const unsigned long long n = *n_cells < cap ? *n_cells : cap;
  const unsigned long long x = (unsigned long long)blockIdx.x * MB + threadIdx.x;
  unsigned long long nt_it = 0;
  if (x < n) {
    long long i, j, k;
    split_node(cells[x], nd, i, j, k);
    T ph[8];
    corners(phi, g.n, i, j, k, ph);
    int nt, it;
    cell_tile<T, MX>(ph, tb, nt, it);
    nt_it = ((unsigned long long)nt << 32) | (unsigned long long)it;
  }
  unsigned long long t;
  cccompact::block_scan<MB>(nt_it, &t);
  if (threadIdx.x == 0) {
    bsum[2 * blockIdx.x] = t >> 32;
    bsum[2 * blockIdx.x + 1] = t & 0xffffffffull;
  }
}

// ---- the edge vertices: one cut node per thread ----------------------------------------------
template <class T>
__global__ void __launch_bounds__(MB) node_emit_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                       const NodeDiv nd, const uint4* __restrict__ nodes, unsigned long long n,
                                                       unsigned* __restrict__ vbase, T* __restrict__ verts,
                                                       unsigned long long vcap, unsigned long long* overflow) {
  const unsigned long long x = (unsigned long long)blockIdx.x * MB + threadIdx.x;
  if (x >= n) return;
  const uint4 e = nodes[x];
  unsigned long long id = e.y;
  long long i, j, k;
  split_node(e.x, nd, i, j, k);
  if (id + __popc(e.z) > vcap) {
    atomicOr(overflow, 1ull);
    return;
  }
  vbase[e.x] = unsigned(id);
  for (int a = 0; a < 3; ++a) {
    if (!(e.z >> a & 1u)) continue;
    T p[3];
    edge_vertex(phi, g, i, j, k, a, p);
    verts[3 * id] = p[0]; verts[3 * id + 1] = p[1]; verts[3 * id + 2] = p[2];
    ++id;
  }
}

// ---- the cells: triangles and interior vertices, one cut cell per thread ----------------------
template <class T, bool MX>
__global__ void __launch_bounds__(MB) cell_emit_kernel(const T* __restrict__ phi, const DevGrid<T> g,
                                                       const NodeDiv nd, const DevTable tb,
                                                       const unsigned* __restrict__ cells, unsigned long long n,
                                                       const unsigned long long* __restrict__ boff,
                                                       const unsigned* __restrict__ vbase,
                                                       unsigned long long n_edge_verts, T* __restrict__ verts,
                                                       unsigned long long vcap, int32_t* __restrict__ tris,
                                                       unsigned long long tcap, int64_t* __restrict__ tri_cells,
                                                       unsigned long long* overflow) {
  const unsigned long long x = (unsigned long long)blockIdx.x * MB + threadIdx.x;
  const unsigned long long tri0 = boff[2 * blockIdx.x], int0 = n_edge_verts + boff[2 * blockIdx.x + 1];
  long long i = 0, j = 0, k = 0;
  T ph[8];
  int nt = 0, it = 0, tile = -1;
  if (x < n) {
    split_node(cells[x], nd, i, j, k);
    corners(phi, g.n, i, j, k, ph);
    tile = cell_tile<T, MX>(ph, tb, nt, it);
  }
  unsigned long long tot;
  const unsigned long long pre = cccompact::block_scan<MB>(((unsigned long long)nt << 32) | (unsigned long long)it, &tot);
  unsigned long long tri_id = tri0 + (pre >> 32);
  const unsigned long long int_id = int0 + (pre & 0xffffffffull);
  if (tile < 0) return;
  if (tri_id + nt > tcap || (it && int_id >= vcap)) {
    atomicOr(overflow, 1ull);
    return;
  }
  const long long c = i + g.n[0] * (j + g.n[1] * k);
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
  const long long nx = g.n[0] + 1, ny = g.n[1] + 1, nn = nx * ny * (g.n[2] + 1);
  const long long W = (nx + 31) / 32, words = W * ny * (g.n[2] + 1);
  const long long nb = (words + BW - 1) / BW;
  // 32-bit node and word indices, with room for the last block's words past the end
  if (nn > 0xffffffffLL || words > 0xffffffffLL - BW)
    return fail(CC_TOO_LARGE, "generate_mesh takes fewer than 2^32 nodes");
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
  // 64-bit words: per word block (cut nodes, edge vertices, cut cells) interleaved, their 3
  // totals, the 2 tile totals (triangles, interior vertices), the overflow flag; then the sign
  // bitmap, 32-bit words
  const size_t head = size_t(3 * nb + 6);
  const size_t scan_n = head + size_t(words + 1) / 2;
  if (scan_n > h->mesh_scan_n) {
    if (h->mesh_scan) cudaFree(h->mesh_scan);
    h->mesh_scan = nullptr;
    h->mesh_scan_n = 0;
    key.valid = false;
    if ((e = cudaMalloc(&h->mesh_scan, scan_n * sizeof(unsigned long long))) != cudaSuccess)
      return cuda_fail(e, "generate_mesh scratch");
    h->mesh_scan_n = scan_n;
  }
  unsigned long long* bsum = h->mesh_scan;  // per word block, then scanned in place
  unsigned long long* tot = bsum + 3 * nb;  // cut nodes, edge vertices, cut cells
  unsigned long long* tot2 = tot + 3;       // triangles, interior vertices
  unsigned long long* overflow = tot2 + 2;
  Signs sg;
  sg.s = reinterpret_cast<unsigned*>(h->mesh_scan + head);
  sg.W = unsigned(W);
  sg.ny = unsigned(ny);
  sg.words = unsigned(words);
  sg.n0 = int(g.n[0]);
  sg.n1 = int(g.n[1]);
  sg.n2 = int(g.n[2]);
  sg.byW = FastDiv::of(unsigned(W));
  sg.byny = FastDiv::of(unsigned(ny));
  const NodeDiv nd{FastDiv::of(unsigned(nx)), FastDiv::of(unsigned(ny))};
  const bool emit = verts || tris;
  bool reuse = emit && key.valid && key.generation == h->generation && key.phi == phi && key.prec == h->prec;
  for (int a = 0; a < 3 && reuse; ++a)
    reuse = key.g.n[a] == gg->n[a] && key.g.x0[a] == gg->x0[a] && key.g.d[a] == gg->d[a];
  unsigned long long t[3] = {key.tot[0], key.tot[1], key.tot[2]};
  unsigned long long n_nodes = key.cut_nodes, n_cells = key.cut_cells;
  // the lists, at the capacities kept on the handle: cut nodes (16 B each), per tile block
  // (triangles, interior vertices), cut cells (4 B each)
  auto lists = [&]() {
    const unsigned long long nc = h->mesh_node_cap, cc = h->mesh_cell_cap, ntb = (cc + MB - 1) / MB;
    return std::make_tuple(reinterpret_cast<uint4*>(h->mesh_list), h->mesh_list + 2 * nc,
                           reinterpret_cast<unsigned*>(h->mesh_list + 2 * nc + 2 * ntb), ntb);
  };
  if (!reuse) {
    key.valid = false;
    const long long rows = ny * (g.n[2] + 1);
    sign_kernel<T><<<unsigned((rows + 7) / 8), 256, 0, s>>>(phi, sg, unsigned(nx), unsigned(rows));
    band_count_kernel<<<unsigned(nb), MB, 0, s>>>(sg, bsum);
    cccompact::scan_series_kernel<512, 3><<<3, 512, 0, s>>>(bsum, nb, tot);
    // the list pass and the tile counts, into the lists as they are; run again below when the
    // surface has outgrown them (the first call on a handle, or a larger surface)
    auto list_pass = [&]() {
      auto [nodes, tsum, cells, ntb] = lists();
      band_list_kernel<<<unsigned(nb), MB, 0, s>>>(sg, unsigned(nx), bsum, tot, nodes, h->mesh_node_cap, cells,
                                                   h->mesh_cell_cap);
      if (ntb > 0) {
        tile_count_kernel<T, MX><<<unsigned(ntb), MB, 0, s>>>(phi, g, nd, h->tb, cells, tot + 2, h->mesh_cell_cap,
                                                             tsum);
        cccompact::scan_series_kernel<512, 2><<<2, 512, 0, s>>>(tsum, (long long)ntb, tot2);
      } else {
        cudaMemsetAsync(tot2, 0, 2 * sizeof(unsigned long long), s);
      }
    };
    unsigned long long c5[5];  // cut nodes, edge vertices, cut cells, triangles, interior vertices
    if (h->mesh_list) list_pass();
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaMemcpyAsync(c5, tot, sizeof c5, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "generate_mesh count");
    n_nodes = c5[0];
    n_cells = c5[2];
    if (!h->mesh_list || n_nodes > h->mesh_node_cap || n_cells > h->mesh_cell_cap) {
      // grow with an eighth to spare, so that a slightly larger surface next time fits
      const unsigned long long nc = n_nodes + n_nodes / 8 + 1024, cc = n_cells + n_cells / 8 + 1024;
      const size_t list_n = size_t(2 * nc + 2 * ((cc + MB - 1) / MB) + (cc + 1) / 2);
      if (h->mesh_list) cudaFree(h->mesh_list);
      h->mesh_list = nullptr;
      h->mesh_node_cap = h->mesh_cell_cap = 0;
      if ((e = cudaMalloc(&h->mesh_list, list_n * sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(e, "generate_mesh scratch");
      h->mesh_node_cap = nc;
      h->mesh_cell_cap = cc;
      list_pass();
      if ((e = cudaGetLastError()) == cudaSuccess)
        e = cudaMemcpyAsync(c5 + 3, tot2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return cuda_fail(e, "generate_mesh count");
    }
    t[0] = c5[1];
    t[1] = c5[3];
    t[2] = c5[4];
    key.valid = true;
    key.generation = h->generation;
    key.phi = phi;
    key.prec = h->prec;
    key.g = *gg;
    for (int q = 0; q < 3; ++q) key.tot[q] = t[q];
    key.cut_nodes = n_nodes;
    key.cut_cells = n_cells;
  }
  const long long n_vert = (long long)(t[0] + t[2]), n_tri = (long long)t[1];
  if (nv) *nv = n_vert;
  if (nt) *nt = n_tri;
  if (!emit) return CC_OK;  // counting only
  if (!verts || !tris || vcap < n_vert || tcap < n_tri)
    return fail(CC_BAD_ARG, "generate_mesh output smaller than the counted surface");
  if (n_vert > 0xffffffffLL) return fail(CC_TOO_LARGE, "generate_mesh numbers at most 2^32 - 1 vertices");
  auto [nodes, tsum, cells, ntb_cap] = lists();
  (void)ntb_cap;
  const unsigned long long ntb = (n_cells + MB - 1) / MB;
  unsigned long long flag = 0;
  e = cudaMemsetAsync(overflow, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess && n_nodes > 0)
    node_emit_kernel<T><<<unsigned((n_nodes + MB - 1) / MB), MB, 0, s>>>(phi, g, nd, nodes, n_nodes, h->mesh_vbase, verts,
                                                                        (unsigned long long)vcap, overflow);
  if (e == cudaSuccess && n_cells > 0)
    cell_emit_kernel<T, MX><<<unsigned(ntb), MB, 0, s>>>(phi, g, nd, h->tb, cells, n_cells, tsum, h->mesh_vbase, t[0],
                                                        verts, (unsigned long long)vcap, tris, (unsigned long long)tcap,
                                                        tri_cells, overflow);
  if (e == cudaSuccess) e = cudaGetLastError();
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
