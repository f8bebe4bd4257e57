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
// Only a thin band of entries draws anything, and its clip (edge crossings, angle sort, fan) is long
// and branchy, so the passes separate the streaming from the clipping. A filter pass reads every
// plane once and writes a bitmap of the entries that may draw (a conservative plane-misses-cell
// test) with per-block counts; after a scan, a list pass writes those entries in order; a clip
// pass counts each listed entry's nodes and elements, one entry per thread, and after a second
// scan the emit pass clips them again and writes at the scanned offsets. The output is in entry
// order with no atomics.
#include <cstdint>
#include <string>
#include <utility>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"
#include "compact.cuh"

namespace {

using namespace ccd;

constexpr int MB = 256;
constexpr int FR = 32;          // filter rounds per thread
constexpr int FBLK = MB * FR;   // entries per filter block (256 bitmap words)
constexpr int LW = 4;           // filter blocks per list block: bitmap words per thread of the list pass

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
    // one strict sign at every corner: no corner on the line and no crossing (m stays 0)
    const bool miss = (s[0] > T(0) && s[1] > T(0) && s[2] > T(0) && s[3] > T(0)) ||
                      (s[0] < T(0) && s[1] < T(0) && s[2] < T(0) && s[3] < T(0));
    for (int k = 0; k < 4 && m < 2 && ok && !miss; ++k) {
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
  bool pos = true, neg = true;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    s[c] = ((nrm[0] * T(c & 1) + nrm[1] * T((c >> 1) & 1)) + nrm[2] * T((c >> 2) & 1)) - a;
    pos = pos && s[c] > T(0);
    neg = neg && s[c] < T(0);
  }
  // one strict sign at every corner: no corner on the plane and no crossing -- most cells
  if (pos || neg) return 0;
  for (int c = 0; c < 8 && m < 6; ++c)
    if (s[c] == T(0)) { xi[m][0] = T(c & 1); xi[m][1] = T((c >> 1) & 1); xi[m][2] = T((c >> 2) & 1); ++m; }
  // the 12 edges, x-edges then y- then z-: edge j of axis ax runs from corner p (bit ax clear,
  // the other two bits j) to p | 1 << ax
  for (int k = 0; k < 12 && m < 6; ++k) {
    const int ax0 = k >> 2, j = k & 3;
    const int p = ((j >> ax0) << (ax0 + 1)) | (j & ((1 << ax0) - 1)), q = p | (1 << ax0);
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

// True when entry k certainly draws nothing: a degenerate fit, or a plane that misses its cell
// by more than rounding (3D), or -- in 2D -- such a miss when the length floor drops the
// zero-length segment it leaves. Conservative: a true here implies clip_cell + cell_counts give no
// node, a false only sends the entry to the full clip. The cube's (square's) corner values
// n . c - a span [sum min(n_i, 0) - a, sum max(n_i, 0) - a]; the full clip's corner sums are
// within 3 u (|n|_1 + |a|) of exact (u the unit roundoff), these bounds within 2 u |n|_1, so a gap
// of 64 u (|n|_1 + |a|) leaves every corner value one strict sign. NaN or inf fails both tests.
template <class T, int D>
__device__ __forceinline__ bool draws_nothing(const PlicIn<T, D>& P, T n0, T n1, T n2, T a, bool ok, T min_d) {
  const T zero = T(0);
  const T lo = (fmin(n0, zero) + fmin(n1, zero)) + fmin(n2, zero);
  const T hi = (fmax(n0, zero) + fmax(n1, zero)) + fmax(n2, zero);
  const T tol = (sizeof(T) == 4 ? T(0x1p-18) : T(0x1p-47)) * (((fabs(n0) + fabs(n1)) + fabs(n2)) + fabs(a));
  const bool miss = (a - hi > tol) || (lo - a > tol);
  if (D == 2) return (!ok || miss) && !(T(0) >= P.min_frac * min_d);
  return !ok || miss;
}

// ---- the filter: a bitmap of the entries that may draw something ------------------------------
// Bit b of word w is set when entry 32 w + b may draw something (draws_nothing is false); bsum gets
// each block's count. Thread t tests entry q*MB + t of its block in round q, so a warp's ballot is
// one word; G rounds' planes are loaded (the index clamped to the block's last entry) before any
// is tested. No clip runs here: the pass streams the planes once.
template <class T, int D>
__global__ void __launch_bounds__(MB) plic_filter_kernel(const PlicIn<T, D> P, T min_d, unsigned* __restrict__ bits,
                                                         unsigned long long* __restrict__ bsum) {
  constexpr int G = 2;
  const long long start = (long long)blockIdx.x * FBLK;
  // this block's entries, addressed by 32-bit offsets
  const int here = P.count - start < FBLK ? int(P.count - start) : FBLK;
  const T* nrm = P.normals + D * start;
  const T* icp = P.intercepts + start;
  const uint8_t* val = P.valid ? P.valid + start : nullptr;
  unsigned* wbits = bits + start / 32;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  unsigned long long cnt = 0;
  for (int q0 = 0; q0 < FR; q0 += G) {
    T n0[G], n1[G], n2[G], a[G];
    bool ok[G];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int r = (q0 + u) * MB + threadIdx.x;
      const int rr = r < here ? r : here - 1;
      n0[u] = nrm[D * rr];
      n1[u] = nrm[D * rr + 1];
      n2[u] = D == 3 ? nrm[D * rr + 2] : T(0);
      a[u] = icp[rr];
      ok[u] = val ? val[rr] != 0 : true;
    }
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int r = (q0 + u) * MB + threadIdx.x;
      const bool okk = val ? ok[u] : (n0[u] != T(0) || n1[u] != T(0) || n2[u] != T(0));
      const unsigned m = __ballot_sync(0xffffffffu, r < here && !draws_nothing<T, D>(P, n0[u], n1[u], n2[u], a[u], okk, min_d));
      const int first = (q0 + u) * MB + wp * 32;  // the word's first entry in the block
      if (lane == 0 && first < here) {
        wbits[first / 32] = m;
        cnt += __popc(m);
      }
    }
  }
  unsigned long long t;
  cccompact::block_scan<MB>(cnt, &t);
  if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

// Writes the surviving entries of LW consecutive filter blocks, in order, at their places in the
// list (as far as its capacity reaches). Thread t takes word q*MB + t in round q, so round q is
// filter block LW * blockIdx.x + q, and boff (the filter blocks' scanned counts) places the first.
__global__ void __launch_bounds__(MB) plic_list_kernel(const unsigned* __restrict__ bits, long long nwords,
                                                       const unsigned long long* __restrict__ boff, long long nb,
                                                       const unsigned long long* __restrict__ total,
                                                       unsigned long long* __restrict__ list, unsigned long long cap) {
  static_assert(FBLK / 32 == MB, "one filter block per round");
  const unsigned long long off = boff[(long long)blockIdx.x * LW];
  // the block's own count, from the next list block's offset (the total after the last)
  const long long nxt = (long long)(blockIdx.x + 1) * LW;
  if ((nxt < nb ? boff[nxt] : *total) == off) return;  // block-uniform: no surviving entry
  const long long w0 = (long long)blockIdx.x * (MB * LW) + threadIdx.x;
  unsigned m[LW];
  unsigned long long cnt[LW], pre[LW];
#pragma unroll
  for (int q = 0; q < LW; ++q) {
    m[q] = w0 + q * MB < nwords ? bits[w0 + q * MB] : 0u;
    cnt[q] = __popc(m[q]);
  }
  cccompact::round_prefix<MB, LW>(cnt, pre);
#pragma unroll
  for (int q = 0; q < LW; ++q) {
    unsigned long long x = off + pre[q];
    const unsigned long long e0 = 32ull * (unsigned long long)(w0 + q * MB);
    while (m[q]) {
      const int b = __ffs(m[q]) - 1;
      m[q] &= m[q] - 1u;
      if (x < cap) list[x] = e0 + unsigned(b);
      ++x;
    }
  }
}

// A listed entry's clip, kept by the clip pass for the emit pass: its polygon, coordinate (v, q) at
// poly[(3 v + q) * cap + x] (one plane per coordinate, so a warp's stores and loads coalesce), and
// a packed word: vertex count m | nodes << 3 | elements << 6 | fan keep bits << 9.
template <class T>
struct Clips {
  T* poly;
  unsigned* info;
  unsigned long long cap;
};

// Per block of MB listed entries: the nodes and elements they draw, packed (nodes high, elements
// low), and each entry's clip kept for the emit. The list holds min(*n_list, cap) entries (the
// count is read on the device; blocks past it write zeros).
template <class T, int D>
__global__ void __launch_bounds__(MB) plic_clip_count_kernel(const PlicIn<T, D> P, T min_d,
                                                             const unsigned long long* __restrict__ list,
                                                             const unsigned long long* __restrict__ n_list,
                                                             const Clips<T> C, unsigned long long* tsum) {
  const unsigned long long n = *n_list < C.cap ? *n_list : C.cap;
  const unsigned long long x = (unsigned long long)blockIdx.x * MB + threadIdx.x;
  unsigned long long packed = 0;
  if (x < n) {
    T p[6][3];
    const int m = clip_cell<T, D>(P, (long long)list[x], p);
    int a, b;
    unsigned keep;
    cell_counts<T, D>(P, m, p, min_d, a, b, keep);
    packed = ((unsigned long long)a << 32) | (unsigned long long)b;
    C.info[x] = unsigned(m) | unsigned(a) << 3 | unsigned(b) << 6 | keep << 9;
    for (int v = 0; v < a; ++v)
#pragma unroll
      for (int q = 0; q < D; ++q) C.poly[(size_t)(3 * v + q) * C.cap + x] = p[v][q];
  }
  unsigned long long t;
  cccompact::block_scan<MB>(packed, &t);
  if (threadIdx.x == 0) {
    tsum[2 * blockIdx.x] = t >> 32;
    tsum[2 * blockIdx.x + 1] = t & 0xffffffffull;
  }
}

// One listed entry per thread: its kept clip written at the scanned offsets of its block. The
// writes are checked against the output capacities: offsets from a count of other planes (a
// caller that changed them between its two calls) raise *overflow instead of writing past the end.
template <class T, int D>
__global__ void __launch_bounds__(MB) plic_emit_kernel(const PlicIn<T, D> P, const unsigned long long* __restrict__ list,
                                                       unsigned long long n, const Clips<T> C,
                                                       const unsigned long long* __restrict__ boff, T* nodes,
                                                       unsigned long long ncap, int32_t* elems, unsigned long long ecap,
                                                       int64_t* cells, unsigned long long* overflow) {
  const unsigned long long x = (unsigned long long)blockIdx.x * MB + threadIdx.x;
  const unsigned long long node0 = boff[2 * blockIdx.x], elem0 = boff[2 * blockIdx.x + 1];
  const unsigned info = x < n ? C.info[x] : 0u;
  const int m = int(info & 7u), a = int(info >> 3 & 7u), b = int(info >> 6 & 7u);
  const unsigned keep = info >> 9;
  unsigned long long t;
  const unsigned long long pre = cccompact::block_scan<MB>(((unsigned long long)a << 32) | (unsigned long long)b, &t);
  const unsigned long long vn = node0 + (pre >> 32);
  unsigned long long ve = elem0 + (pre & 0xffffffffull);
  if (a == 0) return;
  if (vn + a > ncap || ve + b > ecap) {
    atomicOr(overflow, 1ull);
    return;
  }
  const long long k = (long long)list[x];
  const long long ci = P.index ? (long long)P.index[k] : k;
  for (int v = 0; v < a; ++v)
#pragma unroll
    for (int q = 0; q < D; ++q) nodes[D * (vn + v) + q] = C.poly[(size_t)(3 * v + q) * C.cap + x];
  if (D == 2) {
    if (b) {
      elems[2 * ve] = int32_t(vn);
      elems[2 * ve + 1] = int32_t(vn + 1);
      cells[ve] = ci;
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
}

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);
  return s;
}
cc_status cuda_fail(cudaError_t e, const char* where) {
  cci::set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
  return CC_CUDA_ERR;
}

// A surface count kept on a handle between the count call and the emit call of generate_mesh:
// the bitmap, block counts and totals, the list of surviving entries with its per-block clip counts
// (scanned), and what they were counted from. The list keeps its capacity across calls.
struct Stored {
  unsigned long long* bsum = nullptr;  // filter block counts, totals, overflow flag; then the bitmap
  size_t cap = 0;                      // 64-bit words of bsum
  // surviving entries; per list block (nodes, elements); the clips (18 coordinates, 1 info word each)
  unsigned long long* list = nullptr;
  unsigned long long list_cap = 0;     // entries the list holds
  bool valid = false;
  uint64_t generation = 0;
  const void *normals = nullptr, *intercepts = nullptr, *is_valid = nullptr;
  cc_grid g{};
  double min_frac = 0.0;
  int prec = -1;
  unsigned long long tot[2] = {0, 0};
  unsigned long long listed = 0;  // surviving entries of the kept count
  bool same(const cc_handle* h, const cc_grid* gg, const void* n, const void* i, const void* v, double f) const {
    if (!valid || generation != h->generation || normals != n || intercepts != i || is_valid != v ||
        prec != h->prec || min_frac != f || g.dim != gg->dim)
      return false;
    for (int a = 0; a < gg->dim; ++a)
      if (g.n[a] != gg->n[a] || g.x0[a] != gg->x0[a] || g.d[a] != gg->d[a]) return false;
    return true;
  }
  void release() {
    if (bsum) cudaFree(bsum);
    if (list) cudaFree(list);
    bsum = list = nullptr;
    cap = 0;
    list_cap = 0;
  }
};

template <class T, int D>
cc_status run(const cc_grid* g, const void* normals, const void* intercepts, const uint8_t* valid,
              const int64_t* index, int64_t count, double min_frac, void* nodes, int64_t ncap, int32_t* elems,
              int64_t ecap, int64_t* cells, int64_t* n_nodes, int64_t* n_elems, cudaStream_t s, cc_handle* h) {
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
  const long long nb = (nc + FBLK - 1) / FBLK, nwords = (nc + 31) / 32;
  const long long nlb = (nb + LW - 1) / LW;  // list blocks
  // bsum: nb filter block counts, their total, 2 clip totals (nodes, elements), the overflow flag;
  // then the bitmap (FBLK / 32 32-bit words per block, LW blocks per list block)
  const size_t head = size_t(nb) + 4;
  const size_t need = head + size_t(nlb * LW) * (FBLK / 64);
  const bool emit = nodes || elems;
  // With a handle the buffers are kept, and an emit call right after a count of the same planes
  // (same update, arrays, grid and fraction) starts from that count's list and offsets.
  Stored local;
  Stored* st = &local;
  if (h) {
    if (!h->plic_mesh) h->plic_mesh = new Stored();
    st = static_cast<Stored*>(h->plic_mesh);
  }
  auto release = [&]() {
    if (!h) local.release();
  };
  cudaError_t e = cudaSuccess;
  if (st->cap < need) {
    if (st->bsum) cudaFree(st->bsum);
    st->bsum = nullptr;
    st->cap = 0;
    st->valid = false;
    if ((e = cudaMalloc(&st->bsum, need * sizeof(unsigned long long))) != cudaSuccess) {
      release();
      return cuda_fail(e, "generate_mesh scratch");
    }
    st->cap = need;
  }
  const bool reuse = h && emit && st->same(h, g, normals, intercepts, valid, min_frac);
  unsigned long long* bsum = st->bsum;
  unsigned long long* tot1 = bsum + nb;   // surviving entries
  unsigned long long* tot2 = tot1 + 1;    // nodes, elements
  unsigned long long* overflow = tot2 + 2;
  unsigned* bits = reinterpret_cast<unsigned*>(bsum + head);
  // the list: cap entries, 2 * ntb per-block counts, then the clips
  auto ntb_of = [](unsigned long long cap) { return (cap + MB - 1) / MB; };
  auto list_words = [&](unsigned long long cap) {
    return size_t(cap + 2 * ntb_of(cap)) + (size_t(cap) * (18 * sizeof(T) + sizeof(unsigned)) + 7) / 8;
  };
  auto clips = [&]() {
    Clips<T> c;
    c.cap = st->list_cap;
    c.poly = reinterpret_cast<T*>(st->list + c.cap + 2 * ntb_of(c.cap));
    c.info = reinterpret_cast<unsigned*>(c.poly + 18 * c.cap);
    return c;
  };
  unsigned long long tot[2] = {st->tot[0], st->tot[1]};
  unsigned long long listed = st->listed;
  if (!reuse) {
    st->valid = false;
    plic_filter_kernel<T, D><<<unsigned(nb), MB, 0, s>>>(P, min_d, bits, bsum);
    cccompact::scan_series_kernel<512, 1, 16><<<1, 512, 0, s>>>(bsum, nb, tot1);
    // the list and its clip counts, into the list as it is; run again below when the surface has
    // outgrown it (the first call on a handle, or a larger surface)
    auto list_pass = [&]() {
      const unsigned long long ntb = ntb_of(st->list_cap);
      unsigned long long* tsum = st->list + st->list_cap;
      plic_list_kernel<<<unsigned(nlb), MB, 0, s>>>(bits, nwords, bsum, nb, tot1, st->list, st->list_cap);
      plic_clip_count_kernel<T, D><<<unsigned(ntb), MB, 0, s>>>(P, min_d, st->list, tot1, clips(), tsum);
      cccompact::scan_series_kernel<512, 2><<<2, 512, 0, s>>>(tsum, (long long)ntb, tot2);
    };
    unsigned long long c3[3];  // surviving entries, nodes, elements
    if (st->list) list_pass();
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaMemcpyAsync(c3, tot1, sizeof c3, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && (!st->list || c3[0] > st->list_cap)) {
      // grow with an eighth to spare, so that a slightly larger surface next time fits
      const unsigned long long lc = c3[0] + c3[0] / 8 + 1024;
      if (st->list) cudaFree(st->list);
      st->list = nullptr;
      st->list_cap = 0;
      if ((e = cudaMalloc(&st->list, list_words(lc) * sizeof(unsigned long long))) == cudaSuccess) {
        st->list_cap = lc;
        list_pass();
        if ((e = cudaGetLastError()) == cudaSuccess)
          e = cudaMemcpyAsync(c3 + 1, tot2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      }
    }
    if (e != cudaSuccess) {
      release();
      return cuda_fail(e, "generate_mesh count");
    }
    listed = c3[0];
    tot[0] = c3[1];
    tot[1] = c3[2];
    if (h) {
      st->valid = true;
      st->generation = h->generation;
      st->normals = normals;
      st->intercepts = intercepts;
      st->is_valid = valid;
      st->g = *g;
      st->min_frac = min_frac;
      st->prec = h->prec;
      st->tot[0] = tot[0];
      st->tot[1] = tot[1];
      st->listed = listed;
    }
  }
  if (n_nodes) *n_nodes = (int64_t)tot[0];
  if (n_elems) *n_elems = (int64_t)tot[1];
  if (tot[0] > 0x7fffffffull) {
    release();
    return fail(CC_TOO_LARGE, "generate_mesh: more nodes than int32 element indices address");
  }
  if (emit) {
    if (!nodes || !elems || !cells || ncap < (int64_t)tot[0] || ecap < (int64_t)tot[1]) {
      release();
      return fail(CC_BAD_ARG, "generate_mesh output smaller than the counted surface");
    }
    unsigned long long flag = 0;
    if (tot[1] > 0) {
      const unsigned long long* tsum = st->list + st->list_cap;
      e = cudaMemsetAsync(overflow, 0, sizeof(unsigned long long), s);
      if (e == cudaSuccess) {
        plic_emit_kernel<T, D><<<unsigned((listed + MB - 1) / MB), MB, 0, s>>>(
            P, st->list, listed, clips(), tsum, static_cast<T*>(nodes), (unsigned long long)ncap, elems,
            (unsigned long long)ecap, cells, overflow);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, overflow, sizeof flag, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (h) st->valid = false;  // one emit per count
    if (e == cudaSuccess && flag) {
      release();
      return fail(CC_BAD_ARG, "generate_mesh: the planes changed between the count and the emit call");
    }
  }
  release();
  return e == cudaSuccess ? CC_OK : cuda_fail(e, "generate_mesh");
}

cc_status surface(int prec, const cc_grid* g, const void* normals, const void* intercepts, const uint8_t* valid,
                  const int64_t* index, int64_t count, double min_frac, void* nodes, int64_t ncap, int32_t* elems,
                  int64_t ecap, int64_t* cells, int64_t* n_nodes, int64_t* n_elems, cudaStream_t s, cc_handle* h) {
  if (prec == CC_F64)
    return g->dim == 3 ? run<double, 3>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                        cells, n_nodes, n_elems, s, h)
                       : run<double, 2>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                        cells, n_nodes, n_elems, s, h);
  return g->dim == 3 ? run<float, 3>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                     cells, n_nodes, n_elems, s, h)
                     : run<float, 2>(g, normals, intercepts, valid, index, count, min_frac, nodes, ncap, elems, ecap,
                                     cells, n_nodes, n_elems, s, h);
}

}  // namespace

namespace cci {
void free_plic_mesh(cc_handle* h) {
  if (!h || !h->plic_mesh) return;
  Stored* st = static_cast<Stored*>(h->plic_mesh);
  st->release();
  delete st;
  h->plic_mesh = nullptr;
}
}  // namespace cci

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
                 static_cast<cudaStream_t>(stream), nullptr);
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
                               static_cast<cudaStream_t>(stream), h);
  if (old >= 0 && old != h->device) cudaSetDevice(old);
  return st;
}

}  // extern "C"
