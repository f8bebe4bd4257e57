// plic.cu -- PLICCutCell update_cache!, calc_volume and cut_cell_report on sm_100a.
//
// Fit pass (_plic_fit_kernel!, src/plic/cache.jl:96-113): per cell one forward-mode evaluation of
// the op-tape at the centroid gives (dist, normal) -- get_sdf -- and cell_plane
// (src/plic/plic.jl:72-88) turns it into the stored plane. Face pass
// (_plic_face_fraction_kernel!, src/plic/cache.jl:118-162): per cell, per face, the mean of the
// two one-sided candidates evaluated from the two cells' stored planes by the same _face_area
// (src/plic/apertures.jl:112-125), so both cells of a face compute identical bits.
#include <cstdint>
#include "cc_device.cuh"
#include "cc_internal.h"

namespace {

using namespace ccd;
using cci::Cols;
using cci::DevGrid;
using cci::DevTape;

constexpr int NT = 256;
constexpr int VOL_BLOCKS = 148 * 8;

template <class T, int D>
struct PlaneFit {
  T n[D];
  T a;
  T fraction;
  bool valid;
};

// cell_plane, src/plic/plic.jl:72-88 (with MX the plane-cube clip runs in FP64)
template <class T, int D, bool MX>
__device__ __forceinline__ PlaneFit<T, D> cell_plane(const STape<T>& t, const DevGrid<T>& g, const long long idx[3]) {
  Dual<T, D> x[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    x[a].v = centroid_coord(g.x0[a], g.d[a], idx[a]);
#pragma unroll
    for (int b = 0; b < D; ++b) x[a].g[b] = a == b ? T(1) : T(0);
  }
  const Dual<T, D> r = tape_eval<T, D, Dual<T, D>>(t, x);
  T s = r.g[0];
#pragma unroll
  for (int a = 1; a < D; ++a) s = s + r.g[a];
  const T a = T(0.5) * s - r.v / g.d[0];
  bool allzero = true;
#pragma unroll
  for (int q = 0; q < D; ++q) allzero = allzero && (r.g[q] == T(0));
  PlaneFit<T, D> pl;
  if (isnan(a) || allzero) {
#pragma unroll
    for (int q = 0; q < D; ++q) pl.n[q] = T(0);
    pl.a = T(0);
    pl.fraction = r.v <= T(0) ? T(1) : T(0);
    pl.valid = false;
    return pl;
  }
#pragma unroll
  for (int q = 0; q < D; ++q) pl.n[q] = r.g[q];
  pl.a = a;
  if constexpr (D == 2) pl.fraction = gvf2m<T, MX>(r.g[0], r.g[1], a);
  else pl.fraction = gvf3m<T, MX>(r.g[0], r.g[1], r.g[D - 1], a);
  pl.valid = true;
  return pl;
}

// The cell tiles the centroid kernels work in: NT cells, 32 along x (coalesced stores), and the
// tape pruned to the box of each tile's centroids when the body is a union of spheres.
template <int D> struct PTile;
template <> struct PTile<3> { static constexpr int X = 32, Y = 4, Z = 2; };
template <> struct PTile<2> { static constexpr int X = 32, Y = 8, Z = 1; };

// Tile t's first cell, tiles numbered x fastest, from 32-bit quotients (a grid has far fewer
// than 2^32 tiles: that would be 2^40 cells).
template <int D>
__device__ __forceinline__ void tile_origin(unsigned t, unsigned tx, unsigned ty, long long i0[3]) {
  const unsigned a = t / tx, b = a / ty;
  i0[0] = (long long)(t - a * tx) * PTile<D>::X;
  i0[1] = (long long)(a - b * ty) * PTile<D>::Y;
  i0[2] = (long long)b * PTile<D>::Z;
}

// Shared-memory layout of a centroid kernel: the tape, then the pruned ops and the bounds.
struct CentroidSmem {
  int ops_off, ls_off, us_off, bytes;
  __host__ __device__ static CentroidSmem of(const DevTape& tape) {
    CentroidSmem c;
    c.ops_off = ((tape.bytes_len + 15) / 16) * 16;
    c.ls_off = c.ops_off + ((tape.n_ops * int(sizeof(cc_op)) + 15) / 16) * 16;
    c.us_off = c.ls_off + tape.n_ops * 8;
    c.bytes = c.us_off + tape.n_ops * 8;
    return c;
  }
};

// The tape a box of cells (first cell i0, ext cells per axis, clipped to the grid) is evaluated
// with: pruned to the box of their centroids if it can be.
template <class T, int D>
__device__ __forceinline__ STape<T> box_tape(const STape<T>& t, const DevTape& tape, const DevGrid<T>& g,
                                             const long long i0[3], const int ext[3], unsigned char* smem,
                                             int* count) {
  if (!tape.prunable) return t;
  const CentroidSmem L = CentroidSmem::of(tape);
  double lo[D], hi[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const long long last = i0[a] + ext[a] - 1 < g.n[a] - 1 ? i0[a] + ext[a] - 1 : g.n[a] - 1;
    lo[a] = double(g.x0[a]) + (double(i0[a]) + 0.5) * double(g.d[a]);
    hi[a] = double(g.x0[a]) + (double(last) + 0.5) * double(g.d[a]);
  }
  cc_op* ops = reinterpret_cast<cc_op*>(smem + L.ops_off);
  const int m = prune_union<T, D>(t, tape.prunable, lo, hi, reinterpret_cast<double*>(smem + L.ls_off),
                                  reinterpret_cast<double*>(smem + L.us_off), ops, count);
  STape<T> u = t;
  u.ops = ops;
  u.n_ops = m;
  return u;
}

// The tape a tile's cells are evaluated with (a PTile box).
template <class T, int D>
__device__ __forceinline__ STape<T> tile_tape(const STape<T>& t, const DevTape& tape, const DevGrid<T>& g,
                                              const long long i0[3], unsigned char* smem, int* count) {
  const int ext[3] = {PTile<D>::X, PTile<D>::Y, PTile<D>::Z};
  return box_tape<T, D>(t, tape, g, i0, ext, smem, count);
}

template <class T, int D, bool MX>
__global__ void __launch_bounds__(NT) plic_fit_kernel(const DevGrid<T> g, const DevTape tape, const Cols cols,
                                                      T* normals, T* intercepts, uint8_t* valid) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_count;
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  using P = PTile<D>;
  const long long n0 = g.n[0], n1 = g.n[1], n2 = D == 3 ? g.n[2] : 1;
  const long long tx = (n0 + P::X - 1) / P::X, ty = (n1 + P::Y - 1) / P::Y, tz = (n2 + P::Z - 1) / P::Z;
  T* vf = static_cast<T*>(cols.vf);
  const unsigned ntiles = unsigned(tx * ty * tz);
  for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    long long i0[3];
    tile_origin<D>(tile, unsigned(tx), unsigned(ty), i0);
    const STape<T> u = tile_tape<T, D>(t, tape, g, i0, smem, &s_count);
    const int q = threadIdx.x;
    const long long idx[3] = {i0[0] + q % P::X, i0[1] + (q / P::X) % P::Y, i0[2] + q / (P::X * P::Y)};
    if (idx[0] < n0 && idx[1] < n1 && idx[2] < n2) {
      const long long ci = idx[0] + n0 * (idx[1] + n1 * idx[2]);
      const PlaneFit<T, D> pl = cell_plane<T, D, MX>(u, g, idx);
      const T frac = T(1) - pl.fraction;
#pragma unroll
      for (int a = 0; a < D; ++a) normals[D * ci + a] = pl.n[a];
      intercepts[ci] = pl.a;
      valid[ci] = pl.valid ? 1 : 0;
      vf[ci] = frac;
      cols.kind[ci] = frac == T(0) ? 0 : (frac == T(1) ? 1 : 2);
    }
    __syncthreads();  // the next tile's pruning overwrites the ops this one read
  }
}

// _cell_wet + _face_area, src/plic/apertures.jl:73-125 (k is the 0-based direction)
template <class T, int D, bool MX>
__device__ __forceinline__ T face_area(const T* n, T a, T frac, bool valid, const T* cs, int k) {
  const T s = (k & 1) ? T(1) : T(0);
  if constexpr (D == 2) {
    const int c = k < 2 ? 0 : 1, p = k < 2 ? 1 : 0;
    const T len = cs[p];
    if (!valid) return frac < T(0.5) ? T(0) : len;
    const T base = n[c] * s - a;
    return open_fraction<T, MX>(base, base + n[p]) * len;
  } else {
    const int c = k >> 1;
    const int p = c == 0 ? 1 : 0;
    const int q = c == 2 ? 1 : 2;
    const T U = cs[p], V = cs[q];
    if (!valid) return frac < T(0.5) ? T(0) : U * V;
    const T base = n[c] * s - a;
    if (n[p] == T(0) && n[q] == T(0)) return base >= T(0) ? U * V : T(0);
    const T solid = gvf2m<T, MX>(n[p], n[q], -base);
    return (U * V) * (T(1) - solid);
  }
}

// Whether a valid 3D plane misses its cell by more than rounding, and on which side: -1 when
// every face's face_area is 0, +1 when it is the face's full area U V, 0 when it must be computed.
// Over the unit cube n . xi spans [lo, hi] = [sum min(n_i, 0), sum max(n_i, 0)]. If a - hi exceeds
// 64 u (|n|_1 + |a|) (u the unit roundoff of T), every face has n_p x + n_q y < a - n_c s with that
// margin, so gvf2 (whose rounding error is a few u of the same scale, in T or, mixed, in FP64
// from T's base) reaches its alpha >= s return, 1, and the area is (U V) (1 - 1) = 0; if lo - a
// exceeds it, gvf2 returns 0 and the area is U V. A NaN or infinite plane fails both tests.
template <class T>
__device__ __forceinline__ int plane_side(const T n[3], T a) {
  const T zero = T(0);
  const T lo = (fmin(n[0], zero) + fmin(n[1], zero)) + fmin(n[2], zero);
  const T hi = (fmax(n[0], zero) + fmax(n[1], zero)) + fmax(n[2], zero);
  const T tol = (sizeof(T) == 4 ? T(0x1p-18) : T(0x1p-47)) * (((fabs(n[0]) + fabs(n[1])) + fabs(n[2])) + fabs(a));
  return a - hi > tol ? -1 : (lo - a > tol ? 1 : 0);
}

__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

// m / full for a face area m of a face of area full > 0, bit for bit: an area of exactly 0 or
// exactly full (every face the plane misses) gives m itself (0 / full keeps m's sign) or 1
// without the division. The resolved value's halving, (a + b) / 2, is taken as (a + b) * 0.5:
// both round the same real number.
template <class T>
__device__ __forceinline__ T frac_of(T m, T full) { return m == T(0) ? m : (m == full ? T(1) : m / full); }

// The resolved faces (src/plic/cache.jl:118-162) in 2D (3D marches z, plic_face_z_kernel) of one tile: every cell's one-sided areas
// (_face_area, apertures.jl:73-125) computed once into shared memory, with the faces the
// neighbouring cells outside the tile show it; each shared face is then resolved from its two
// one-sided areas, (left / full + right / full) / 2, the same expression in the same order from
// either side, so the face is single-valued bit for bit. Boundary faces are one-sided.
template <class T, int D, bool MX>
__global__ void __launch_bounds__(NT, 6) plic_face_kernel(const DevGrid<T> g, const Cols cols, const T* __restrict__ normals,
                                                       const T* __restrict__ intercepts, const uint8_t* __restrict__ valid) {
  using P = PTile<D>;
  constexpr int NF = 2 * D;
  constexpr int EXT[3] = {P::X, P::Y, P::Z};
  constexpr int E0 = P::Y * P::Z, E1 = P::X * P::Z, E2 = P::X * P::Y;  // halo face sizes per axis
  constexpr int HB[3] = {0, 2 * E0, 2 * E0 + 2 * E1};                  // halo base per axis
  constexpr int NH = D == 3 ? 2 * (E0 + E1 + E2) : 2 * (E0 + E1);
  static_assert(P::X * P::Y * P::Z == NT, "one cell per thread");
  static_assert((P::X & (P::X - 1)) == 0 && (P::Y & (P::Y - 1)) == 0 && (P::Z & (P::Z - 1)) == 0, "powers of two");
  constexpr int LX = ilog2(P::X), LY = ilog2(P::Y), LZ = ilog2(P::Z);
  constexpr int LE0 = LY + LZ, LE1 = LX + LZ, LE2 = LX + LY;  // log2 of the halo face sizes
  __shared__ T own[NF][NT];                  // one-sided areas, face-major (no bank conflicts)
  __shared__ T halo[NH];
  __shared__ __align__(16) T res[NT * NF];   // resolved fractions, cell-major as in the column
  const long long n[3] = {g.n[0], g.n[1], D == 3 ? g.n[2] : 1};
  const T* vf = static_cast<const T*>(cols.vf);
  T* ff = static_cast<T*>(cols.ff);
  const T cs[3] = {g.d[0], g.d[1], D == 3 ? g.d[2] : T(1)};
  const long long tx = (n[0] + P::X - 1) / P::X, ty = (n[1] + P::Y - 1) / P::Y, tz = (n[2] + P::Z - 1) / P::Z;
  const unsigned ntiles = unsigned(tx * ty * tz);
  for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    long long i0[3];
    tile_origin<D>(tile, unsigned(tx), unsigned(ty), i0);
    const int q = threadIdx.x;
    const int lq[3] = {q % P::X, (q / P::X) % P::Y, q / (P::X * P::Y)};
    const long long idx[3] = {i0[0] + lq[0], i0[1] + lq[1], i0[2] + lq[2]};
    const bool in = idx[0] < n[0] && idx[1] < n[1] && idx[2] < n[2];
    const long long ci = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
    if (in) {  // this cell's plane, read once, on all its faces
      T nrm[D];
#pragma unroll
      for (int a = 0; a < D; ++a) nrm[a] = normals[D * ci + a];
      const T a = intercepts[ci], frac = vf[ci];
      const bool ok = valid[ci] != 0;
#pragma unroll
      for (int k = 0; k < NF; ++k) own[k][q] = face_area<T, D, MX>(nrm, a, frac, ok, cs, k);
    }
    // the halo: for each axis and side, the cell beyond the tile shows its face toward the tile
    for (int h = threadIdx.x; h < NH; h += NT) {
      int ax = 0;
      if (D == 3 && h >= HB[2]) ax = 2;
      else if (h >= HB[1]) ax = 1;
      // the extents are powers of two: shifts and masks, not divisions
      const int lE = ax == 0 ? LE0 : (ax == 1 ? LE1 : LE2);
      const int side = (h - HB[ax]) >> lE, pos = (h - HB[ax]) & ((1 << lE) - 1);
      const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;  // the other two axes, increasing
      const int lX = o1 == 0 ? LX : LY;
      long long nb[3];
      nb[ax] = side == 0 ? i0[ax] - 1 : i0[ax] + EXT[ax];
      nb[o1] = i0[o1] + (pos & ((1 << lX) - 1));
      nb[o2] = i0[o2] + (pos >> lX);
      if (nb[ax] >= 0 && nb[ax] < n[ax] && nb[o1] < n[o1] && nb[o2] < n[o2]) {
        const long long cj = nb[0] + n[0] * (nb[1] + n[1] * nb[2]);
        halo[h] = face_area<T, D, MX>(normals + D * cj, intercepts[cj], vf[cj], valid[cj] != 0, cs,
                                      side == 0 ? 2 * ax + 1 : 2 * ax);
      }
    }
    __syncthreads();
    if (in) {
#pragma unroll
      for (int k = 0; k < NF; ++k) {
        const int c = k >> 1;
        const int o1 = c == 0 ? 1 : 0, o2 = c == 2 ? 1 : 2;
        T full;
        if constexpr (D == 2) full = cs[1 - c];
        else full = (T(1) * cs[o1]) * cs[o2];
        const int lstride = c == 0 ? 1 : (c == 1 ? P::X : P::X * P::Y);
        const int hpos = lq[o1] + EXT[o1] * (D == 3 ? lq[o2] : 0);
        const T mine = own[k][q];
        T r;
        if ((k & 1) == 0) {
          const bool has = idx[c] >= 1;
          const T below = lq[c] > 0 ? own[k + 1][q - lstride] : halo[HB[c] + hpos];
          r = has ? (frac_of(below, full) + frac_of(mine, full)) * T(0.5) : frac_of(mine, full);
        } else {
          const bool has = idx[c] <= n[c] - 2;
          const int Ec = c == 0 ? E0 : (c == 1 ? E1 : E2);
          const T above = lq[c] < EXT[c] - 1 ? own[k - 1][q + lstride] : halo[HB[c] + Ec + hpos];
          r = has ? (frac_of(mine, full) + frac_of(above, full)) * T(0.5) : frac_of(mine, full);
        }
        res[q * NF + k] = r;
      }
    }
    __syncthreads();
    // the tile's rows leave whole: a row is P::X cells x NF values, contiguous in the column
    const int rowcells = (int)(n[0] - i0[0] < P::X ? n[0] - i0[0] : P::X);
    constexpr int RV = P::X * NF * int(sizeof(T)) / 16;  // 16-byte vectors per full row
    for (int w = threadIdx.x; w < P::Y * P::Z * RV; w += NT) {
      const int row = w / RV, v = w - row * RV;
      const long long j = i0[1] + row % P::Y, k = i0[2] + row / P::Y;
      if (j >= n[1] || k >= n[2]) continue;
      const long long c0 = i0[0] + n[0] * (j + n[1] * k);
      if (rowcells == P::X && (reinterpret_cast<uintptr_t>(ff + NF * c0) & 15u) == 0) {
        reinterpret_cast<uint4*>(ff + NF * c0)[v] = reinterpret_cast<const uint4*>(res + row * P::X * NF)[v];
      } else {
        constexpr int PER = 16 / int(sizeof(T));
        for (int e = v * PER; e < (v + 1) * PER; ++e)
          if (e < rowcells * NF) ff[NF * c0 + e] = res[row * P::X * NF + e];
      }
    }
    __syncthreads();  // the next tile reuses own, halo and res
  }
}

// What the fit records per cell for the 3D face pass (cell_side): -1 when every face_area of the
// cell's plane is 0, +1 when every one is the full face, 0 when they must be clipped. A valid plane
// is classified by plane_side; an invalid one has face areas 0 (fraction < 1/2) or full (any other
// fraction, NaN included), _face_area's rule for an invalid plane.
template <class T>
__device__ __forceinline__ int8_t cell_side(bool valid, const T n[3], T a, T frac) {
  if (!valid) return frac < T(0.5) ? int8_t(-1) : int8_t(1);
  return int8_t(plane_side<T>(n, a));
}

// The resolved faces in 3D, marching z: a CTA owns a column of FZ_X x FZ_Y cells and FZ_KZ slices.
// Per slice it forms the next slice's one-sided fractions (area / full face, frac_of; whose -z face
// is this slice's +z neighbour) and this slice's x and y halo, then resolves the slice and writes
// its rows; this slice's +z fractions are kept as the next slice's -z neighbours. A cell's six
// one-sided fractions come from its side byte alone (all 0 or all 1) unless the fit marked its
// plane as crossing the cell, and only then is the plane read and clipped. Every side byte is read
// once (the column's first slice also reads the one below it), in one barrier per slice, and each
// one-sided fraction is formed once rather than by both cells of its face. The areas, fractions
// and resolve expression are plic_face_kernel's, so the faces are the same bits.
constexpr int FZ_X = 32, FZ_Y = 8, FZ_KZ = 32;

template <class T, bool MX>
__global__ void __launch_bounds__(NT, MX ? 4 : 5) plic_face_z_kernel(const DevGrid<T> g, const Cols cols,
                                                            const T* __restrict__ normals,
                                                            const T* __restrict__ intercepts,
                                                            const int8_t* __restrict__ sides) {
  constexpr int X = FZ_X, Y = FZ_Y, NF = 6;
  static_assert(X * Y == NT, "one cell of the slice per thread");
  // One-sided fractions of the slices k % 3, warp-blocked: row w (one warp) keeps its six faces
  // over its 32 lanes, [w][f][lane], so a warp's own writes stay in its own block.
  __shared__ __align__(16) T bufs[3][Y][NF][X];
  __shared__ T prev5[NT];                    // the slice below's +z fractions (own slot only)
  __shared__ T hx[2][2][Y], hy[2][2][X];     // the x and y halo of slices of each parity
  const long long n[3] = {g.n[0], g.n[1], g.n[2]};
  T* ff = static_cast<T*>(cols.ff);
  const T cs[3] = {g.d[0], g.d[1], g.d[2]};
  const unsigned ntx = unsigned((n[0] + X - 1) / X), nty = unsigned((n[1] + Y - 1) / Y);
  unsigned b = blockIdx.x;
  const unsigned bx = b % ntx;
  b /= ntx;
  const unsigned by = b % nty;
  b /= nty;
  const long long i0 = (long long)bx * X, j0 = (long long)by * Y, k0 = (long long)b * FZ_KZ;
  const long long k1 = k0 + FZ_KZ < n[2] ? k0 + FZ_KZ : n[2];
  const int q = threadIdx.x, lx = q % X, ly = q / X;
  const long long ix = i0 + lx, jy = j0 + ly;
  const bool inxy = ix < n[0] && jy < n[1];
  // the full area of a face of direction f
  auto full_of = [&](int f) {
    const int c = f >> 1;
    return (T(1) * cs[c == 0 ? 1 : 0]) * cs[c == 2 ? 1 : 2];
  };
  // the clipped one-sided fraction of face f of cell ci, whose plane crosses it (side 0, so valid)
  auto clip_frac = [&](const T nn[3], T a, int f) {
    return frac_of(face_area<T, 3, MX>(nn, a, T(0), true, cs, f), full_of(f));
  };
  auto own6 = [&](T (*buf)[NF][X], int side, long long ci) {  // this thread's cell: six one-sided fractions
    if (side != 0) {
      const T v = side > 0 ? T(1) : T(0);
#pragma unroll
      for (int f = 0; f < NF; ++f) buf[ly][f][lx] = v;
    } else {
      const T nn[3] = {normals[3 * ci], normals[3 * ci + 1], normals[3 * ci + 2]};
      const T a = intercepts[ci];
#pragma unroll
      for (int f = 0; f < NF; ++f) buf[ly][f][lx] = clip_frac(nn, a, f);
    }
  };
  // The x and y halo of a slice: 2Y + 2X faces, one on every third thread (all eight warps share
  // them). Item h: the cell beyond the tile's -x / +x edge at row h (h < 2Y), or beyond its -y / +y
  // edge at column h - 2Y; the face it shows the tile.
  constexpr int NH = 2 * Y + 2 * X;
  static_assert(3 * (NH - 1) < NT, "one halo face per third thread");
  const int hitem = (q % 3 == 0) ? q / 3 : NH;
  long long hcell = -1;
  int hface = 0;
  if (hitem < 2 * Y) {
    const int side = hitem / Y, y = hitem % Y;
    const long long ii = side == 0 ? i0 - 1 : i0 + X, jj = j0 + y;
    if (ii >= 0 && ii < n[0] && jj < n[1]) hcell = ii + n[0] * jj;
    hface = side == 0 ? 1 : 0;
  } else if (hitem < NH) {
    const int side = (hitem - 2 * Y) / X, x = (hitem - 2 * Y) % X;
    const long long ii = i0 + x, jj = side == 0 ? j0 - 1 : j0 + Y;
    if (jj >= 0 && jj < n[1] && ii < n[0]) hcell = ii + n[0] * jj;
    hface = side == 0 ? 3 : 2;
  }
  // a halo cell's face hface (one of the x and y directions), clipped with a constant direction
  auto halo_frac = [&](int side, long long ci) -> T {
    if (side != 0) return side > 0 ? T(1) : T(0);
    const T nn[3] = {normals[3 * ci], normals[3 * ci + 1], normals[3 * ci + 2]};
    const T a = intercepts[ci];
    switch (hface) {
      case 0: return clip_frac(nn, a, 0);
      case 1: return clip_frac(nn, a, 1);
      case 2: return clip_frac(nn, a, 2);
      default: return clip_frac(nn, a, 3);
    }
  };
  const long long nxy = n[0] * n[1];
  const long long cxy = ix + n[0] * jy;
  // One barrier per slice. Slice k's fractions live in bufs[(k - k0) % 3]: the next slice's are
  // written (own slots) while this one's are read, and the buffer they overwrite was last read in
  // slice k - 2, whose readers all passed the previous barrier. The halo alternates by slice
  // parity on the same argument. The third buffer, free during slice k (it was slice k - 1's and
  // becomes slice k + 2's), takes each warp's resolved row in the warp's own block: only that
  // warp writes or reads its block until it fills it with slice k + 2's fractions itself, and it
  // copies the row out in between. Side bytes are read a slice ahead of their use.
  if (inxy) own6(bufs[0], sides[cxy + nxy * k0], cxy + nxy * k0);
  if (inxy && k0 >= 1) {
    const long long cb = cxy + nxy * (k0 - 1);
    const int sb = sides[cb];
    T v;
    if (sb != 0) {
      v = sb > 0 ? T(1) : T(0);
    } else {
      const T nn[3] = {normals[3 * cb], normals[3 * cb + 1], normals[3 * cb + 2]};
      v = clip_frac(nn, intercepts[cb], 5);
    }
    prev5[q] = v;
  }
  // Slice bookkeeping in 32-bit counters and running offsets: kk = k - k0, kn = n[2] - k0 slices
  // to the grid's top; the offsets advance one slice (nxy cells) per step.
  const int nk = int(k1 - k0), kn = int(n[2] - k0);
  const bool x_lo = ix >= 1, x_hi = ix <= n[0] - 2, y_lo = jy >= 1, y_hi = jy <= n[1] - 2;
  long long cn = cxy + nxy * (k0 + 1);  // the cell own6 builds next (slice k + 1)
  long long hc = hcell + nxy * k0;      // this slice's halo cell
  int snext = (inxy && kn > 1) ? sides[cn] : 0;
  int hsnext = hcell >= 0 ? sides[hc] : 0;
  const int lane = q & 31, wrow = q >> 5;
  static_assert(X == 32, "a warp is one row of the slice");
  const int rowcells = (int)(n[0] - i0 < X ? n[0] - i0 : X);
  T* frow = ff + NF * (i0 + n[0] * (jy + n[1] * k0));
  const long long fstep = NF * nxy;
  int r3 = 0;
  for (int kk = 0; kk < nk; ++kk) {
    const int par = kk & 1;
    T (*cur)[NF][X] = bufs[r3];
    T (*nxt)[NF][X] = bufs[r3 == 2 ? 0 : r3 + 1];
    T* const res = &bufs[r3 == 0 ? 2 : r3 - 1][wrow][0][0];  // this warp's row, cell-major
    T (*hxp)[Y] = hx[par];
    T (*hyp)[X] = hy[par];
    const int scur = snext, hscur = hsnext;
    if (inxy && kk + 2 < kn) snext = sides[cn + nxy];
    if (hcell >= 0 && kk + 1 < nk) hsnext = sides[hc + nxy];
    if (inxy && kk + 1 < kn) own6(nxt, scur, cn);
    if (hcell >= 0) {
      const T v = halo_frac(hscur, hc);
      if (hitem < 2 * Y) hxp[hitem / Y][hitem % Y] = v;
      else hyp[(hitem - 2 * Y) / X][(hitem - 2 * Y) % X] = v;
    }
    cn += nxy;
    hc += nxy;
    __syncthreads();
    if (inxy) {
      const bool lo[3] = {x_lo, y_lo, k0 + kk >= 1}, hi[3] = {x_hi, y_hi, kk + 1 < kn};
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const int c = f >> 1;
        const T mine = cur[ly][f][lx];
        T r;
        if ((f & 1) == 0) {
          const bool has = lo[c];
          T below = T(0);
          if (has) below = c == 0 ? (lx > 0 ? cur[ly][1][lx - 1] : hxp[0][ly])
                                  : c == 1 ? (ly > 0 ? cur[ly - 1][3][lx] : hyp[0][lx]) : prev5[q];
          r = has ? (below + mine) * T(0.5) : mine;
        } else {
          const bool has = hi[c];
          T above = T(0);
          if (has) above = c == 0 ? (lx < X - 1 ? cur[ly][0][lx + 1] : hxp[1][ly])
                                  : c == 1 ? (ly < Y - 1 ? cur[ly + 1][2][lx] : hyp[1][lx]) : nxt[ly][4][lx];
          r = has ? (mine + above) * T(0.5) : mine;
        }
        res[lx * NF + f] = r;
      }
    }
    __syncwarp();
    // the warp's row leaves whole (16-byte vectors where the row is full and aligned)
    if (jy < n[1]) {
      constexpr int RV = X * NF * int(sizeof(T)) / 16;
      const T* src = res;
      if (rowcells == X && (reinterpret_cast<uintptr_t>(frow) & 15u) == 0) {
        for (int v = lane; v < RV; v += 32)
          reinterpret_cast<uint4*>(frow)[v] = reinterpret_cast<const uint4*>(src)[v];
      } else {
        for (int e = lane; e < rowcells * NF; e += 32) frow[e] = src[e];
      }
    }
    frow += fstep;
    if (inxy) prev5[q] = cur[ly][5][lx];
    __syncwarp();  // every lane has copied the row out before any writes the next slice's fractions here
    r3 = r3 == 2 ? 0 : r3 + 1;
  }
}

// The fit pass in 3D, marching z: a CTA owns a column of FZ_X x FZ_Y cells and FZ_KZ slices, and
// prunes a union of spheres once per slab of tape.slab slices (the box of the slab's centroids;
// the depth is chosen on the host from the spheres' radii, prune_slab) instead of once per 256
// cells. The pruning drops only spheres strictly above the minimum over the box and keeps op
// order, so the planes are the same bits whatever the depth.

// At Float32 a bound of 3 CTAs per SM lets the fit keep its values in registers (62, no spills;
// 64-sphere cloud at 512^3: 3.64 -> 3.61 ms per update); Float64 keeps the compiler's own choice
// (a bound of 1 CTA doubled its registers and cost 0.19 ms).
template <class T, bool MX>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 3 : 0) plic_fit_z_kernel(const DevGrid<T> g, const DevTape tape, const Cols cols,
                                                        T* normals, T* intercepts, uint8_t* valid, int8_t* sides) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_count;
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  constexpr int X = FZ_X, Y = FZ_Y;
  const long long n[3] = {g.n[0], g.n[1], g.n[2]};
  const unsigned ntx = unsigned((n[0] + X - 1) / X), nty = unsigned((n[1] + Y - 1) / Y);
  unsigned b = blockIdx.x;
  const unsigned bx = b % ntx;
  b /= ntx;
  const unsigned by = b % nty;
  b /= nty;
  const long long i0 = (long long)bx * X, j0 = (long long)by * Y, k0 = (long long)b * FZ_KZ;
  const long long k1 = k0 + FZ_KZ < n[2] ? k0 + FZ_KZ : n[2];
  const int q = threadIdx.x;
  const long long ix = i0 + q % X, jy = j0 + q / X;
  const bool inxy = ix < n[0] && jy < n[1];
  T* vf = static_cast<T*>(cols.vf);
  const int fit_s = tape.slab > 0 ? tape.slab : 8;
  for (long long ks = k0; ks < k1; ks += fit_s) {
    const long long first[3] = {i0, j0, ks};
    const int ext[3] = {X, Y, fit_s};
    const STape<T> u = box_tape<T, 3>(t, tape, g, first, ext, smem, &s_count);
    const long long ke = ks + fit_s < k1 ? ks + fit_s : k1;
    for (long long k = ks; k < ke; ++k) {
      if (!inxy) continue;
      const long long idx[3] = {ix, jy, k};
      const long long ci = ix + n[0] * (jy + n[1] * k);
      const PlaneFit<T, 3> pl = cell_plane<T, 3, MX>(u, g, idx);
      const T frac = T(1) - pl.fraction;
#pragma unroll
      for (int a = 0; a < 3; ++a) normals[3 * ci + a] = pl.n[a];
      intercepts[ci] = pl.a;
      valid[ci] = pl.valid ? 1 : 0;
      vf[ci] = frac;
      cols.kind[ci] = frac == T(0) ? 0 : (frac == T(1) ? 1 : 2);
      sides[ci] = cell_side<T>(pl.valid, pl.n, pl.a, frac);
    }
    __syncthreads();  // the next slab's pruning overwrites the ops this one read
  }
}

// Neumaier-compensated accumulation in Float64.
struct KSum {
  double s, c;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
};

// calc_volume, src/volume.jl:29-40: every cell's cell_plane solid fraction, summed.
template <class T, int D, bool MX>
__global__ void __launch_bounds__(NT) calc_volume_kernel(const DevGrid<T> g, const DevTape tape, double* partial) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_count;
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  using P = PTile<D>;
  const long long n0 = g.n[0], n1 = g.n[1], n2 = D == 3 ? g.n[2] : 1;
  const long long tx = (n0 + P::X - 1) / P::X, ty = (n1 + P::Y - 1) / P::Y, tz = (n2 + P::Z - 1) / P::Z;
  KSum acc{0.0, 0.0};
  const unsigned ntiles = unsigned(tx * ty * tz);
  for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    long long i0[3];
    tile_origin<D>(tile, unsigned(tx), unsigned(ty), i0);
    const STape<T> u = tile_tape<T, D>(t, tape, g, i0, smem, &s_count);
    const int q = threadIdx.x;
    const long long idx[3] = {i0[0] + q % P::X, i0[1] + (q / P::X) % P::Y, i0[2] + q / (P::X * P::Y)};
    if (idx[0] < n0 && idx[1] < n1 && idx[2] < n2) acc.add(double(cell_plane<T, D, MX>(u, g, idx).fraction));
    __syncthreads();
  }
  __shared__ double ss[NT], sc[NT];
  ss[threadIdx.x] = acc.s;
  sc[threadIdx.x] = acc.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    KSum b{0.0, 0.0};
    double cc = 0.0;
    for (int i = 0; i < NT; ++i) { b.add(ss[i]); cc += sc[i]; }
    partial[2 * blockIdx.x] = b.s;
    partial[2 * blockIdx.x + 1] = b.c + cc;
  }
}

// calc_volume in 3D, marching z: persistent CTAs take FZ_X x FZ_Y x FZ_KZ columns and prune a union
// of spheres once per slab of tape.slab slices, as the 3D fit pass does (the same fractions; the sum
// is the same compensated accumulation, in another order).
template <class T, bool MX>
__global__ void __launch_bounds__(NT) calc_volume_z_kernel(const DevGrid<T> g, const DevTape tape, double* partial) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_count;
  const STape<T> t = load_tape<T>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  constexpr int X = FZ_X, Y = FZ_Y;
  const long long n[3] = {g.n[0], g.n[1], g.n[2]};
  const unsigned ntx = unsigned((n[0] + X - 1) / X), nty = unsigned((n[1] + Y - 1) / Y);
  const unsigned ncol = ntx * nty * unsigned((n[2] + FZ_KZ - 1) / FZ_KZ);
  const int q = threadIdx.x;
  KSum acc{0.0, 0.0};
  for (unsigned col = blockIdx.x; col < ncol; col += gridDim.x) {
    unsigned b = col;
    const unsigned bx = b % ntx;
    b /= ntx;
    const unsigned by = b % nty;
    b /= nty;
    const long long i0 = (long long)bx * X, j0 = (long long)by * Y, k0 = (long long)b * FZ_KZ;
    const long long k1 = k0 + FZ_KZ < n[2] ? k0 + FZ_KZ : n[2];
    const long long ix = i0 + q % X, jy = j0 + q / X;
    const bool inxy = ix < n[0] && jy < n[1];
    const int fit_s = tape.slab > 0 ? tape.slab : 8;
    for (long long ks = k0; ks < k1; ks += fit_s) {
      const long long first[3] = {i0, j0, ks};
      const int ext[3] = {X, Y, fit_s};
      const STape<T> u = box_tape<T, 3>(t, tape, g, first, ext, smem, &s_count);
      const long long ke = ks + fit_s < k1 ? ks + fit_s : k1;
      if (inxy)
        for (long long k = ks; k < ke; ++k) {
          const long long idx[3] = {ix, jy, k};
          acc.add(double(cell_plane<T, 3, MX>(u, g, idx).fraction));
        }
      __syncthreads();  // the next slab's pruning overwrites the ops this one read
    }
  }
  __shared__ double ss[NT], sc[NT];
  ss[threadIdx.x] = acc.s;
  sc[threadIdx.x] = acc.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    KSum r{0.0, 0.0};
    double cc = 0.0;
    for (int i = 0; i < NT; ++i) { r.add(ss[i]); cc += sc[i]; }
    partial[2 * blockIdx.x] = r.s;
    partial[2 * blockIdx.x + 1] = r.c + cc;
  }
}

__global__ void calc_volume_final(const double* partial, int nb, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum b{0.0, 0.0};
  double cc = 0.0;
  for (int i = 0; i < nb; ++i) { b.add(partial[2 * i]); cc += partial[2 * i + 1]; }
  out[0] = b.s + (b.c + cc);
}

// cut_cell_report, src/cut_cell.jl:302-319: counts by kind, ambiguous, smallest cut fraction.
// Each thread takes 16 cells at a time with 16-byte loads of the kind and ambiguous columns (the
// caller guarantees 16-byte aligned columns for the vector part; the tail is scalar).
template <class T>
__device__ __forceinline__ void report_cell(int k, int a, T v, unsigned long long& cut, unsigned long long& ins,
                                            unsigned long long& out, unsigned long long& am, T& vmin) {
  cut += k == 2;
  ins += k == 0;
  out += k == 1;
  am += a != 0;
  if (k == 2 && v > T(0) && v < vmin) vmin = v;
}

// 0x80 in each byte of x that is zero, nothing elsewhere (no carry crosses a byte: (b & 0x7f) +
// 0x7f <= 0xfe).
__device__ __forceinline__ unsigned zero_bytes(unsigned x) {
  return ~(((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x | 0x7f7f7f7fu);
}

template <class T>
__global__ void __launch_bounds__(NT) report_kernel(long long ncell, const int8_t* __restrict__ kind,
                                                    const uint8_t* __restrict__ amb, const T* __restrict__ vf,
                                                    unsigned long long* counts, unsigned long long* vmin_bits,
                                                    int vec_ok) {
  unsigned long long cut = 0, ins = 0, out = 0, am = 0;
  T vmin = T(1);
  const long long nvec = vec_ok ? ncell / 16 : 0;
  const uint4* kind4 = reinterpret_cast<const uint4*>(kind);
  const uint4* amb4 = reinterpret_cast<const uint4*>(amb);
  // sixteen cells: the bytes of each word equal to 2 (cut), 0 (inside), 1 (outside), and the
  // nonzero ambiguous bytes, counted exactly whatever the byte values; the fraction is only read
  // for cut cells, which are few
  auto sixteen = [&](const uint4 kk, const uint4 aa, long long g) {
    const unsigned kw[4] = {kk.x, kk.y, kk.z, kk.w};
    const unsigned aw[4] = {aa.x, aa.y, aa.z, aa.w};
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const unsigned cutm = zero_bytes(kw[w] ^ 0x02020202u);
      cut += __popc(cutm);
      ins += __popc(zero_bytes(kw[w]));
      out += __popc(zero_bytes(kw[w] ^ 0x01010101u));
      am += 4 - __popc(zero_bytes(aw[w]));
      for (unsigned m = cutm; m; m &= m - 1) {
        const T v = vf[16 * g + 4 * w + ((__ffs(m) - 1) >> 3)];
        if (v > T(0) && v < vmin) vmin = v;
      }
    }
  };
  const long long stride = (long long)gridDim.x * NT;
  long long g = blockIdx.x * (long long)NT + threadIdx.x;
  for (; g + 3 * stride < nvec; g += 4 * stride) {  // four strides' loads in flight before any test
    uint4 kk[4], aa[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      kk[u] = kind4[g + u * stride];
      aa[u] = amb4[g + u * stride];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) sixteen(kk[u], aa[u], g + u * stride);
  }
  for (; g < nvec; g += stride) sixteen(kind4[g], amb4[g], g);
  for (long long i = 16 * nvec + blockIdx.x * (long long)NT + threadIdx.x; i < ncell; i += (long long)gridDim.x * NT)
    report_cell<T>(kind[i], amb[i], kind[i] == 2 ? vf[i] : T(1), cut, ins, out, am, vmin);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cut += __shfl_down_sync(0xffffffffu, cut, o);
    ins += __shfl_down_sync(0xffffffffu, ins, o);
    out += __shfl_down_sync(0xffffffffu, out, o);
    am += __shfl_down_sync(0xffffffffu, am, o);
    const T w = __shfl_down_sync(0xffffffffu, vmin, o);
    vmin = w < vmin ? w : vmin;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counts + 0, cut);
    atomicAdd(counts + 1, ins);
    atomicAdd(counts + 2, out);
    atomicAdd(counts + 3, am);
    // non-negative floats order as their bit patterns; the slot keeps the complement's maximum, so
    // it starts from 0 like the counters and the host zeroes all five with one memset
    const double dv = double(vmin);
    atomicMax(vmin_bits, ~(unsigned long long)__double_as_longlong(dv));
  }
}

int blocks_for(long long work, int per_sm) {
  long long b = (work + NT - 1) / NT;
  const long long cap = 148LL * per_sm;
  return int(b < 1 ? 1 : (b > cap ? cap : b));
}

// Monte Carlo volume of {phi < 0} in the box lo..hi: point p's coordinates are three
// successive splitmix64 outputs of (seed, 3p + a), 53 random bits each, mapped to [lo, hi);
// the body is evaluated in Float64. Counts accumulate per thread, then per CTA, then into
// out[0] with one atomic add per CTA.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void __launch_bounds__(NT) monte_carlo_kernel(const DevTape tape, double lo0, double lo1, double lo2,
                                                         double hi0, double hi1, double hi2, long long npts,
                                                         unsigned long long seed, unsigned long long* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const STape<double> t = load_tape<double>(tape.bytes, tape.n_ops, tape.n_params, smem);
  __syncthreads();
  const double lo[3] = {lo0, lo1, lo2}, span[3] = {hi0 - lo0, hi1 - lo1, hi2 - lo2};
  unsigned long long inside = 0;
  for (long long p = blockIdx.x * (long long)NT + threadIdx.x; p < npts; p += (long long)gridDim.x * NT) {
    double x[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const unsigned long long r = splitmix64(seed ^ (unsigned long long)(3 * p + a));
      x[a] = lo[a] + double(r >> 11) * 0x1.0p-53 * span[a];
    }
    inside += tape_eval<double, 3, double>(t, x) < 0.0 ? 1 : 0;
  }
  __shared__ unsigned long long part[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) inside += __shfl_xor_sync(0xffffffffu, inside, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x / 32] = inside;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < NT / 32; ++w) s += part[w];
    atomicAdd(out, s);
  }
}

}  // namespace

namespace cci {

cudaError_t launch_monte_carlo(const DevTape& tape, const double lo[3], const double hi[3], long long npts,
                               unsigned long long seed, unsigned long long* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || npts <= 0) return e;
  const int sm = ((tape.bytes_len + 15) / 16) * 16;
  monte_carlo_kernel<<<blocks_for(npts, 16), NT, sm, s>>>(tape, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], npts, seed,
                                                          out);
  return cudaGetLastError();
}

template <class T, int D>
cudaError_t launch_plic(const DevGrid<T>& g, const DevTape& tape, const Cols& cols, T* normals, T* intercepts,
                        uint8_t* valid, int8_t* sides, cudaStream_t s, bool mixed) {
  if (D == 3 && !sides) return cudaErrorInvalidValue;
  const long long total = g.n[0] * g.n[1] * (D == 3 ? g.n[2] : 1);
  const int sm = CentroidSmem::of(tape).bytes;
  if (sm > 48 * 1024) {
    cudaError_t e;
    if constexpr (D == 3) {
      e = cudaFuncSetAttribute(plic_fit_z_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(plic_fit_z_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    } else {
      e = cudaFuncSetAttribute(plic_fit_kernel<T, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(plic_fit_kernel<T, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    if (e != cudaSuccess) return e;
  }
  // 3D fit and faces march z, one CTA per FZ_X x FZ_Y x FZ_KZ column; 2D works in tiles
  const long long zcols = ((g.n[0] + FZ_X - 1) / FZ_X) * ((g.n[1] + FZ_Y - 1) / FZ_Y) * ((g.n[2] + FZ_KZ - 1) / FZ_KZ);
  if (mixed && sizeof(T) == 4) {
    if constexpr (D == 3) {
      plic_fit_z_kernel<T, true><<<unsigned(zcols), NT, sm, s>>>(g, tape, cols, normals, intercepts, valid, sides);
      plic_face_z_kernel<T, true><<<unsigned(zcols), NT, 0, s>>>(g, cols, normals, intercepts, sides);
    } else {
      plic_fit_kernel<T, D, true><<<blocks_for(total, 16), NT, sm, s>>>(g, tape, cols, normals, intercepts, valid);
      plic_face_kernel<T, D, true><<<blocks_for(total, 16), NT, 0, s>>>(g, cols, normals, intercepts, valid);
    }
  } else {
    if constexpr (D == 3) {
      plic_fit_z_kernel<T, false><<<unsigned(zcols), NT, sm, s>>>(g, tape, cols, normals, intercepts, valid, sides);
      plic_face_z_kernel<T, false><<<unsigned(zcols), NT, 0, s>>>(g, cols, normals, intercepts, sides);
    } else {
      plic_fit_kernel<T, D, false><<<blocks_for(total, 16), NT, sm, s>>>(g, tape, cols, normals, intercepts, valid);
      plic_face_kernel<T, D, false><<<blocks_for(total, 16), NT, 0, s>>>(g, cols, normals, intercepts, valid);
    }
  }
  return cudaGetLastError();
}

int calc_volume_blocks() { return VOL_BLOCKS; }

template <class T, int D>
cudaError_t launch_calc_volume(const DevGrid<T>& g, const DevTape& tape, double* partial, double* out,
                               cudaStream_t s, bool mixed) {
  const int sm = CentroidSmem::of(tape).bytes;
  if constexpr (D == 3) {
    if (sm > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(calc_volume_z_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(calc_volume_z_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e != cudaSuccess) return e;
    }
    if (mixed && sizeof(T) == 4) calc_volume_z_kernel<T, true><<<VOL_BLOCKS, NT, sm, s>>>(g, tape, partial);
    else calc_volume_z_kernel<T, false><<<VOL_BLOCKS, NT, sm, s>>>(g, tape, partial);
  } else {
    if (sm > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(calc_volume_kernel<T, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(calc_volume_kernel<T, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      if (e != cudaSuccess) return e;
    }
    if (mixed && sizeof(T) == 4) calc_volume_kernel<T, D, true><<<VOL_BLOCKS, NT, sm, s>>>(g, tape, partial);
    else calc_volume_kernel<T, D, false><<<VOL_BLOCKS, NT, sm, s>>>(g, tape, partial);
  }
  calc_volume_final<<<1, 32, 0, s>>>(partial, VOL_BLOCKS, out);
  return cudaGetLastError();
}

cudaError_t launch_report(long long ncell, const int8_t* kind, const uint8_t* amb, const void* vf, int is_f64,
                          unsigned long long* counts, double* vmin, cudaStream_t s) {
  // four CTAs of 256 per SM (the unrolled loop's registers), each thread with eight 16-byte
  // loads in flight: 128 KB per SM
  const int nb = blocks_for((ncell + 15) / 16, 4);
  unsigned long long* vb = reinterpret_cast<unsigned long long*>(vmin);
  const int vec_ok = ((reinterpret_cast<uintptr_t>(kind) | reinterpret_cast<uintptr_t>(amb)) & 15u) == 0;
  if (is_f64)
    report_kernel<double><<<nb, NT, 0, s>>>(ncell, kind, amb, static_cast<const double*>(vf), counts, vb, vec_ok);
  else
    report_kernel<float><<<nb, NT, 0, s>>>(ncell, kind, amb, static_cast<const float*>(vf), counts, vb, vec_ok);
  return cudaGetLastError();
}

#define INST(T, D)                                                                                      \
  template cudaError_t launch_plic<T, D>(const DevGrid<T>&, const DevTape&, const Cols&, T*, T*, uint8_t*, int8_t*, \
                                         cudaStream_t, bool);                                           \
  template cudaError_t launch_calc_volume<T, D>(const DevGrid<T>&, const DevTape&, double*, double*, cudaStream_t, \
                                                bool);
INST(float, 2)
INST(float, 3)
INST(double, 2)
INST(double, 3)
#undef INST

}  // namespace cci
