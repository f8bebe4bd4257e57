// mc.cu -- MarchingCubesCutCell update_cache! on sm_100a.
//
// Two kernels replace the reference's two KernelAbstractions launches
// (_sample_nodes_kernel! and _nodal_cells_kernel!, src/marching_squares/cache.jl:55-78):
//
//   * mc_fill_kernel: a CTA owns a pencil of TX x TY cells in (x, y) and marches up to KZ slices
//     along z. Node slabs of (TX+1) x (TY+1) values are sampled from the op-tape NS at a time into
//     a shared-memory ring, so a node is evaluated once per CTA and written to phi once, by the
//     CTA that owns it. Every thread classifies one cell from its eight corners. Uncut cells (all
//     corners of one sign) get their fields directly -- their face centroids are half the lattice
//     edge lengths, a cheap affine fill -- into a double-buffered shared-memory staging tile that
//     leaves as one TMA tensor store per StructArray column (cp.async.bulk.tensor, shared ->
//     global), so the SM's threads never issue the column stores. Cut cells are compacted with a
//     warp ballot into a global work list.
//   * mc_cut_kernel: one lane per listed cut cell runs the full construction of
//     src/marching_cubes/moments.jl:275-346 densely and writes that cell's fields.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <cuda.h>
#include "cc_device.cuh"
#include "cc_internal.h"
#include "mc_cell.cuh"

namespace {

using namespace ccd;
using namespace ccmc;
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
  static constexpr int MINB = sizeof(T) == 4 ? 3 : 3;  // Float64 at 4 spills
};
constexpr int NS = 4;   // node slabs sampled per round (one op-major tape pass per thread)
constexpr int KZ = 31;  // most z slices marched per CTA: KZ + 1 = 32 node slabs, 8 sampling rounds
constexpr int CUT_NT = 256;  // 512^3 CSG body, Float32 update: 2.73 ms at 128, 2.71-2.72 at 256, 2.75 at 64

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
  int kz;  // z slices per pencil (pencil_slices)
  int tma_mask;  // bit c: column c leaves through TMA tensor stores (its map below is valid)
  int byte_words;  // kind/ambiguous rows start on 4-byte boundaries
  int thread_cols;  // bit c: column c is copied element by element by the threads (no TMA, no words)
  // a union of spheres: each CTA's kept ops (stride tape.n_ops) and their count, or null
  const cc_op* pruned_ops;
  const int* pruned_count;
};

// One TMA tensor map per output column: kind, ambiguous, volume_fraction (n0 x n1 x n2), centroid
// and interface_centroid (3 n0 x n1 x n2), face_fraction (6 n0 x n1 x n2), face_centroid_local
// (12 x n0 x n1 x n2). A staged tile is exactly one box of each.
struct ColumnMaps {
  CUtensorMap m[7];
};

// TMA bulk-group bookkeeping (the tensor stores below commit into bulk groups).
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
  // an uncut cell's interface centroid is its centroid, and a cut cell's staged values are
  // overwritten by the cut kernel: the interface_centroid box is sent from the centroid column
  static constexpr int ic = c;
  static constexpr int stage_bytes = ((fcl + 12 * NC * int(sizeof(T)) + 127) / 128) * 128;
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

// For a union of spheres: each fill CTA's pencil (cells i0.., j0.., k0..k1) gets the tape pruned to
// the box of its nodes (prune_union), written to out[cta * n_ops ..] with its count.
template <class T>
__global__ void __launch_bounds__(256) prune_pencils_kernel(const McArgs<T> A, cc_op* __restrict__ out,
                                                            int* __restrict__ count) {
  extern __shared__ __align__(128) unsigned char smem[];  // one alignment for every extern declaration
  __shared__ int s_count;
  using TL = Tile<T>;
  const STape<T> t = load_tape<T>(A.tape.bytes, A.tape.n_ops, A.tape.n_params, smem);
  __syncthreads();
  const PruneSmem ps = PruneSmem::of(A.tape, 0);
  int b = blockIdx.x;
  const int it = b % A.n_itiles; b /= A.n_itiles;
  const int jt = b % A.n_jtiles; b /= A.n_jtiles;
  const long long n0 = A.g.n[0], n1 = A.g.n[1], n2 = A.g.n[2];
  const long long i0 = (long long)it * TL::TX, j0 = (long long)jt * TL::TY, k0 = (long long)b * A.kz;
  const long long i1 = i0 + TL::TX < n0 ? i0 + TL::TX : n0, j1 = j0 + TL::TY < n1 ? j0 + TL::TY : n1;
  const long long k1 = k0 + A.kz < n2 ? k0 + A.kz : n2;
  const double lo[3] = {double(A.g.x0[0]) + double(i0) * double(A.g.d[0]),
                        double(A.g.x0[1]) + double(j0) * double(A.g.d[1]),
                        double(A.g.x0[2]) + double(k0) * double(A.g.d[2])};
  const double hi[3] = {double(A.g.x0[0]) + double(i1) * double(A.g.d[0]),
                        double(A.g.x0[1]) + double(j1) * double(A.g.d[1]),
                        double(A.g.x0[2]) + double(k1) * double(A.g.d[2])};
  cc_op* kept = reinterpret_cast<cc_op*>(smem + ps.ops);
  const int m = prune_union<T, 3>(t, A.tape.prunable, lo, hi, reinterpret_cast<double*>(smem + ps.ls),
                                  reinterpret_cast<double*>(smem + ps.us), kept, &s_count);
  for (int q = threadIdx.x; q < m; q += blockDim.x) out[(long long)blockIdx.x * A.tape.n_ops + q] = kept[q];
  if (threadIdx.x == 0) count[blockIdx.x] = m;
}

// An uncut cell whose staging slot held an uncut cell of the same kind at the slot's previous use
// (two slices earlier, in the same column): kind, flag, fraction, face fractions and the x, y
// parts are the same values, so only what depends on the slice is written -- the centroid's and
// interface centroid's z and the face centroids' half-height entries (slots 1, 3, 5, 7, written
// with their neighbours as two 16-byte vectors). The slot then holds exactly what put_cell leaves.
// 512^3 CSG body: Float32 update 2.78 -> 2.74 ms.
__device__ __forceinline__ void put_uncut_z(const Stage<float>& st, int lc, float cz, float hx, float hy, float hz) {
  st.c[3 * lc + 2] = cz;
  float4* d4 = reinterpret_cast<float4*>(st.fcl + 12 * lc);
  d4[0] = make_float4(hy, hz, hy, hz);
  d4[1] = make_float4(hx, hz, hx, hz);
}

template <class T, bool SAMPLE, bool PRUNED>
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
  const long long k0 = (long long)b * A.kz;
  const long long k1 = (k0 + A.kz < n2) ? k0 + A.kz : n2;

  STape<T> tape;
  if (SAMPLE) {
    tape = load_tape<T>(A.tape.bytes, A.tape.n_ops, A.tape.n_params, smem + L::tape);
    if (PRUNED) {  // this pencil's kept ops over the loaded ones (same places, fewer)
      const int m = A.pruned_count[blockIdx.x];
      cc_op* ops = reinterpret_cast<cc_op*>(smem + L::tape);
      __syncthreads();
      for (int q = tid; q < m; q += NT) ops[q] = A.pruned_ops[(long long)blockIdx.x * A.tape.n_ops + q];
      tape.n_ops = m;
    }
  }
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


  const int tx = tid % TX, ty = tid / TX;
  const long long ci = i0 + tx, cj = j0 + ty;
  const bool valid = ci < n0 && cj < n1;
  const T xa = node_coord(x0, dx, ci), xb = node_coord(x0, dx, ci + 1);
  const T ya = node_coord(y0, dy, cj), yb = node_coord(y0, dy, cj + 1);
  const T hx = T(0.5) * (xb - xa), hy = T(0.5) * (yb - ya);
  const T cx = xa + T(0.5) * dx, cy = ya + T(0.5) * dy;
  const int lc = ty * TX + tx;
  const int s00 = ty * NSX + tx;
  const bool fast = A.tma_mask != 0;
  const int rows = (int)((n1 - j0) < TY ? (n1 - j0) : TY);
  const int cnt = (int)((n0 - i0) < TX ? (n0 - i0) : TX);
  unsigned char* gcol[7] = {reinterpret_cast<unsigned char*>(A.cols.kind), A.cols.amb,
                            reinterpret_cast<unsigned char*>(A.cols.vf), reinterpret_cast<unsigned char*>(A.cols.c),
                            reinterpret_cast<unsigned char*>(A.cols.ff), reinterpret_cast<unsigned char*>(A.cols.fcl),
                            reinterpret_cast<unsigned char*>(A.cols.ic)};

  // What this thread's slot of each staging buffer holds: 0 not known (first use, or a cut cell,
  // whose slot the fill leaves alone), 1 an uncut cell outside, 2 inside (2 bits per buffer).
  int slots = 0;
  for (long long k = k0; k < k1; ++k) {
    const int sb = (int)((k - k0) & 1);
    unsigned char* sbase = smem + sb * L::stage_bytes;
    {
      // round r samples slabs k0 + NS r .. k0 + NS r + NS - 1 before the slice that first needs its
      // first slab; the slabs it overwrites were last read before the previous slice's barriers
      const int kk = (int)(k - k0);
      if (kk == 0) sample_round(k0, k1, false);
      else if (kk % NS == NS - 1) sample_round(k + 1, k1, false);
    }
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
      const int state = nout == 8 ? 2 : (nout == 0 ? 1 : 0);
      if (state != 0) {
        const T hz = T(0.5) * (zb - za);
        const T one = nout == 8 ? T(1) : T(0);
        const T cen[3] = {cx, cy, za + T(0.5) * dz};
        // (Float32 only: at Float64 the split cost more than the stores it saved, 4.91 vs 4.76 ms)
        if (sizeof(T) == 4 && ((slots >> (2 * sb)) & 3) == state) {
          if constexpr (sizeof(T) == 4) put_uncut_z(stage_at<T>(sbase), lc, cen[2], hx, hy, hz);
        } else {
          const T ff[6] = {one, one, one, one, one, one};
          const T fcl[12] = {hy, hz, hy, hz, hx, hz, hx, hz, hx, hy, hx, hy};
          const Stage<T> st = stage_at<T>(sbase);
          st.kind[lc] = int8_t(nout == 8 ? 1 : 0);
          st.amb[lc] = 0;
          st.vf[lc] = one;
          st.c[3 * lc] = cen[0]; st.c[3 * lc + 1] = cen[1]; st.c[3 * lc + 2] = cen[2];
          put_vec<T>(st.ff + 6 * lc, ff, 6);
          put_vec<T>(st.fcl + 12 * lc, fcl, 12);
        }
      } else {
        is_cut = true;
      }
      slots = (slots & ~(3 << (2 * sb))) | (state << (2 * sb));
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
    if (fast && tid == 0) {
      // one thread stores the TMA-addressable columns: one box each (clipped at the grid's edge)
      const int ci0 = (int)i0, cj0 = (int)j0, ck = (int)k;
      if (A.tma_mask & 1) tma_store3(&maps.m[0], sbase + col_offset<T>(0), ci0, cj0, ck);
      if (A.tma_mask & 2) tma_store3(&maps.m[1], sbase + col_offset<T>(1), ci0, cj0, ck);
      if (A.tma_mask & 4) tma_store3(&maps.m[2], sbase + col_offset<T>(2), ci0, cj0, ck);
      if (A.tma_mask & 8) tma_store3(&maps.m[3], sbase + col_offset<T>(3), 3 * ci0, cj0, ck);
      if (A.tma_mask & 16) tma_store3(&maps.m[4], sbase + col_offset<T>(4), 6 * ci0, cj0, ck);
      if (A.tma_mask & 32) tma_store4(&maps.m[5], sbase + col_offset<T>(5), 0, ci0, cj0, ck);
      if (A.tma_mask & 64) tma_store3(&maps.m[6], sbase + col_offset<T>(6), 3 * ci0, cj0, ck);
      bulk_commit();
    }
    if (A.tma_mask != 0x7f) {
      // the columns TMA cannot address, copied by every thread: kind / ambiguous as one 32-bit word
      // per thread where every row starts on a 4-byte boundary (rows x 2 columns x TX/4 words fit
      // in the CTA), else bytes; T columns by element
      static_assert(2 * TY * (TX / 4) <= NT, "one word of kind / ambiguous per thread");
      if (A.byte_words) {
        const int wpr = (cnt + 3) / 4;  // words per row (cnt is a multiple of 4 here)
        const int w = tid % wpr, rest = tid / wpr, r = rest % TY, col = rest / TY;
        if (col < 2 && r < rows && !(A.tma_mask & (1 << col))) {
          const long long rowc = row0 + (long long)r * n0;
          reinterpret_cast<uint32_t*>(gcol[col] + rowc)[w] =
              reinterpret_cast<const uint32_t*>(sbase + col_offset<T>(col) + r * col_bytes<T>(col))[w];
        }
      }
      // the rest element by element; most grids have none (every float column TMA-addressed and
      // the byte columns copied as words), and the row loop is then skipped whole (200^3: 31.4 ->
      // 18.3 warp instructions per cell, 0.383 -> 0.244 ms per update)
      for (int r = 0; A.thread_cols && r < rows; ++r) {
        const long long rowc = row0 + (long long)r * n0;
#pragma unroll
        for (int col = 0; col < 7; ++col) {
          if (!(A.thread_cols & (1 << col))) continue;
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

template <class T, bool SAMPLE, bool MX>
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
    mc_cut_cell<T, MX>(ph, l, org, cs, A.tb, st, ci);
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

// The column maps of a marching-cubes cache: bit c of the result is set when column c (kind,
// ambiguous, volume_fraction, centroid, face_fraction, face_centroid_local, interface_centroid) can
// be written by TMA tensor stores -- its base 16-byte aligned, its row pitch (x extent x bytes per
// cell) a multiple of 16 bytes, every dimension below 2^31. The CTA's threads copy the others.
template <class T>
int make_column_maps(const DevGrid<T>& g, const Cols& cols, ColumnMaps* maps) {
  using TL = Tile<T>;
  const long long n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  if (12 * n0 >= 0x7fffffffLL || n1 >= 0x7fffffffLL || n2 >= 0x7fffffffLL) return 0;
  EncodeTiledFn enc = encode_fn();
  if (!enc) return 0;
  void* base[7] = {cols.kind, cols.amb, cols.vf, cols.c, cols.ff, cols.fcl, cols.ic};
  const CUtensorMapDataType tt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint64_t es = sizeof(T);
  const int width[7] = {1, 1, 1, 3, 6, 12, 3};
  int mask = 0;
  for (int c = 0; c < 7; ++c) {
    const CUtensorMapDataType dt = c < 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : tt;
    const cuuint64_t e = c < 2 ? 1 : es;
    const cuuint64_t w = width[c];
    if ((reinterpret_cast<uintptr_t>(base[c]) & 15u) || ((w * e * (cuuint64_t)n0) & 15u)) continue;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r;
    if (c == 5) {
      const cuuint64_t dims[4] = {12, (cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
      const cuuint64_t strides[3] = {12 * e, 12 * e * n0, 12 * e * n0 * n1};
      const cuuint32_t box[4] = {12, (cuuint32_t)TL::TX, (cuuint32_t)TL::TY, 1};
      r = enc(&maps->m[c], dt, 4, base[c], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
      const cuuint64_t dims[3] = {w * n0, (cuuint64_t)n1, (cuuint64_t)n2};
      const cuuint64_t strides[2] = {w * e * n0, w * e * n0 * n1};
      const cuuint32_t box[3] = {(cuuint32_t)(w * TL::TX), (cuuint32_t)TL::TY, 1};
      r = enc(&maps->m[c], dt, 3, base[c], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (r == CUDA_SUCCESS) mask |= 1 << c;
  }
  return mask;
}

}  // namespace

namespace cci {

namespace {
constexpr long long DEFAULT_WAIT_LIMIT = 1ll << 22;  // mbarrier polls of the learned kernels' waits
long long g_wait_limit = DEFAULT_WAIT_LIMIT;
}  // namespace
long long set_wait_limit(long long polls) {
  const long long old = g_wait_limit;
  g_wait_limit = polls < 0 ? DEFAULT_WAIT_LIMIT : polls;
  return old;
}
long long wait_limit() { return g_wait_limit; }

namespace {
// SMs of the current device (read once per device).
long long device_sms() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::atomic<int>* c = dev >= 0 && dev < 64 ? &cache[dev] : nullptr;
  int v = c ? c->load(std::memory_order_relaxed) : 0;
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    if (c) c->store(v, std::memory_order_relaxed);
  }
  return v;
}
}  // namespace

// Slices per fill pencil for an n0 x n1 x n2 grid. The CTAs are launched x-tile fastest and
// z-layer slowest, so every layer of pencils but the last is kz slices deep and the last is the
// remainder. Each candidate depth (kz + 1 a whole number of NS-slab sampling rounds) is scored by
// list-scheduling the launch on the resident CTAs (each pencil to the earliest free one, in launch
// order), a pencil taking its slices plus PENCIL_OVERHEAD slice-times (its tape load, first
// sampling round and last drain). Few waves of deep pencils leave SMs idle in the last wave: at
// 256^3, 31-slice pencils make 5.2 waves of the 444 resident CTAs; 27-slice pencils fill 5.8.
int pencil_slices(long long n0, long long n1, long long n2, bool f64) {
  const long long tx = f64 ? Tile<double>::TX : Tile<float>::TX, ty = Tile<float>::TY;
  const long long tiles = ((n0 + tx - 1) / tx) * ((n1 + ty - 1) / ty);
  const long long slots = device_sms() * (f64 ? Tile<double>::MINB : Tile<float>::MINB);
  constexpr double PENCIL_OVERHEAD = 2.0;
  int best = KZ;
  double best_t = 0;
  for (int kz = KZ; kz >= NS - 1; kz -= NS) {
    const long long layers = (n2 + kz - 1) / kz;
    const long long rem = n2 - (layers - 1) * kz;
    // groups of resident CTAs that become free at the same time: (time, count), times increasing
    double gt[8];
    long long gc[8];
    int ng = 1;
    gt[0] = 0;
    gc[0] = slots;
    double end = 0;
    const long long batch[2] = {tiles * (layers - 1), tiles};
    const double dur[2] = {kz + PENCIL_OVERHEAD, rem + PENCIL_OVERHEAD};
    for (int bi = 0; bi < 2; ++bi) {
      long long m = batch[bi];
      while (m > 0) {
        // the earliest group takes as many pencils as it has CTAs; they free up dur later
        const long long k = gc[0] < m ? gc[0] : m;
        const double t = gt[0] + dur[bi];
        end = t > end ? t : end;
        m -= k;
        if (k == gc[0]) {
          for (int q = 1; q < ng; ++q) { gt[q - 1] = gt[q]; gc[q - 1] = gc[q]; }
          --ng;
        } else {
          gc[0] -= k;
        }
        int q = 0;
        while (q < ng && gt[q] < t) ++q;
        if (q < ng && gt[q] == t) {
          gc[q] += k;
        } else if (ng < 8) {
          for (int r = ng; r > q; --r) { gt[r] = gt[r - 1]; gc[r] = gc[r - 1]; }
          gt[q] = t;
          gc[q] = k;
          ++ng;
        } else {
          gc[ng - 1] += k;  // out of groups: merge into the latest (a later free time, never earlier)
          gt[ng - 1] = t > gt[ng - 1] ? t : gt[ng - 1];
        }
      }
    }
    if (kz == KZ || end < best_t * 0.995) {  // a shallower pencil only for a clear gain
      best = kz;
      best_t = end;
    }
  }
  return best;
}

size_t mc_prune_bytes(long long n0, long long n1, long long n2, int n_ops, bool f64) {
  const long long tx = f64 ? Tile<double>::TX : Tile<float>::TX, ty = Tile<float>::TY;
  const long long kz = pencil_slices(n0, n1, n2, f64);
  const long long blocks = ((n0 + tx - 1) / tx) * ((n1 + ty - 1) / ty) * ((n2 + kz - 1) / kz);
  return size_t(((blocks * 4 + 15) / 16) * 16 + blocks * (long long)n_ops * (long long)sizeof(cc_op));
}

namespace {
// One fill launch. (4 CTAs per SM at Float32 was measured too: faster only while grids whose x
// extent is not a multiple of 16 still walked a per-row copy loop; without it 3 is faster at
// every size: 500^3 2.85 against 3.18 ms, 260^3 0.468 against 0.496.)
template <class T, bool SAMPLE, bool PRUNED>
cudaError_t launch_fill(const McArgs<T>& a, const ColumnMaps& maps, unsigned blocks, int sm, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(mc_fill_kernel<T, SAMPLE, PRUNED>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  mc_fill_kernel<T, SAMPLE, PRUNED><<<blocks, Tile<T>::NT, sm, s>>>(a, maps);
  return cudaSuccess;
}
}  // namespace

template <class T>
cudaError_t launch_mc(const DevGrid<T>& g, const DevTape& tape, const T* phi_in, T* phi_out,
                      const Cols& cols, const DevTable& tb, unsigned* cut_list, unsigned* cut_count,
                      cudaStream_t s, bool with_cut, bool mixed, void* prune_scratch, size_t prune_bytes) {
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
  a.tma_mask = make_column_maps<T>(g, cols, &maps);
  a.byte_words = (g.n[0] % 4 == 0 && (reinterpret_cast<uintptr_t>(cols.kind) & 3u) == 0 &&
                  (reinterpret_cast<uintptr_t>(cols.amb) & 3u) == 0) ? 1 : 0;
  a.thread_cols = ~a.tma_mask & 0x7f & ~(a.byte_words ? 3 : 0);
  a.n_itiles = int((g.n[0] + TL::TX - 1) / TL::TX);
  a.n_jtiles = int((g.n[1] + TL::TY - 1) / TL::TY);
  a.kz = pencil_slices(g.n[0], g.n[1], g.n[2], sizeof(T) == 8);
  const long long nk = (g.n[2] + a.kz - 1) / a.kz;
  const long long blocks = (long long)a.n_itiles * a.n_jtiles * nk;
  if (blocks <= 0 || blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaMemsetAsync(cut_count, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  const bool sample = phi_in == nullptr;
  a.pruned_ops = nullptr;
  a.pruned_count = nullptr;
  if (sample && tape.prunable && prune_scratch && prune_bytes >= mc_prune_bytes(g.n[0], g.n[1], g.n[2], tape.n_ops, sizeof(T) == 8)) {
    int* cnt = static_cast<int*>(prune_scratch);
    cc_op* ops = reinterpret_cast<cc_op*>(static_cast<unsigned char*>(prune_scratch) + ((blocks * 4 + 15) / 16) * 16);
    const int psm = PruneSmem::of(tape, 0).end;
    if (psm > 48 * 1024) {
      e = cudaFuncSetAttribute(prune_pencils_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, psm);
      if (e != cudaSuccess) return e;
    }
    prune_pencils_kernel<T><<<unsigned(blocks), 256, psm, s>>>(a, ops, cnt);
    a.pruned_ops = ops;
    a.pruned_count = cnt;
  }
  const int sm = smem_bytes<T>(sample ? tape.bytes_len : 0);
  const int cut_blocks = 148 * 8;
  // the FP64 islands of mixed precision exist for Float32 caches only
  const bool mx = mixed && sizeof(T) == 4;
  if (sample && a.pruned_ops) {
    e = launch_fill<T, true, true>(a, maps, unsigned(blocks), sm, s);
    if (e != cudaSuccess) return e;
    if (with_cut && mx) mc_cut_kernel<T, true, true><<<cut_blocks, CUT_NT, 0, s>>>(a);
    else if (with_cut) mc_cut_kernel<T, true, false><<<cut_blocks, CUT_NT, 0, s>>>(a);
  } else if (sample) {
    e = launch_fill<T, true, false>(a, maps, unsigned(blocks), sm, s);
    if (e != cudaSuccess) return e;
    if (with_cut && mx) mc_cut_kernel<T, true, true><<<cut_blocks, CUT_NT, 0, s>>>(a);
    else if (with_cut) mc_cut_kernel<T, true, false><<<cut_blocks, CUT_NT, 0, s>>>(a);
  } else {
    e = launch_fill<T, false, false>(a, maps, unsigned(blocks), sm, s);
    if (e != cudaSuccess) return e;
    if (with_cut && mx) mc_cut_kernel<T, false, true><<<cut_blocks, CUT_NT, 0, s>>>(a);
    else if (with_cut) mc_cut_kernel<T, false, false><<<cut_blocks, CUT_NT, 0, s>>>(a);
  }
  return cudaGetLastError();
}

template cudaError_t launch_mc<float>(const DevGrid<float>&, const DevTape&, const float*, float*,
                                      const Cols&, const DevTable&, unsigned*, unsigned*, cudaStream_t, bool, bool,
                                      void*, size_t);
template cudaError_t launch_mc<double>(const DevGrid<double>&, const DevTape&, const double*, double*,
                                       const Cols&, const DevTable&, unsigned*, unsigned*, cudaStream_t, bool, bool,
                                       void*, size_t);

}  // namespace cci
