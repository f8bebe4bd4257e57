// batch.cu -- many marching-squares updates in one persistent launch over a work list, captured
// in a CUDA graph, with an autotuner for the launch shape.
//
// A batch holds any number of updates, each with its own body and cache:
// MarchingSquaresCutCell on a CartesianGrid (update_cache!, src/marching_squares/cache.jl:49-78)
// or on the leaves of an AdaptiveMesh{2} (:115-137). The work list is the concatenation of
// every update's tiles: tile_x x tile_y cells of a grid, or `threads` leaves of a tree. A
// persistent grid of CTAs (ctas_per_sm per SM) takes `chunk` tiles at a time from one atomic
// counter. No CTA ever waits on another, so a pop cannot spin. Per grid tile the CTA samples the
// tile's (tile_x + 1) x (tile_y + 1) nodes once into shared memory (each node's phi written by
// the one tile that owns it), then builds every cell from those values. Per leaf chunk each
// thread samples its leaf's four corners and builds the leaf. Every cell's arithmetic is the
// single-update kernels' (ms.cu), so a batched update is bit-identical to the same update run
// alone, whatever the launch shape.
//
// cc_batch_run replays a CUDA graph: the upload of the bodies' op-tapes (from pinned staging, so a
// body moved with cc_batch_set_body is picked up by the next replay), the counter reset and the
// kernel. It runs on the batch's own stream, ordered after and before the caller's stream by
// events. cc_batch_autotune times the candidate launch shapes on the batch as it stands and keeps
// the fastest.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"
#include "cc_device.cuh"
#include "cc_internal.h"
#include "ms_cell.cuh"

namespace {

using namespace ccd;
using namespace ccms;

// get_node's coordinate x0 + T(i) d from a 32-bit index: T(i) is the same value as from 64 bits.
template <class T> __device__ __forceinline__ T node_coord_i(T x0, T d, int i) { return x0 + T(i) * d; }
using cci::Cols;

// One update as the kernel sees it.
struct BatchItem {
  long long tile_begin;  // its first tile in the work list
  long long n0, n1;      // grid: cells per axis; tree: n0 = leaves
  int kind;              // 0 = grid, 1 = tree
  int tiles_x;           // grid: tiles along x
  int tape_off, n_ops, n_params, pad_;
  double x0[2], d[2];    // grid: origin, cell size; tree: origin, base cell size
  const int32_t* level;  // tree
  const int32_t* coord;  // tree
  void* phi;
  Cols cols;
};

struct BatchArgs {
  const BatchItem* items;
  int n_items;
  int tx, ty;   // grid tile in cells
  int chunk;    // tiles per pop
  const unsigned char* tapes;
  unsigned long long* counter;
  long long total_tiles;
  int tape_smem;  // bytes reserved for one op-tape in shared memory
  int band;       // band compaction: percent of a tile's cells (0 never, 100 always)
};

__device__ __forceinline__ int find_item(const BatchItem* items, int n, long long tile) {
  int lo = 0, hi = n - 1;  // the last item whose tile_begin <= tile
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Whether a cell of corner values ph is cut: ms_cell's own test (not every corner on one side).
template <class T>
__device__ __forceinline__ bool ms_is_cut(const T* node, int nxn, int a, int b) {
  const int nout = (node[a + nxn * b] >= T(0)) + (node[a + 1 + nxn * b] >= T(0)) +
                   (node[a + 1 + nxn * (b + 1)] >= T(0)) + (node[a + nxn * (b + 1)] >= T(0));
  return nout != 0 && nout != 4;
}

// BAND: the instantiation with band compaction (A.band > 0); without it the kernel carries none of
// that code, so a batch that does not compact runs exactly as before the option existed.
template <class T, bool MX, bool BAND>
__global__ void __launch_bounds__(256) ms_batch_kernel(const BatchArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* node = reinterpret_cast<T*>(smem + A.tape_smem);
  // band compaction: the tile's cut cells (a + tile_x * b), after the node values
  uint16_t* band = reinterpret_cast<uint16_t*>(smem + A.tape_smem + ((A.tx + 1) * (A.ty + 1) * int(sizeof(T)) + 15) / 16 * 16);
  __shared__ long long s_first;
  __shared__ int s_ncut, s_nlist;
  const int nt = blockDim.x;
  const int nxn = A.tx + 1, nyn = A.ty + 1;
  int cur = -1;
  STape<T> tp;
  for (;;) {
    __syncthreads();  // every thread is done with the previous chunk (s_first, node, the tape)
    if (threadIdx.x == 0) s_first = (long long)atomicAdd(A.counter, (unsigned long long)A.chunk);
    __syncthreads();
    const long long first = s_first;
    if (first >= A.total_tiles) break;
    const long long last = first + A.chunk < A.total_tiles ? first + A.chunk : A.total_tiles;
    for (long long tile = first; tile < last; ++tile) {
      const int it = find_item(A.items, A.n_items, tile);
      const BatchItem& I = A.items[it];
      if (it != cur) {
        __syncthreads();
        tp = load_tape<T>(A.tapes + I.tape_off, I.n_ops, I.n_params, smem);
        __syncthreads();
        cur = it;
      }
      const long long lt = tile - I.tile_begin;
      if (I.kind == 0) {
        // one grid tile: its nodes into shared memory (owned ones to phi), then its cells
        // 32-bit node and cell coordinates (a batch grid has fewer than 2^31 cells per axis, checked
        // when it is added); only the linear cell and node indices are 64-bit
        const int n0 = int(I.n0), n1 = int(I.n1);
        const T gx0 = T(I.x0[0]), gy0 = T(I.x0[1]), dx = T(I.d[0]), dy = T(I.d[1]);
        const unsigned ltu = unsigned(lt), row = ltu / unsigned(I.tiles_x);  // 32-bit: tiles of one grid
        const int i0 = int(ltu - row * unsigned(I.tiles_x)) * A.tx, j0 = int(row) * A.ty;
        T* phi = static_cast<T*>(I.phi);
        if (BAND && threadIdx.x == 0) {
          s_ncut = 0;
          s_nlist = 0;
        }
        for (int v = threadIdx.x; v < nxn * nyn; v += nt) {
          const int a = v % nxn, b = v / nxn;
          const int i = i0 + a, j = j0 + b;
          if (i <= n0 && j <= n1) {
            const T x[2] = {node_coord_i(gx0, dx, i), node_coord_i(gy0, dy, j)};
            const T val = tape_eval<T, 2, T>(tp, x);
            node[v] = val;
            if ((a < A.tx || i == n0) && (b < A.ty || j == n1)) phi[(long long)i + (long long)(n0 + 1) * j] = val;
          }
        }
        __syncthreads();
        const T cs[2] = {dx, dy};
        auto cell = [&](int a, int b) {
          const int i = i0 + a, j = j0 + b;
          if (i < n0 && j < n1) {
            const T xa = node_coord_i(gx0, dx, i), xb = node_coord_i(gx0, dx, i + 1);
            const T ya = node_coord_i(gy0, dy, j), yb = node_coord_i(gy0, dy, j + 1);
            const T nd[4][2] = {{xa, ya}, {xb, ya}, {xb, yb}, {xa, yb}};
            const T ph[4] = {node[a + nxn * b], node[a + 1 + nxn * b], node[a + 1 + nxn * (b + 1)],
                             node[a + nxn * (b + 1)]};
            ms_cell<T, MX>(nd, ph, cs, I.cols, (long long)i + (long long)n0 * j);
          }
        };
        const bool rowwise = sizeof(T) == 4 && nt % A.tx == 0;
        if constexpr (!BAND) {
          if (rowwise) {
            // the block covers whole tile rows: a thread keeps its column and steps through rows
            // (Float32 only: measured, the Float64 instantiation runs 6% slower this way)
            const int a = threadIdx.x % A.tx, step = nt / A.tx;
            for (int b = threadIdx.x / A.tx; b < A.ty; b += step) cell(a, b);
          } else {
            for (int c = threadIdx.x; c < A.tx * A.ty; c += nt) cell(c % A.tx, c / A.tx);
          }
        } else {
          // Band compaction (A.band percent): when few enough of the tile's cells are cut, the
          // threads fill the uncut cells and list the cut ones, then build the listed cells densely,
          // so the long construction runs on full warps instead of on the few lanes whose cell
          // happens to be cut. The same ms_cell runs for every cell either way: the same bits.
          bool compact = A.band >= 100;
          if (A.band < 100) {
            int mine = 0;
            if (rowwise) {
              const int a = threadIdx.x % A.tx, step = nt / A.tx;
              for (int b = threadIdx.x / A.tx; b < A.ty; b += step)
                mine += (i0 + a < n0 && j0 + b < n1 && ms_is_cut(node, nxn, a, b)) ? 1 : 0;
            } else {
              for (int c = threadIdx.x; c < A.tx * A.ty; c += nt) {
                const int a = c % A.tx, b = c / A.tx;
                mine += (i0 + a < n0 && j0 + b < n1 && ms_is_cut(node, nxn, a, b)) ? 1 : 0;
              }
            }
            if (mine) atomicAdd(&s_ncut, mine);
            __syncthreads();
            compact = s_ncut * 100 <= A.band * A.tx * A.ty;
          }
          auto visit = [&](int a, int b) {
            if (compact && i0 + a < n0 && j0 + b < n1 && ms_is_cut(node, nxn, a, b))
              band[atomicAdd(&s_nlist, 1)] = uint16_t(a + A.tx * b);
            else
              cell(a, b);
          };
          if (rowwise) {
            const int a = threadIdx.x % A.tx, step = nt / A.tx;
            for (int b = threadIdx.x / A.tx; b < A.ty; b += step) visit(a, b);
          } else {
            for (int c = threadIdx.x; c < A.tx * A.ty; c += nt) visit(c % A.tx, c / A.tx);
          }
          if (compact) {
            __syncthreads();
            const int m = s_nlist;
            for (int c = threadIdx.x; c < m; c += nt) cell(band[c] % A.tx, band[c] / A.tx);
          }
        }
      } else {
        // one chunk of tree leaves, a leaf per thread (as ms_tree_kernel)
        const long long l = lt * nt + threadIdx.x;
        if (l < I.n0) {
          const T x00 = T(I.x0[0]), x01 = T(I.x0[1]);
          const int lv = I.level[l];
          const T scale = T(ldexp(1.0, -lv));
          const T h[2] = {T(I.d[0]) * scale, T(I.d[1]) * scale};
          const long long cx = I.coord[2 * l], cy = I.coord[2 * l + 1];
          const T xa = x00 + T(cx) * h[0], xb = x00 + T(cx + 1) * h[0];
          const T ya = x01 + T(cy) * h[1], yb = x01 + T(cy + 1) * h[1];
          const T nd[4][2] = {{xa, ya}, {xb, ya}, {xb, yb}, {xa, yb}};
          T* phi4 = static_cast<T*>(I.phi);
          T ph[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            ph[q] = tape_eval<T, 2, T>(tp, nd[q]);
            phi4[4 * l + q] = ph[q];
          }
          ms_cell<T, MX>(nd, ph, h, I.cols, l);
        }
      }
      __syncthreads();  // the next tile overwrites the node values this one's cells read
    }
  }
}

struct HostItem {
  int kind;
  cc_grid g;
  cc_tree t;
  std::vector<cc_op> ops;
  std::vector<double> params;
  void* phi;
  cc_cells cells;
};

}  // namespace

struct cc_batch {
  int device = 0;
  int prec = CC_F32;
  std::vector<HostItem> items;
  cc_batch_config cfg{32, 8, 256, 4, 2, 1, 0};
  bool layout_ok = false;  // device items and tapes match `items` and `cfg`
  bool graph_ok = false;   // `exec` replays the current layout
  BatchItem* items_dev = nullptr;
  size_t items_cap = 0;
  unsigned char* tapes_dev = nullptr;
  size_t tapes_cap = 0;
  unsigned char* tapes_host = nullptr;  // pinned staging
  size_t tapes_host_cap = 0;
  size_t tapes_bytes = 0;
  int max_tape = 0;
  std::vector<int> tape_off;
  unsigned long long* counter = nullptr;
  long long total_tiles = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t in_ready = nullptr, done = nullptr;
  bool pending = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

cc_status fail(cc_status s, const std::string& m) {
  cci::set_last_error(m);
  return s;
}
cc_status cuda_fail(cudaError_t e, const char* where) {
  cci::set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
  return CC_CUDA_ERR;
}

struct Dev {
  int old = -1;
  explicit Dev(int d) {
    cudaGetDevice(&old);
    if (old != d) cudaSetDevice(d);
  }
  ~Dev() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (old >= 0 && cur != old) cudaSetDevice(old);
  }
};

size_t elem_size(int prec) { return prec == CC_F64 ? 8 : 4; }

size_t pack(int prec, const cc_optape* t, unsigned char* out, int* np) {
  return prec == CC_F64 ? cci::pack_tape<double>(t, 2, out, np) : cci::pack_tape<float>(t, 2, out, np);
}

cc_optape tape_of(const HostItem& it) {
  cc_optape t;
  t.ops = it.ops.data();
  t.n_ops = int(it.ops.size());
  t.n_params = int(it.params.size());
  t.params = it.params.data();
  return t;
}

cc_status wait_pending(cc_batch* b) {
  if (!b->pending) return CC_OK;
  const cudaError_t e = cudaEventSynchronize(b->done);
  if (e != cudaSuccess) return cuda_fail(e, "batch");
  b->pending = false;
  return CC_OK;
}

void drop_graph(cc_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_ok = false;
}

int tape_smem_of(const cc_batch* b) { return ((b->max_tape + 15) / 16) * 16; }
int smem_of(const cc_batch* b) {
  const int nodes = (b->cfg.tile_x + 1) * (b->cfg.tile_y + 1) * int(elem_size(b->prec));
  const int list = b->cfg.band_percent > 0 ? b->cfg.tile_x * b->cfg.tile_y * int(sizeof(uint16_t)) : 0;
  return tape_smem_of(b) + (nodes + 15) / 16 * 16 + list;
}

// Pack every body into the staging buffer and lay the work list out for the current config.
cc_status build_layout(cc_batch* b) {
  if (b->layout_ok) return CC_OK;
  cc_status st = wait_pending(b);
  if (st != CC_OK) return st;
  drop_graph(b);
  const size_t cap = cci::tape_pack_capacity();
  std::vector<unsigned char> tmp(cap);
  b->tape_off.assign(b->items.size(), 0);
  std::vector<BatchItem> dev(b->items.size());
  size_t off = 0;
  int max_tape = 0;
  long long tiles = 0;
  const int tx = b->cfg.tile_x, ty = b->cfg.tile_y, nt = b->cfg.threads;
  // sizes first, so the staging buffer is grown once
  std::vector<size_t> sz(b->items.size());
  std::vector<int> nps(b->items.size());
  for (size_t k = 0; k < b->items.size(); ++k) {
    const cc_optape t = tape_of(b->items[k]);
    sz[k] = pack(b->prec, &t, tmp.data(), &nps[k]);
    b->tape_off[k] = int(off);
    off += ((sz[k] + 15) / 16) * 16;
    if (int(sz[k]) > max_tape) max_tape = int(sz[k]);
  }
  if (off > 0x7fffffffULL) return fail(CC_TOO_LARGE, "the batch's op-tapes exceed 2 GiB");
  if (off > b->tapes_host_cap) {
    if (b->tapes_host) cudaFreeHost(b->tapes_host);
    b->tapes_host = nullptr;
    b->tapes_host_cap = 0;
    const cudaError_t e = cudaMallocHost(&b->tapes_host, off);
    if (e != cudaSuccess) return cuda_fail(e, "batch staging");
    b->tapes_host_cap = off;
  }
  if (off > b->tapes_cap) {
    if (b->tapes_dev) cudaFree(b->tapes_dev);
    b->tapes_dev = nullptr;
    b->tapes_cap = 0;
    const cudaError_t e = cudaMalloc(&b->tapes_dev, off);
    if (e != cudaSuccess) return cuda_fail(e, "batch tapes");
    b->tapes_cap = off;
  }
  for (size_t k = 0; k < b->items.size(); ++k) {
    const HostItem& h = b->items[k];
    const cc_optape t = tape_of(h);
    int np = 0;
    pack(b->prec, &t, b->tapes_host + b->tape_off[k], &np);
    BatchItem& d = dev[k];
    std::memset(&d, 0, sizeof d);
    d.tile_begin = tiles;
    d.kind = h.kind;
    d.tape_off = b->tape_off[k];
    d.n_ops = t.n_ops;
    d.n_params = np;
    d.phi = h.phi;
    d.cols = Cols{h.cells.kind, h.cells.ambiguous, h.cells.volume_fraction, h.cells.centroid, h.cells.face_fraction,
                  h.cells.face_centroid_local, h.cells.interface_centroid};
    if (h.kind == 0) {
      d.n0 = h.g.n[0];
      d.n1 = h.g.n[1];
      d.x0[0] = h.g.x0[0]; d.x0[1] = h.g.x0[1];
      d.d[0] = h.g.d[0]; d.d[1] = h.g.d[1];
      const long long txs = (d.n0 + tx - 1) / tx, tys = (d.n1 + ty - 1) / ty;
      if (txs > 0x7fffffffLL) return fail(CC_TOO_LARGE, "grid too wide for the batch's tiles");
      d.tiles_x = int(txs);
      tiles += txs * tys;
    } else {
      d.n0 = h.t.nleaves;
      d.x0[0] = h.t.x0[0]; d.x0[1] = h.t.x0[1];
      d.d[0] = h.t.base_d[0]; d.d[1] = h.t.base_d[1];
      d.level = h.t.level;
      d.coord = h.t.coord;
      tiles += (d.n0 + nt - 1) / nt;
    }
  }
  b->tapes_bytes = off;
  b->max_tape = max_tape;
  b->total_tiles = tiles;
  if (smem_of(b) > 200 * 1024) return fail(CC_TOO_LARGE, "batch tile and op-tape exceed shared memory");
  const size_t ib = dev.size() * sizeof(BatchItem);
  if (ib > b->items_cap) {
    if (b->items_dev) cudaFree(b->items_dev);
    b->items_dev = nullptr;
    b->items_cap = 0;
    const cudaError_t e = cudaMalloc(&b->items_dev, ib);
    if (e != cudaSuccess) return cuda_fail(e, "batch items");
    b->items_cap = ib;
  }
  if (ib > 0) {
    const cudaError_t e = cudaMemcpy(b->items_dev, dev.data(), ib, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "batch items");
  }
  b->layout_ok = true;
  return CC_OK;
}

// The work of one run, issued on s: tapes up, counter reset, the persistent kernel.
cudaError_t issue(cc_batch* b, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(b->tapes_dev, b->tapes_host, b->tapes_bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  BatchArgs a;
  a.items = b->items_dev;
  a.n_items = int(b->items.size());
  a.tx = b->cfg.tile_x;
  a.ty = b->cfg.tile_y;
  a.chunk = b->cfg.chunk;
  a.tapes = b->tapes_dev;
  a.counter = b->counter;
  a.total_tiles = b->total_tiles;
  a.tape_smem = tape_smem_of(b);
  a.band = b->cfg.band_percent;
  const int sm = smem_of(b);
  const int grid = 148 * b->cfg.ctas_per_sm;
  const int nt = b->cfg.threads;
  const bool bd = a.band > 0;
  if (b->prec == CC_F64) {
    if (bd) ms_batch_kernel<double, false, true><<<grid, nt, sm, s>>>(a);
    else ms_batch_kernel<double, false, false><<<grid, nt, sm, s>>>(a);
  } else if (b->prec == CC_MIXED) {
    if (bd) ms_batch_kernel<float, true, true><<<grid, nt, sm, s>>>(a);
    else ms_batch_kernel<float, true, false><<<grid, nt, sm, s>>>(a);
  } else {
    if (bd) ms_batch_kernel<float, false, true><<<grid, nt, sm, s>>>(a);
    else ms_batch_kernel<float, false, false><<<grid, nt, sm, s>>>(a);
  }
  return cudaGetLastError();
}

// The kernel's dynamic shared-memory limit for the current layout (set outside any capture).
cudaError_t prepare_kernel(const cc_batch* b) {
  const int sm = smem_of(b);
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  const bool bd = b->cfg.band_percent > 0;
  if (b->prec == CC_F64)
    return bd ? cudaFuncSetAttribute(ms_batch_kernel<double, false, true>, at, sm)
              : cudaFuncSetAttribute(ms_batch_kernel<double, false, false>, at, sm);
  if (b->prec == CC_MIXED)
    return bd ? cudaFuncSetAttribute(ms_batch_kernel<float, true, true>, at, sm)
              : cudaFuncSetAttribute(ms_batch_kernel<float, true, false>, at, sm);
  return bd ? cudaFuncSetAttribute(ms_batch_kernel<float, false, true>, at, sm)
            : cudaFuncSetAttribute(ms_batch_kernel<float, false, false>, at, sm);
}

cc_status check_config(const cc_batch_config* c) {
  if (!c) return fail(CC_BAD_ARG, "null config");
  if (c->tile_x < 1 || c->tile_x > 256 || c->tile_y < 1 || c->tile_y > 256 || c->tile_x * c->tile_y > 4096)
    return fail(CC_BAD_ARG, "batch tile must be 1..256 x 1..256 cells, at most 4096");
  if (c->threads < 32 || c->threads > 256 || c->threads % 32 != 0)
    return fail(CC_BAD_ARG, "batch threads must be a multiple of 32 in 32..256");
  if (c->ctas_per_sm < 1 || c->ctas_per_sm > 32) return fail(CC_BAD_ARG, "batch ctas_per_sm must be 1..32");
  if (c->chunk < 1 || c->chunk > 1024) return fail(CC_BAD_ARG, "batch chunk must be 1..1024");
  if (c->band_percent < 0 || c->band_percent > 100) return fail(CC_BAD_ARG, "batch band_percent must be 0..100");
  return CC_OK;
}

bool same_structure(const HostItem& it, const cc_optape* t) {
  if (int(it.ops.size()) != t->n_ops || int(it.params.size()) != t->n_params) return false;
  for (int i = 0; i < t->n_ops; ++i)
    if (it.ops[i].opcode != t->ops[i].opcode || it.ops[i].combine != t->ops[i].combine ||
        it.ops[i].poff != t->ops[i].poff || it.ops[i].kparam != t->ops[i].kparam)
      return false;
  return true;
}

cc_status add_item(cc_batch* b, HostItem&& it, const cc_optape* body, int32_t* item) {
  it.ops.assign(body->ops, body->ops + body->n_ops);
  it.params.assign(body->params, body->params + body->n_params);
  cc_status st = wait_pending(b);
  if (st != CC_OK) return st;
  b->items.push_back(std::move(it));
  b->layout_ok = false;
  b->graph_ok = false;
  if (item) *item = int32_t(b->items.size() - 1);
  return CC_OK;
}

bool cells_ok(const cc_cells* c) {
  return c && c->kind && c->ambiguous && c->volume_fraction && c->centroid && c->face_fraction &&
         c->face_centroid_local && c->interface_centroid;
}

}  // namespace

extern "C" {

cc_status cc_batch_create(int32_t device, int32_t prec, cc_batch** out) {
  if (!out) return fail(CC_BAD_ARG, "null argument");
  *out = nullptr;
  if (prec != CC_F32 && prec != CC_F64 && prec != CC_MIXED) return fail(CC_BAD_ARG, "unsupported precision");
  Dev dg(device);
  cc_batch* b = new cc_batch();
  b->device = device;
  b->prec = prec;
  cudaError_t e = cudaMalloc(&b->counter, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->in_ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cc_batch_destroy(b);
    return cuda_fail(e, "cc_batch_create");
  }
  *out = b;
  return CC_OK;
}

cc_status cc_batch_destroy(cc_batch* b) {
  if (!b) return CC_OK;
  Dev dg(b->device);
  if (b->pending) cudaEventSynchronize(b->done);
  drop_graph(b);
  if (b->items_dev) cudaFree(b->items_dev);
  if (b->tapes_dev) cudaFree(b->tapes_dev);
  if (b->tapes_host) cudaFreeHost(b->tapes_host);
  if (b->counter) cudaFree(b->counter);
  if (b->in_ready) cudaEventDestroy(b->in_ready);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CC_OK;
}

cc_status cc_batch_add_ms_grid(cc_batch* b, const cc_grid* g, const cc_optape* body, void* phi, const cc_cells* cells,
                               int32_t* item) {
  if (!b || !g || !phi || !cells_ok(cells)) return fail(CC_BAD_ARG, "null argument");
  if (g->dim != 2) return fail(CC_DIM_MISMATCH, "marching squares is 2D");
  if (g->n[0] < 1 || g->n[1] < 1) return fail(CC_BAD_ARG, "every axis needs at least one cell");
  if (g->n[0] >= 0x7fffffffLL || g->n[1] >= 0x7fffffffLL)  // the kernel indexes an axis's nodes in 32 bits
    return fail(CC_TOO_LARGE, "a batched grid has fewer than 2^31 - 1 cells per axis");
  cc_status st = cci::validate_body(body, 2);
  if (st != CC_OK) return st;
  HostItem it;
  it.kind = 0;
  it.g = *g;
  std::memset(&it.t, 0, sizeof it.t);
  it.phi = phi;
  it.cells = *cells;
  return add_item(b, std::move(it), body, item);
}

cc_status cc_batch_add_ms_tree(cc_batch* b, const cc_tree* t, const cc_optape* body, void* phi4,
                               const cc_cells* cells, int32_t* item) {
  if (!b || !t || !phi4 || !cells_ok(cells)) return fail(CC_BAD_ARG, "null argument");
  if (t->nleaves < 0 || (t->nleaves > 0 && (!t->level || !t->coord))) return fail(CC_BAD_ARG, "bad tree");
  cc_status st = cci::validate_body(body, 2);
  if (st != CC_OK) return st;
  HostItem it;
  it.kind = 1;
  std::memset(&it.g, 0, sizeof it.g);
  it.t = *t;
  it.phi = phi4;
  it.cells = *cells;
  return add_item(b, std::move(it), body, item);
}

cc_status cc_batch_set_body(cc_batch* b, int32_t item, const cc_optape* body) {
  if (!b) return fail(CC_BAD_ARG, "null batch");
  if (item < 0 || size_t(item) >= b->items.size()) return fail(CC_BAD_ARG, "no such batch item");
  cc_status st = cci::validate_body(body, 2);
  if (st != CC_OK) return st;
  HostItem& it = b->items[item];
  if (!same_structure(it, body))
    return fail(CC_BAD_TAPE, "a batch item's body may move, not change its op structure; build a new batch");
  Dev dg(b->device);
  if ((st = wait_pending(b)) != CC_OK) return st;
  it.params.assign(body->params, body->params + body->n_params);
  if (b->layout_ok) {  // repack in place: same structure, same packed size
    const cc_optape t = tape_of(it);
    int np = 0;
    pack(b->prec, &t, b->tapes_host + b->tape_off[item], &np);
  }
  return CC_OK;
}

cc_status cc_batch_set_config(cc_batch* b, const cc_batch_config* cfg) {
  if (!b) return fail(CC_BAD_ARG, "null batch");
  cc_status st = check_config(cfg);
  if (st != CC_OK) return st;
  if ((st = wait_pending(b)) != CC_OK) return st;
  const bool layout = cfg->tile_x != b->cfg.tile_x || cfg->tile_y != b->cfg.tile_y || cfg->threads != b->cfg.threads;
  b->cfg = *cfg;
  if (layout) b->layout_ok = false;
  b->graph_ok = false;
  return CC_OK;
}

cc_status cc_batch_get_config(const cc_batch* b, cc_batch_config* cfg) {
  if (!b || !cfg) return fail(CC_BAD_ARG, "null argument");
  *cfg = b->cfg;
  return CC_OK;
}

cc_status cc_batch_info(const cc_batch* b, int64_t* n_items, int64_t* total_tiles) {
  if (!b) return fail(CC_BAD_ARG, "null batch");
  if (n_items) *n_items = int64_t(b->items.size());
  if (total_tiles) *total_tiles = b->layout_ok ? b->total_tiles : -1;
  return CC_OK;
}

cc_status cc_batch_run(cc_batch* b, void* stream) {
  if (!b) return fail(CC_BAD_ARG, "null batch");
  Dev dg(b->device);
  cc_status st = build_layout(b);
  if (st != CC_OK) return st;
  const cudaStream_t user = static_cast<cudaStream_t>(stream);
  if (b->total_tiles == 0) return CC_OK;
  cudaError_t e = prepare_kernel(b);
  if (e == cudaSuccess) e = cudaEventRecord(b->in_ready, user);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->in_ready, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cc_batch_run");
  if (b->cfg.use_graph) {
    if (!b->graph_ok) {
      drop_graph(b);
      e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
      const cudaError_t ie = issue(b, b->stream);
      e = cudaStreamEndCapture(b->stream, &b->graph);
      if (ie != cudaSuccess) {
        drop_graph(b);
        return cuda_fail(ie, "batch graph capture");
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      if (e != cudaSuccess) {
        drop_graph(b);
        return cuda_fail(e, "batch graph instantiate");
      }
      b->graph_ok = true;
    }
    e = cudaGraphLaunch(b->exec, b->stream);
  } else {
    e = issue(b, b->stream);
  }
  if (e == cudaSuccess) e = cudaEventRecord(b->done, b->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(user, b->done, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cc_batch_run");
  b->pending = true;
  return CC_OK;
}

cc_status cc_batch_autotune(cc_batch* b, int32_t reps, cc_batch_config* best, float* best_ms, void* stream) {
  if (!b || reps < 1) return fail(CC_BAD_ARG, "bad arguments");
  Dev dg(b->device);
  static const int tiles[][2] = {{32, 4}, {32, 8}, {64, 4}, {64, 8}, {128, 2}, {32, 16}, {16, 16}};
  static const int threads[] = {128, 256};
  static const int ctas[] = {2, 4, 8};
  static const int chunks[] = {1, 4};
  static const int bands[] = {0, 25, 100};
  const cudaStream_t user = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  // time one candidate: two warm-up runs, then `reps` runs between events on the caller's stream
  auto time_one = [&](const cc_batch_config& c, float* ms) -> cc_status {
    cc_status st = cc_batch_set_config(b, &c);
    for (int w = 0; w < 2 && st == CC_OK; ++w) st = cc_batch_run(b, stream);
    if (st != CC_OK) return st;
    cudaError_t ce = cudaEventRecord(e0, user);
    for (int r = 0; r < reps && st == CC_OK && ce == cudaSuccess; ++r) st = cc_batch_run(b, stream);
    if (st != CC_OK) return st;
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, user);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(ms, e0, e1);
    if (ce != cudaSuccess) return cuda_fail(ce, "cc_batch_autotune");
    *ms /= float(reps);
    return CC_OK;
  };
  cc_status st = e == cudaSuccess ? CC_OK : cuda_fail(e, "cc_batch_autotune");
  const int use_graph = b->cfg.use_graph;
  cc_batch_config top = b->cfg;
  float top_ms = -1.0f;
  for (const auto& tl : tiles) {
    for (int nt : threads) {
      for (int c : ctas) {
        for (int ch : chunks) {
          for (int bd : bands) {
            if (st != CC_OK) break;
            const cc_batch_config cand{tl[0], tl[1], nt, c, ch, use_graph, bd};
            float ms = 0.0f;
            st = time_one(cand, &ms);
            if (st == CC_OK && (top_ms < 0.0f || ms < top_ms)) {
              top_ms = ms;
              top = cand;
            }
          }
        }
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st != CC_OK) return st;
  if ((st = cc_batch_set_config(b, &top)) != CC_OK) return st;
  if (best) *best = top;
  if (best_ms) *best_ms = top_ms;
  return CC_OK;
}

}  // extern "C"
